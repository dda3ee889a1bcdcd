"""The coupled source generated for a mechanism (peregrine_b200/csrc/rategen.cu),
on the CPU: for every shipped mechanism the generated CUDA source holds one
straight-line block per reaction, with the rate state and production rates as
named scalars (no array the species index), and NVRTC compiles it for sm_100a
with nothing loaded on a device.  Its results against the table-driven kernel
are checked on the GPU (tests/test_rategen_gpu.py).
"""

import ctypes
import re
from types import SimpleNamespace

import numpy as np
import pytest

from peregrine_b200 import cases, native


def unfinalized_case(mechanism):
    """A case of the reacting configuration's physics with the mechanism's
    tables and reactions set, never finalized (no device memory)."""
    from peregrine_b200.mixture import Mixture
    from peregrine_b200.solver import Solver

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, tables=mechanism)
    mix = Mixture(cfg["mixture"])
    phys = native.Physics(simulator=native.NAVIER_STOKES, eos=native.EOS_TPG, primary=native.FLUX_HLLC,
                          recon=native.RECON_MUSCL, limiter=native.LIMITERS["koren"], trans=native.TRANS_KINETIC,
                          ns=mix.ns, nregs=2, alpha=1.0, chemistry=native.CHEM_COUPLED)
    h = ctypes.c_void_p()
    native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(h))
    tables = Solver.species_tables(SimpleNamespace(mixture=mix, cfg=cfg))
    for name, values in tables.items():
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        native.call("pgb_case_set_table", h, name.encode(), v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), v.size)
    mech, keep = native.mechanism(mix.constants())
    native.call("pgb_case_set_mechanism", h, ctypes.byref(mech))
    return h, mix, keep


MECHS = ["h2o2_gri30", "h2o2_gri30_oneway", "ch4_o2_ffcmy"]


@pytest.mark.parametrize("mechanism", MECHS)
def test_the_generated_source_is_straight_line_and_compiles(mechanism):
    h, mix, keep = unfinalized_case(mechanism)
    try:
        n = ctypes.c_longlong()
        native.call("pgb_case_rates_source", h, None, 0, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        native.call("pgb_case_rates_source", h, buf, n.value + 1, ctypes.byref(n))
        src = buf.value.decode()
        consts = mix.constants()
        nr = int(consts["rxn_nr"])
        assert len(re.findall(r"// reaction \d+\n", src)) == nr
        # every species quantity a scalar of its own: nothing indexes a per-species array
        assert not re.search(r"\b(omega|gRT|logc|cG|ctb|logtb)\[", src)
        for k in range(mix.ns):
            assert f"double omega{k} = 0.0;" in src
        log = ctypes.create_string_buffer(1 << 16)
        rc = native.load().pgb_case_rates_compile(h, log, len(log))
        if rc == native.ERR_UNSUPPORTED and b"could not be opened" in log.value:
            pytest.skip(log.value.decode())
        assert rc == 0, log.value.decode()
    finally:
        native.call("pgb_case_destroy", h)


def test_the_generated_source_follows_the_mechanism():
    h, mix, keep = unfinalized_case("h2o2_gri30")
    try:
        n = ctypes.c_longlong()
        native.call("pgb_case_rates_source", h, None, 0, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        native.call("pgb_case_rates_source", h, buf, n.value + 1, ctypes.byref(n))
        src = buf.value.decode()
        consts = mix.constants()
        blocks = re.split(r"  \{  // reaction \d+\n", src)[1:]
        for k, body in enumerate(blocks):
            kind = int(consts["rxn_kind"][k])
            # a falloff's pressure ratio, a Troe centre's fit, a plain three-body's concentration
            assert ("logpr" in body) == (kind >= 2), k
            assert ("lfc" in body) == (kind == 3), k
            # the reverse rate only where the reaction is reversible
            assert ("rev" in body) == bool(consts["rxn_reversible"][k]), k
            # its net stoichiometry's species, each once
            net = [int(s) for s, nu in zip(consts["rxn_netsp"][k], consts["rxn_netnu"][k]) if nu != 0]
            assert sorted(int(s) for s in re.findall(r"omega(\d+) \+=", body)) == sorted(net), k
    finally:
        native.call("pgb_case_destroy", h)
