"""Host-side logic with no GPU: the C ABI's symbols, config, meshes, halo maps,
and the multi-rank timing over gloo."""

import ctypes
import os
import re
import socket

import numpy as np
import pytest

from peregrine_b200 import native
from peregrine_b200.config import Config, ConfigError
from peregrine_b200.mesher import CubeMesher, uneven_cuts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "pgb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgb_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = native.load()
    names = header_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    # and the Python binding types every one of them
    assert set(names) <= set(native.SIGNATURES), set(names) - set(native.SIGNATURES)


def test_no_kernel_is_defined_by_two_units():
    # every unit keeps its own constant memory, so a kernel template two units
    # instantiate is two kernels behind one linked launch stub
    from peregrine_b200 import build

    objs = [o for _, o, _ in build.units()]
    if not all(os.path.exists(o) for o in objs):
        pytest.skip("the library's objects are not built here")
    assert build.shared_kernels(objs) == []


def test_errors_carry_the_library_message():
    lib = native.load()
    rc = lib.pgb_case_create(None, None)
    assert rc == native.ERR_ARG
    assert b"null" in lib.pgb_last_error()
    with pytest.raises(native.PgbArgumentError):
        native.check(rc)


def test_config_refuses_unknown_keys_and_bad_choices():
    cfg = Config()
    with pytest.raises(KeyError):
        cfg["simulation"]["simulatr"] = "euler"
    cfg["time-integration"]["integrator"] = "rk5"
    with pytest.raises(ConfigError):
        cfg.validate()
    cfg = Config()
    cfg["mixture"]["trans"] = None
    with pytest.raises(ConfigError):
        cfg.validate()  # navier-stokes needs a transport model
    cfg = Config.from_dict({"simulation": {"simulator": "euler", "dt": "1e-7"}})
    assert cfg["simulation"]["dt"] == 1e-7


def double_flux(simulator="navier-stokes-df", eos="real-gas-df", primary="rusanov", **more):
    given = {"simulation": {"simulator": simulator},
             "mixture": {"species": "o2_h2_pr", "eos": eos, "trans": "kinetic-theory"},
             "adv-flux": {"primary": primary, **more}}
    return Config.from_dict(given)


def test_the_double_flux_takes_its_eos_and_its_flux_functions():
    # peregrine/simulator/eulerdf/simulator.py:15-20 and eulerdf/kernels/flux/function/
    assert double_flux()["simulation"]["simulator"] == "navier-stokes-df"
    assert double_flux(primary="ausmup", recon="muscl", limiter="koren")
    for bad in (dict(eos="real-gas"), dict(simulator="navier-stokes"), dict(primary="hllc")):
        with pytest.raises(ConfigError):
            double_flux(**bad)
    # the library refuses the same before it touches a device
    phys = native.Physics()
    phys.simulator, phys.eos, phys.ns, phys.nregs = native.NAVIER_STOKES_DF, native.EOS_REALGAS_DF, 2, 3
    phys.primary, phys.trans = native.FLUX_HLLC, native.TRANS_KINETIC
    handle = ctypes.c_void_p()
    with pytest.raises(native.PgbUnsupported):
        native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(handle))
    phys.primary, phys.eos = native.FLUX_RUSANOV, native.EOS_REALGAS
    with pytest.raises(native.PgbArgumentError):
        native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(handle))


def test_uneven_cuts_are_seeded_and_bounded():
    for seed in range(5):
        cuts = uneven_cuts(128, 3, 30, 56, np.random.default_rng(seed))
        assert sum(cuts) == 128 and all(30 <= c <= 56 for c in cuts)
    a = uneven_cuts(128, 3, 30, 56, np.random.default_rng(0))
    b = uneven_cuts(128, 3, 30, 56, np.random.default_rng(0))
    assert a == b


def test_lattice_connectivity_and_periodic_node_halo():
    mesh = CubeMesher(mbdims=[3, 2, 1], cells=[[4, 5, 6], [3, 4], [5]], lengths=[1.0, 1.0, 1.0],
                      periodic=[True, True, False])
    blocks = mesh.make_blocks(2)
    assert [b.cells for b in blocks][:3] == [(4, 3, 5), (5, 3, 5), (6, 3, 5)]
    b0 = blocks[0]
    lo, hi = b0.get_intface(1), b0.get_intface(2)
    assert lo.nbr == 2 and lo.periodic and hi.nbr == 1 and not hi.periodic
    assert b0.get_intface(5).nbr is None  # k is not periodic
    # the i-low halo nodes of block 0 are block 2's nodes one in from its high face, moved down one length
    g = b0.ng
    x0 = b0.nodes[g - 1, g:-g, g:-g, 0]
    x2 = blocks[2].nodes[g + blocks[2].ni - 2, g:-g, g:-g, 0]
    assert np.allclose(x0, x2 - 1.0)


def test_halo_map_covers_every_face_halo_cell_once():
    from oracle.oracle import halo_map

    mesh = CubeMesher(mbdims=[2, 2, 2], cells=[[3, 4], [4, 3], [2, 5]], lengths=[1.0] * 3, periodic=[True] * 3)
    blocks = mesh.make_blocks(2)
    m = halo_map(blocks)
    expect = sum(2 * 2 * (b.cells[1] * b.cells[2] + b.cells[0] * b.cells[2] + b.cells[0] * b.cells[1]) for b in blocks)
    assert m.size == expect
    keys = set(zip(m["dblk"], m["di"], m["dj"], m["dk"]))
    assert len(keys) == expect
    # every source is an interior cell of its block
    for r in m[:200]:
        sb = blocks[r["sblk"]]
        for a, c in enumerate((r["si"], r["sj"], r["sk"])):
            assert 2 <= c < 2 + sb.cells[a]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    from peregrine_b200.replicas import max_over_ranks, weak_throughput

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = max_over_ranks(10.0 + rank, dist, device="cpu")
    out[rank] = (ms, weak_throughput(1000, 4, 10, ms, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_report_the_slowest_time_and_the_whole_job():
    import torch.multiprocessing as mp

    # the manager's server process spawned, as the ranks are: no fork of a threaded process
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    assert out[0] == out[1]
    ms, value = out[0]
    assert ms == 11.0
    assert value == pytest.approx(1000 * 4 * 10 * 2 / 0.011)


def test_reacting_tables_and_mechanism_structs_build_on_the_host():
    import types

    from peregrine_b200 import cases, native
    from peregrine_b200.mixture import Mixture
    from peregrine_b200.solver import Solver

    cfg = cases.reacting_config()
    mix = Mixture(cfg["mixture"])
    tables = Solver.species_tables(types.SimpleNamespace(mixture=mix, cfg=cfg))
    assert "cp0" not in tables and tables["cppolyR"].shape == (9, 7) and tables["mupoly"].shape[0] == 9
    consts = mix.constants()
    mech, keep = native.mechanism(consts)
    assert mech.nr == 28 and mech.ntb == 5 and mech.ntroe == 1 and mech.ng == 8
    kinds = [mech.rxn[k].kind for k in range(mech.nr)]
    assert kinds.count(native.RXN_TROE if hasattr(native, "RXN_TROE") else 3) == 1
    # every species index on the device's sides lies within the mixture
    for k in range(mech.nr):
        r = mech.rxn[k]
        for j in range(r.nnet):
            assert 0 <= r.netsp[j] < 9
        assert 0 < r.nnet <= native.MAXNET and r.nreact <= native.MAXSIDE and r.nprod <= native.MAXSIDE


class _FakePool:
    """A pool of fixed cell capacity that finishes a case after its steps."""

    def __init__(self, cap):
        self.cap, self.used, self.slots, self.next = cap, 0, {}, 0
        self.admitted = []

    def admit(self, req):
        need = int(np.prod([c + 4 for c in req.cells]))
        if self.used + need > self.cap:
            return None
        s = self.next
        self.next += 1
        self.used += need
        self.slots[s] = [req, req.steps, need]
        self.admitted.append(req.rid)
        return s

    def step(self, dt, n=1):
        for v in self.slots.values():
            v[1] -= 1
        return 0.5, 14

    def done(self):
        return [s for s, v in self.slots.items() if v[1] <= 0]

    def take(self, slot, cells, kind="1d"):
        req, _, need = self.slots.pop(slot)
        assert kind == req.kind
        self.used -= need
        return np.full(cells, float(req.rid))


def test_server_admits_in_order_as_room_frees_and_times_each_request():
    from peregrine_b200 import serving

    spn, MW = ["H2", "O2", "N2"], [2.016, 31.998, 28.014]
    reqs = serving.requests(12, 0.0, spn, MW, seed=4, steps=3, nmin=8, nmax=16)
    t = [0.0]

    def clock():
        t[0] += 1e-3
        return t[0]

    pool = _FakePool(cap=3 * 20 * 6 * 6)
    out = serving.Server(pool, 1e-8).run(reqs, 3, clock=clock, sleep=lambda s: None)
    # first come, first admitted; every request finished with its own result
    assert pool.admitted == sorted(pool.admitted)
    assert all(r.finished is not None and r.finished >= r.admitted >= r.arrival for r in out)
    assert all(np.all(r.result == r.rid) for r in out)
    st = serving.latency_stats(out)
    assert st["n"] == 12 and st["p99_ms"] >= st["p50_ms"] > 0


def test_serving_requests_follow_the_workload():
    from peregrine_b200 import serving

    spn, MW = ["H2", "H", "O2", "N2"], [2.016, 1.008, 31.998, 28.014]
    reqs = serving.requests(400, 50.0, spn, MW, seed=1)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and abs(arr[-1] / 400 - 1 / 50.0) < 0.3 / 50.0
    zero = [r for r in reqs if r.kind == "0d"]
    one = [r for r in reqs if r.kind == "1d"]
    assert 150 < len(zero) < 250 and all(r.cells == (2, 2, 2) for r in zero)
    assert all(64 <= r.cells[0] <= 2048 for r in one)
    for r in zero:
        p, T = r.prims[0, 0, 0, 0], r.prims[0, 0, 0, 4]
        assert 900 <= T <= 1400 and 1 * 101325 <= p <= 40 * 101325
        Y = np.append(r.prims[0, 0, 0, 5:], 1 - r.prims[0, 0, 0, 5:].sum())
        X = Y / np.array(MW)
        phi = X[0] / X[2] / 2.0
        assert 0.5 - 1e-9 <= phi <= 2.0 + 1e-9


def test_the_stage_registers_are_the_references():
    # peregrine/integrators/rungekutta.py:9-14: each stage reads start then
    # stage, and writes stage, the last writing start
    from peregrine_b200.integrators import Integrator

    cfg = Config()
    cfg["simulation"]["simulator"] = "euler"
    for name, regs in (("tvd-rk3", ("Q", "Q1", "Q2")), ("rk2", ("Q", "Q1", "Q2")), ("rk4", ("Q", "Q1", "Q2", "Q3"))):
        cfg["time-integration"]["integrator"] = name
        st = Integrator(cfg.validate()).stageregs(regs)
        assert st[0].Q == "Q" and all(s.Q == "Q1" for s in st[1:])
        assert all(s.dQ == regs[-1] for s in st)
        assert st[-1].Qout == "Q" and all(s.Qout == "Q1" for s in st[:-1])
