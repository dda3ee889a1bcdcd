"""Binary diffusion on the device against the CPU oracle: the reacting
H2/O2/N2 configuration with the mixture-averaged coefficients of the pair
fits (peregrine/simulator/mixture/diffusion/kernels/binary.mako) in place of
Lewis numbers, the oracle pinned in tests/test_binary_cpu.py.  The bars are
the reacting tests' (tests/test_reacting_gpu.py): the right-hand side within
5e-10 of the flux summands, the state after steps within 1e-9 of each
component's largest.
"""

import numpy as np
import pytest

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu


def build(chemistry=True, integrator="tvd-rk3", cells=12, seed=7):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.reacting_config("navier-stokes", integrator, "hllc", "muscl", "koren", chemistry,
                                tables="h2o2_gri30_binary")
    cfg["mixture"]["diffusion"] = "binary"
    cfg.validate()
    mesh = cases.reacting_mesh(cells, (2, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], cells, seed=seed, width=2.0, dT=600.0,
                                 radicals=2e-3)
    mb.set_prims(prims)
    orc = Oracle(consts, mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, integrator, primary="hllc",
                 recon="muscl", limiter="koren", eos="tpg", trans="kinetic-theory",
                 chemistry="finite-rate" if chemistry else None)
    orc.set_prims(prims)
    return mb, orc


def summand_err(mb, orc, dq):
    want = [np.zeros_like(r) for r in orc.regs[0]]
    F = orc.rhs(orc.regs[0], want, faces=True)
    out = []
    for b, w, (iF, jF, kF), m in zip(mb.blocks, want, F, mb.metrics):
        g = b.mesh.ng
        ne = w.shape[-1]
        s = (np.abs(iF[g:-g - 1, g:-g, g:-g]) + np.abs(iF[g + 1:-g, g:-g, g:-g]) +
             np.abs(jF[g:-g, g:-g - 1, g:-g]) + np.abs(jF[g:-g, g + 1:-g, g:-g]) +
             np.abs(kF[g:-g, g:-g, g:-g - 1]) + np.abs(kF[g:-g, g:-g, g + 1:-g])) * \
            m["detJinv"][b.mesh.interior][..., None]
        wi = w[b.mesh.interior]
        scale = s.reshape(-1, ne).max(axis=0) + np.abs(wi).reshape(-1, ne).max(axis=0)
        # a row with no flux at all (a species absent everywhere) is held to zero
        scale[scale == 0.0] = 1.0
        got = getattr(b, dq).get()[b.mesh.interior]
        out.append(np.abs(got - wi).reshape(-1, ne).max(axis=0) / scale)
    return np.max(out, axis=0)


@pytest.mark.parametrize("chemistry", [False, True])
def test_the_rhs_with_binary_diffusion_matches_the_oracle(chemistry):
    mb, orc = build(chemistry)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    assert summand_err(mb, orc, dq).max() < 5e-10


def test_steps_with_binary_diffusion_match_the_oracle():
    mb, orc = build(True)
    dt = 2e-8
    mb.step(dt, 3)
    for _ in range(3):
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = b.Q.get()[b.mesh.interior], w[b.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        scale[scale == 0.0] = 1.0
        assert (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max() < 1e-9


def test_binary_diffusion_differs_from_lewis():
    # the same field through the Lewis-number tables: the species rows differ
    import peregrine_b200 as pg

    mb, _ = build(False)
    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", False)
    lewis = pg.get_solver(cfg, cases.reacting_mesh(12, (2, 1, 1)), pg.get_backend("cuda", cfg))
    consts = lewis.mixture.constants()
    lewis.set_prims(cases.reacting_prims(lewis.metrics, lewis.mixture.spnames, consts["MW"], 12, seed=7, width=2.0,
                                         dT=600.0, radicals=2e-3))
    for m in (mb, lewis):
        m.rhs(Q="Q", dQ=m.regs[-1])
    a = getattr(mb.blocks[0], mb.regs[-1]).get()[mb.mesh_blocks[0].interior][..., 5:]
    b = getattr(lewis.blocks[0], lewis.regs[-1]).get()[lewis.mesh_blocks[0].interior][..., 5:]
    assert np.isfinite(a).all() and not np.allclose(a, b, rtol=1e-3)


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_traces_beside_a_pure_species_match_the_oracle(sign):
    # tests/transport/test_diffusion.py:31-57 on the device: pure N2 with
    # traces of both signs, each species' coefficient through the pure cell's
    # branches (the lone species' self coefficient, the others' pairs with it)
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", False,
                                tables="h2o2_gri30_binary")
    cfg["mixture"]["diffusion"] = "binary"
    cfg.validate()
    mesh = cases.reacting_mesh(12, (2, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    names = list(mb.mixture.spnames)
    prims = cases.reacting_prims(mb.metrics, names, consts["MW"], 12, seed=7, width=2.0, dT=600.0)
    for q in prims:
        q[..., 5:] = 0.0
        q[..., 5 + names.index("O2")] = -3e-44
        q[..., 5 + names.index("OH")] = sign * 5e-44
        q[..., 5 + names.index("H2O")] = -0.8e-44
    mb.set_prims(prims)
    orc = Oracle(consts, mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3", primary="hllc",
                 recon="muscl", limiter="koren", eos="tpg", trans="kinetic-theory")
    orc.set_prims(prims)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    err = summand_err(mb, orc, dq)
    assert np.all(np.isfinite(err)) and err.max() < 5e-10, err


def test_herning_viscosity_matches_the_oracle():
    # Herning's mixing rule in place of Wilke's (peregrine/simulator/mixture/mixrule/herning.py)
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", False)
    cfg["mixture"]["mixing-rule"] = "herning"
    cfg.validate()
    mesh = cases.reacting_mesh(12, (2, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], 12, seed=5, width=2.0, dT=600.0,
                                 radicals=2e-3)
    mb.set_prims(prims)
    orc = Oracle(consts, mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3", primary="hllc",
                 recon="muscl", limiter="koren", eos="tpg", trans="kinetic-theory", mixrule="herning")
    orc.set_prims(prims)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    assert summand_err(mb, orc, dq).max() < 5e-10
