"""The cubic real gas and its double flux on the device against the CPU
oracle: the transcritical O2/H2 mixing layer at 60 bar, small, inviscid and
viscous (kinetic-theory transport), the double flux with kepaec, Rusanov and
AUSM+-up (on the cells as they are and on MUSCL's Koren sides).

Bars as the reacting tests': the right-hand side within 5e-10 of the
largest sum of each component's face-flux magnitudes times 1 / volume (the
iterative eos fixes T to its fit's rounding band), the state after steps
within 1e-9 of each component's largest.
"""

import numpy as np
import pytest
from totals import totals

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu


def build(cubic="pr", simulator="euler-df", integrator="tvd-rk3", nx=24, ny=16, blocks=2, seed=2, **flux):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.mixing_layer_config(cubic, simulator, integrator, **flux)
    mesh = cases.mixing_layer_mesh(nx, ny, 2, blocks, seed=seed, low=nx // blocks - 3, high=nx // blocks + 3)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.mixing_layer_prims(mb.metrics, ny, seed=seed, width=1.5)
    mb.set_prims(prims)
    eos = cfg["mixture"]["eos"]
    adv = cfg["adv-flux"]
    orc = Oracle(mb.mixture.constants(), mb.ns, simulator, mb.mesh_blocks, mb.metrics, integrator, eos=eos,
                 trans=cfg["mixture"]["trans"], primary=adv["primary"], recon=adv["recon"], limiter=adv["limiter"])
    orc.set_prims(prims)
    return mb, orc


def summand_err(mb, orc, dq):
    want = [np.zeros_like(r) for r in orc.regs[0]]
    F = orc.rhs(orc.regs[0], want, faces=True)
    out = []
    for b, w, (iF, jF, kF), m in zip(mb.blocks, want, F, mb.metrics):
        g = b.mesh.ng
        ne = w.shape[-1]
        # the double flux's two energy rows: each cell's own is F[ne] on its low faces
        lo = lambda A: A[..., :ne]
        s = (np.abs(lo(iF[g:-g - 1, g:-g, g:-g])) + np.abs(lo(iF[g + 1:-g, g:-g, g:-g])) +
             np.abs(lo(jF[g:-g, g:-g - 1, g:-g])) + np.abs(lo(jF[g:-g, g + 1:-g, g:-g])) +
             np.abs(lo(kF[g:-g, g:-g, g:-g - 1])) + np.abs(lo(kF[g:-g, g:-g, g + 1:-g]))) * \
            m["detJinv"][b.mesh.interior][..., None]
        wi = w[b.mesh.interior]
        scale = s.reshape(-1, ne).max(axis=0) + np.abs(wi).reshape(-1, ne).max(axis=0)
        got = getattr(b, dq).get()[b.mesh.interior]
        out.append(np.abs(got - wi).reshape(-1, ne).max(axis=0) / scale)
    return np.max(out, axis=0)


@pytest.mark.parametrize("cubic", ["srk", "pr"])
@pytest.mark.parametrize("simulator", ["euler", "euler-df", "navier-stokes", "navier-stokes-df"])
def test_realgas_rhs_matches_oracle(simulator, cubic):
    mb, orc = build(cubic, simulator)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    err = summand_err(mb, orc, dq)
    assert err.max() < 5e-10, err


@pytest.mark.parametrize("simulator", ["euler", "euler-df", "navier-stokes", "navier-stokes-df"])
def test_realgas_steps_match_oracle(simulator):
    mb, orc = build("pr", simulator)
    dt = 2e-9
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = b.Q.get()[b.mesh.interior], w[b.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        # the momentum is a vector: its rows share its largest component's scale
        # (a row the flow leaves at rest carries the device's rounding alone)
        scale[1:4] = scale[1:4].max()
        assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-9 * scale)


FLUXES = [("rusanov", "constant", None), ("ausmup", "constant", None), ("rusanov", "muscl", "koren"),
          ("ausmup", "muscl", "koren")]


@pytest.mark.parametrize("primary,recon,limiter", FLUXES, ids=lambda v: str(v))
@pytest.mark.parametrize("simulator", ["euler-df", "navier-stokes-df"])
def test_double_flux_riemann_rhs_matches_oracle(simulator, primary, recon, limiter):
    mb, orc = build("srk", simulator, primary=primary, recon=recon, limiter=limiter)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    err = summand_err(mb, orc, dq)
    assert err.max() < 5e-10, err


@pytest.mark.parametrize("primary,recon,limiter", FLUXES[:2] + FLUXES[3:], ids=lambda v: str(v))
def test_double_flux_riemann_steps_match_oracle(primary, recon, limiter):
    mb, orc = build("pr", "euler-df", primary=primary, recon=recon, limiter=limiter)
    dt = 2e-9
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = b.Q.get()[b.mesh.interior], w[b.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        # the momentum is a vector: its rows share its largest component's scale
        # (a row the flow leaves at rest carries the device's rounding alone)
        scale[1:4] = scale[1:4].max()
        assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-9 * scale)


def test_the_double_flux_refuses_hllc():
    from peregrine_b200.config import ConfigError

    with pytest.raises(ConfigError):
        cases.mixing_layer_config("pr", "euler-df", primary="hllc", recon="muscl", limiter="koren")


def test_double_flux_keeps_mass_and_species():
    mb, _ = build("pr", "euler-df")

    before = totals(mb)
    mb.step(2e-9, 5)
    after = totals(mb)
    for row in (0, 5):
        assert abs(after[row] - before[row]) <= 1e-14 * abs(before[row]), row


@pytest.mark.parametrize("simulator", ["euler-df", "navier-stokes"])
def test_the_packed_path_steps_as_the_per_block_path(simulator):
    # the same kernels, each pass one launch over every block: the same bits
    from peregrine_b200 import native

    mb, _ = build("pr", simulator)
    ref, _ = build("pr", simulator)
    mb.path = native.PATH_PACKED
    mb.step(2e-9, 3)
    ref.step(2e-9, 3)
    assert mb.launches_per_step() < ref.launches_per_step()
    for a, b in zip(mb.blocks, ref.blocks):
        assert np.array_equal(a.Q.get()[a.mesh.interior], b.Q.get()[b.mesh.interior])


def test_the_double_flux_batched_path_is_the_per_block_paths():
    # the inviscid double flux with kepaec on the batched path: the frozen
    # planes each step (each pass one launch over every block), then per
    # stage Q's halo, the state off the planes and one kernel of a cell's six
    # faces, divergence and combines
    from peregrine_b200 import native

    mb, orc = build("pr", "euler-df", nx=24, ny=16, blocks=3)
    ref, _ = build("pr", "euler-df", nx=24, ny=16, blocks=3)
    mb.path = native.PATH_BATCHED
    assert mb.batched_form() == 2
    dt = 2e-9
    mb.step(dt, 3)
    ref.step(dt, 3)
    for _ in range(3):
        orc.step(dt)
    # the freeze (3 launches: the interior's state, the freeze, then Q's and
    # the state's halo in one pass) and three stages of three (the
    # interior's state off the planes, Q's halo with the state's copy, and
    # the faces, divergence and combines)
    assert mb.launches_per_step() == 3 + 3 * 3
    for a, b, w in zip(mb.blocks, ref.blocks, orc.regs[0]):
        got, same = a.Q.get()[a.mesh.interior], b.Q.get()[b.mesh.interior]
        scale = np.abs(same).reshape(-1, same.shape[-1]).max(axis=0)
        assert np.all(np.abs(got - same).reshape(-1, same.shape[-1]).max(axis=0) <= 1e-12 * scale)
        want = w[a.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        scale[1:4] = scale[1:4].max()
        assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-9 * scale)


def test_the_double_flux_batched_rhs_is_the_per_block_rhs():
    from peregrine_b200 import native

    mb, _ = build("pr", "euler-df")
    ref, _ = build("pr", "euler-df")
    mb.path = native.PATH_BATCHED
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    ref.rhs(Q="Q", dQ=dq)
    for a, b in zip(mb.blocks, ref.blocks):
        got, want = getattr(a, dq).get()[a.mesh.interior], getattr(b, dq).get()[b.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-12 * scale)
