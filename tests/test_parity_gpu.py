"""Device path against the CPU oracle: the right-hand side and whole steps.

The reference's tolerance convention: a component's error is measured
against that component's largest magnitude over the block
(tests/simulator/test_facefluxes.py:53-56).  Bars: RHS 1e-12, state after
steps 1e-9, conservation to rounding.
"""

import numpy as np
import pytest
from totals import totals

from peregrine_b200 import cases
from peregrine_b200 import native

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
STATE_TOL = 1e-9


def rowmax_err(got, want):
    """max |got - want| per component over the max |want| of that component."""
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


def build(simulator="navier-stokes", integrator="rk4", cells=16, blocks=(2, 2, 1), launch="batched", seed=3,
          low=None, high=None, jostle=False):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.tgv_config(simulator, integrator, launch)
    mesh = cases.tgv_mesh(cells, blocks, seed=seed, low=low, high=high, jostle=0.15 if jostle else 0.0)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=seed, noise=1e-3)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 1, simulator, mb.mesh_blocks, mb.metrics, integrator)
    orc.set_prims(prims)
    return mb, orc


def interiors(mb, arrays):
    return [a[b.interior] for a, b in zip(arrays, mb.mesh_blocks)]


@pytest.mark.parametrize("launch", ["batched", "per-block", "packed"])
@pytest.mark.parametrize("jostle", [False, True])
@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
def test_rhs_matches_oracle(simulator, jostle, launch):
    # on the batched path the right-hand side is the fused stage kernel's own
    # (the uniform-metric kernel on the even grid, the metric-array kernel on
    # the jostled one), written at unit step with no register term
    mb, orc = build(simulator, cells=16, blocks=(2, 2, 1), jostle=jostle, launch=launch)
    assert mb.path == {"batched": native.PATH_BATCHED, "per-block": native.PATH_PER_BLOCK,
                       "packed": native.PATH_PACKED}[launch]
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    got = [getattr(b, dq).get() for b in mb.blocks]
    want = [np.zeros_like(r) for r in orc.regs[0]]
    orc.rhs(orc.regs[0], want)
    for g, w in zip(interiors(mb, got), interiors(mb, want)):
        assert rowmax_err(g, w) < RHS_TOL
    if launch == "batched":
        assert all(mb.uniform(n) != jostle for n in range(len(mb.blocks)))


@pytest.mark.parametrize("jostle", [False, True])
@pytest.mark.parametrize("launch", ["batched", "per-block"])
@pytest.mark.parametrize("integrator", ["rk4", "tvd-rk3", "rk1", "rk34"])
def test_steps_match_oracle(launch, integrator, jostle):
    mb, orc = build("navier-stokes", integrator, cells=16, blocks=(2, 1, 2), launch=launch, low=5, high=11,
                    jostle=jostle)
    _, g = cases.tgv_gas()
    dt = 0.2 * (2 * np.pi / 16) / (g["U0"] + np.sqrt(g["gamma"] * g["R"] * cases.T0))
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    got = [b.Q.get() for b in mb.blocks]
    errs = [rowmax_err(gq, w) for gq, w in zip(interiors(mb, got), interiors(mb, orc.regs[0]))]
    assert max(errs) < STATE_TOL, errs


def test_batched_equals_per_block():
    a, _ = build("navier-stokes", "rk4", cells=16, blocks=(2, 2, 2), launch="batched", low=6, high=10)
    b, _ = build("navier-stokes", "rk4", cells=16, blocks=(2, 2, 2), launch="per-block", low=6, high=10)
    for s in (a, b):
        s.step(1e-5, 4)
    for x, y in zip(a.blocks, b.blocks):
        gx, gy = x.Q.get()[x.mesh.interior], y.Q.get()[y.mesh.interior]
        assert rowmax_err(gx, gy) < STATE_TOL


def test_mass_is_conserved():
    mb, _ = build("navier-stokes", "rk4", cells=16, blocks=(2, 2, 2), low=6, high=10)

    before = totals(mb)
    mb.step(1e-5, 10)
    after = totals(mb)
    assert abs(after[0] - before[0]) <= 1e-14 * abs(before[0])
    assert abs(after[4] - before[4]) <= 1e-14 * abs(before[4])


@pytest.mark.parametrize("jostle", [False, True])
def test_uniform_blocks_are_detected(jostle):
    mb, _ = build("navier-stokes", "rk4", cells=16, blocks=(2, 1, 1), jostle=jostle)
    mb.step(1e-6)
    assert all(mb.uniform(n) != jostle for n in range(len(mb.blocks)))


@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
def test_batched_euler_and_ns_on_both_kernels(simulator):
    for jostle in (False, True):
        mb, orc = build(simulator, "rk4", cells=12, blocks=(2, 2, 2), jostle=jostle)
        mb.step(2e-5, 2)
        orc.step(2e-5)
        orc.step(2e-5)
        for b, w in zip(mb.blocks, orc.regs[0]):
            assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < STATE_TOL


@pytest.mark.parametrize("shape", range(6))
@pytest.mark.parametrize("simulator,integrator", [("navier-stokes", "rk4"), ("euler", "tvd-rk3"),
                                                  ("navier-stokes", "tvd-rk3")])
def test_every_uniform_kernel_shape_matches_the_oracle(shape, simulator, integrator):
    # each launch shape the library has, on ragged tiles (blocks of uneven
    # widths) and several k runs a block, two steps against the oracle
    from peregrine_b200 import autotune

    shapes = autotune.shapes()
    if shape >= len(shapes):
        pytest.skip("the library has fewer shapes")
    threads, minb, width, _ = shapes[shape]
    mb, orc = build(simulator, integrator, cells=24, blocks=(2, 1, 2), low=9, high=15)
    mb.step(1e-6)
    orc.step(1e-6)
    assert all(mb.uniform(n) for n in range(len(mb.blocks)))
    native.call("pgb_set_fused_shape", mb.case, threads, minb, width)
    for n, (tw, th, kc) in enumerate(autotune._tiles(mb, threads, 3)):
        mb.set_tile(n, tw, th, kc)
    dt = 2e-5
    mb.step(dt, 2)
    orc.step(dt)
    orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < STATE_TOL


def test_unsupported_physics_is_refused():
    import peregrine_b200 as pg

    cfg = cases.tgv_config()
    cfg["mixture"]["eos"] = "tpg"
    with pytest.raises((ValueError, native.PgbUnsupported)):
        pg.get_solver(cfg.validate(), cases.tgv_mesh(8), pg.get_backend("cuda", cfg))


def test_the_tgv_after_100_steps_matches_the_oracle():
    """The single-block 32^3 Taylor-Green vortex (air, Mach 0.1, Re 1600,
    kepaec + alpha damping, RK4) after 100 steps of the batched path: each
    component within 1e-9 of its largest, the bar on the state after 100
    steps; and mass and energy conserved to the rounding of 400 stages."""
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.tgv_config("navier-stokes", "rk4", "batched")
    mesh = cases.tgv_mesh(32, (1, 1, 1), seed=0)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=0)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "rk4")
    orc.set_prims(prims)
    _, g = cases.tgv_gas()
    dt = 0.3 * (2 * np.pi / 32) / (g["U0"] + np.sqrt(g["gamma"] * g["R"] * cases.T0))
    start = totals(mb)
    mb.step(dt, 100)
    for _ in range(100):
        orc.step(dt)
    got = mb.blocks[0].Q.get()[mb.mesh_blocks[0].interior]
    want = orc.regs[0][0][mb.mesh_blocks[0].interior]
    assert rowmax_err(got, want) < STATE_TOL
    # the face fluxes cancel pair by pair, so the exact totals move only by
    # each cell's rounding of its update, of random sign: over 32768 cells x
    # 400 stages about 1e-16 / sqrt(32768 / 400) of the total; the bar is far
    # above that and far below any flux a face gave one side and not the other
    end = totals(mb)
    assert abs(end[0] - start[0]) <= 1e-14 * abs(start[0])
    assert abs(end[4] - start[4]) <= 1e-14 * abs(start[4])


@pytest.mark.parametrize("integrator", ["tvd-rk3", "rk4"])
def test_the_stages_by_hand_are_a_step(integrator):
    # the reference's hand-rolled step (tests/integrators/test_postrhs.py:73-80):
    # each stage's right-hand side, then its advance
    mb, _ = build("navier-stokes", integrator, cells=12, blocks=(2, 1, 1), launch="per-block")
    ref, _ = build("navier-stokes", integrator, cells=12, blocks=(2, 1, 1), launch="per-block")
    dt = 2e-5
    ref.step(dt)
    mb.dt.set(dt)
    for n, stage in enumerate(mb.integ.stageregs(mb.regs)):
        mb.rhs(Q=stage.Q, dQ=stage.dQ)
        mb.advance(n)
    for a, b in zip(mb.blocks, ref.blocks):
        assert np.array_equal(a.Q.get()[a.mesh.interior], b.Q.get()[b.mesh.interior])
    assert mb.dt.get() == dt


def _pull_case(simulator, mesh, seed=5):
    import peregrine_b200 as pg

    cfg = cases.tgv_config(simulator, "tvd-rk3", "batched")
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    mb.set_prims(cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=seed, noise=1e-3))
    return mb


def _pulls(mb):
    import ctypes

    on = ctypes.c_int(-1)
    native.call("pgb_case_halo_pull", mb.case, ctypes.byref(on))
    return on.value


@pytest.mark.parametrize("shape", [(256, 1, 24), (256, 1, 30), (128, 2, 14)])
@pytest.mark.parametrize("blocks,low,high", [((3, 3, 3), 6, 11), ((2, 1, 2), 5, 19), ((1, 3, 1), 2, 14)])
@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
def test_reading_across_faces_gives_the_halo_fills_bits(simulator, blocks, low, high, shape):
    # the uniform stage reading its tiles' ring and the planes past a block's
    # k ends straight from the neighbouring blocks (i first, then j, then k:
    # the order a halo cell's source is found in) gives the bits the halo fill
    # before each stage gives, on uneven blocks two cells thick and up, tiles
    # of several k runs, a block that is its own neighbour across j
    runs = []
    for pull in (1, 0):
        mb = _pull_case(simulator, cases.tgv_mesh(24, blocks, seed=7, low=low, high=high))
        native.call("pgb_case_set_halo_pull", mb.case, pull)
        mb.step(1e-6)
        native.call("pgb_set_fused_shape", mb.case, *shape)
        mb.step(2e-5, 3)
        assert all(mb.uniform(n) for n in range(len(mb.blocks)))
        assert _pulls(mb) == pull
        runs.append([b.Q.get()[b.mesh.interior] for b in mb.blocks])
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def test_a_block_thinner_than_the_halo_keeps_the_fill():
    # a halo cell past a block one cell thick comes from two faces away, so
    # the stage keeps the halo fill, and matches the oracle
    from oracle.oracle import Oracle
    from peregrine_b200.mesher import CubeMesher

    mesh = CubeMesher(mbdims=[3, 1, 1], cells=[[10, 1, 13], [16], [16]], lengths=[2 * np.pi] * 3,
                      periodic=[True] * 3)
    mb = _pull_case("navier-stokes", mesh)
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=5, noise=1e-3)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3")
    orc.set_prims(prims)
    mb.step(2e-5, 2)
    orc.step(2e-5)
    orc.step(2e-5)
    assert _pulls(mb) == 0
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < STATE_TOL
