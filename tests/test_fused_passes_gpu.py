"""The fused passes (the batched path for every ideal-gas case the fused
stage kernel does not take): a cell pass (fromQ and transport), the coupled
chemistry source, the gradients, a face pass per axis (the advective and
diffusive flux in one thread) and one pass of the divergence and the
stage's combines.  Each face and cell runs the per-block kernels' own device
functions in the same order, so the batched path gives the per-block path's
results to rounding; and against the CPU oracle it holds the per-block
path's bars.
"""

import numpy as np
import pytest

from peregrine_b200 import cases, native

pytestmark = pytest.mark.gpu


def rowmax(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale


def reacting(launch, simulator="navier-stokes", integrator="tvd-rk3", primary="hllc", recon="muscl",
             limiter="koren", chemistry=True, cells=12, blocks=(2, 1, 1), seed=7):
    import peregrine_b200 as pg

    cfg = cases.reacting_config(simulator, integrator, primary, recon, limiter, chemistry, launch=launch)
    mb = pg.get_solver(cfg, cases.reacting_mesh(cells, blocks), pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], cells, seed=seed, width=2.0,
                                 dT=600.0, radicals=2e-3)
    mb.set_prims(prims)
    return mb, prims


def mixed(launch, simulator="navier-stokes", integrator="rk4", primary="kepaec", recon="constant", limiter=None,
          ns=3, seed=4):
    import peregrine_b200 as pg

    cfg = cases.mixing_config(simulator, integrator, primary, recon, limiter, ns=ns, launch=launch)
    mesh = cases.tgv_mesh(12, (2, 2, 1), seed=seed, low=5, high=7)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.rough_prims(mb.metrics, ns, seed=seed)
    mb.set_prims(prims)
    return mb, prims


def same_results(a, b):
    # the same device functions in the same order; where the compiler contracts
    # a multiply and an add differently in the two kernels, the last bits of a
    # face flux differ, so the bar is rounding: 1e-12 of each component's largest
    for x, y in zip(a.blocks, b.blocks):
        gx, gy = x.Q.get()[x.mesh.interior], y.Q.get()[y.mesh.interior]
        err = rowmax(gx, gy).max()
        assert err < 1e-12, err


def test_the_batched_forms():
    import peregrine_b200 as pg

    tgv = pg.get_solver(cases.tgv_config(), cases.tgv_mesh(8), pg.get_backend("cuda"))
    assert tgv.batched_form() == 1
    mb, _ = reacting("batched")
    assert mb.batched_form() == 2 and mb.path == native.PATH_BATCHED
    cfg = cases.mixing_layer_config("pr", "euler-df", "tvd-rk3", launch="batched")
    mesh = cases.mixing_layer_mesh(16, 8, 2, 2, seed=0, low=6, high=10)
    df = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    assert df.batched_form() == 2 and df.path == native.PATH_BATCHED
    cfg = cases.mixing_layer_config("pr", "navier-stokes-df", "tvd-rk3", launch="batched")
    rg = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    assert rg.batched_form() == 0 and rg.path == native.PATH_PACKED


@pytest.mark.parametrize("simulator,chemistry", [("navier-stokes", True), ("navier-stokes", False), ("euler", True)])
def test_reacting_steps_are_the_per_block_paths(simulator, chemistry):
    a, _ = reacting("batched", simulator, chemistry=chemistry)
    b, _ = reacting("per-block", simulator, chemistry=chemistry)
    assert a.path == native.PATH_BATCHED and b.path == native.PATH_PER_BLOCK
    for mb in (a, b):
        mb.step(2e-8, 3)
    same_results(a, b)


@pytest.mark.parametrize("primary,recon,limiter", [("hllc", "constant", None), ("rusanov", "muscl", "vanleer"),
                                                   ("ausmup", "muscl", "minmod"), ("hllc", "muscl", "superbee"),
                                                   ("kepaec", "constant", None)])
@pytest.mark.parametrize("integrator", ["rk4", "tvd-rk3"])
def test_every_flux_function_is_the_per_block_paths(primary, recon, limiter, integrator):
    a, _ = mixed("batched", "navier-stokes", integrator, primary, recon, limiter)
    b, _ = mixed("per-block", "navier-stokes", integrator, primary, recon, limiter)
    assert a.batched_form() == 2
    for mb in (a, b):
        mb.step(1e-6, 3)
    same_results(a, b)


def test_the_right_hand_side_is_the_per_block_paths():
    a, _ = reacting("batched")
    b, _ = reacting("per-block")
    dq = a.regs[-1]
    a.rhs(Q="Q", dQ=dq)
    b.rhs(Q="Q", dQ=dq)
    for x, y in zip(a.blocks, b.blocks):
        gx, gy = getattr(x, dq).get()[x.mesh.interior], getattr(y, dq).get()[y.mesh.interior]
        assert rowmax(gx, gy).max() < 1e-12


@pytest.mark.parametrize("blocks", [(2, 1, 1), (1, 2, 2), (2, 2, 1)])
def test_uneven_blocks(blocks):
    # every pass one launch over blocks of unequal extents
    a, _ = reacting("batched", cells=12, blocks=blocks)
    b, _ = reacting("per-block", cells=12, blocks=blocks)
    for mb in (a, b):
        mb.step(2e-8, 3)
    same_results(a, b)


def test_the_fused_passes_match_the_oracle():
    from test_reacting_gpu import build

    mb, orc = build("navier-stokes", "tvd-rk3")
    mb.path = native.PATH_BATCHED
    assert mb.batched_form() == 2
    dt = 2e-8
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax(b.Q.get()[b.mesh.interior], w[b.mesh.interior]).max() < 1e-9


def interior_cell_pass(mb):
    """Whether the case's blocks take the interior cell pass (their cells with
    the halo over 1.3 times the interior), which copies the cell fields into
    the halo after: the state's, and the transport's and enthalpies' when
    viscous."""
    full = sum(np.prod([n + 4 for n in b.cells]) for b in mb.mesh_blocks)
    inner = sum(np.prod(b.cells) for b in mb.mesh_blocks)
    return full > 1.3 * inner


def test_launches_per_stage():
    # Q's halo, the cell pass, the source, the gradients and their halo, a
    # face pass per axis, the divergence and combines; inviscid, no gradients
    mb, _ = reacting("batched")
    mb.step(2e-8)
    assert mb.launches_per_step() == 3 * (9 + (3 if interior_cell_pass(mb) else 0))
    inv, _ = reacting("batched", "euler")
    inv.step(2e-8)
    assert inv.launches_per_step() == 3 * (7 + (1 if interior_cell_pass(inv) else 0))
