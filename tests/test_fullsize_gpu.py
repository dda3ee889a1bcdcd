"""The benchmarked workloads themselves against the CPU oracle, at their own
sizes and on the inputs the benchmark builds.

* The multiblock Taylor-Green vortex: 128^3 cells in 27 blocks of seeded
  uneven sizes (30-56 cells a side), Navier-Stokes, kepaec + alpha damping,
  RK4.  The fused stage kernel's right-hand side within 1e-12 of its
  summands: each component's largest device-oracle difference over the
  largest sum of its six face fluxes' magnitudes times 1 / volume plus its
  own largest value.  (The reference's convention, each component against
  its own largest, tests/simulator/test_facefluxes.py:53-63, holds the small
  fields of tests/test_parity_gpu.py to 1e-12; on this field, at Mach 0.1
  with 1e-6 noise, the mass row's divergence is ~1e-7 of its face fluxes, so
  against its own largest it reads the fluxes' last bits: 8e-11 measured,
  the per-block kernels alike.)  Then two RK4 steps on the launch shapes the
  library has (the autotuner's pick among them), each k run split in two,
  three and four, within 1e-9; mass and energy conserved.
* The reacting field: 96^3 cells of H2/air, 9 species and 28 reactions,
  MUSCL-koren + HLLC, Navier-Stokes, TVD-RK3: one step within 1e-9 of each
  component's largest; the right-hand side within 1e-9 of its summands.
  The thermally perfect temperature is fixed only to its fit's rounding band
  (tests/test_reacting_gpu.py states why), and on this field the oracle's
  own right-hand side moves by 3.4e-10 of its summands when nothing but its
  Newton's starting guesses change (cold, or drifted by 1e-6 or 3e-4:
  3.3e-10, 3.2e-10, 3.9e-10 at the worst row).  Two implementations that
  each land in that band differ by up to twice it; the bar is three times it.
* The transcritical mixing layer: 256 x 128 x 4 cells in 8 blocks of seeded
  uneven widths, Peng-Robinson with the double flux, kepaec, TVD-RK3: three
  steps within 1e-9.
"""

import numpy as np
import pytest
from totals import totals

import bench
from peregrine_b200 import cases
from peregrine_b200 import native

pytestmark = pytest.mark.gpu


def rowmax(got, want, vector=False):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    if vector:
        scale[1:4] = scale[1:4].max()
    scale[scale == 0.0] = 1.0
    return np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale


@pytest.fixture(scope="module")
def tgv():
    """The benchmark's case and the oracle's right-hand side and two RK4 steps."""
    from oracle.oracle import Oracle

    mb, mesh, prims = bench.build_case("batched")
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "rk4")
    orc.set_prims(prims)
    rhs = [np.zeros_like(r) for r in orc.regs[0]]
    F = orc.rhs(orc.regs[0], rhs, faces=True)
    # each block's summand scale per component
    scales = []
    for b, w, (iF, jF, kF), m in zip(mb.mesh_blocks, rhs, F, mb.metrics):
        g = b.ng
        sm = (np.abs(iF[g:-g - 1, g:-g, g:-g]) + np.abs(iF[g + 1:-g, g:-g, g:-g]) +
              np.abs(jF[g:-g, g:-g - 1, g:-g]) + np.abs(jF[g:-g, g + 1:-g, g:-g]) +
              np.abs(kF[g:-g, g:-g, g:-g - 1]) + np.abs(kF[g:-g, g:-g, g + 1:-g])) * m["detJinv"][b.interior][..., None]
        scales.append(sm.reshape(-1, 5).max(axis=0) + np.abs(w[b.interior]).reshape(-1, 5).max(axis=0))
    del F
    dt = bench.stable_dt()
    for _ in range(2):
        orc.step(dt)
    return mb, prims, (rhs, scales), [r.copy() for r in orc.regs[0]], dt


def test_the_benchmark_tgv_is_the_benchmark(tgv):
    mb = tgv[0]
    sizes = [b.cells for b in mb.mesh_blocks]
    assert len(sizes) == 27 and sum(np.prod(s) for s in sizes) == 128 ** 3
    assert min(min(s) for s in sizes) >= 30 and max(max(s) for s in sizes) <= 56


@pytest.mark.parametrize("launch", ["batched", "per-block"])
def test_the_rhs_of_the_benchmark_tgv_matches_the_oracle(tgv, launch):
    mb, prims, (rhs, scales), _, _ = tgv
    mb.path = native.PATH_BATCHED if launch == "batched" else native.PATH_PER_BLOCK
    try:
        mb.set_prims(prims)
        dq = mb.regs[-1]
        mb.rhs(Q="Q", dQ=dq)
        # every block in the uniform-metric form: the benchmark's kernel
        assert all(mb.uniform(n) for n in range(len(mb.blocks)))
        for b, w, sc in zip(mb.blocks, rhs, scales):
            got = getattr(b, dq).get()[b.mesh.interior]
            err = np.abs(got - w[b.mesh.interior]).reshape(-1, 5).max(axis=0) / sc
            assert err.max() < 1e-12, err
    finally:
        mb.path = native.PATH_BATCHED


@pytest.mark.parametrize("ksplit", [2, 3, 4])
def test_two_steps_of_the_benchmark_tgv_match_the_oracle_on_every_shape(tgv, ksplit):
    from peregrine_b200 import autotune

    mb, prims, _, want, dt = tgv
    for threads, minb, width, _ in autotune.shapes():
        mb.set_prims(prims)
        native.call("pgb_set_fused_shape", mb.case, threads, minb, width)
        for n, (tw, th, kc) in enumerate(autotune._tiles(mb, threads, ksplit)):
            mb.set_tile(n, tw, th, kc)
        mb.step(dt, 2)
        for b, w in zip(mb.blocks, want):
            err = rowmax(b.Q.get()[b.mesh.interior], w[b.mesh.interior]).max()
            assert err < 1e-9, (threads, minb, width, ksplit, err)


def test_the_benchmark_tgv_conserves_mass_and_energy(tgv):
    mb, prims, _, _, dt = tgv
    mb.set_prims(prims)

    before = totals(mb)
    mb.step(dt, 4)
    after = totals(mb)
    assert abs(after[0] - before[0]) <= 1e-14 * abs(before[0])
    assert abs(after[4] - before[4]) <= 1e-14 * abs(before[4])


def test_one_step_of_the_benchmark_reacting_field_matches_the_oracle():
    import peregrine_b200 as pg
    from oracle.oracle import Oracle
    from test_reacting_gpu import summand_err

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="per-block")
    mb = pg.get_solver(cfg, cases.reacting_mesh(bench.REACT_CELLS, (1, 1, 1)), pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], bench.REACT_CELLS, seed=bench.SEED)
    mb.set_prims(prims)
    orc = Oracle(consts, mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3", primary="hllc",
                 recon="muscl", limiter="koren", eos="tpg", trans="kinetic-theory", chemistry="finite-rate")
    orc.set_prims(prims)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    assert summand_err(mb, orc, dq).max() < 1e-9
    mb.set_prims(prims)
    orc.set_prims(prims)
    mb.step(2e-8)
    orc.step(2e-8)
    b, w = mb.blocks[0], orc.regs[0][0]
    assert rowmax(b.Q.get()[b.mesh.interior], w[b.mesh.interior]).max() < 1e-9


@pytest.mark.parametrize("launch", ["batched", "per-block"])
def test_three_steps_of_the_benchmark_mixing_layer_match_the_oracle(launch):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.mixing_layer_config("pr", "euler-df", "tvd-rk3", launch=launch)
    mesh = cases.mixing_layer_mesh(256, 128, 4, 8, seed=bench.SEED)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.mixing_layer_prims(mb.metrics, 128, seed=bench.SEED)
    mb.set_prims(prims)
    assert len(mb.blocks) == 8 and sum(b.ncells for b in mb.mesh_blocks) == 256 * 128 * 4
    assert mb.path == (native.PATH_BATCHED if launch == "batched" else native.PATH_PER_BLOCK)
    adv = cfg["adv-flux"]
    orc = Oracle(mb.mixture.constants(), mb.ns, "euler-df", mb.mesh_blocks, mb.metrics, "tvd-rk3",
                 eos=cfg["mixture"]["eos"], trans=cfg["mixture"]["trans"], primary=adv["primary"],
                 recon=adv["recon"], limiter=adv["limiter"])
    orc.set_prims(prims)
    for _ in range(3):
        mb.step(2e-9)
        orc.step(2e-9)
    for b, w in zip(mb.blocks, orc.regs[0]):
        # the momentum is a vector: its rows share its largest component's scale
        assert rowmax(b.Q.get()[b.mesh.interior], w[b.mesh.interior], vector=True).max() < 1e-9
