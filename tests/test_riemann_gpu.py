"""The Riemann solvers and MUSCL on the device against the CPU oracle.

hllc, rusanov and ausmup on the cells as they are and on MUSCL's sides
under each limiter (peregrine/simulator/euler/kernels/flux/function/,
recon/muscl.mako), for two and three species, on jostled blocks, through
the per-block path; the oracle is pinned to the reference's numpy oracle for
the same face fluxes.  Bars as the other parity tests: a component's error
over its largest magnitude, 1e-12 for the right-hand side, 1e-9 for the
state after steps.
"""

import numpy as np
import pytest
from totals import totals

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
STATE_TOL = 1e-9


def rowmax_err(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


def build(simulator, primary, recon, limiter, ns, integrator="rk4", seed=5):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.mixing_config(simulator, integrator, primary, recon, limiter, ns)
    mesh = cases.tgv_mesh(12, (2, 1, 2), seed=seed, low=4, high=8, jostle=0.15)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.rough_prims(mb.metrics, ns, seed=seed)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), ns, simulator, mb.mesh_blocks, mb.metrics, integrator, primary=primary,
                 recon=recon, limiter=limiter)
    orc.set_prims(prims)
    return mb, orc


def rhs_err(mb, orc):
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    want = [np.zeros_like(r) for r in orc.regs[0]]
    orc.rhs(orc.regs[0], want)
    return max(rowmax_err(getattr(b, dq).get()[b.mesh.interior], w[b.mesh.interior])
               for b, w in zip(mb.blocks, want))


SCHEMES = [(p, "constant", None) for p in ("hllc", "rusanov", "ausmup")] + \
          [(p, "muscl", "koren") for p in ("hllc", "rusanov", "ausmup")] + \
          [("hllc", "muscl", lim) for lim in ("minmod", "mc", "superbee", "vanleer")]


@pytest.mark.parametrize("primary,recon,limiter", SCHEMES, ids=["-".join(filter(None, s)) for s in SCHEMES])
@pytest.mark.parametrize("ns", [2, 3])
def test_euler_rhs_matches_oracle(primary, recon, limiter, ns):
    mb, orc = build("euler", primary, recon, limiter, ns)
    assert rhs_err(mb, orc) < RHS_TOL


@pytest.mark.parametrize("ns", [1, 2, 3])
def test_navier_stokes_rhs_with_muscl_hllc_matches_oracle(ns):
    mb, orc = build("navier-stokes", "hllc", "muscl", "koren", ns)
    assert rhs_err(mb, orc) < RHS_TOL


@pytest.mark.parametrize("integrator", ["tvd-rk3", "rk4"])
def test_steps_with_muscl_hllc_match_oracle(integrator):
    mb, orc = build("navier-stokes", "hllc", "muscl", "koren", 2, integrator)
    dt = 0.1 * (2 * np.pi / 12) / (420.0 + 450.0)
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    errs = [rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) for b, w in zip(mb.blocks, orc.regs[0])]
    assert max(errs) < STATE_TOL, errs


def test_muscl_hllc_conserves_mass_and_species():
    mb, _ = build("euler", "hllc", "muscl", "vanleer", 3)

    before = totals(mb)
    mb.step(1e-6, 5)
    after = totals(mb)
    for row in (0, 4, 5, 6):
        assert abs(after[row] - before[row]) <= 1e-14 * abs(before[row]), row
