"""Two live cases of different gases, stepped in turn with no wait between.

The species and mechanism tables sit in each translation unit's constant
memory, one case's at a time.  A case's launches are queued on its own
stream and may still be waiting when another case's call uploads its own
tables; the upload is ordered after everything the previous owner has
queued, so each case's steps read its own gas.  Each case against its own
oracle, after both have run: within 1e-9 of each component's largest.
"""

import numpy as np
import pytest

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu


def rowmax(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


def tgv_case(gas, launch, seed):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.tgv_config("navier-stokes", "rk4", launch)
    cfg["mixture"]["species"] = gas
    cfg.validate()
    mesh = cases.tgv_mesh(16, (2, 1, 1), seed=seed)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=seed, noise=1e-3)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "rk4")
    orc.set_prims(prims)
    return mb, orc


def mixed_case(names, seed):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.mixing_config("navier-stokes", "rk4", "hllc", "muscl", "koren", ns=2)
    cfg["mixture"]["species"] = {k: cases.MIXED[k] for k in names}
    cfg.validate()
    mesh = cases.tgv_mesh(12, (2, 1, 1), seed=seed)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.rough_prims(mb.metrics, 2, seed=seed)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 2, "navier-stokes", mb.mesh_blocks, mb.metrics, "rk4", primary="hllc",
                 recon="muscl", limiter="koren")
    orc.set_prims(prims)
    return mb, orc


def alternate(a, b, dt, rounds, steps):
    for _ in range(rounds):
        for mb, _ in (a, b):
            mb.step(dt, steps)  # queued; no wait
    for _, orc in (a, b):
        for _ in range(rounds * steps):
            orc.step(dt)


def check(case):
    mb, orc = case
    for blk, want in zip(mb.blocks, orc.regs[0]):
        assert rowmax(blk.Q.get()[blk.mesh.interior], want[blk.mesh.interior]) < 1e-9


def test_two_gases_on_the_batched_path_each_read_their_own_tables():
    air = cases.tgv_gas()[0]
    mu, kappa = air["Air"]["mu0"], air["Air"]["kappa0"]
    heavy = {"Ar": {"MW": 39.948, "cp0": 520.3, "mu0": 1.6 * mu, "kappa0": 0.7 * kappa}}
    a = tgv_case(air, "batched", 1)
    b = tgv_case(heavy, "batched", 2)
    alternate(a, b, 2e-4, 3, 20)
    check(a)
    check(b)


def test_two_gases_on_the_per_block_path_each_read_their_own_tables():
    a = mixed_case(("A", "B"), 3)
    b = mixed_case(("A", "C"), 4)
    alternate(a, b, 2e-6, 3, 10)
    check(a)
    check(b)
