"""Two ranks' shards of one grid on one GPU, stepped a stage at a time with
their halos traded between stages through the device pack and unpack
(pgb_exchange_pack, pgb_exchange_unpack, pgb_step_stage), against one case
holding every block: the same bits, on the batched path's both forms and
on the per-block path.

The two shards run one after the other on the one device, and neither
waits on the other inside a kernel: a trade is two packs, two device
copies and two unpacks between stages, as two GPUs would post them.
"""

import ctypes

import numpy as np
import pytest

from peregrine_b200 import cases, native, shard

pytestmark = pytest.mark.gpu


def build(kind, launch, simulator="navier-stokes"):
    if kind == "tgv":
        cfg = cases.tgv_config(simulator, "rk4", launch)
        mesh = cases.tgv_mesh(18, (3, 2, 1), seed=4, low=5, high=9)
    else:
        cfg = cases.mixing_config(simulator, "tvd-rk3", "hllc", "muscl", "koren", ns=2, launch=launch)
        mesh = cases.tgv_mesh(12, (3, 2, 1), seed=4, low=3, high=6)
    return cfg, mesh


def prims_of(kind, blocks, mets):
    if kind == "tgv":
        return cases.tgv_prims(blocks, mets, seed=2, noise=1e-3)
    return cases.rough_prims(mets, 2, seed=2)


def shards(cfg, mesh, allprims):
    import peregrine_b200 as pg

    blocks = mesh.make_blocks(2)
    owner = shard.partition(blocks, 2)
    parts = []
    for r in range(2):
        plan = shard.ExchangePlan(blocks, owner, r)
        mb = pg.get_solver(cfg, shard.LocalMesh(mesh, owner, r), pg.get_backend("cuda", cfg))
        mb.set_prims([allprims[g] for g in plan.local])
        s, rv = plan.flat("send"), plan.flat("recv")
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        sb, si, rb, ri = i32(s[:, 0]), i32(s[:, 1]), i32(rv[:, 0]), i32(rv[:, 1])
        native.call("pgb_case_set_exchange", mb.case, len(s), p(sb), p(si), len(rv), p(rb), p(ri))
        parts.append((plan, mb))
    return parts


# the viscous Taylor-Green vortex on the fused stage kernel; the inviscid
# two-species gas on the per-block kernels and the fused passes
@pytest.mark.parametrize("kind,launch,simulator", [("tgv", "batched", "navier-stokes"), ("tgv", "per-block", "euler"),
                                                   ("mixed", "batched", "euler"), ("mixed", "per-block", "euler")])
def test_two_shards_step_as_one_case(kind, launch, simulator):
    import torch

    import peregrine_b200 as pg

    cfg, mesh = build(kind, launch, simulator)
    whole = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    allprims = prims_of(kind, whole.mesh_blocks, whole.metrics)
    whole.set_prims(allprims)
    parts = shards(cfg, mesh, allprims)
    assert all(len(pl.send[1 - r]) > 0 for r, (pl, _) in enumerate(parts))
    from peregrine_b200.integrators import stages

    nstages = len(stages(whole.integrator)[0])
    dt = 2e-5 if kind == "tgv" else 1e-6
    dev = torch.device("cuda:0")
    ne = whole.ne
    for mb in [whole] + [m for _, m in parts]:
        native.call("pgb_set_dt", mb.case, dt)
    for _ in range(3):
        whole.step(dt)
        for s in range(nstages):
            packs = []
            for plan, mb in parts:
                ns, _ = plan.counts()
                buf = torch.zeros((ne, max(1, sum(ns))), dtype=torch.float64, device=dev)
                native.call("pgb_exchange_pack", mb.case, s, mb.path, ctypes.c_void_p(buf.data_ptr()))
                native.call("pgb_device_sync")
                packs.append(buf)
            for r, (plan, mb) in enumerate(parts):
                _, nr = plan.counts()
                rbuf = torch.zeros((ne, max(1, sum(nr))), dtype=torch.float64, device=dev)
                off = 0
                for q in range(2):
                    # what q packed for r: its send list to r, after its sends to the ranks before r
                    qs, _ = parts[q][0].counts()
                    start = sum(qs[:r])
                    rbuf[:, off:off + nr[q]] = packs[q][:, start:start + qs[r]]
                    off += nr[q]
                native.call("pgb_exchange_unpack", mb.case, s, mb.path, ctypes.c_void_p(rbuf.data_ptr()))
                native.call("pgb_step_stage", mb.case, s, mb.path)
                native.call("pgb_device_sync")
    for plan, mb in parts:
        for n, g in enumerate(plan.local):
            a = mb.blocks[n].Q.get()[mb.mesh_blocks[n].interior]
            b = whole.blocks[g].Q.get()[whole.mesh_blocks[g].interior]
            assert np.array_equal(a, b), (g, np.abs(a - b).max())
    if kind == "tgv" and launch == "batched":
        # the whole grid's stage reads across its blocks' faces; a shard,
        # whose halo at the cut comes from the exchange, fills its halo
        def pulls(mb):
            on = ctypes.c_int(-1)
            native.call("pgb_case_halo_pull", mb.case, ctypes.byref(on))
            return on.value

        assert pulls(whole) == 1
        assert all(pulls(mb) == 0 for _, mb in parts)


def test_a_stage_out_of_order_is_refused():
    import peregrine_b200 as pg

    cfg, mesh = build("tgv", "batched")
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    mb.set_prims(prims_of("tgv", mb.mesh_blocks, mb.metrics))
    native.call("pgb_set_dt", mb.case, 1e-5)
    with pytest.raises(native.PgbStateError):
        native.call("pgb_step_stage", mb.case, 1, mb.path)
    native.call("pgb_step_stage", mb.case, 0, mb.path)
    # a whole step waits for the staged one to finish
    with pytest.raises(native.PgbStateError):
        mb.step(1e-5)
    for s in range(1, 4):
        native.call("pgb_step_stage", mb.case, s, mb.path)
    mb.step(1e-5)


def test_a_viscous_shard_off_the_fused_stage_kernel_is_refused():
    import peregrine_b200 as pg

    cfg, mesh = build("mixed", "per-block")
    whole = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    parts = shards(cfg, mesh, prims_of("mixed", whole.mesh_blocks, whole.metrics))
    _, mb = parts[0]
    native.call("pgb_set_dt", mb.case, 1e-6)
    with pytest.raises(native.PgbUnsupported):
        native.call("pgb_step_stage", mb.case, 0, mb.path)


def test_the_shards_cfl_numbers_make_the_whole_grids():
    # each shard's own blocks' maxima, a MAX over the shards: the whole grid's
    # numbers, and so the cfl controller's step, to the bit (the MAX across
    # ranks itself is shard.reduce_cfl, checked over gloo ranks on the CPU)
    import peregrine_b200 as pg

    cfg, mesh = build("tgv", "batched")
    whole = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    allprims = prims_of("tgv", whole.mesh_blocks, whole.metrics)
    whole.set_prims(allprims)
    parts = shards(cfg, mesh, allprims)
    mine = [mb.cflmax() for _, mb in parts]
    got = {k: max(m[k] for m in mine) for k in shard.CFL_KEYS}
    assert got == whole.cflmax()
    assert shard.cfl_stepsize(0.8, 1.0, got) == min(0.8 / whole.cflmax()["combined"], 1.0)
