"""Blocks over ranks (peregrine_b200/shard.py), on the CPU.

The partition weighs blocks as the reference does (peregrine/partition/base.py:56-62);
the exchange plans of every pair of ranks pair up cell for cell and, with
each rank's own fill, cover every halo cell; and two gloo ranks, each
stepping its blocks with the CPU oracle and trading halos through the plan
before every stage (host-staged, the reference's default,
peregrine/multiblock/collections/exchange/message/hoststaged.py), end where
one rank stepping every block ends, to the bit.
"""

import os
import socket

import numpy as np
import pytest

from peregrine_b200 import cases, shard


def tgv_blocks(cells=16, blocks=(2, 2, 1), seed=3):
    mesh = cases.tgv_mesh(cells, blocks, seed=seed, low=cells // 2 - 3, high=cells // 2 + 3)
    return mesh, mesh.make_blocks(2)


def test_weights_follow_the_reference():
    mesh, blocks = tgv_blocks()
    w = shard.block_weights(blocks)
    for b in blocks:
        nx, ny, nz = b.cells
        planes = 2 * (ny * nz + nx * nz + nx * ny)
        # every face of the periodic lattice is an interface, traded or not
        assert w[b.nblki] == pytest.approx(nx * ny * nz + (0.25 + 0.06) * 2 * planes)


@pytest.mark.parametrize("nranks", [2, 3, 4])
def test_the_partition_places_every_block_and_balances(nranks):
    mesh = cases.tgv_mesh(128, (3, 3, 3), seed=0, low=30, high=56)
    blocks = mesh.make_blocks(2)
    owner = shard.partition(blocks, nranks)
    assert set(owner.tolist()) == set(range(nranks))
    w = shard.block_weights(blocks)
    load = np.bincount(owner, weights=w, minlength=nranks)
    assert load.max() <= 1.2 * load.mean()


@pytest.mark.parametrize("nranks", [2, 3])
def test_the_plans_pair_up_and_cover_every_halo_cell(nranks):
    mesh, blocks = tgv_blocks(16, (3, 2, 1))
    owner = shard.partition(blocks, nranks)
    plans = [shard.ExchangePlan(blocks, owner, r) for r in range(nranks)]
    glob = shard.halo_entries(blocks)
    source = {(int(d), int(i)): (int(s), int(j)) for d, i, s, j in glob[:, :4]}
    for r, pr in enumerate(plans):
        for q, pq in enumerate(plans):
            assert len(pr.send[q]) == len(pq.recv[r])
            # q's receive list, in order, is filled from r's send list, in order
            got = [(pr.local[b], int(i)) for b, i in pr.send[q]]
            want = [source[(pq.local[b], int(i))] for b, i in pq.recv[r]]
            assert got == want
    # each rank's own fill and its receives are every halo cell of its blocks
    for r, p in enumerate(plans):
        mine = set(p.local)
        every = {(int(d), int(i)) for d, i in glob[:, :2] if int(d) in mine}
        order = p.local
        lid = {g: n for n, g in enumerate(order)}
        local = shard._scratch_case(shard._Renumbered([blocks[g] for g in order]),
                                    lambda b, f: lid.get(f.nbr) if f.nbr is not None else None)
        filled = {(order[int(d)], int(i)) for d, i in local[:, :2]}
        got = {(order[int(b)], int(i)) for q in range(nranks) for b, i in p.recv[q]}
        assert filled | got == every and not (filled & got)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle(blocks, which=None):
    """The oracle over blocks (a rank's, numbered from 0) with the field of the
    whole grid's blocks which[n] (every block's field drawn once, in order)."""
    from oracle.oracle import Oracle
    from peregrine_b200.grid import metrics as make_metrics
    from peregrine_b200.mixture import Mixture

    _, every = tgv_blocks()
    allmets = [make_metrics(b.nodes, 2) for b in every]
    allprims = cases.tgv_prims(every, allmets, seed=5, noise=1e-3)
    which = list(range(len(every))) if which is None else which
    consts = Mixture(cases.tgv_config("euler")["mixture"]).constants()
    orc = Oracle(consts, 1, "euler", blocks, [allmets[g] for g in which], "rk4")
    orc.set_prims([allprims[g] for g in which])
    return orc


STEPS, DT = 3, 2e-4


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mesh, blocks = tgv_blocks()
    owner = shard.partition(blocks, world)
    plan = shard.ExchangePlan(blocks, owner, rank)
    local = shard.LocalMesh(mesh, owner, rank).make_blocks(2)
    orc = _oracle(local, plan.local)

    def ijk(b, idx):
        X, Y = local[b].cells[0] + 4, local[b].cells[1] + 4
        return idx % X, (idx // X) % Y, idx // (X * Y)

    def trade(reg):
        packed = {}
        for q in range(world):
            rows = [reg[b][ijk(b, i)] for b, i in plan.send[q]]
            packed[q] = torch.from_numpy(np.array(rows).T.copy() if rows else np.zeros((5, 0)))
        got = shard.trade(plan, packed)
        for q in range(world):
            vals = got[q].numpy()
            for e, (b, i) in enumerate(plan.recv[q]):
                reg[b][ijk(b, i)] = vals[:, e]

    for _ in range(STEPS):
        orc.step(DT, before_stage=trade)
    out[rank] = {int(g): orc.regs[0][n][local[n].interior].copy() for n, g in enumerate(plan.local)}
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_step_as_one_rank_to_the_bit():
    import torch.multiprocessing as mp

    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    _, blocks = tgv_blocks()
    one = _oracle(blocks)
    for _ in range(STEPS):
        one.step(DT)
    got = {}
    for r in range(2):
        got.update(out[r])
    assert sorted(got) == list(range(len(blocks)))
    for b, blk in enumerate(blocks):
        assert np.array_equal(got[b], one.regs[0][b][blk.interior]), b


def _cfl_rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mesh, blocks = tgv_blocks()
    owner = shard.partition(blocks, world)
    plan = shard.ExchangePlan(blocks, owner, rank)
    local = shard.LocalMesh(mesh, owner, rank).make_blocks(2)
    orc = _oracle(local, plan.local)
    mine = {k: float(v) for k, v in orc.cflmax().items()}
    out[rank] = (mine, shard.reduce_cfl(mine))
    dist.barrier()
    dist.destroy_process_group()


def test_the_cfl_numbers_reduce_over_the_ranks():
    # each rank's own blocks' maxima, a MAX over the ranks: the one-rank
    # maxima over every block, and so the cfl controller's step, to the bit
    import torch.multiprocessing as mp

    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_cfl_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    _, blocks = tgv_blocks()
    whole = {k: float(v) for k, v in _oracle(blocks).cflmax().items()}
    for r in range(2):
        mine, reduced = out[r]
        assert reduced == whole
        assert all(mine[k] <= whole[k] for k in shard.CFL_KEYS)
    assert shard.cfl_stepsize(0.8, 1.0, out[0][1]) == min(0.8 / whole["combined"], 1.0)
