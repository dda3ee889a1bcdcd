"""The serving pool on the device: a case's result is the same alone, in a
mix of cases that come and go around it, and on the ordinary per-block
path; and a closed reactor's result matches the CPU oracle."""

import numpy as np
import pytest

from peregrine_b200 import cases, serving

pytestmark = pytest.mark.gpu

DT = 2e-8


def proto():
    import peregrine_b200 as pg

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True)
    mb = pg.get_solver(cfg, cases.reacting_mesh(4), pg.get_backend("cuda", cfg))
    return mb


def some_requests(mb, n=9, steps=12, seed=3):
    consts = mb.mixture.constants()
    return serving.requests(n, 0.0, mb.mixture.spnames, consts["MW"], seed=seed, steps=steps, nmin=16, nmax=96)


def run_alone(pool, req):
    slot = pool.admit(req)
    while True:
        pool.step(DT, 1)
        if slot in pool.done():
            return pool.take(slot, req.cells, req.kind)


def test_a_case_is_the_same_alone_and_in_the_mix():
    mb = proto()
    reqs = some_requests(mb)
    pool = serving.Pool(mb, 2_000_000, 64)
    alone = [run_alone(pool, r) for r in reqs]
    # the mix: cases admitted at different steps, finishing at different
    # steps, the arena's ranges reused as they free up
    mixed = {}
    running = {}
    order = list(range(len(reqs)))[::-1]
    step = 0
    while order or running:
        if order and step % 3 == 0:
            for _ in range(2):
                if order:
                    k = order.pop()
                    running[pool.admit(reqs[k])] = k
        pool.step(DT, 1)
        step += 1
        for slot in pool.done():
            k = running.pop(slot)
            mixed[k] = pool.take(slot, reqs[k].cells, reqs[k].kind)
    for k, a in enumerate(alone):
        assert np.array_equal(a, mixed[k]), k
    assert any(r.kind == "0d" for r in reqs) and any(r.kind == "1d" for r in reqs)
    pool.close()


def test_a_pooled_case_equals_the_per_block_path():
    import peregrine_b200 as pg
    from peregrine_b200.mesher import CubeMesher

    mb = proto()
    req = [r for r in some_requests(mb, n=12) if r.kind == "1d"][0]
    pool = serving.Pool(mb, 1_000_000, 8)
    got = run_alone(pool, req)
    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True)
    mesh = CubeMesher(cells=[[c] for c in req.cells], lengths=list(req.lengths), periodic=[True] * 3)
    one = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    one.set_prims([req.prims])
    one.step(DT, req.steps)
    want = one.blocks[0].Q.get()[one.mesh_blocks[0].interior]
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-13 * scale)
    pool.close()


def test_a_closed_reactor_matches_the_oracle():
    from oracle.oracle import Oracle

    mb = proto()
    req = [r for r in some_requests(mb, n=12, steps=20) if r.kind == "0d"][0]
    pool = serving.Pool(mb, 100_000, 4)
    got = run_alone(pool, req)
    m = serving.box_metrics(req.cells, req.lengths)
    from peregrine_b200.mesher import CubeMesher

    blk = CubeMesher(cells=[[c] for c in req.cells], lengths=list(req.lengths), periodic=[True] * 3).make_blocks(2)[0]
    orc = Oracle(mb.mixture.constants(), mb.ns, "navier-stokes", [blk], [m], "tvd-rk3", primary="hllc", recon="muscl",
                 limiter="koren", eos="tpg", trans="kinetic-theory", chemistry="finite-rate")
    full = np.zeros(tuple(c + 4 for c in req.cells) + (mb.ne,))
    full[...] = req.prims[0, 0, 0]
    orc.set_prims([full])
    for _ in range(req.steps):
        orc.step(DT)
    want = orc.regs[0][0][blk.interior]
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-9 * scale)
    # a uniform closed box: the state stays uniform, the chemistry moves it
    assert np.abs(got - got[:1, :1, :1]).max() == 0.0
    assert np.abs(got - req.prims).max() > 0.0


def test_a_reactor_equals_its_box_on_the_per_block_path():
    """The pool's reactor (one cell, no flux) against the 2 x 2 x 2 closed box
    stepped on the ordinary per-block path, whose fluxes of a uniform state
    cancel."""
    import peregrine_b200 as pg
    from peregrine_b200.mesher import CubeMesher

    mb = proto()
    reqs = [r for r in some_requests(mb, n=16, steps=15, seed=5) if r.kind == "0d"][:3]
    pool = serving.Pool(mb, 100_000, 8)
    for req in reqs:
        got = run_alone(pool, req)
        cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="per-block")
        # the reactor kernel walks the mechanism's tables, as this kernel does
        cfg["backend-b200"]["chemistry-kernel"] = "tables"
        mesh = CubeMesher(cells=[[c] for c in req.cells], lengths=list(req.lengths), periodic=[True] * 3)
        one = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
        one.set_prims([req.prims])
        one.step(DT, req.steps)
        want = one.blocks[0].Q.get()[one.mesh_blocks[0].interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        err = np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0)
        assert np.all(err <= 1e-13 * np.maximum(scale, 1e-300)), err / scale
    pool.close()


def test_reactors_and_blocks_share_the_slots_and_come_back_free():
    mb = proto()
    reqs = some_requests(mb, n=10, steps=4, seed=7)
    pool = serving.Pool(mb, 400_000, 5)
    free0, _, _ = pool.info()
    slots = [pool.admit(r) for r in reqs[:5]]
    assert None not in slots and len(set(slots)) == 5
    # every slot taken: a sixth case, reactor or block, waits
    assert pool.admit(reqs[5]) is None
    while pool.info()[1]:
        pool.step(DT, 1)
    for s, r in zip(slots, reqs[:5]):
        pool.take(s, r.cells, r.kind)
    assert pool.info() == (free0, 0, 0)
    pool.close()
