"""The CFL reduction and the device-side cfl controller against the CPU oracle.

The device's cflmax against the oracle's (pinned to the reference's checks in
tests/test_cfl_cpu.py) on jostled multiblock cases of every eos, the closed
form of the walled box on the device, steps under the controller against the
oracle stepping at the sizes its own cflmax gives, and the scheme-limit
bracket run through the solver's own loop.

Bars: the CFL numbers within 1e-12 (1e-10 where an iterative eos's T enters
the sound speed), the state after steps within 1e-9 of each component's
largest, the clock within 1e-13.
"""

import numpy as np
import pytest

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu


def rowmax_err(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


def tgv(launch="batched", integrator="rk4"):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.tgv_config("navier-stokes", integrator, launch)
    mesh = cases.tgv_mesh(16, (2, 2, 1), seed=3, jostle=0.15)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=3, noise=1e-3, mach=0.3)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, integrator)
    orc.set_prims(prims)
    return mb, orc


def close(got, want, rel):
    for name in want:
        assert got[name] == pytest.approx(want[name], rel=rel), name


@pytest.mark.parametrize("launch", ["batched", "per-block"])
def test_cflmax_matches_the_oracle_on_a_jostled_multiblock_case(launch):
    mb, orc = tgv(launch)
    close(mb.cflmax(), orc.cflmax(), 1e-12)


def test_cflmax_on_uniform_blocks_matches_the_oracle():
    # the batched path's first step finds the blocks uniform; the reduction
    # then takes the uniform form (the axes as normals, the spacing as lengths)
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.tgv_config("navier-stokes", "rk4", "batched")
    mesh = cases.tgv_mesh(16, (2, 1, 2), seed=3)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=3, noise=1e-3, mach=0.3)
    mb.set_prims(prims)
    mb.step(0.0, 1)
    assert all(mb.uniform(n) for n in range(len(mb.blocks)))
    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "rk4")
    orc.set_prims(prims)
    close(mb.cflmax(), orc.cflmax(), 1e-12)


@pytest.mark.parametrize("kind,ns,eos", [("sub-in-fvt", 3, "cpg"), ("slp-adia-wall", 1, "cpg"),
                                         ("sup-out-fn", 2, "real-gas")])
def test_cflmax_matches_the_oracle_on_a_boundary_box(kind, ns, eos):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    tables = "o2_h2_pr" if eos == "real-gas" else None
    cfg = cases.bc_box_config(kind, ns=ns, eos=eos, tables=tables)
    mb = pg.get_solver(cfg, cases.bc_box_mesh(), pg.get_backend("cuda", cfg))
    prims = cases.bc_box_prims(mb.metrics, mb.ns)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), mb.ns, "euler", mb.mesh_blocks, mb.metrics, "rk4", eos=eos,
                 trans="constant", bcvals=cfg["bcvals"], species=mb.mixture.spnames)
    orc.set_prims(prims)
    close(mb.cflmax(), orc.cflmax(), 1e-10 if eos == "real-gas" else 1e-12)


def test_cflmax_is_the_fastest_oblique_mode_on_the_device():
    import peregrine_b200 as pg
    from peregrine_b200.config import Config
    from peregrine_b200.mesher import CubeMesher
    from peregrine_b200.mixture import Ru

    air = {"Air": {"MW": 28.96, "cp0": 1005.0}}
    R = Ru / 28.96
    gamma = 1005.0 / (1005.0 - R)
    lengths, cells, u = (0.6, 0.9, 1.5), (6, 5, 4), np.array([50.0, -30.0, 20.0])
    cfg = Config()
    cfg["simulation"]["simulator"] = "euler"
    cfg["mixture"]["species"] = air
    cfg["bcvals"]["wall"] = {"kind": "slp-adia-wall"}
    cfg.validate()
    mesh = CubeMesher(cells=[[c] for c in cells], lengths=list(lengths), defaultbc="wall")
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    blk = mb.mesh_blocks[0]
    q = np.zeros(tuple(n + 4 for n in cells) + (5,))
    q[..., 0] = 101325.0
    q[..., 1:4] = u
    q[..., 4] = 300.0 * (1.0 + 0.1 * np.sin(2 * np.pi * np.arange(q.shape[0])[:, None, None] / 6.0))
    mb.set_prims([q])
    cmax = np.sqrt(gamma * R * q[blk.interior][..., 4]).max()
    d = np.asarray(lengths) / np.asarray(cells)
    acoustic = cmax * np.sqrt((1.0 / d ** 2).sum())
    convective = (np.abs(u) / d).sum()
    close(mb.cflmax(), dict(acoustic=acoustic, convective=convective, combined=acoustic + convective), 1e-12)


def oracle_steps(orc, cfl, dtmax, n):
    dts = []
    for _ in range(n):
        dt = min(cfl / orc.cflmax()["combined"], dtmax)
        orc.step(dt)
        dts.append(dt)
    return dts


@pytest.mark.parametrize("launch,graph", [("batched", True), ("batched", False), ("per-block", True)])
def test_steps_under_the_controller_match_the_oracle(launch, graph):
    mb, orc = tgv(launch)
    mb.graph = graph
    mb.tme = orc.tme = 0.25
    cfl, dtmax = 0.6, 1.0
    mb.step_cfl(cfl, dtmax, 12)
    dts = oracle_steps(orc, cfl, dtmax, 12)
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < 1e-9
    assert mb.tme == pytest.approx(orc.tme, rel=1e-13)
    assert mb.last_dt() == pytest.approx(dts[-1], rel=1e-9)
    assert mb.nrt == 12


def test_dt_max_caps_the_step():
    mb, orc = tgv("batched")
    free = 0.6 / mb.cflmax()["combined"]
    mb.step_cfl(0.6, 0.5 * free, 3)
    assert mb.last_dt() == 0.5 * free
    assert mb.tme == pytest.approx(1.5 * free, rel=1e-13)


def test_the_solvers_run_loop_takes_the_controller():
    import peregrine_b200 as pg

    cfg = cases.tgv_config("navier-stokes", "rk4", "batched")
    cfg["simulation"]["controller"] = "cfl"
    cfg["simulation"]["cfl"] = 0.5
    cfg["simulation"]["dt-max"] = 1.0
    cfg["simulation"]["niter"] = 5
    mesh = cases.tgv_mesh(16, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    mb.set_prims(cases.tgv_prims(mb.mesh_blocks, mb.metrics))
    first = mb.integ.controller.stepsize(mb)
    assert first == 0.5 / mb.cflmax()["combined"]
    mb.run()
    assert mb.nrt == 5
    # the flow changes little over five steps: each took about the first's size
    assert mb.tme == pytest.approx(5 * first, rel=1e-3)


@pytest.mark.parametrize("cfl, bounded", [(1.6, True), (1.7, True), (1.8, False), (2.0, False)])
def test_the_target_brackets_the_schemes_limit_on_the_device(cfl, bounded):
    # tests/integrators/test_cfl.py:123-151: a line of forty cells, tvd-rk3
    # over the two-point central flux, 300 steps under the controller
    import peregrine_b200 as pg
    from peregrine_b200.config import Config
    from peregrine_b200.mesher import CubeMesher

    dx, seed = 1e-3, 1e-6
    cfg = Config()
    cfg["simulation"]["simulator"] = "euler"
    cfg["simulation"].update(controller="cfl", cfl=cfl, niter=300)
    cfg["simulation"]["dt-max"] = 1.0
    cfg["mixture"]["species"] = {"Air": {"MW": 28.96, "cp0": 1005.0}}
    cfg["bcvals"]["slip"] = {"kind": "slp-adia-wall"}
    cfg.validate()
    mesh = CubeMesher(cells=[[40], [1], [1]], lengths=[40 * dx, dx, dx], periodic=[True, False, False],
                      bcnames={n: "slip" for n in (3, 4, 5, 6)})
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    x = mb.metrics[0]["xcc"][..., 0]
    q = np.zeros(x.shape + (5,))
    q[..., 0] = 101325.0 * (1.0 + seed * np.sin(2 * np.pi * x / (4 * dx)))
    q[..., 4] = 300.0 * (1.0 + 0.1 * np.sin(2 * np.pi * x / (40 * dx)))
    mb.set_prims([q])
    assert mb.integ.controller.stepsize(mb) == cfl / mb.cflmax()["combined"]
    mb.run()
    from oracle.oracle import Oracle

    orc = Oracle(mb.mixture.constants(), 1, "euler", mb.mesh_blocks, mb.metrics, "tvd-rk3",
                 bcvals=cfg["bcvals"], species=mb.mixture.spnames)
    Q = np.ascontiguousarray(mb.blocks[0].Q.get()[mb.mesh_blocks[0].interior].reshape(-1, 5))
    p = orc.fromQ(Q, np.zeros(len(Q)))[:, 0]
    scatter = np.abs(p / 101325.0 - 1.0).max()
    assert np.isfinite(scatter)
    if bounded:
        assert scatter < seed
    else:
        assert scatter > 10 * seed
