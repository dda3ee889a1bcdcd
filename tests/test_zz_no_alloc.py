"""The right-hand side entry point that allocates no device memory.

Some callers cannot allocate device memory themselves: code running inside
another framework's memory pool or a fixed arena, or a host application
that owns all of the device's memory.  pgb_rhs_block_noalloc serves them:
the caller passes its own device arrays (Q with its halo, the metrics, dQ)
and the call works in a static device array of the library's.  This test
holds it to the case API's right-hand side (pgb_rhs) and to the CPU oracle's
on the same block, on two calls in a row, for the euler and navier-stokes
simulators and one to three species.  The test allocates its arrays through
torch; the entry point under test allocates nothing.

This file is collected last, so a run that stops at the first failure has
run every other test before it.
"""

import ctypes

import numpy as np
import pytest

from peregrine_b200 import cases, native

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12


def rowmax_err(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


def tables(consts, ns):
    names = ("Rsp", "cp0", "h298R", "MWinv", None, "h298", "mu0", "kappa0", "MWqinv", "lewis")
    rows = []
    for name in names:
        if name is None:
            rows.append(np.asarray(consts["hpoly"], dtype=np.float64)[:, 0])
        else:
            rows.append(np.asarray(consts.get(name, np.ones(ns)), dtype=np.float64).ravel())
    # an inviscid gas carries no transport tables; the call reads them all the same
    rows.append(np.asarray(consts.get("wilkepair", np.full((ns, ns), 0.25)), dtype=np.float64).ravel())
    return np.ascontiguousarray(np.concatenate(rows))


def packed_metrics(m, X, Y, Z):
    """The 31 metric components of one block, F order with the case's halo."""
    comps = [m["xcc"], m["detJinv"][..., None], m["Jinv"].reshape(X, Y, Z, 9)]
    for name in ("iS", "jS", "kS", "ixc", "jxc", "kxc"):
        comps.append(m[name][:X, :Y, :Z])
    met = np.concatenate([np.asarray(c, dtype=np.float64).reshape(X, Y, Z, -1) for c in comps], axis=-1)
    assert met.shape[-1] == 31
    return np.ascontiguousarray(np.transpose(met, (3, 2, 1, 0)))


def physics(simulator, ns):
    return native.Physics(simulator=simulator, eos=native.EOS_CPG, primary=native.FLUX_KEPAEC,
                          recon=native.RECON_CONSTANT, limiter=0,
                          trans=native.TRANS_CONSTANT if simulator == native.NAVIER_STOKES else native.TRANS_NONE,
                          ns=ns, nregs=4, alpha=1.0)


@pytest.mark.parametrize("ns", [1, 2, 3])
@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
def test_noalloc_rhs_matches_the_case_rhs_and_the_oracle_twice(simulator, ns):
    import torch

    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    if ns == 1:
        cfg = cases.tgv_config(simulator, "rk4", "per-block")
    else:
        cfg = cases.mixing_config(simulator, "rk4", "kepaec", "constant", None, ns=ns)
    mesh = cases.tgv_mesh(16, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    if ns == 1:
        prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=5, noise=1e-3)
    else:
        prims = cases.rough_prims(mb.metrics, ns, seed=5, speed=120.0)
    consts = mb.mixture.constants()
    orc = Oracle(consts, ns, simulator, mb.mesh_blocks, mb.metrics, "rk4")
    orc.set_prims(prims)
    blk = mb.blocks[0]
    inner = blk.mesh.interior
    # the oracle's state on both sides, so the three right-hand sides read one Q
    Qi = orc.regs[0][0][inner]
    blk.Q.set(Qi)
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    case_rhs = getattr(blk, dq).get()[inner]
    want = [np.zeros_like(r) for r in orc.regs[0]]
    orc.rhs(orc.regs[0], want)
    oracle_rhs = want[0][inner]
    assert rowmax_err(case_rhs, oracle_rhs) < RHS_TOL

    nx, ny, nz = blk.mesh.cells
    g = 2
    X, Y, Z = nx + 2 * g, ny + 2 * g, nz + 2 * g
    ne = 4 + ns
    # Q with its halo: one periodic block's halo is its own far side
    Qfull = np.pad(Qi, ((g, g), (g, g), (g, g), (0, 0)), mode="wrap")
    dev = torch.device("cuda:0")
    Qd = torch.from_numpy(np.ascontiguousarray(np.transpose(Qfull, (3, 2, 1, 0)))).to(dev)
    metd = torch.from_numpy(packed_metrics(mb.metrics[0], X, Y, Z)).to(dev)
    tab = tables(consts, ns)
    phys = physics(native.NAVIER_STOKES if simulator == "navier-stokes" else native.EULER, ns)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    tptr = tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for call in range(2):
        dQd = torch.full((ne, Z, Y, X), float("nan"), dtype=torch.float64, device=dev)
        native.call("pgb_rhs_block_noalloc", ctypes.byref(phys), tptr, nx, ny, nz, ctypes.c_void_p(Qd.data_ptr()),
                    ctypes.c_void_p(metd.data_ptr()), ctypes.c_void_p(dQd.data_ptr()), stream)
        torch.cuda.synchronize(dev)
        got = np.transpose(dQd.cpu().numpy(), (3, 2, 1, 0))[g:-g, g:-g, g:-g]
        assert rowmax_err(got, case_rhs) < RHS_TOL, (call, "case")
        assert rowmax_err(got, oracle_rhs) < RHS_TOL, (call, "oracle")


@pytest.mark.parametrize("simulator", [native.EULER_DF, native.NAVIER_STOKES_DF, 7])
def test_noalloc_refuses_a_simulator_it_does_not_take(simulator):
    import torch

    phys = physics(native.NAVIER_STOKES, 1)
    phys.simulator = simulator
    tab = np.ones(11)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(dummy.data_ptr())
    with pytest.raises(native.PgbUnsupported):
        native.call("pgb_rhs_block_noalloc", ctypes.byref(phys), tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                    8, 8, 8, p, p, p, ctypes.c_void_p(0))


def test_noalloc_refuses_a_block_past_its_scratch():
    import torch

    cap = native.load().pgb_rhs_block_noalloc_max_cells(1)
    assert cap >= 36 ** 3
    phys = physics(native.NAVIER_STOKES, 1)
    tab = np.ones(11)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(dummy.data_ptr())
    with pytest.raises(native.PgbArgumentError):
        native.call("pgb_rhs_block_noalloc", ctypes.byref(phys), tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                    64, 64, 64, p, p, p, ctypes.c_void_p(0))
