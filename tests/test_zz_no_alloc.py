"""The right-hand side entry point that allocates no device memory.

Some callers cannot allocate device memory themselves: code running inside
another framework's memory pool or a fixed arena, or a host application
that owns all of the device's memory.  pgb_rhs_block_noalloc serves them:
the caller passes its own device arrays (Q with its halo, the metrics, dQ)
and the call works in a static device array of the library's.  This test
holds it to the case API's right-hand side (pgb_rhs) on the same block, on
two calls in a row.  The test allocates its arrays through torch; the entry
point under test allocates nothing.

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
    rows.append(np.asarray(consts["wilkepair"], dtype=np.float64).ravel())
    return np.ascontiguousarray(np.concatenate(rows))


def packed_metrics(m, X, Y, Z):
    """The 31 metric components of one block, F order with the case's halo."""
    comps = [m["xcc"], m["detJinv"][..., None], m["Jinv"].reshape(X, Y, Z, 9)]
    for name in ("iS", "jS", "kS", "ixc", "jxc", "kxc"):
        comps.append(m[name][:X, :Y, :Z])
    met = np.concatenate([np.asarray(c, dtype=np.float64).reshape(X, Y, Z, -1) for c in comps], axis=-1)
    assert met.shape[-1] == 31
    return np.ascontiguousarray(np.transpose(met, (3, 2, 1, 0)))


def test_noalloc_rhs_matches_the_case_rhs_twice():
    import torch

    import peregrine_b200 as pg

    cfg = cases.tgv_config("navier-stokes", "rk4", "per-block")
    mesh = cases.tgv_mesh(16, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    mb.set_prims(cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=5, noise=1e-3))
    blk = mb.blocks[0]
    inner = blk.mesh.interior
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    want = getattr(blk, dq).get()[inner]

    nx, ny, nz = blk.mesh.cells
    g = 2
    X, Y, Z = nx + 2 * g, ny + 2 * g, nz + 2 * g
    # Q with its halo: one periodic block's halo is its own far side
    Qi = blk.Q.get()[inner]
    Qfull = np.pad(Qi, ((g, g), (g, g), (g, g), (0, 0)), mode="wrap")
    dev = torch.device("cuda:0")
    Qd = torch.from_numpy(np.ascontiguousarray(np.transpose(Qfull, (3, 2, 1, 0)))).to(dev)
    metd = torch.from_numpy(packed_metrics(mb.metrics[0], X, Y, Z)).to(dev)
    tab = tables(mb.mixture.constants(), 1)

    phys = native.Physics(simulator=native.NAVIER_STOKES, eos=native.EOS_CPG, primary=native.FLUX_KEPAEC,
                          recon=native.RECON_CONSTANT, limiter=0, trans=native.TRANS_CONSTANT, ns=1,
                          nregs=4, alpha=1.0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    tptr = tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for call in range(2):
        dQd = torch.full((5, Z, Y, X), float("nan"), dtype=torch.float64, device=dev)
        native.call("pgb_rhs_block_noalloc", ctypes.byref(phys), tptr, nx, ny, nz, ctypes.c_void_p(Qd.data_ptr()),
                    ctypes.c_void_p(metd.data_ptr()), ctypes.c_void_p(dQd.data_ptr()), stream)
        torch.cuda.synchronize(dev)
        got = np.transpose(dQd.cpu().numpy(), (3, 2, 1, 0))[g:-g, g:-g, g:-g]
        err = rowmax_err(got, want)
        assert err < RHS_TOL, (call, err)


def test_noalloc_refuses_a_block_past_its_scratch():
    import torch

    cap = native.load().pgb_rhs_block_noalloc_max_cells(1)
    assert cap >= 36 ** 3
    phys = native.Physics(simulator=native.NAVIER_STOKES, eos=native.EOS_CPG, primary=native.FLUX_KEPAEC,
                          recon=native.RECON_CONSTANT, limiter=0, trans=native.TRANS_CONSTANT, ns=1,
                          nregs=4, alpha=1.0)
    tab = np.ones(11)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(dummy.data_ptr())
    with pytest.raises(native.PgbArgumentError):
        native.call("pgb_rhs_block_noalloc", ctypes.byref(phys), tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                    64, 64, 64, p, p, p, ctypes.c_void_p(0))
