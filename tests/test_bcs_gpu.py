"""Boundary conditions on the device against the CPU oracle.

Every kind on a jostled box whose every face carries it (the reference's
boundary test box, tests/bcs/bcblock.py): the halo layers the device's
boundary pass writes and the right-hand side they feed, against the oracle,
whose kinds are pinned to the reference's halo rules and wall known answers
(tests/test_bcs_cpu.py).  Then steps with boundary values that move with the
clock, the viscous walls' known answers on the device, and the path choice.

Bars: a halo component within 1e-12 of that component's largest over the
halos; the right-hand side within 1e-12 of the largest sum of each
component's face-flux magnitudes times 1 / volume (the measure the other
per-block parity tests use where a face flux can cancel); the state after
steps within 1e-9 of each component's largest.
"""

import numpy as np
import pytest

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu

WALLS = ["slp-adia-wall", "slp-isot-wall", "no-slp-adia-wall", "mov-adia-wall", "no-slp-isot-wall", "mov-isot-wall"]
FLOWS = ["sub-in-fvt", "sup-in-fa", "sub-in-ftptt", "sub-in-fmt", "sub-out-fp", "sup-out-fn"]
VISCOUS_ONLY = ["no-slp-adia-wall", "mov-adia-wall", "no-slp-isot-wall", "mov-isot-wall"]


def build(kind, ns=1, simulator="euler", primary="kepaec", recon="constant", limiter=None, integrator="rk4", seed=0,
          entry=None, cells=(7, 5, 3), eos="cpg", tables=None, mesh=None, bcvals=None, prims=None):
    import peregrine_b200 as pg
    from oracle.oracle import Oracle

    cfg = cases.bc_box_config(kind, ns=ns, simulator=simulator, primary=primary, recon=recon, limiter=limiter,
                              integrator=integrator, seed=seed, entry=entry, eos=eos, tables=tables)
    if bcvals is not None:
        cfg["bcvals"] = bcvals
    mesh = mesh or cases.bc_box_mesh(cells=cells)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = prims(mb) if prims else cases.bc_box_prims(mb.metrics, mb.ns, seed=seed)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), mb.ns, simulator, mb.mesh_blocks, mb.metrics, integrator, primary=primary,
                 recon=recon, limiter=limiter, eos=eos, trans=cfg["mixture"]["trans"] or "constant",
                 bcvals=cfg["bcvals"], species=mb.mixture.spnames)
    orc.set_prims(prims)
    return mb, orc


def halo_slabs(blk, Q):
    """Every boundary face's two halo layers over the face's cells."""
    g = blk.ng
    out = []
    for face in blk.intfaces:
        if face.nbr is not None:
            continue
        n = blk.cells[face.axis]
        planes = np.moveaxis(Q, face.axis, 0)
        for l in range(g):
            k = g - 1 - l if face.is_low else g + n + l
            out.append(planes[k][g:-g, g:-g].reshape(-1, Q.shape[-1]))
    return np.concatenate(out)


def halo_err(mb, orc):
    errs = []
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = halo_slabs(b.mesh, b.Q.get()), halo_slabs(b.mesh, w)
        scale = np.abs(want).max(axis=0)
        scale[scale == 0.0] = 1.0
        errs.append((np.abs(got - want).max(axis=0) / scale).max())
    return max(errs)


def rhs_err(mb, orc, t=None):
    """The right-hand side's error over the largest sum of each component's
    face-flux magnitudes times 1 / volume."""
    dq = mb.regs[-1]
    mb.rhs(Q="Q", dQ=dq)
    want = [np.zeros_like(r) for r in orc.regs[0]]
    F = orc.rhs(orc.regs[0], want, faces=True, t=t)
    out = []
    for b, w, (iF, jF, kF), m in zip(mb.blocks, want, F, mb.metrics):
        g = b.mesh.ng
        # the double flux's faces carry a second energy row: the summands are the first ne
        ne = w.shape[-1]
        iF, jF, kF = iF[..., :ne], jF[..., :ne], kF[..., :ne]
        s = (np.abs(iF[g:-g - 1, g:-g, g:-g]) + np.abs(iF[g + 1:-g, g:-g, g:-g]) +
             np.abs(jF[g:-g, g:-g - 1, g:-g]) + np.abs(jF[g:-g, g + 1:-g, g:-g]) +
             np.abs(kF[g:-g, g:-g, g:-g - 1]) + np.abs(kF[g:-g, g:-g, g + 1:-g])) * \
            m["detJinv"][b.mesh.interior][..., None]
        ne = w.shape[-1]
        wi = w[b.mesh.interior]
        scale = s.reshape(-1, ne).max(axis=0) + np.abs(wi).reshape(-1, ne).max(axis=0)
        got = getattr(b, dq).get()[b.mesh.interior]
        out.append((np.abs(got - wi).reshape(-1, ne).max(axis=0) / scale).max())
    return max(out)


def rowmax_err(got, want):
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    scale[scale == 0.0] = 1.0
    return (np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) / scale).max()


@pytest.mark.parametrize("ns", [1, 3])
@pytest.mark.parametrize("kind", WALLS + FLOWS)
def test_each_kind_matches_the_oracle(kind, ns):
    sim = "navier-stokes" if kind in VISCOUS_ONLY else "euler"
    mb, orc = build(kind, ns=ns, simulator=sim)
    assert mb.path == 1  # the per-block path: the batched kernel's halo is the block-to-block fill alone
    assert rhs_err(mb, orc) < 1e-12
    assert halo_err(mb, orc) < 1e-12


@pytest.mark.parametrize("kind", WALLS + FLOWS)
def test_each_kind_on_the_viscous_path_matches_the_oracle(kind):
    # the viscous walls' own face flux and the inflows' and outflows' image gradients
    mb, orc = build(kind, ns=3, simulator="navier-stokes")
    assert rhs_err(mb, orc) < 1e-12
    assert halo_err(mb, orc) < 1e-12


@pytest.mark.parametrize("kind", ["slp-adia-wall", "sub-in-fvt", "sup-out-fn", "sub-in-ftptt"])
def test_muscl_and_hllc_read_both_halo_layers(kind):
    mb, orc = build(kind, ns=3, primary="hllc", recon="muscl", limiter="koren")
    assert rhs_err(mb, orc) < 1e-12
    assert halo_err(mb, orc) < 1e-12


@pytest.mark.parametrize("kind", ["slp-adia-wall", "slp-isot-wall", "sub-in-fvt", "sup-in-fa", "sub-out-fp",
                                  "sup-out-fn"])
def test_the_real_gas_boundaries_match_the_oracle(kind):
    mb, orc = build(kind, eos="real-gas", tables="o2_h2_pr")
    # the real gas's Newton fixes T to its rounding band (about 1e-11), which
    # the halo's energy and the fluxes carry
    assert rhs_err(mb, orc) < 5e-10
    assert halo_err(mb, orc) < 5e-10


@pytest.mark.parametrize("kind", WALLS + FLOWS)
def test_the_viscous_real_gas_boundaries_match_the_oracle(kind):
    mb, orc = build(kind, simulator="navier-stokes", eos="real-gas", tables="o2_h2_pr")
    assert rhs_err(mb, orc) < 5e-10
    assert halo_err(mb, orc) < 5e-10


@pytest.mark.parametrize("kind", WALLS + FLOWS)
@pytest.mark.parametrize("simulator", ["euler-df", "navier-stokes-df"])
def test_the_double_flux_boundaries_match_the_oracle(simulator, kind):
    # a boundary's halo cells are frozen at the step's start from the state the
    # halo pass gives them; a slip wall's halo carries its image's record whole
    if simulator == "euler-df" and kind in VISCOUS_ONLY:
        pytest.skip("the inviscid simulator has no viscous walls")
    mb, orc = build(kind, simulator=simulator, eos="real-gas-df", tables="o2_h2_pr")
    assert rhs_err(mb, orc) < 5e-10
    assert halo_err(mb, orc) < 5e-10


@pytest.mark.parametrize("simulator", ["euler-df", "navier-stokes-df"])
def test_double_flux_steps_with_boundaries_match_the_oracle(simulator):
    # every face a different kind of boundary: an inflow, an exit, walls
    viscous = simulator == "navier-stokes-df"
    bcvals = {"in": {"kind": "sub-in-fvt", "u": "40.0 + 5.0 * z", "v": 0.0, "w": 0.0, "T": 290.0, "O2": 0.6},
              "out": {"kind": "sub-out-fp", "p": 101325.0},
              "wall": {"kind": "no-slp-isot-wall", "T": 300.0} if viscous else {"kind": "slp-adia-wall"},
              "lid": {"kind": "slp-isot-wall", "T": 310.0}}
    mesh = cases.bc_box_mesh(cells=(8, 5, 4), bcnames={1: "in", 2: "out", 6: "lid"}, defaultbc="wall")
    mb, orc = build("sub-in-fvt", simulator=simulator, eos="real-gas-df", tables="o2_h2_pr", mesh=mesh,
                    bcvals=bcvals, integrator="tvd-rk3")
    dt = 2e-7
    for _ in range(3):
        mb.step(dt)
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = b.Q.get()[b.mesh.interior], w[b.mesh.interior]
        scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
        scale[1:4] = scale[1:4].max()
        assert np.all(np.abs(got - want).reshape(-1, want.shape[-1]).max(axis=0) <= 1e-9 * scale)


def channel(integrator="rk4", simulator="navier-stokes", ns=3):
    """A box with an inflow whose velocity and temperature move with x, z and
    the clock, a pressure exit, and walls: no-slip and moving where viscous."""
    inflow = {"kind": "sub-in-fvt", "u": "40.0 + 20.0 * sin(3.0 * z) * cos(2000.0 * t)", "v": "5.0 * x",
              "w": "0.0", "T": "300.0 + 40.0 * z**2 + max(x, 0.5) + 1e4 * t", "A": "0.3 + 0.05 * z", "B": 0.2}
    viscous = simulator == "navier-stokes"
    bcvals = {"in": inflow, "out": {"kind": "sub-out-fp", "p": "101325.0 + 500.0 * z"},
              "wall": {"kind": "no-slp-isot-wall", "T": 320.0} if viscous else {"kind": "slp-adia-wall"},
              "lid": {"kind": "mov-adia-wall", "u": "10.0 * z", "v": 0.0, "w": 0.0} if viscous else
              {"kind": "slp-isot-wall", "T": "310.0 + 5.0 * x"}}
    mesh = cases.bc_box_mesh(cells=(10, 6, 5), bcnames={1: "in", 2: "out", 6: "lid"}, defaultbc="wall")

    def prims(mb):
        out = cases.bc_box_prims(mb.metrics, mb.ns, seed=4, speed=30.0)
        for q in out:
            q[..., 1] += 40.0
        return out

    return build("sub-in-fvt", ns=ns, simulator=simulator, integrator=integrator, mesh=mesh, bcvals=bcvals,
                 prims=prims)


@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
@pytest.mark.parametrize("integrator", ["rk4", "tvd-rk3"])
def test_steps_with_moving_boundary_values_match_the_oracle(integrator, simulator):
    mb, orc = channel(integrator, simulator)
    mb.graph = False
    mb.tme = orc.tme = 1.0e-4
    dt = 2e-7
    mb.step(dt, 20)
    for _ in range(20):
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < 1e-9
    # the device's clock is the step's end: start + dt per step
    import ctypes

    from peregrine_b200 import native

    t = ctypes.c_double()
    native.call("pgb_get_time", mb.case, ctypes.byref(t))
    assert abs(t.value - orc.tme) <= 1e-15 * orc.tme


def test_a_graph_replays_the_moving_boundary_values():
    # the CUDA graph of a step captures the clock by address: a replay reads
    # the step's own time
    mb, orc = channel()
    mb.graph = True
    dt = 2e-7
    mb.step(dt, 8)
    for _ in range(8):
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        assert rowmax_err(b.Q.get()[b.mesh.interior], w[b.mesh.interior]) < 1e-9


def test_a_boundary_case_asked_for_the_batched_path_runs_per_block():
    # the per-block kernels, packed: each pass one launch over every block
    import peregrine_b200 as pg
    from peregrine_b200 import native

    cfg = cases.bc_box_config("slp-adia-wall", launch="batched")
    mb = pg.get_solver(cfg, cases.bc_box_mesh(), pg.get_backend("cuda", cfg))
    assert mb.path == native.PATH_PACKED


# -- the viscous walls' known answers on the device (tests/bcs/test_viscwalls.py)

N, H = 16, 1e-3
DY = H / N
CP, MW = 1005.0, 28.96
MU0 = 0.5 * DY * 347.0 * 1.17
KAPPA0 = MU0 * CP
T0, U = 300.0, 100.0


def column(low, high, u0=0.0):
    import peregrine_b200 as pg
    from peregrine_b200.config import Config
    from peregrine_b200.mesher import CubeMesher

    cfg = Config()
    cfg["simulation"]["simulator"] = "navier-stokes"
    cfg["mixture"]["species"] = {"Air": {"MW": MW, "cp0": CP, "mu0": MU0, "kappa0": KAPPA0}}
    cfg["mixture"]["trans"] = "constant"
    cfg["ics"]["u"], cfg["ics"]["T"], cfg["ics"]["p"] = u0, T0, 101325.0
    cfg["bcvals"]["low"], cfg["bcvals"]["high"] = low, high
    cfg.validate()
    mesh = CubeMesher(cells=[[1], [N], [1]], lengths=[DY, H, DY], periodic=[True, False, True],
                      bcnames={3: "low", 4: "high"})
    return pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))


def settle(mb, steps=8000):
    from oracle.oracle import Oracle

    orc = Oracle(mb.mixture.constants(), 1, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3",
                 bcvals=mb.cfg["bcvals"])
    g = 2
    Q = mb.blocks[0].Q.get()[mb.mesh_blocks[0].interior].reshape(-1, 5)
    dt = 0.3 * DY / orc.fromQ(Q, np.zeros(len(Q)))[:, 7].max()
    mb.step(dt, steps)
    Q = np.ascontiguousarray(mb.blocks[0].Q.get()[g, g:-g, g])
    return Q, orc.fromQ(Q, np.zeros(N)), mb.metrics[0]["xcc"][g, g:-g, g, 1]


def test_couette_flow_is_linear_on_the_device():
    mb = column({"kind": "no-slp-isot-wall", "T": T0}, {"kind": "mov-isot-wall", "u": U, "v": 0.0, "w": 0.0, "T": T0},
                u0=0.5 * U)
    Q, st, y = settle(mb)
    u = Q[:, 1:4] / Q[:, :1]
    assert np.allclose(u[:, 0], U * y / H, rtol=0.0, atol=1e-12 * U)
    assert np.allclose(u[:, 1:], 0.0, atol=1e-12 * U)
    peak = MU0 * U * U / (8.0 * KAPPA0)
    want = T0 + MU0 * U * U / (2.0 * KAPPA0) * (y / H) * (1.0 - y / H)
    assert np.abs(st[:, 1] - want).max() <= 2.0 / N ** 2 * peak


def test_conduction_is_linear_on_the_device():
    T1, T2 = 300.0, 400.0
    mb = column({"kind": "no-slp-isot-wall", "T": T1}, {"kind": "no-slp-isot-wall", "T": T2})
    Q, st, _ = settle(mb)
    want = T1 + (T2 - T1) * (np.arange(N) + 0.5) / N
    assert np.allclose(st[:, 1], want, rtol=0.0, atol=1e-12 * (T2 - T1))
    assert np.allclose(Q[:, 1:4] / Q[:, :1], 0.0, atol=1e-11)


def test_the_packed_path_steps_as_the_per_block_path():
    # the channel's boundaries on the packed path: the same bits
    from peregrine_b200 import native

    mb, _ = channel()
    ref, _ = channel()
    mb.path = native.PATH_PACKED
    mb.step(2e-7, 3)
    ref.step(2e-7, 3)
    for a, b in zip(mb.blocks, ref.blocks):
        assert np.array_equal(a.Q.get()[a.mesh.interior], b.Q.get()[b.mesh.interior])
