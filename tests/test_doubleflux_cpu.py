"""The double flux's Riemann forms and its viscous simulator on the CPU
oracle, pinned to the reference's own checks of them
(tests/doubleflux/test_doubleflux.py:83-112, 243-265): a real-gas contact of
CH4 in O2 at 59.8 MPa, advected at 20 m/s through a periodic line of forty
cells, keeps its pressure to 1e-9 under the double flux's Rusanov and
AUSM+-up, on the cells as they are and on MUSCL's Koren sides, where the
plain fluxes scatter it; mass and species are kept to 1e-12.  Under
navier-stokes-df a diffusing layer at rest keeps the plain simulator's
temperature within 0.1 K and its pressure within 1e-4 of P0.  Behind
isothermal no-slip walls the double flux heats a box at rest as the plain
simulator does (dQ's energy row to 1e-12), both sides alike, and a hot box
against cold walls stays finite and cools.

The reference walls its line's one-cell-thick cross-section with slip walls;
a flow along the line alone sees the same halo cells through a periodic
cross-section, which this restatement uses.  The CH4/O2 tables are the
reference's own mixture constants (the Soave-Redlich-Kwong real gas as it
ships, kinetic-theory transport, fits over 100-1500 K).
"""

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import CubeMesher
from peregrine_b200.mixture import load_tables

P0, CELLS, DX = 59.8e6, 40, 5e-5


def line(simulator, primary="kepaec", recon="constant", limiter=None, dx=DX, trans=None):
    t = load_tables("ch4_o2_srk")
    mesh = CubeMesher(cells=[[CELLS], [1], [1]], lengths=[CELLS * dx, dx, dx], periodic=[True] * 3)
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    df = simulator.endswith("-df")
    orc = Oracle(t, 2, simulator, blocks, mets, "tvd-rk3", primary=primary, recon=recon, limiter=limiter,
                 eos="real-gas-df" if df else "real-gas", trans=trans)
    return orc, blocks[0]


def slab(orc, blk, u0=20.0, Tin=162.7, Tout=111.7, smear=1.5):
    """tanh edges, so the central flux carries a profile rather than a jump
    (tests/doubleflux/test_doubleflux.py:47-60)"""
    shape = tuple(n + 4 for n in blk.cells)
    q = np.zeros(shape + (6,))
    i = np.arange(shape[0]) - 2 + 0.5
    f = (0.5 * (np.tanh((i - CELLS // 4) / smear) - np.tanh((i - CELLS // 2) / smear)))[:, None, None]
    q[..., 0], q[..., 1] = P0, u0
    q[..., 4] = Tout + f * (Tin - Tout)
    q[..., 5] = f
    orc.set_prims([q])
    return (slice(2, -2), 2, 2)


def sound(orc, Q):
    return orc.realgas_fromQ(np.ascontiguousarray(Q), np.full(len(Q), 130.0))[:, 7]


def pressure(orc, inner):
    """the state's p: the double flux's from the last right-hand side's
    planes, the plain real gas's from the eos of Q"""
    if orc.df:
        return orc.pst[0][inner][:, 0]
    Q = np.ascontiguousarray(orc.regs[0][0][inner])
    return orc.realgas_fromQ(Q, np.full(len(Q), 130.0))[:, 0]


def advect(orc, blk, cfl, steps, u0=20.0):
    inner = slab(orc, blk, u0=u0)
    Q0 = orc.regs[0][0][inner].copy()
    dt = cfl * DX / sound(orc, Q0).max()
    totals0 = Q0.sum(axis=0)
    scatter = 0.0
    for _ in range(steps):
        orc.step(dt)
        p = pressure(orc, inner)
        assert np.all(np.isfinite(p))
        scatter = max(scatter, np.abs(p / P0 - 1.0).max())
    Q = orc.regs[0][0][inner]
    change = Q.sum(axis=0) - totals0
    drift = np.divide(change, np.abs(totals0), out=np.zeros_like(change), where=totals0 != 0)
    return scatter, drift


@pytest.mark.parametrize(
    "primary, recon, limiter, plainabove",
    [
        ("rusanov", "constant", None, 1e-3),
        ("ausmup", "constant", None, 1e-4),
        ("rusanov", "muscl", "koren", 1e-5),
        ("ausmup", "muscl", "koren", 1e-5),
    ],
    ids=["rusanov", "ausmup", "muscl-koren-rusanov", "muscl-koren-ausmup"],
)
def test_the_riemann_solvers_keep_the_pressure(primary, recon, limiter, plainabove):
    flux = dict(primary=primary, recon=recon, limiter=limiter)
    plain, _ = advect(*line("euler", **flux), 0.4, 200)
    scatter, drift = advect(*line("euler-df", **flux), 0.4, 200)
    assert plain > plainabove and scatter < 1e-9
    assert abs(drift[0]) < 1e-12 and abs(drift[5]) < 1e-12


def diffusing(simulator, dx=1e-7, steps=2000):
    orc, blk = line(simulator, dx=dx, trans="kinetic-theory")
    inner = slab(orc, blk, u0=0.0, Tin=140.0, Tout=140.0, smear=3.0)
    Q0 = orc.regs[0][0][inner].copy()
    dt = 0.4 * dx / sound(orc, Q0).max()
    E0 = Q0[:, 4].sum()
    for _ in range(steps):
        orc.step(dt)
    Q = np.ascontiguousarray(orc.regs[0][0][inner])
    drift = (Q[:, 4].sum() - E0) / abs(E0)
    if orc.df:
        rec = orc.pst[0][inner]
    else:
        rec = orc.realgas_fromQ(Q, np.full(len(Q), 140.0))
    return rec[:, 1], rec[:, 0], drift


def test_a_diffusing_layer_keeps_its_temperature():
    # 2000 steps let the edges mix a few thousandths; the volume of mixing moves
    # the pressure by 1e-4 P0 under the plain physics too, so the double flux is
    # held to the plain simulator's state
    Tplain, pplain, _ = diffusing("navier-stokes")
    T, p, drift = diffusing("navier-stokes-df")
    assert np.abs(T - Tplain).max() < 0.1
    assert np.abs(p - pplain).max() / P0 < 1e-4
    assert abs(drift) < 1e-4


def heated(simulator, Tbox=300.0, Twall=400.0, steps=0):
    """A closed box of CH4/O2 at rest behind isothermal no-slip walls
    (tests/doubleflux/test_doubleflux.py:268-288): dQ's energy row on the
    first and last layer along each axis after steps."""
    t = load_tables("ch4_o2_srk")
    mesh = CubeMesher(cells=[[5], [4], [3]], lengths=[2.5e-4, 2e-4, 1.5e-4], defaultbc="walls")
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    df = simulator.endswith("-df")
    orc = Oracle(t, 2, simulator, blocks, mets, "tvd-rk3", eos="real-gas-df" if df else "real-gas",
                 trans="kinetic-theory", bcvals={"walls": {"kind": "no-slp-isot-wall", "T": Twall}},
                 species=[str(n) for n in t["spnames"]])
    q = np.zeros((9, 8, 7, 6))
    q[..., 0], q[..., 4], q[..., 5] = P0, Tbox, 0.5
    orc.set_prims([q])
    inner = blocks[0].interior
    dt = 0.3 * 5e-5 / sound(orc, np.ascontiguousarray(orc.regs[0][0][inner].reshape(-1, 6))).max()
    for _ in range(steps):
        orc.step(dt)
    dQ = [np.zeros_like(orc.regs[0][0])]
    orc.rhs(orc.regs[0], dQ)
    e = dQ[0][inner][..., 4]
    return [(np.take(e, 0, axis=a), np.take(e, -1, axis=a)) for a in range(3)]


def test_a_wall_heats_both_sides_of_the_box_alike():
    plain, df = heated("navier-stokes"), heated("navier-stokes-df")
    for (low, high), (lowdf, highdf) in zip(plain, df):
        assert np.allclose(lowdf, low, rtol=1e-12)
        assert np.allclose(highdf, high, rtol=1e-12)
        assert np.allclose(lowdf.mean(), highdf.mean(), rtol=1e-12)


def test_a_hot_box_against_cold_walls_stays_finite():
    # a mirrored halo at 2 Twall - Tbox would have no real-gas state; the halo holds the wall's own
    for low, high in heated("navier-stokes-df", Tbox=1400.0, Twall=300.0, steps=30):
        assert np.isfinite(low).all() and np.isfinite(high).all()
        assert (low < 0.0).all() and (high < 0.0).all()
