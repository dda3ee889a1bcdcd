"""The CFL reduction and the cfl controller on the CPU oracle, pinned to the
reference's own checks of them (tests/integrators/test_cfl.py): the closed
form of the fastest oblique mode on a walled box of unequal cells, the
acoustic number alone at rest, invariance to turning the box, and a target
that brackets the central scheme's stability limit on a line of cells.
"""

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200 import integrators
from peregrine_b200.config import Config
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import CubeMesher
from peregrine_b200.mixture import Mixture, Ru

AIR = {"Air": {"MW": 28.96, "cp0": 1005.0, "mu0": 1.8591191080521142e-05, "kappa0": 0.026}}
R = Ru / AIR["Air"]["MW"]
GAMMA = AIR["Air"]["cp0"] / (AIR["Air"]["cp0"] - R)

# a box of unequal cells, walled, and a velocity along every axis
LENGTHS, CELLS, U = (0.6, 0.9, 1.5), (6, 5, 4), np.array([50.0, -30.0, 20.0])


def rotabout(axis, degrees):
    """The rotation by degrees about axis (Rodrigues' formula)."""
    k = np.asarray(axis, float) / np.linalg.norm(axis)
    t = np.radians(degrees)
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return np.eye(3) + np.sin(t) * K + (1.0 - np.cos(t)) * (K @ K)


class TurnedCube(CubeMesher):
    """The lattice turned by rot about the origin, its halo nodes built after."""

    def __init__(self, rot, **kwargs):
        super().__init__(**kwargs)
        self.rot = np.asarray(rot, float)

    def _shape(self, blk, ijk):
        super()._shape(blk, ijk)
        blk.nodes[blk.interior] = blk.nodes[blk.interior] @ self.rot.T


def walled(mesher=CubeMesher, cells=CELLS, lengths=LENGTHS, periodic=(False, False, False), integrator="tvd-rk3",
           **kw):
    mix = Mixture({"species": AIR, "eos": "cpg", "trans": None})
    mesh = mesher(cells=[[c] for c in cells], lengths=list(lengths), periodic=list(periodic), defaultbc="wall", **kw)
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    orc = Oracle(mix.constants(), 1, "euler", blocks, mets, integrator, bcvals={"wall": {"kind": "slp-adia-wall"}},
                 species=mix.spnames)
    return orc, blocks, mets


def flowing(orc, blocks, u, rot=None):
    prims = []
    for blk in blocks:
        shape = tuple(n + 2 * blk.ng for n in blk.cells)
        q = np.zeros(shape + (5,))
        i = np.arange(shape[0])[:, None, None]
        q[..., 0] = 101325.0
        q[..., 1:4] = u if rot is None else rot @ u
        # the wave is by cell index, not position, so a turned box carries the same values
        q[..., 4] = 300.0 * (1.0 + 0.1 * np.sin(2 * np.pi * i / 6.0))
        prims.append(q)
    orc.set_prims(prims)
    return prims


def closed_form(prims, blk, lengths, u):
    T = prims[0][blk.interior][..., 4]
    cmax = np.sqrt(GAMMA * R * T).max()
    d = np.asarray(lengths) / np.asarray(blk.cells)
    acoustic = cmax * np.sqrt((1.0 / d ** 2).sum())
    convective = (np.abs(u) / d).sum()
    return dict(acoustic=acoustic, convective=convective, combined=acoustic + convective)


def test_cflmax_is_the_fastest_oblique_mode():
    orc, blocks, mets = walled()
    prims = flowing(orc, blocks, U)
    want, got = closed_form(prims, blocks[0], LENGTHS, U), orc.cflmax()
    for name in want:
        assert got[name] == pytest.approx(want[name], rel=1e-12)


def test_cflmax_at_rest_is_acoustic_alone():
    orc, blocks, mets = walled()
    prims = flowing(orc, blocks, np.zeros(3))
    T = prims[0][blocks[0].interior][..., 4].max()
    d = np.asarray(LENGTHS) / np.asarray(CELLS)
    got = orc.cflmax()
    assert got["acoustic"] == pytest.approx(np.sqrt(GAMMA * R * T) * np.sqrt((1.0 / d ** 2).sum()), rel=1e-12)
    assert got["convective"] == 0.0 and got["combined"] == got["acoustic"]


def test_cflmax_is_invariant_to_turning_the_box():
    orc, blocks, _ = walled()
    flowing(orc, blocks, U)
    rot = rotabout([1.0, 1.0, 1.0], 30.0)
    torc, tblocks, _ = walled(mesher=lambda **kw: TurnedCube(rot, **kw))
    flowing(torc, tblocks, U, rot)
    want, got = orc.cflmax(), torc.cflmax()
    for name in want:
        assert got[name] == pytest.approx(want[name], rel=1e-12)


def test_an_axis_one_cell_thick_limits_nothing():
    # dijk is infinite along an axis one cell thick (multiblock/block/grid.py:173-175)
    orc, blocks, _ = walled(cells=(12, 1, 1), lengths=(12e-3, 1e-3, 1e-3))
    prims = flowing(orc, blocks, np.zeros(3))
    c = np.sqrt(GAMMA * R * prims[0][blocks[0].interior][..., 4].max())
    assert orc.cflmax()["acoustic"] == pytest.approx(c / 1e-3, rel=1e-12)


class FakeSolver:
    def __init__(self, combined):
        self.combined = combined

    def cflmax(self):
        return {"combined": self.combined}


def test_the_controllers_step_sizes():
    cfg = Config()
    cfg["simulation"]["simulator"] = "euler"
    cfg["simulation"]["controller"] = "cfl"
    cfg["simulation"]["cfl"] = 0.5
    cfg["simulation"]["dt-max"] = 1.0
    ctrl = integrators.Integrator(cfg.validate()).controller
    assert ctrl.stepsize(FakeSolver(2.0e4)) == 0.5 / 2.0e4
    cfg["simulation"]["dt-max"] = 1e-5
    assert ctrl.stepsize(FakeSolver(2.0e4)) == 1e-5
    cfg["simulation"]["controller"] = "fixed"
    assert integrators.Integrator(cfg).controller.stepsize(FakeSolver(1.0)) == cfg["simulation"]["dt"]


def line_case(cfl, dx=1e-3, seed=1e-6):
    """A line of forty cells, periodic along it and one cell thick and walled
    across, at rest: the four-cell mode seeded in the pressure over a
    temperature wave."""
    mix = Mixture({"species": AIR, "eos": "cpg", "trans": None})
    mesh = CubeMesher(cells=[[40], [1], [1]], lengths=[40 * dx, dx, dx], periodic=[True, False, False],
                      bcnames={n: "slip" for n in (3, 4, 5, 6)})
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    orc = Oracle(mix.constants(), 1, "euler", blocks, mets, "tvd-rk3", bcvals={"slip": {"kind": "slp-adia-wall"}},
                 species=mix.spnames)
    x = mets[0]["xcc"][..., 0]
    q = np.zeros(x.shape + (5,))
    q[..., 0] = 101325.0 * (1.0 + seed * np.sin(2 * np.pi * x / (4 * dx)))
    q[..., 4] = 300.0 * (1.0 + 0.1 * np.sin(2 * np.pi * x / (40 * dx)))
    orc.set_prims([q])
    return orc, blocks[0]


@pytest.mark.parametrize("cfl, bounded", [(1.6, True), (1.7, True), (1.8, False), (2.0, False)])
def test_the_target_brackets_the_schemes_limit(cfl, bounded):
    # tvd-rk3 over the two-point central flux reaches sqrt(3) along the
    # imaginary axis: the seeded mode decays under it and grows past it
    seed = 1e-6
    orc, blk = line_case(cfl, seed=seed)
    for _ in range(300):
        orc.step(min(cfl / orc.cflmax()["combined"], 1.0))
    Q = orc.regs[0][0][blk.interior].reshape(-1, 5)
    p = orc.fromQ(np.ascontiguousarray(Q), np.zeros(len(Q)))[:, 0]
    scatter = np.abs(p / 101325.0 - 1.0).max()
    assert np.isfinite(scatter)
    if bounded:
        assert scatter < seed
    else:
        assert scatter > 10 * seed
