"""The sub-stepped chemistry on the CPU oracle, pinned to the reference's own
checks of it (tests/chemint/test_integration.py, test_equilibrium.py): one
walled cell of CH4/O2 under the FFCM-Y mechanism, its right-hand side's
species rows the integrator's mean rates.

* one substep within the fastest species' bound is the finite-rate source,
  to the bit;
* where the explicit source overshoots the mass fractions' bounds, the
  substeps keep them in [0, 1];
* a settled cell (cold reactants) finishes in one relaxed move within 1e-6
  of the finite-rate source, and without the exit is that source to the bit;
  a right-hand side before any step (dt 0) is the source to the bit;
* ignited products never settle: with and without the exit they substep
  alike, to the bit;
* the ignition delay at 20 bar and 1500 K is within 1 % of the 3.175e-5 s the
  reference's test quotes for Cantera, and the exit leaves the run unchanged.
"""

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import CubeMesher
from peregrine_b200.mixture import Mixture

GAS = "ch4_o2_ffcmy"


def mixture():
    return Mixture({"species": GAS, "eos": "tpg", "trans": None})


def stoichiometric(mix):
    """CH4 + 2 O2 by moles, as mass fractions of every species."""
    X = np.zeros(mix.ns)
    X[mix.spnames.index("CH4")], X[mix.spnames.index("O2")] = 1.0, 2.0
    Y = X * np.asarray(mix.constants()["MW"])
    return Y / Y.sum()


def cell(kind, p, T, Y, dt=1e-9, cap=200, eqtol=1e-7, stepset=True):
    mix = mixture()
    blocks = CubeMesher(cells=[[1], [1], [1]], lengths=[0.01] * 3, defaultbc="walls").make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    orc = Oracle(mix.constants(), mix.ns, "euler", blocks, mets, "tvd-rk3", eos="tpg", trans="constant",
                 chemistry="finite-rate", chemint=kind, max_substeps=cap, eqtol=eqtol,
                 bcvals={"walls": {"kind": "slp-adia-wall"}}, species=mix.spnames)
    q = np.zeros((5, 5, 5, 4 + mix.ns))
    q[..., 0], q[..., 4], q[..., 5:] = p, T, np.asarray(Y)[:-1]
    orc.set_prims([q])
    if stepset:
        orc.dt = dt
    return orc, mix


def rhs(orc):
    dQ = [np.zeros_like(orc.regs[0][0])]
    orc.rhs(orc.regs[0], dQ)
    return dQ[0][2, 2, 2]


def Qcell(orc):
    return orc.regs[0][0][2, 2, 2].copy()


def temperature(orc):
    Q = Qcell(orc)
    return orc.fromQ(Q[None, :], np.array([orc.Tg[0][2, 2, 2]]))[0, 1]


def test_one_substep_within_the_bound_is_the_finite_rate_source():
    rng = np.random.default_rng(5)
    mix = mixture()
    Y = rng.random(mix.ns)
    Y /= Y.sum()
    explicit, _ = cell("coupled", 10e5, 1800.0, Y)
    Q = Qcell(explicit)
    rho = Q[0]
    omega = explicit.production(np.array([rho]), Y[None, :], np.array([1800.0]))[0]
    # the fastest species' way to its bound, in time
    headroom = np.where(omega < 0, Y, 1.0 - Y)
    dt = 0.5 * (rho * headroom / np.abs(omega)).min()
    explicit, _ = cell("coupled", 10e5, 1800.0, Y, dt=dt)
    substepped, _ = cell("sub-stepped", 10e5, 1800.0, Y, dt=dt, cap=1)
    assert np.array_equal(rhs(explicit)[5:], rhs(substepped)[5:])


@pytest.mark.parametrize("cap", [1, 10, 50])
def test_substeps_keep_the_state_in_bounds(cap):
    mix = mixture()
    Y, dt = stoichiometric(mix), 1e-5
    explicit, _ = cell("coupled", 10e5, 2500.0, Y, dt=dt)
    Q, r = Qcell(explicit), rhs(explicit)
    after = (Q[5:] + r[5:] * dt) / Q[0]
    assert after.min() < -0.1 or after.max() > 1.1
    sub, _ = cell("sub-stepped", 10e5, 2500.0, Y, dt=dt, cap=cap)
    Q, r = Qcell(sub), rhs(sub)
    after = (Q[5:] + r[5:] * dt) / Q[0]
    assert np.isfinite(r).all()
    assert after.min() > -1e-12 and after.sum() < 1.0 + 1e-12


def reactants(kind, tolerance, dt=1e-6, **kw):
    mix = mixture()
    return cell(kind, 10e5, 400.0, stoichiometric(mix), dt=dt, cap=200, eqtol=tolerance, **kw)[0]


def test_a_settled_cell_finishes_in_one_relaxed_move():
    explicit = rhs(reactants("coupled", 0.0))[5:]
    withexit = reactants("sub-stepped", 1e-7)
    source = rhs(withexit)[5:]
    assert int(withexit.subs[0][2, 2, 2]) == 1
    scale = np.abs(explicit).max()
    assert np.abs(source - explicit).max() < 1e-6 * scale
    assert not np.array_equal(source, explicit)
    # without the exit the one substep covers the step: the finite-rate source to the bit
    assert np.array_equal(rhs(reactants("sub-stepped", 0.0))[5:], explicit)


def test_a_right_hand_side_before_any_step_is_the_finite_rate_source():
    # the step scalar is nothing until a step sets it, so the exit is not judged over no time
    explicit = rhs(reactants("coupled", 0.0))[5:]
    bare = reactants("sub-stepped", 1e-7, stepset=False)
    assert np.array_equal(rhs(bare)[5:], explicit)


def products(tolerance, relax=2, dt=1e-6):
    mix = mixture()
    orc, _ = cell("sub-stepped", 10e5, 2500.0, stoichiometric(mix), dt=dt, cap=200, eqtol=tolerance)
    for _ in range(relax):
        orc.step(dt)
    return orc


def test_an_unsettled_cell_substeps_as_the_one_pass_form():
    # ignited products never settle: each substep throws the fast radicals off
    # their quasi-steady values, so their rates are large at a step's start
    withexit, without = products(1e-7), products(0.0)
    withexit.step(1e-6)
    without.step(1e-6)
    assert np.array_equal(withexit.subs[0], without.subs[0])
    assert withexit.subs[0][2, 2, 2] > 1
    assert np.array_equal(Qcell(withexit), Qcell(without))


def delay(orc, dt, T0, rise, until):
    t = 0.0
    while t < until:
        orc.step(dt)
        t += dt
        if temperature(orc) > T0 + rise:
            return t
    return None


def test_ignition_follows_the_reference_delay():
    # the reference's test quotes Cantera's 3.175e-5 s (and its own 3.180e-5 s)
    # at 20 bar and 1500 K, stoichiometric, dt 1e-8 with a ten-substep cap
    theirs = 3.175e-5
    p0, T0, dt = 20e5, 1500.0, 1e-8
    mix = mixture()
    orc, _ = cell("sub-stepped", p0, T0, stoichiometric(mix), dt=dt, cap=10, eqtol=0.0)
    ours = delay(orc, dt, T0, 400.0, 4 * theirs)
    assert ours is not None and abs(ours / theirs - 1.0) < 0.01
    # the exit never takes an igniting cell: the run with it is this one to the bit
    withexit, _ = cell("sub-stepped", p0, T0, stoichiometric(mix), dt=dt, cap=10, eqtol=1e-7)
    assert delay(withexit, dt, T0, 400.0, 4 * theirs) == ours
    assert np.array_equal(Qcell(withexit), Qcell(orc))
