"""The oracle's cubic real gas and its double-flux plane, pinned to the
reference.

The cubic's constants come from the reference's own RealGasModel
(peregrine_b200/data/o2_h2_{srk,pr}.npz, written by its mixture code; the
Peng-Robinson set with the reference's model class given PR's constants).
tests/golden/realgas_<cubic>.npz holds tests/eos/support.py's textbook
density (numpy's roots of the cubic and the least Gibbs energy phase) at
random states and through liquid oxygen.  The rest restates the reference's
own checks of its real gas and plane (tests/eos/test_coldstart.py,
tests/doubleflux/test_plane.py) and thermodynamic identities the cubic must
satisfy.
"""

import os

import numpy as np
import pytest

from oracle import oracle as orc
from peregrine_b200.mixture import load_tables

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
F = ("p", "T", "rhoinv", "rho", "e", "cp", "gamma", "c")


def gas(cubic, df=False):
    t = load_tables(f"o2_h2_{cubic}")
    return t, orc.Oracle(t, 2, "euler", [], [], eos="real-gas-df" if df else "real-gas")


def Q_of(rec, Y0, u=(0.0, 0.0, 0.0)):
    rho, e = rec[:, 3], rec[:, 4]
    u = np.asarray(u, dtype=float)
    Q = np.zeros((len(rec), 6))
    Q[:, 0] = rho
    Q[:, 1:4] = rho[:, None] * u
    Q[:, 4] = rho * (e + 0.5 * (u * u).sum())
    Q[:, 5] = rho * Y0
    return Q


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_density_is_the_textbook_cubics(cubic):
    g = np.load(os.path.join(GOLD, f"realgas_{cubic}.npz"))
    _, o = gas(cubic)
    rec = o.realgas_frompT(g["p"], g["T"], g["Y"])
    # Cardano against numpy's companion-matrix roots: the roots' rounding
    assert np.abs(rec[:, 3] / g["rho"] - 1.0).max() < 1e-10


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_fromrhoE_recovers_the_state_from_cold_and_warm_starts(cubic):
    g = np.load(os.path.join(GOLD, f"realgas_{cubic}.npz"))
    _, o = gas(cubic)
    rec = o.realgas_frompT(g["p"], g["T"], g["Y"])
    Q = Q_of(rec, g["Y"][:, 0])
    for guess in (g["T"], g["T"] * 1.01, np.zeros_like(g["T"])):
        back = o.realgas_fromQ(Q, guess)
        # p and T within the Newton's tolerance of the state set
        # (tests/eos/test_coldstart.py: 1e-6 K from cold starts)
        assert np.abs(back[:, 1] - g["T"]).max() < 1e-6
        assert np.abs(back[:, 0] / g["p"] - 1.0).max() < 1e-8


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_cp_is_the_enthalpys_slope_at_fixed_pressure(cubic):
    _, o = gas(cubic)
    rng = np.random.default_rng(2)
    n = 32
    p, T, Y = rng.uniform(2e6, 6e7, n), rng.uniform(200.0, 600.0, n), rng.uniform(0.0, 1.0, (n, 1))
    h = lambda rec: rec[:, 4] + rec[:, 0] / rec[:, 3]
    dT = 1e-3 * T
    up, dn, at = (o.realgas_frompT(p, T + s * dT, Y) for s in (1.0, -1.0, 0.0))
    assert np.abs((h(up) - h(dn)) / (2 * dT) / at[:, 5] - 1.0).max() < 1e-5


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_sound_speed_is_the_isentropic_pressure_slope(cubic):
    # at fixed entropy de = p / rho^2 drho, so c^2 = dp/drho along it, p from fromrhoE
    _, o = gas(cubic)
    rng = np.random.default_rng(4)
    n = 32
    p, T, Y = rng.uniform(2e6, 6e7, n), rng.uniform(200.0, 600.0, n), rng.uniform(0.0, 1.0, (n, 1))
    rec = o.realgas_frompT(p, T, Y)
    rho, e = rec[:, 3], rec[:, 4]
    d = 1e-5 * rho

    def p_at(r, ee):
        q = np.zeros((n, 6))
        q[:, 0], q[:, 4], q[:, 5] = r, r * ee, r * Y[:, 0]
        return o.realgas_fromQ(q, T)[:, 0]

    slope = (p_at(rho + d, e + p / rho ** 2 * d) - p_at(rho - d, e - p / rho ** 2 * d)) / (2 * d)
    assert np.abs(slope / rec[:, 7] ** 2 - 1.0).max() < 1e-5


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_the_plane_is_tangent_to_the_eos(cubic):
    # tests/doubleflux/test_plane.py:55-76: the residual of rho e off the frozen
    # plane differs across a perturbation by second order, the energy by first
    _, o = gas(cubic, df=True)
    P0, T0, Y0 = 59.8e6, 130.0, 0.5

    def at(p, T, Y):
        rec = np.ascontiguousarray(o.realgas_frompT([p], [T], [[Y]]))
        return rec, np.ascontiguousarray(Q_of(rec, Y))

    rec, Q = at(P0, T0, Y0)
    o.freeze(Q, rec)
    theta, eps, kappa, zeta = rec[0, 9], rec[0, 10], rec[0, 11], rec[0, 12]

    def residual(p, T, Y):
        r, q = at(p, T, Y)
        E = q[0, 0] * r[0, 4]
        return E - (theta * p + eps * q[0, 0] + zeta * q[0, 5] + kappa), E

    h = 1e-3
    for k in range(3):
        up, dn = [P0, T0, Y0], [P0, T0, Y0]
        up[k] *= 1.0 + h
        dn[k] *= 1.0 - h
        Ru, Eu = residual(*up)
        Rd, Ed = residual(*dn)
        assert abs(Ru - Rd) < 1e-5 * abs(Eu - Ed), k


@pytest.mark.parametrize("cubic", ["srk", "pr"])
def test_the_frozen_state_is_the_eoss(cubic):
    # tests/doubleflux/test_plane.py:79-93: the state off the plane at the
    # point it froze is the eos's state, within 1e-12
    _, o = gas(cubic, df=True)
    rng = np.random.default_rng(6)
    n = 16
    p, T, Y = rng.uniform(5e6, 6e7, n), rng.uniform(110.0, 400.0, n), rng.uniform(0.0, 1.0, (n, 1))
    rec = np.ascontiguousarray(o.realgas_frompT(p, T, Y))
    Q = np.ascontiguousarray(Q_of(rec, Y[:, 0], u=(20.0, 0.0, 0.0)))
    eos = np.ascontiguousarray(o.realgas_fromQ(Q, T))
    frozen = eos.copy()
    o.freeze(Q, frozen)
    # the plane's pressure at the frozen point, and the state there
    rhoinv = 1.0 / Q[:, 0]
    pp = (Q[:, 4] - 0.5 * (Q[:, 1:4] ** 2).sum(1) * rhoinv - frozen[:, 10] * Q[:, 0] - frozen[:, 12] * Q[:, 5]
          - frozen[:, 11]) / frozen[:, 9]
    assert np.abs(pp / eos[:, 0] - 1.0).max() < 1e-12
    for k, name in enumerate(F):
        assert np.abs(frozen[:, k] / eos[:, k] - 1.0).max() < 1e-12, name
