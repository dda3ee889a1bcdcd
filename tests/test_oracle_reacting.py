"""The oracle's thermally perfect gas, kinetic-theory transport and
finite-rate chemistry against fixtures made by the reference itself.

tests/golden/make_golden.py recorded the reference's table log and exp
(peregrine/backend/base/mathfns.py and the numpy twins of
tests/mixture/rates.py), its production rates in the kernels' form
(tests/mixture/rates.py:169-185), its Gibbs functions
(peregrine/simulator/mixture/eos/base.py:62-67) and the species' cp and h by
its own polynomial evaluation, for the 9-species H2/O2/N2 subset of GRI-Mech
3.0, the same subset with every reaction irreversible (the reference's
one-way twin), and CH4_O2_FFCMY.  The mixtures' tables come from
peregrine_b200/data, written by the reference's mixture code.  Bars are the
reference's: 3e-14 of the largest rate for the rates against the numpy twin
(tests/chemint/test_rates.py:34-35), bit for bit for the tables.
"""

import os

import numpy as np
import pytest

from oracle import oracle as orc
from peregrine_b200.mixture import load_tables

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MECHS = ["h2o2_gri30", "ch4_o2_ffcmy"]


def gold(name):
    return np.load(os.path.join(GOLD, name))


def reacting(name):
    consts = load_tables(name)
    ns = int(consts["ns"])
    return consts, orc.Oracle(consts, ns, "euler", [], [], eos="tpg", trans="kinetic-theory", chemistry="finite-rate")


def test_the_math_tables_are_the_references_bit_for_bit():
    m = gold("mathfns.npz")
    lt, rt, et, sc = orc.mathtables()
    assert np.array_equal(lt, m["LOGTAB"]) and np.array_equal(rt, m["RCPTAB"]) and np.array_equal(et, m["EXPTAB"])
    assert np.array_equal(sc, m["scalars"])


def test_tlog_and_texp_are_the_numpy_twins_bit_for_bit():
    # the oracle is built without contraction, as numpy evaluates, so the
    # twins agree to the bit
    m = gold("mathfns.npz")
    assert np.array_equal(orc.tlog(m["xlog"]), m["tlog"])
    assert np.array_equal(orc.texp(m["xexp"]), m["texp"])


def test_the_table_functions_are_the_librarys_to_rounding():
    # the reference's claims: tlog within 3e-14 absolute, texp within two ulps
    # (peregrine/backend/base/kernels/mathfns.mako:4-5, 28-29)
    rng = np.random.default_rng(3)
    x = np.exp(rng.uniform(-690.0, 690.0, 20000))
    assert np.abs(orc.tlog(x) - np.log(x)).max() < 3e-14 * 10
    y = rng.uniform(-700.0, 700.0, 20000)
    assert (np.abs(orc.texp(y) / np.exp(y) - 1.0)).max() < 4.5e-16


@pytest.mark.parametrize("mech", MECHS)
def test_gibbs_functions_match_the_reference(mech):
    g = gold(f"rates_{mech}.npz")
    _, o = reacting(mech)
    got = o.gibbs(g["T"])
    # the same Horner in the same order; numpy's polyval may round its
    # products otherwise
    assert np.abs(got - g["gRT"]).max() <= 1e-13 * np.abs(g["gRT"]).max()


@pytest.mark.parametrize("mech", MECHS)
def test_species_cp_and_h_match_the_references_fits(mech):
    g = gold(f"rates_{mech}.npz")
    consts, o = reacting(mech)
    u = np.log(g["Ts"])
    for n in range(int(consts["ns"])):
        cp, h = o.species_cph(n, g["Ts"])
        Rsp = consts["Rsp"][n]
        # the fits alternate in sign in ln T, so a Horner loses digits to
        # cancellation: the bar is rounding on the sum of the terms' magnitudes
        mag = sum(np.abs(c) * u ** m for m, c in enumerate(consts["cppoly"][n])) * Rsp
        assert np.all(np.abs(cp - g["cpR"][:, n] * Rsp) <= 8 * np.finfo(float).eps * mag)
        hmag = sum(np.abs(c) * u ** m for m, c in enumerate(consts["hpoly"][n])) * Rsp * g["Ts"]
        hmag += np.abs(consts["h298"][n]) * Rsp
        assert np.all(np.abs(h - g["hR"][:, n] * Rsp) <= 16 * np.finfo(float).eps * hmag)


@pytest.mark.parametrize("mech", MECHS + ["h2o2_gri30_oneway"])
def test_production_rates_match_the_references_numpy_twin(mech):
    g = gold(f"rates_{mech}.npz")
    _, o = reacting(mech)
    got = o.production(g["rho"], g["Y"], g["T"])
    want = g["omega"]
    for q in range(len(want)):
        scale = np.abs(want[q]).max()
        # (a state whose present species react with nothing has every rate
        # exactly zero on both sides)
        assert np.abs(got[q] - want[q]).max() <= 3e-14 * scale, q
    # mass is conserved: the rates sum to nothing
    assert np.all(np.abs(got.sum(axis=1)) <= 1e-12 * np.abs(want).max(axis=1))


def test_tpg_converges_from_cold_starts():
    # the reference's cold-start check (tests/eos/test_coldstart.py:11-18): pure N2 at
    # 1 bar and 1200 K from guesses a thousand kelvin off, to 1e-6 K
    consts, o = reacting("h2o2_gri30")
    ns = int(consts["ns"])
    y = np.zeros(ns)
    y[list(consts["spnames"]).index("N2")] = 1.0
    q = np.zeros((1, 4 + ns))
    q[0, 0], q[0, 4], q[0, 5:] = 1e5, 1200.0, y[:-1]
    Q = prims_to_Q(o, q)
    for guess in (3400.0, 320.0, 0.0):
        st = o.fromQ(Q, np.array([guess]))
        assert abs(st[0, 1] - 1200.0) < 1e-6


def test_tpg_warm_start_is_the_same_state():
    # from the exact T and from T a stage's drift away, the Newton lands on the
    # same state (tests/eos/test_tpg.py:42-58: within 1e-10)
    consts, o = reacting("h2o2_gri30")
    ns = int(consts["ns"])
    rng = np.random.default_rng(5)
    q = np.zeros((64, 4 + ns))
    Y = rng.random((64, ns))
    Y /= Y.sum(axis=1, keepdims=True)
    q[:, 0], q[:, 4], q[:, 5:] = rng.uniform(1e4, 1e5, 64), rng.uniform(300.0, 2500.0, 64), Y[:, :-1]
    q[:, 1:4] = rng.uniform(-50.0, 50.0, (64, 3))
    Q = prims_to_Q(o, q)
    exact = o.fromQ(Q, q[:, 4])
    drift = o.fromQ(Q, q[:, 4] * 1.01)
    assert np.abs(exact[:, 1] / q[:, 4] - 1.0).max() < 1e-10
    assert np.abs(exact[:, 0] / q[:, 0] - 1.0).max() < 1e-10
    assert np.abs(drift / exact - 1.0).max() < 1e-10
    # rho is p / (R T) with the mixture's R: Ru and every weight pinned
    R = (np.c_[Y[:, :-1], 1.0 - Y[:, :-1].sum(1)] * consts["Rsp"]).sum(1)
    assert np.abs(Q[:, 0] / (q[:, 0] / (R * q[:, 4])) - 1.0).max() < 1e-15


def prims_to_Q(o, q):
    """Q of prims rows through the oracle's fromprims."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    Q = np.zeros_like(q)
    Tg = np.zeros(len(q))
    o.lib.oracle_fromprims(orc.ctypes.byref(o.case), orc._ptr(q), orc._ptr(Q), orc.ctypes.c_long(len(q)), orc._ptr(Tg))
    return Q


def test_the_oneway_mechanism_is_the_mechanism_without_its_reverse_rates():
    # the one-way twin's columns are the mechanism's, every reaction
    # irreversible; its rates are the forward halves of the mechanism's
    a, b = load_tables("h2o2_gri30"), load_tables("h2o2_gri30_oneway")
    assert not b["rxn_reversible"].any() and a["rxn_reversible"].all()
    for k in ("rxn_logA", "rxn_b", "rxn_EaR", "rxn_netnuMW", "rxn_netsp", "gpoly"):
        assert np.array_equal(a[k], b[k]), k
    g = gold("rates_h2o2_gri30_oneway.npz")
    _, o = reacting("h2o2_gri30_oneway")
    got = o.production(g["rho"], g["Y"], g["T"])
    _, two = reacting("h2o2_gri30")
    both = two.production(g["rho"], g["Y"], g["T"])
    # no reverse rate cancels a forward one: the one-way rates differ
    assert np.abs(got - both).max() > 1e-3 * np.abs(got).max()
