"""Herning's viscosity mixing rule on the CPU oracle, against the rule
written out in numpy as the reference's own check does
(tests/transport/test_mixrule.py:37-49): mu = sum X_n sqrt(MW_n) mu_n /
sum X_n sqrt(MW_n), the species viscosities from the kinetic-theory fits,
on the 9-species H2/O2/N2 gas at random compositions; and within a few
percent of Wilke's for air-like mixtures, as the reference says of it.
"""

import numpy as np

from oracle.oracle import Oracle
from peregrine_b200.mixture import load_tables


def horner(coeffs, u):
    out = np.zeros_like(u)
    for c in coeffs[::-1]:
        out = out * u + c
    return out


def states(t, Y, T, p):
    MW = t["MW"]
    R = 8314.46261815324 / (1.0 / (Y / MW).sum(axis=1))
    rho = p / (R * T)
    ns = Y.shape[1]
    Q = np.zeros((len(T), 4 + ns))
    Q[:, 0] = rho
    Q[:, 5:] = rho[:, None] * Y[:, :-1]
    st = np.zeros((len(T), 8))
    st[:, 0], st[:, 1], st[:, 3], st[:, 2] = p, T, rho, 1.0 / rho
    st[:, 5] = 1000.0
    return Q, st


def mixture(rule):
    t = load_tables("h2o2_gri30")
    return t, Oracle(t, int(t["ns"]), "navier-stokes", [], [], eos="tpg", trans="kinetic-theory", mixrule=rule)


def test_herning_is_the_rule_written_out():
    t, orc = mixture("herning")
    ns = int(t["ns"])
    rng = np.random.default_rng(11)
    Y = rng.random((32, ns))
    Y /= Y.sum(axis=1, keepdims=True)
    T, p = rng.uniform(300.0, 2800.0, 32), rng.uniform(1e5, 3e6, 32)
    Q, st = states(t, Y, T, p)
    mu = orc.transport(Q, st)[:, 0]
    MW = t["MW"]
    X = Y / MW / (Y / MW).sum(axis=1, keepdims=True)
    mun = np.stack([(horner(t["mupoly"][n], np.log(T)) * T ** 0.25) ** 2 for n in range(ns)], axis=1)
    w = X * np.sqrt(MW)
    want = (w * mun).sum(axis=1) / w.sum(axis=1)
    assert np.abs(mu / want - 1.0).max() < 1e-12


def test_herning_is_near_wilke_for_like_molecules():
    # O2 and N2 alone: like molecules, where the two rules agree within a few percent
    th, herning = mixture("herning")
    _, wilke = mixture("wilke")
    names = [str(n) for n in th["spnames"]]
    ns = len(names)
    Y = np.zeros((4, ns))
    Y[:, names.index("O2")] = [0.1, 0.23, 0.5, 0.9]
    Y[:, names.index("N2")] = 1.0 - Y[:, names.index("O2")]
    T, p = np.array([300.0, 600.0, 1200.0, 2000.0]), np.full(4, 1e5)
    Q, st = states(th, Y, T, p)
    a, b = herning.transport(Q, st)[:, 0], wilke.transport(Q, st)[:, 0]
    assert np.abs(a / b - 1.0).max() < 0.03
    assert not np.array_equal(a, b)
