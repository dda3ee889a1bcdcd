"""Binary diffusion on the CPU oracle, pinned to the reference.

tests/golden/binary_h2o2.npz holds the reference's own pair coefficients
(peregrine/simulator/mixture/diffusion/binary.py, T^(3/2) / D at unit
pressure) for the 9-species H2/O2/N2 gas at its fit's sample temperatures,
before the refit.  The exported table set's fits reproduce them within the
refit tolerance; the oracle's mixture average (binary.mako:13-62) reduces to
the pair's coefficient in a two-species mixture and to the self-diffusion
coefficient for a species alone, and matches a numpy restatement of the
kernel's sums on random compositions.
"""

import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200.mixture import load_tables

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def horner(coeffs, u):
    out = np.zeros_like(u)
    for c in coeffs[::-1]:
        out = out * u + c
    return out


@pytest.fixture(scope="module")
def gas():
    t = load_tables("h2o2_gri30_binary")
    orc = Oracle(t, int(t["ns"]), "navier-stokes", [], [], eos="tpg", trans="kinetic-theory")
    return t, orc


def test_the_fits_are_the_references_pair_coefficients():
    g = np.load(os.path.join(GOLD, "binary_h2o2.npz"))
    t = load_tables("h2o2_gri30_binary")
    u = np.log(g["Ts"])
    fits = np.array([horner(row, u) for row in t["dijinv"]])
    assert fits.shape == g["diffinv"].shape
    assert np.abs(fits / g["diffinv"] - 1.0).max() < float(g["tol"])


def states(orc, t, Y, T, p):
    """Q rows and 8-wide state rows at mass fractions Y (every species), T, p."""
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


def pair_D(t, n, m, T, p):
    """The pair's coefficient at T and p from the pair fits: 1 / (p fit T^-3/2)."""
    ns = int(t["ns"])
    k, j = min(n, m), max(n, m)
    slot = {(a, b): q for q, (a, b) in enumerate(zip(*np.triu_indices(ns)))}[(k, j)]
    return 1.0 / (p * horner(t["dijinv"][slot], np.log(T)) * (1.0 / (T * np.sqrt(T))))


def test_a_two_species_mixture_diffuses_at_its_pair_coefficient(gas):
    t, orc = gas
    ns = int(t["ns"])
    rng = np.random.default_rng(3)
    n, m = 0, 8  # H2 in N2
    x = rng.uniform(0.05, 0.95, 16)
    Y = np.zeros((16, ns))
    Y[:, n], Y[:, m] = x, 1.0 - x
    T, p = rng.uniform(300.0, 2500.0, 16), rng.uniform(1e5, 3e6, 16)
    Q, st = states(orc, t, Y, T, p)
    D = orc.transport(Q, st)[:, 2:]
    want = pair_D(t, n, m, T, p)
    assert np.abs(D[:, n] / want - 1.0).max() < 1e-13
    assert np.abs(D[:, m] / want - 1.0).max() < 1e-13


def test_a_species_alone_takes_its_self_diffusion_coefficient(gas):
    t, orc = gas
    ns = int(t["ns"])
    T, p = np.array([400.0, 1500.0]), np.array([1e5, 2e6])
    for n in (0, 3, ns - 1):
        Y = np.zeros((2, ns))
        Y[:, n] = 1.0
        Q, st = states(orc, t, Y, T, p)
        D = orc.transport(Q, st)[:, 2 + n]
        assert np.abs(D / pair_D(t, n, n, T, p) - 1.0).max() < 1e-13


def test_the_mixture_average_is_the_kernels_sums(gas):
    t, orc = gas
    ns = int(t["ns"])
    rng = np.random.default_rng(7)
    Y = rng.random((32, ns))
    Y[rng.random((32, ns)) < 0.3] = 0.0
    Y[:, 0] += 0.05
    Y /= Y.sum(axis=1, keepdims=True)
    T, p = rng.uniform(300.0, 2800.0, 32), rng.uniform(1e5, 3e6, 32)
    Q, st = states(orc, t, Y, T, p)
    D = orc.transport(Q, st)[:, 2:]
    # the kernel's sums restated: over a species' partners X_m / D_nm and
    # X_m MW_m / D_nm, D_n = rest / (p (rest sum1 + X_n sum2))
    MW = t["MW"]
    Yc = Q[:, 5:] / Q[:, :1]
    Yall = np.concatenate([Yc, np.maximum(1.0 - Yc.sum(axis=1, keepdims=True), 0.0)], axis=1)
    X = Yall / MW / (Yall / MW).sum(axis=1, keepdims=True)
    want = np.zeros_like(D)
    for q in range(len(T)):
        for n in range(ns):
            Dinv = np.array([1.0 / pair_D(t, n, m, T[q], 1.0) for m in range(ns)])
            others = [m for m in range(ns) if m != n]
            sum1 = sum(X[q, m] * Dinv[m] for m in others)
            sum2 = sum(X[q, m] * MW[m] * Dinv[m] for m in others)
            rest = sum(X[q, m] * MW[m] for m in others)
            want[q, n] = rest / (p[q] * (rest * sum1 + X[q, n] * sum2))
    assert np.abs(D / want - 1.0).max() < 1e-12


@pytest.mark.parametrize("trace, counts", [(1e-44, 1e-9)])
def test_traces_of_either_sign_read_as_the_pure_cell(gas, trace, counts):
    # tests/transport/test_diffusion.py:31-57: traces of both signs beside a
    # pure species, the negative ones absent and the positive ones under the
    # kernel's tolerance of 64 epsilon too, leave the pure cell; a trace over
    # the tolerance is what the dominant species diffuses in
    t, orc = gas
    ns = int(t["ns"])
    names = [str(n) for n in t["spnames"]]
    lone, up = ns - 1, names.index("OH")
    T, p = np.array([700.0, 1900.0]), np.array([2e5, 1.5e6])

    def D_of(Y):
        Q, st = states(orc, t, np.tile(Y, (2, 1)), T, p)
        return orc.transport(Q, st)[:, 2:]

    Y = np.zeros(ns)
    Y[lone] = 1.0
    Y[names.index("O2")], Y[up], Y[names.index("H2O")] = -3 * trace, 5 * trace, -0.8 * trace
    others = np.arange(ns) != lone
    for sign in (1.0, -1.0):
        Y[up] = sign * 5 * trace
        D = D_of(Y)
        assert np.all(np.isfinite(D))
        for q in range(2):
            assert np.abs(D[q, lone] / pair_D(t, lone, lone, T[q], p[q]) - 1.0) < 1e-12
            want = np.array([pair_D(t, n, lone, T[q], p[q]) for n in np.flatnonzero(others)])
            assert np.abs(D[q, others] / want - 1.0).max() < 1e-12
    # a trace that counts sets the direction: the dominant species' pair with it
    Y[up] = counts
    D = D_of(Y)
    for q in range(2):
        assert np.abs(D[q, lone] / pair_D(t, lone, up, T[q], p[q]) - 1.0) < 1e-8
