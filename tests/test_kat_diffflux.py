"""Known answers for the diffusive face flux, on the CPU oracle.

The reference's own checks of its alpha-damping flux
(tests/navstokes/test_diffflux.py): on linear fields of velocity,
temperature and composition the face flux is the Newtonian stress, Fick's
law with the correction velocity, and Fourier's law plus the species'
enthalpy flux; on a checkerboard temperature, whose central gradients all
vanish, the face gradient is alpha times the two-point jump.  The same
fields, gas and bars (1e-12 of the largest value) as the reference's.
"""

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import CubeMesher
from peregrine_b200.mixture import Mixture, Tref

# three species differing in weight, heat capacity, formation enthalpy, Lewis
# number, viscosity and conductivity (the reference's test gas)
MIXED = {
    "A": {"MW": 28.0, "cp0": 1000.0, "dHf298": 0.0, "lewis": 1.0, "mu0": 1.8e-5, "kappa0": 0.026},
    "B": {"MW": 32.0, "cp0": 900.0, "dHf298": 1.0e7, "lewis": 1.4, "mu0": 2.0e-5, "kappa0": 0.025},
    "C": {"MW": 16.0, "cp0": 2200.0, "dHf298": -7.5e7, "lewis": 0.7, "mu0": 1.1e-5, "kappa0": 0.034},
}
A = np.array([[3.0, -2.0, 1.0], [0.5, 4.0, -1.5], [-2.0, 1.0, 2.5]])
aT = np.array([20.0, -30.0, 10.0])
aY = np.array([[0.05, 0.1, -0.08], [-0.03, 0.06, 0.07]])
Y0 = np.array([0.5, 0.25])


def setup(cells=(8, 7, 6), periodic=(False, False, False), alpha=1.0, lengths=(1.0, 1.0, 1.0)):
    mix = Mixture({"species": MIXED, "eos": "cpg", "trans": "constant"})
    mesh = CubeMesher(cells=[[c] for c in cells], lengths=lengths, periodic=periodic)
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, b.ng) for b in blocks]
    orc = Oracle(mix.constants(), 3, "navier-stokes", blocks, mets, alpha=alpha)
    return mix, blocks, mets, orc


def transport(mix, Q):
    """trstate (mu, kappa, D) of constant transport, Wilke and Lewis, per cell."""
    c = mix.constants()
    rho = Q[..., 0]
    Y = np.concatenate([Q[..., 5:] / rho[..., None], 1.0 - (Q[..., 5:] / rho[..., None]).sum(-1, keepdims=True)], -1)
    X = Y * c["MWinv"] / (Y * c["MWinv"]).sum(-1, keepdims=True)
    sq = np.sqrt(c["mu0"])
    s = sq * c["MWqinv"]
    phi = ((1.0 + s[:, None] / s[None, :]) ** 2 * c["wilkepair"]) @ X[..., :, None]
    mu = (sq * sq * X / phi[..., 0]).sum(-1)
    kappa = 0.5 * ((X * c["kappa0"]).sum(-1) + 1.0 / (X / c["kappa0"]).sum(-1))
    cp = Y @ c["cp0"]
    D = (kappa / (rho * cp))[..., None] / c["lewis"]
    return mu, kappa, D


def linear_fields(mix, blocks, mets, orc, velocity):
    m, blk = mets[0], blocks[0]
    x = m["xcc"]
    q = np.zeros(x.shape[:3] + (7,))
    q[..., 0] = 101325.0
    q[..., 1:4] = 10.0 + x @ A.T if velocity else 0.0
    q[..., 4] = 300.0 + x @ aT
    q[..., 5:] = Y0 + x @ aY.T
    orc.set_prims([q])
    dQ = [np.zeros_like(orc.regs[0][0])]
    return orc.rhs(orc.regs[0], dQ, faces=True, diffusive_only=True)[0]


def faces_of(blk, mets, Fs, Q, axis, mix):
    ng = blk.ng
    F, S = Fs[axis], mets[0]["ijk"[axis] + "S"]
    nf = F.shape[axis]
    fs, left, right = ([slice(ng + 1, -ng - 1)] * 3 for _ in range(3))
    fs[axis] = slice(ng + 2, nf - ng - 2)
    left[axis] = slice(ng + 1, nf - ng - 3)
    right[axis] = slice(ng + 2, nf - ng - 2)
    fs, L, R = tuple(fs), tuple(left), tuple(right)
    mu, kappa, D = transport(mix, Q)
    Y = Q[..., 5:] / Q[..., :1]
    Yall = np.concatenate([Y, 1.0 - Y.sum(-1, keepdims=True)], -1)
    u = Q[..., 1:4] / Q[..., :1]
    e = (Q[..., 4] - 0.5 * (Q[..., 1:4] ** 2).sum(-1) / Q[..., 0]) / Q[..., 0]
    c = mix.constants()
    cv = Yall @ c["cp0"] - Yall @ c["Rsp"]
    T = (e - Yall @ c["h298R"]) / cv

    def mean(a):
        return 0.5 * (a[L] + a[R])

    return dict(F=F[fs], S=S[fs], rho=mean(Q[..., 0]), T=mean(T), u=mean(u), Y=mean(Yall), mu=mean(mu),
                kappa=mean(kappa), D=mean(D))


def expected(f, mix, work):
    S = f["S"]
    mu = f["mu"][..., None, None]
    tau = -mu * (A + A.T) + 2.0 / 3.0 * mu * np.trace(A) * np.eye(3)
    momentum = np.einsum("...ij,...j->...i", tau, S)
    gY = S @ np.vstack([aY, -aY.sum(axis=0)]).T
    J = -f["rho"][..., None] * f["D"] * gY
    Vc = (f["D"] * gY).sum(axis=-1)
    J += f["Y"] * (f["rho"] * Vc)[..., None]
    sp = [MIXED[n] for n in mix.spnames]
    cp = np.array([s["cp0"] for s in sp])
    hf = np.array([s["dHf298"] / s["MW"] for s in sp])
    h = cp * (f["T"][..., None] - Tref) + hf
    energy = -f["kappa"] * (S @ aT) + (J * h).sum(axis=-1)
    if work:
        energy += np.einsum("...i,...ij,...j->...", f["u"], tau, S)
    return momentum, energy, J[..., :-1]


def rel(got, want):
    return np.abs(got - want).max() / np.abs(want).max()


@pytest.mark.parametrize("axis", range(3))
def test_momentum_rows_are_the_newtonian_stress(axis):
    mix, blocks, mets, orc = setup()
    Fs = linear_fields(mix, blocks, mets, orc, True)
    f = faces_of(blocks[0], mets, Fs, orc.regs[0][0], axis, mix)
    momentum, _, _ = expected(f, mix, True)
    assert rel(f["F"][..., 1:4], momentum) < 1e-12


@pytest.mark.parametrize("axis", range(3))
def test_species_rows_are_ficks_law_with_the_correction(axis):
    mix, blocks, mets, orc = setup()
    Fs = linear_fields(mix, blocks, mets, orc, True)
    f = faces_of(blocks[0], mets, Fs, orc.regs[0][0], axis, mix)
    _, _, species = expected(f, mix, True)
    assert rel(f["F"][..., 5:], species) < 1e-12


@pytest.mark.parametrize("velocity", [False, True])
@pytest.mark.parametrize("axis", range(3))
def test_energy_row_is_fourier_species_enthalpy_and_stress_work(axis, velocity):
    mix, blocks, mets, orc = setup()
    Fs = linear_fields(mix, blocks, mets, orc, velocity)
    f = faces_of(blocks[0], mets, Fs, orc.regs[0][0], axis, mix)
    _, energy, _ = expected(f, mix, velocity)
    assert rel(f["F"][..., 4], energy) < 1e-12


@pytest.mark.parametrize("alpha", [0.0, 1.0])
def test_alpha_damps_toward_the_two_point_gradient(alpha):
    nx, L = 8, 1e-3
    mix, blocks, mets, orc = setup(cells=(nx, 2, 2), periodic=(True, True, True), alpha=alpha,
                                   lengths=(L, L / nx * 2, L / nx * 2))
    blk = blocks[0]
    ng = blk.ng
    q = np.zeros(tuple(n + 2 * ng for n in blk.cells) + (7,))
    q[..., 0] = 101325.0
    T = 300.0 + 10.0 * (-1.0) ** np.arange(q.shape[0])
    q[..., 4] = T[:, None, None]
    q[..., 5:] = Y0
    orc.set_prims([q])
    dQ = [np.zeros_like(orc.regs[0][0])]
    F = orc.rhs(orc.regs[0], dQ, faces=True, diffusive_only=True)[0][0]
    nf = F.shape[0]
    got = F[ng:nf - ng, ng, ng, 4]
    area = np.abs(mets[0]["iS"][ng:nf - ng, ng, ng, 0])
    kappa = transport(mix, orc.regs[0][0])[1][ng, ng, ng]
    dx = L / nx
    jump = T[ng:nf - ng] - T[ng - 1:nf - ng - 1]
    want = -alpha * kappa * jump / dx * area
    scale = kappa * 20.0 / dx * area.max()
    assert np.abs(got - want).max() < 1e-12 * scale
