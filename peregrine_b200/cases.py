"""Synthetic benchmark cases: configs, meshes and seeded initial fields.

The Taylor-Green vortex is the reference's own example
(examples/threeDTaylorGreen.py:30-66): a periodic cube of side 2 pi, the
analytic velocity and pressure field, here at Mach 0.1 and Re 1600 with a
seeded 1e-6 white-noise perturbation of the velocity.  The gas is air as a
calorically perfect gas with gamma 1.4 (cp0 = 3.5 Ru / MW), at 300 K and
1 atm; mu = rho0 U0 L / Re with L = 1, kappa = mu cp / Pr with Pr = 0.71.
"""

import numpy as np

from peregrine_b200.config import Config
from peregrine_b200.mesher import CubeMesher, uneven_cuts
from peregrine_b200.mixture import Ru

MW_AIR = 28.97
CP_AIR = 3.5 * Ru / MW_AIR
T0, P0 = 300.0, 101325.0


def tgv_gas(mach=0.1, reynolds=1600.0, prandtl=0.71):
    R = Ru / MW_AIR
    gamma = CP_AIR / (CP_AIR - R)
    rho0 = P0 / (R * T0)
    U0 = mach * np.sqrt(gamma * R * T0)
    mu = rho0 * U0 * 1.0 / reynolds
    kappa = mu * CP_AIR / prandtl
    gas = {"Air": {"MW": MW_AIR, "cp0": CP_AIR, "mu0": mu, "kappa0": kappa}}
    return gas, dict(R=R, gamma=gamma, rho0=rho0, U0=U0)


def tgv_config(simulator="navier-stokes", integrator="rk4", launch="batched"):
    gas, _ = tgv_gas()
    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"]["species"] = gas
    cfg["mixture"]["trans"] = "constant" if simulator == "navier-stokes" else None
    cfg["time-integration"]["integrator"] = integrator
    cfg["adv-flux"]["primary"] = "kepaec"
    cfg["backend-b200"]["launch"] = launch
    return cfg.validate()


def tgv_mesh(cells=32, blocks=(1, 1, 1), seed=0, low=None, high=None, jostle=0.0):
    """A periodic 2 pi cube of cells^3, cut into blocks; uneven cuts drawn from seed."""
    rng = np.random.default_rng(seed)
    cuts = []
    for n in blocks:
        if n == 1:
            cuts.append([cells])
        elif low is None:
            base = cells // n
            cuts.append([base + (1 if m < cells - base * n else 0) for m in range(n)])
        else:
            cuts.append(uneven_cuts(cells, n, low, high, rng))
    return CubeMesher(mbdims=list(blocks), cells=cuts, lengths=[2 * np.pi] * 3, periodic=[True] * 3, jostle=jostle)


def tgv_prims(blocks, metrics, ne=5, seed=0, noise=1e-6, mach=0.1):
    """Primitives p, u, v, w, T per block (full shape, halo included)."""
    _, g = tgv_gas(mach=mach)
    rng = np.random.default_rng(seed)
    out = []
    for b, m in zip(blocks, metrics):
        xc = m["xcc"]
        x, y, z = xc[..., 0], xc[..., 1], xc[..., 2]
        q = np.zeros(x.shape + (ne,))
        U0, rho0 = g["U0"], g["rho0"]
        q[..., 0] = P0 + rho0 * U0 ** 2 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
        q[..., 1] = U0 * np.sin(x) * np.cos(y) * np.cos(z)
        q[..., 2] = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
        q[..., 1:4] += noise * U0 * rng.standard_normal(x.shape + (3,))
        q[..., 4] = T0 * q[..., 0] / P0
        out.append(q)
    return out


# three species differing in weight, heat capacity, formation enthalpy, Lewis
# number, viscosity and conductivity
MIXED = {
    "A": {"MW": 28.0, "cp0": 1000.0, "dHf298": 0.0, "lewis": 1.0, "mu0": 1.8e-5, "kappa0": 0.026},
    "B": {"MW": 32.0, "cp0": 900.0, "dHf298": 1.0e7, "lewis": 1.4, "mu0": 2.0e-5, "kappa0": 0.025},
    "C": {"MW": 16.0, "cp0": 2200.0, "dHf298": -7.5e7, "lewis": 0.7, "mu0": 1.1e-5, "kappa0": 0.034},
}


def mixing_config(simulator="navier-stokes", integrator="rk4", primary="hllc", recon="muscl", limiter="koren", ns=2,
                  launch="per-block"):
    """A gas of ns of the MIXED species through one advective scheme."""
    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"]["species"] = {k: MIXED[k] for k in list(MIXED)[:ns]}
    cfg["mixture"]["trans"] = "constant" if simulator == "navier-stokes" else None
    cfg["time-integration"]["integrator"] = integrator
    cfg["adv-flux"]["primary"] = primary
    cfg["adv-flux"]["recon"] = recon
    cfg["adv-flux"]["limiter"] = limiter if recon == "muscl" else None
    cfg["backend-b200"]["launch"] = launch
    return cfg.validate()


def rough_prims(metrics, ns, seed=0, speed=420.0):
    """Primitives p, u, v, w, T, Y[ns - 1] per block on the 2 pi cube: waves
    with a step in pressure, temperature and composition across x = pi, so
    the slope ratios take every sign and size and, at this speed, some faces
    are supersonic each way."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2 * np.pi, 8)
    out = []
    for m in metrics:
        x, y, z = (m["xcc"][..., d] for d in range(3))
        step = (np.mod(x, 2 * np.pi) > np.pi).astype(float)
        q = np.zeros(x.shape + (4 + ns,))
        q[..., 0] = P0 * (1.0 + 0.2 * np.sin(x + ph[0]) * np.cos(y + ph[1]) + 0.5 * step)
        q[..., 1] = speed * np.sin(x + ph[2]) * np.cos(z + ph[3])
        q[..., 2] = 0.4 * speed * np.cos(y + ph[4])
        q[..., 3] = 0.3 * speed * np.sin(z + ph[5]) * np.cos(x)
        q[..., 1:4] += 5.0 * rng.standard_normal(x.shape + (3,))
        q[..., 4] = T0 * (1.0 + 0.2 * np.cos(x + ph[6]) * np.sin(z + ph[7]) + 0.4 * step)
        for n in range(ns - 1):
            q[..., 5 + n] = (0.6 - 0.2 * step) / (ns - 1) * (1.0 + 0.3 * np.sin((n + 1) * x + y + ph[n]))
        out.append(q)
    return out


# the reacting homogeneous field: stoichiometric H2/air (H2 : O2 : N2 = 2 : 1 : 3.76
# by moles) at 1 atm and 1000 K, Gaussian hot spots and a divergence-free velocity
H2O2_TABLES = "h2o2_gri30"


def reacting_config(simulator="navier-stokes", integrator="tvd-rk3", primary="hllc", recon="muscl", limiter="koren",
                    chemistry=True, tables=H2O2_TABLES, launch="per-block"):
    """The 9-species H2/O2/N2 mixture (the GRI-Mech 3.0 subset, thermally
    perfect, kinetic-theory transport, finite-rate chemistry coupled)."""
    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"]["species"] = tables
    cfg["mixture"]["eos"] = "tpg"
    cfg["mixture"]["trans"] = "kinetic-theory" if simulator == "navier-stokes" else None
    cfg["mixture"]["chemistry"] = "finite-rate" if chemistry else None
    cfg["chem-integration"]["kind"] = "coupled" if chemistry else None
    cfg["time-integration"]["integrator"] = integrator
    cfg["adv-flux"]["primary"] = primary
    cfg["adv-flux"]["recon"] = recon
    cfg["adv-flux"]["limiter"] = limiter if recon == "muscl" else None
    cfg["backend-b200"]["launch"] = launch
    return cfg.validate()


def stoichiometric_h2_air(spnames, MW):
    X = np.zeros(len(spnames))
    for name, moles in (("H2", 2.0), ("O2", 1.0), ("N2", 3.76)):
        X[spnames.index(name)] = moles
    Y = X * np.asarray(MW)
    return Y / Y.sum()


def reacting_mesh(cells=96, blocks=(1, 1, 1), length=0.01):
    """A periodic cube of side length (m) in cells^3, evenly cut."""
    cuts = []
    for n in blocks:
        base = cells // n
        cuts.append([base + (1 if m < cells - base * n else 0) for m in range(n)])
    return CubeMesher(mbdims=list(blocks), cells=cuts, lengths=[length] * 3, periodic=[True] * 3)


def reacting_prims(metrics, spnames, MW, cells, length=0.01, seed=0, spots=4, dT=400.0, width=8.0, urms=10.0,
                   T0=1000.0, p0=101325.0, radicals=0.0):
    """Primitives of the reacting field: seeded Gaussian hot spots (peak
    dT, standard deviation width cells, periodic images) on T0, and the curl
    of a seeded random vector potential of a few Fourier modes scaled to
    u_rms, so the velocity is divergence free.  radicals > 0 seeds every
    species absent from the mixture with random mass fractions up to that,
    taken from the last species, so every reaction runs both ways."""
    rng = np.random.default_rng(seed)
    ns = len(spnames)
    Y = stoichiometric_h2_air(list(spnames), MW)
    centres = rng.uniform(0.0, length, (spots, 3))
    amps = rng.uniform(0.5, 1.0, spots) * dT
    sigma = width * length / cells
    nk = 6
    kvec = rng.integers(1, 4, (nk, 3)) * rng.choice([-1, 1], (nk, 3))
    avec = rng.normal(0.0, 1.0, (nk, 3))
    phase = rng.uniform(0.0, 2 * np.pi, nk)
    out = []
    vel = []
    for m in metrics:
        x = m["xcc"]
        T = np.full(x.shape[:3], T0)
        for c, a in zip(centres, amps):
            d = x - c
            d -= length * np.round(d / length)
            T += a * np.exp(-0.5 * (d ** 2).sum(-1) / sigma ** 2)
        # u = curl A, A = sum_k a_k sin(2 pi k.x / L + phi_k)
        u = np.zeros(x.shape)
        for k, a, ph in zip(kvec, avec, phase):
            arg = 2 * np.pi * (x @ k) / length + ph
            grad = np.cos(arg)[..., None] * (2 * np.pi * k / length)
            u += np.cross(grad, a)
        vel.append(u)
        q = np.zeros(x.shape[:3] + (4 + ns,))
        q[..., 0] = p0
        q[..., 4] = T
        q[..., 5:] = Y[:-1]
        if radicals > 0.0:
            for n in range(ns - 1):
                if Y[n] == 0.0:
                    q[..., 5 + n] = radicals * rng.uniform(0.0, 1.0, x.shape[:3])
        out.append(q)
    rms = np.sqrt(np.mean(np.concatenate([(u ** 2).sum(-1).ravel() / 3 for u in vel])))
    for q, u in zip(out, vel):
        q[..., 1:4] = u * (urms / rms)
    return out


# the transcritical mixing layer: O2 (dense, 120 K) and H2 (300 K) at 60 bar,
# the real gas with the double flux
def mixing_layer_config(cubic="pr", simulator="euler-df", integrator="tvd-rk3", launch="per-block", primary="kepaec",
                        recon="constant", limiter=None):
    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"]["species"] = f"o2_h2_{cubic}"
    cfg["mixture"]["eos"] = "real-gas-df" if simulator.endswith("-df") else "real-gas"
    cfg["mixture"]["trans"] = "kinetic-theory" if simulator.startswith("navier-stokes") else None
    cfg["time-integration"]["integrator"] = integrator
    cfg["adv-flux"].update(primary=primary, recon=recon, limiter=limiter)
    cfg["backend-b200"]["launch"] = launch
    return cfg.validate()


def mixing_layer_mesh(nx=256, ny=128, nz=4, blocks=8, dx=2e-5, seed=0, low=None, high=None):
    """A periodic box of nx x ny x nz cells of dx, cut along i into blocks of
    seeded uneven widths (low..high cells)."""
    rng = np.random.default_rng(seed)
    if blocks == 1:
        cuts = [nx]
    else:
        lo = low if low is not None else int(0.75 * nx / blocks)
        hi = high if high is not None else int(1.25 * nx / blocks)
        cuts = uneven_cuts(nx, blocks, lo, hi, rng)
    return CubeMesher(mbdims=[blocks, 1, 1], cells=[cuts, [ny], [nz]], lengths=[nx * dx, ny * dx, nz * dx],
                      periodic=[True] * 3)


def mixing_layer_prims(metrics, ny, dx=2e-5, seed=0, p=6e6, Tcold=120.0, Thot=300.0, dU=50.0, noise=0.01,
                       width=4.0):
    """Primitives (p, u, v, w, T, Y_O2): a band of cold O2 between two tanh
    interfaces (width cells thick) in a periodic H2 stream, the streams at
    +-dU/2, with seeded noise of noise * dU on u and v."""
    rng = np.random.default_rng(seed)
    Ly = ny * dx
    out = []
    for m in metrics:
        y = m["xcc"][..., 1]
        d = width * dx
        f = 0.5 * (np.tanh((y - 0.25 * Ly) / d) - np.tanh((y - 0.75 * Ly) / d))
        q = np.zeros(y.shape + (6,))
        q[..., 0] = p
        q[..., 1] = -0.5 * dU + dU * f + noise * dU * rng.standard_normal(y.shape)
        q[..., 2] = noise * dU * rng.standard_normal(y.shape)
        q[..., 4] = Thot + (Tcold - Thot) * f
        q[..., 5] = np.clip(f, 0.0, 1.0)
        out.append(q)
    return out


# the boundary test box: one jostled block whose every face carries the same
# boundary entry at seeded values (the reference's own boundary tests run
# such a box, tests/bcs/bcblock.py), the velocity random cell by cell so an
# exit sees flow both ways, p, T and Y smooth so an extrapolated halo stays
# physical
def bc_box_config(kind, ns=1, simulator="euler", primary="kepaec", recon="constant", limiter=None, eos="cpg",
                  integrator="rk4", seed=0, entry=None, launch="per-block", tables=None):
    """tables: a mixture's stored tables (the real gases) instead of ns of the MIXED species."""
    rng = np.random.default_rng(seed)
    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    if tables is not None:
        cfg["mixture"]["species"] = tables
    elif ns == 1:
        cfg["mixture"]["species"] = {"Air": {"MW": MW_AIR, "cp0": CP_AIR, "mu0": 1.8e-5, "kappa0": 0.026}}
    else:
        cfg["mixture"]["species"] = {k: MIXED[k] for k in list(MIXED)[:ns]}
    cfg["mixture"]["eos"] = eos
    # the real gases' stored tables carry the kinetic-theory fits
    viscous = simulator.startswith("navier-stokes")
    cfg["mixture"]["trans"] = ("kinetic-theory" if tables is not None else "constant") if viscous else None
    cfg["time-integration"]["integrator"] = integrator
    cfg["adv-flux"]["primary"] = primary
    cfg["adv-flux"]["recon"] = recon
    cfg["adv-flux"]["limiter"] = limiter if recon == "muscl" else None
    cfg["backend-b200"]["launch"] = launch

    def rounded(v):
        return float(f"{v:.6g}")

    values = {"kind": kind, "p": rounded(rng.uniform(0.9, 1.1) * P0), "u": rounded(rng.uniform(1, 300)),
              "v": rounded(rng.uniform(1, 300)), "w": rounded(rng.uniform(1, 300)),
              "T": rounded(rng.uniform(270.0, 330.0)), "mflux": rounded(rng.uniform(1, 300))}
    values["pt"], values["Tt"] = rounded(1.3 * values["p"]), rounded(1.1 * values["T"])
    if tables is not None:
        from peregrine_b200.mixture import Mixture

        names = Mixture(cfg["mixture"]).spnames
        ns = len(names)
    else:
        names = list(cfg["mixture"]["species"])
    if ns > 1:
        Y = rng.uniform(0.2, 1.0, ns)
        values.update(zip(names[:-1], map(rounded, Y[:-1] / Y.sum())))
    values.update(entry or {})
    cfg["bcvals"]["outer"] = values
    return cfg.validate()


def bc_box_mesh(cells=(7, 5, 3), jostle=0.1, bcnames=None, defaultbc="outer", periodic=(False, False, False),
                lengths=(1.0, 1.0, 1.0)):
    return CubeMesher(cells=[[c] for c in cells], lengths=list(lengths), periodic=list(periodic),
                      bcnames=bcnames, defaultbc=defaultbc, jostle=jostle)


def bc_box_prims(metrics, ns, seed=0, speed=200.0):
    rng = np.random.default_rng(seed + 1)
    ph = rng.uniform(0.0, 2 * np.pi, 6)
    out = []
    for m in metrics:
        x, y, z = (m["xcc"][..., d] for d in range(3))
        smooth = np.cos(2.0 * x + ph[0]) * np.cos(1.5 * y + ph[1]) * np.cos(z + ph[2])
        q = np.zeros(x.shape + (4 + ns,))
        q[..., 0] = P0 * (1.0 + 0.3 * smooth)
        q[..., 1:4] = rng.uniform(-speed, speed, x.shape + (3,))
        q[..., 4] = 1000.0 * (1.0 + 0.3 * np.cos(x + ph[3]) * np.cos(2.0 * z + ph[4]))
        for n in range(ns - 1):
            q[..., 5 + n] = 0.9 / (ns - 1) * (0.5 + 0.4 * np.cos((n + 1) * x + y + ph[5]) ** 2)
        out.append(q)
    return out


# the bounded channel: a box of air and a second gas between a still
# isothermal wall and a moving lid, periodic across, a velocity inflow whose
# profile and temperature move with position and time, and a pressure exit;
# Navier-Stokes with MUSCL-koren and HLLC, TVD-RK3 under the cfl controller
CHANNEL_CELLS = (192, 96, 96)
CHANNEL_BLOCKS = (2, 2, 2)
CHANNEL_LENGTHS = (0.04, 0.02, 0.02)


def channel_config(launch="per-block", cfl=0.8):
    cfg = Config()
    cfg["simulation"]["simulator"] = "navier-stokes"
    cfg["simulation"]["controller"] = "cfl"
    cfg["simulation"]["cfl"] = cfl
    cfg["simulation"]["dt-max"] = 1e-5
    cfg["mixture"]["species"] = {k: MIXED[k] for k in ("A", "B")}
    cfg["mixture"]["trans"] = "constant"
    cfg["time-integration"]["integrator"] = "tvd-rk3"
    cfg["adv-flux"]["primary"] = "hllc"
    cfg["adv-flux"]["recon"] = "muscl"
    cfg["adv-flux"]["limiter"] = "koren"
    cfg["backend-b200"]["launch"] = launch
    cfg["ics"].update(p=P0, u=30.0, T=T0, Y={"A": 0.5})
    h = CHANNEL_LENGTHS[1]
    cfg["bcvals"]["inflow"] = {"kind": "sub-in-fvt", "u": f"60.0 * (y / {h}) * (1.0 - y / {h}) * 4.0 + 5.0 * sin(2000.0 * t)",
                               "v": 0.0, "w": "2.0 * sin(300.0 * z)", "T": "300.0 + 20.0 * cos(300.0 * z)", "A": 0.6}
    cfg["bcvals"]["exit"] = {"kind": "sub-out-fp", "p": P0}
    cfg["bcvals"]["floor"] = {"kind": "no-slp-isot-wall", "T": 320.0}
    cfg["bcvals"]["lid"] = {"kind": "mov-adia-wall", "u": 20.0, "v": 0.0, "w": 0.0}
    return cfg.validate()


def channel_mesh(cells=CHANNEL_CELLS, blocks=CHANNEL_BLOCKS):
    cuts = [[n // b + (1 if m < n - (n // b) * b else 0) for m in range(b)] for n, b in zip(cells, blocks)]
    return CubeMesher(mbdims=list(blocks), cells=cuts, lengths=list(CHANNEL_LENGTHS), periodic=[False, False, True],
                      bcnames={1: "inflow", 2: "exit", 3: "floor", 4: "lid"})
