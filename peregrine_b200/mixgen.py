"""The mixture's constant tables, worked out here from a Cantera-format
mechanism file (and a species library for what a mechanism leaves out),
with no reference checkout: the thermally perfect gas's cp, h and s in ln T,
the kinetic theory's mu and kappa fits, Wilke's and Herning's pair
constants, Lewis numbers or the binary diffusion's pair fits, the cubic real
gas's constants and the finite-rate reaction columns, third-body sets and
Troe fits.

Each table is the reference's, made by the same floating-point operations in
the same order, so the kernels read the doubles the reference writes into its
rendered kernels (tests/test_mixgen_cpu.py regenerates every table set under
peregrine_b200/data and compares it key by key):

* mechanism reading: peregrine/simulator/mixture/parser/base.py:22-263,
  parser/cantera.py, parser/units.py (units to SI, the Arrhenius A scaled by
  the reaction's order, falloff colliders and explicit third bodies);
* species data and the library's supplement: simulator/mixture/species.py;
* thermally perfect caloric model: caloric/tdepcp/model.py (cp/R sampled off
  the NASA-7 or JANAF data, padded to the T-range, fitted in ln T at the
  lowest degree whose relative error meets the tolerance, polyfit.py), and
  the eos tables, eos/base.py:33-62;
* kinetic theory: transport/kinetic.py, on the Stockmayer collision integrals
  of transport/integrals.py (natural cubic splines in ln T*, a quadratic in
  delta*), whose table ships as peregrine_b200/data/collision_integrals.npz;
* mixing rules and diffusion: mixrule/wilke.py, mixrule/herning.py,
  diffusion/lewis.py, diffusion/binary.py;
* cubic real gas: eos/realgas/model.py (Soave-Redlich-Kwong, or
  Peng-Robinson's constants);
* finite-rate chemistry: chemistry/finiterate.py and reaction.py.

Physical constants are CODATA's (exact where SI defines them); atomic weights
are the IUPAC standard values Cantera uses.
"""

import math
import os
import re
from types import SimpleNamespace

import numpy as np
from numpy.polynomial import chebyshev

# J/kmol/K, J/K, 1/kmol, F/m, m/s
RU = 8314.46261815324
KB = 1.380649e-23
AVOGADRO = 6.02214076e26
EPS0 = 8.854187812773345e-12
CLIGHT = 299792458.0
# C m (Cantera's debye)
DEBYE = 1.0e-21 / CLIGHT
TREF = 298.15

# kg/kmol
ATOMIC_WEIGHTS = {
    "H": 1.008, "He": 4.002602, "Li": 6.94, "Be": 9.0121831, "B": 10.81, "C": 12.011, "N": 14.007,
    "O": 15.999, "F": 18.998403163, "Ne": 20.1797, "Na": 22.98976928, "Mg": 24.305, "Al": 26.9815384,
    "Si": 28.085, "P": 30.973761998, "S": 32.06, "Cl": 35.45, "Ar": 39.95, "K": 39.0983, "Ca": 40.078,
    "Sc": 44.955908, "Ti": 47.867, "V": 50.9415, "Cr": 51.9961, "Mn": 54.938043, "Fe": 55.845,
    "Co": 58.933194, "Ni": 58.6934, "Cu": 63.546, "Zn": 65.38, "Ga": 69.723, "Ge": 72.630,
    "As": 74.921595, "Se": 78.971, "Br": 79.904, "Kr": 83.798,
}
# the rotational degrees of freedom over two, by shape
ROTDOF = {"atom": 0.0, "linear": 1.0, "nonlinear": 1.5}

# units to SI: energy per kmol, length, amount, and a species' transport data
ENERGY = {"cal/mol": 4184.0, "kcal/mol": 4.184e6, "J/mol": 1.0e3, "kJ/mol": 1.0e6, "J/kmol": 1.0, "K": RU}
LENGTH = {"cm": 1.0e-2, "m": 1.0, "angstrom": 1.0e-10}
QUANTITY = {"mol": 1.0e-3, "kmol": 1.0, "molec": 1.0 / AVOGADRO}
TRANSPORT = {"well-depth": ("well", KB), "diameter": ("diam", 1.0e-10), "dipole": ("dipole", DEBYE),
             "polarizability": ("polarize", 1.0e-30)}
# a Cantera file with no units section is SI
SI_UNITS = {"length": "m", "quantity": "kmol", "activation-energy": "J/kmol"}

# cubic forms: p = Ru T / (v - b) - a / (v^2 + u b v + w b^2)
CUBICS = {
    "srk": dict(u=1.0, w=0.0, omega_a=0.4274802, omega_b=0.0866403, m=(0.480, 1.574, -0.176)),
    "pr": dict(u=2.0, w=-1.0, omega_a=0.45724, omega_b=0.07780, m=(0.37464, 1.54226, -0.26992)),
}
CRITICAL = ("Tcrit", "pcrit", "Vcrit", "acentric")
KINDS = {"elementary": 0, "three-body": 1, "lindemann": 2, "troe": 3}

LOG10E = 0.4342944819032518
LN10 = 2.302585092994046
EXPBOUND = 680.0

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


# -- the mechanism file ------------------------------------------------------


def _load_yaml(path):
    import yaml

    # YAML 1.1 reads NO, YES, ON, OFF as booleans: species NO must stay a name
    class Loader(yaml.SafeLoader):
        pass

    Loader.yaml_implicit_resolvers = {
        k: [(tag, rx) for tag, rx in v if tag != "tag:yaml.org,2002:bool"]
        for k, v in yaml.SafeLoader.yaml_implicit_resolvers.items()
    }
    with open(path) as f:
        return yaml.load(f, Loader=Loader)


def _molwt(comp, weights):
    return sum(weights[e] * n for e, n in comp.items())


def _molar(text):
    value, unit = str(text).split()
    return float(value) / QUANTITY[unit.split("/")[1]]


def _species_entry(raw, weights):
    sp = {}
    if "composition" in raw:
        sp["comp"] = {k: float(v) for k, v in raw["composition"].items()}
        sp["MW"] = _molwt(sp["comp"], weights)
    thermo = raw.get("thermo")
    if thermo and thermo["model"] == "constant-cp":
        cp0 = _molar(thermo["cp0"])
        sp["cp0"] = cp0 / sp["MW"]
        T0 = float(str(thermo.get("T0", "298.15 K")).split()[0])
        h0 = _molar(thermo["h0"]) if "h0" in thermo else 0.0
        sp["dHf298"] = h0 + cp0 * (TREF - T0)
    elif thermo:
        if thermo["model"].upper() != "NASA7":
            raise ValueError(f"{raw['name']}: thermo model {thermo['model']} (NASA7 or constant-cp)")
        ranges = [float(r) for r in thermo["temperature-ranges"]]
        data = [list(map(float, c)) for c in thermo["data"]]
        low, high = (data[0], data[0]) if len(data) == 1 else data[:2]
        mid = ranges[1] if len(data) > 1 else ranges[-1]
        sp["NASA7"] = {"T-range": [ranges[0], mid, ranges[-1]], "high": high, "low": low}
    if "transport" in raw:
        tr = raw["transport"]
        sp["geometry"] = tr["geometry"]
        for key, (ours, unit) in TRANSPORT.items():
            sp[ours] = float(tr.get(key, 0.0)) * unit
        sp["zrot"] = float(tr.get("rotational-relaxation", 0.0))
        if "acentric-factor" in tr:
            sp["acentric"] = float(tr["acentric-factor"])
    return sp


def _side(text):
    out, third = {}, False
    text = re.sub(r"\(\s*\+[^)]+\)", "", text).strip()
    for term in text.split("+"):
        term = term.strip()
        if not term:
            continue
        if term == "M":
            if third:
                raise ValueError("more than one generic third body M on a side")
            third = True
            continue
        m = re.match(r"^(\d+\.?\d*)\s+(.+)$", term)
        nu, name = (float(m.group(1)), m.group(2).strip()) if m else (1.0, term)
        out[name] = out.get(name, 0.0) + nu
    return out, third


def _arrhenius(sect, order, units):
    e, l, q = ENERGY[units["activation-energy"]], LENGTH[units["length"]], QUANTITY[units["quantity"]]
    return float(sect["A"]) * (l**3 / q) ** (order - 1), float(sect["b"]), float(sect["Ea"]) * e / RU


def _flag(raw, key):
    v = raw.get(key, False)
    return v.strip().lower() in ("true", "yes", "on") if isinstance(v, str) else bool(v)


def _reaction(raw, units):
    eq = raw["equation"].split("#")[0].strip()
    colliders = {c.strip() for c in re.findall(r"\(\s*\+([^)]+)\)", eq)}
    if len(colliders) > 1:
        raise ValueError(f"inconsistent falloff colliders in {eq!r}")
    collider = colliders.pop() if colliders else None
    if "<=>" in eq:
        lhs, rhs = eq.split("<=>")
        reversible = True
    elif "=>" in eq:
        lhs, rhs = eq.split("=>")
        reversible = False
    else:
        raise ValueError(f"no arrow in {eq!r}")
    reactants, lm = _side(lhs)
    products, rm = _side(rhs)
    if lm != rm:
        raise ValueError(f"a third body M on one side of {eq!r}")
    kind = {"Arrhenius": "elementary", "three-body-Arrhenius": "three-body", "Lindemann": "falloff",
            "Troe": "falloff"}.get(raw.get("type"), raw.get("type"))
    effs = {k: float(v) for k, v in raw.get("efficiencies", {}).items()}
    defeff = float(raw.get("default-efficiency", 1.0))
    troe = "Troe" in raw
    if kind == "falloff":
        rtype = "troe" if troe else "lindemann"
        if collider is None:
            raise ValueError(f"a falloff reaction without its (+M) collider: {eq!r}")
        if collider != "M":
            if "default-efficiency" in raw and defeff != 0.0:
                raise ValueError(f"a default efficiency beside an explicit collider: {eq!r}")
            if effs and (len(effs) != 1 or collider not in effs):
                raise ValueError(f"third-body colliders that disagree: {eq!r}")
            defeff = 0.0
            effs = effs or {collider: 1.0}
    elif kind == "three-body" or (kind is None and lm):
        rtype = "three-body"
        if collider is not None:
            raise ValueError(f"a (+{collider}) collider on a reaction not typed falloff: {eq!r}")
        if not lm:
            if len(effs) != 1:
                raise ValueError(f"an explicit third body needs its one efficiency: {eq!r}")
            (sp,) = effs
            for side in (reactants, products):
                if side.get(sp, 0) < 1:
                    raise ValueError(f"the third body {sp} on both sides: {eq!r}")
                if side[sp] == 1:
                    del side[sp]
                else:
                    side[sp] -= 1
            defeff = 0.0
    elif kind in (None, "elementary"):
        rtype = "elementary"
        if lm or collider is not None:
            raise ValueError(f"an elementary reaction with a third body: {eq!r}")
        if "efficiencies" in raw or "default-efficiency" in raw:
            raise ValueError(f"efficiencies on a reaction with no third body: {eq!r}")
    else:
        raise ValueError(f"reaction type {kind!r} in {eq!r}")
    orders = {sp: float(v) for sp, v in raw.get("orders", {}).items()}
    if orders:
        if reversible:
            raise ValueError(f"orders on a reversible reaction: {eq!r}")
        if any(sp not in reactants for sp in orders) and not _flag(raw, "nonreactant-orders"):
            raise ValueError(f"an order for a species that is not a reactant: {eq!r}")
        if any(v < 0 for v in orders.values()) and not _flag(raw, "negative-orders"):
            raise ValueError(f"a negative order: {eq!r}")
    fwd = dict(reactants)
    fwd.update(orders)
    bodyorder = 1 if rtype == "three-body" else 0
    order = sum(fwd.values()) + bodyorder
    rxn = dict(equation=eq, type=rtype, reversible=reversible, reactants=reactants, products=products, fwd=fwd,
               efficiencies=effs, defeff=defeff)
    if rtype in ("lindemann", "troe"):
        rxn["rate"] = _arrhenius(raw["high-P-rate-constant"], order, units)
        rxn["lowrate"] = _arrhenius(raw["low-P-rate-constant"], order + 1, units)
    else:
        rxn["rate"] = _arrhenius(raw["rate-constant"], order, units)
    if troe:
        t = {"T2": 0.0, **raw["Troe"]}
        rxn["troe"] = [float(t[k]) for k in ("A", "T3", "T1", "T2")]
    return rxn


def read_mechanism(path, species=None):
    """A Cantera-format mechanism's species (name -> data, SI) and reactions,
    species the phase's list unless given."""
    data = _load_yaml(path)
    if species is None:
        if "phases" not in data:
            raise ValueError(f"{path} has no phases: name the species")
        species = list(data["phases"][0]["species"])
    lookup = {sp["name"]: sp for sp in data.get("species", [])}
    weights = dict(ATOMIC_WEIGHTS)
    for el in data.get("elements", []):
        weights[el["symbol"]] = float(el["atomic-weight"])
    out = {}
    for name in species:
        if name not in lookup:
            raise KeyError(f"species {name!r} is not in {path}")
        out[name] = _species_entry(lookup[name], weights)
    reactions = []
    units = {**SI_UNITS, **data.get("units", {})}
    for raw in data.get("reactions") or []:
        r = _reaction(raw, units)
        unknown = (set(r["reactants"]) | set(r["products"]) | set(r["efficiencies"])) - set(out)
        if unknown:
            raise KeyError(f"{r['equation']!r} names species outside the phase: {sorted(unknown)}")
        reactions.append(r)
    return out, reactions


def supplement(species, library):
    """Each species' missing data from the library by name, as the reference
    builds its species: a species that has one of the thermo data forms takes
    none of the library's."""
    thermo = ("janaf", "NASA7")
    out = {}
    for name, data in species.items():
        sp = {k: v for k, v in data.items() if v is not None}
        known = (library or {}).get(name) or {}
        has_thermo = any(k in sp for k in thermo)
        for k, v in known.items():
            if v is None or (has_thermo and k in thermo):
                continue
            sp.setdefault(k, v)
        if "MW" not in sp and "comp" in sp:
            sp["MW"] = _molwt(sp["comp"], ATOMIC_WEIGHTS)
        out[name] = sp
    return out


# -- fits in ln T ------------------------------------------------------------


def fit(x, y, tol, maxdeg):
    """Coefficients rising in the power, at the lowest degree whose relative
    error reaches tol (weights 1/y^2), and that error."""
    w = 1.0 / y**2
    for degree in range(maxdeg + 1):
        c = np.polyfit(x, y, degree, w=w)
        err = np.abs(np.polyval(c, x) / y - 1).max()
        if err <= tol:
            break
    return np.flip(c), err


def evaluate(poly, x):
    return np.polyval(np.flip(poly), x)


def expintegral(P):
    """Q with the integral of P(u) e^u du equal to e^u Q(u) (u = ln T), by
    parts: Q = P - P' + P'' - ..."""
    Q = np.zeros(len(P))
    D = np.flip(P)
    for k in range(len(P)):
        Q[: len(D)] += (-1) ** k * np.flip(D)
        D = np.polyder(D)
    return Q


def integral(P):
    return np.flip(np.polyint(np.flip(P)))


def padded(rows, dtype=np.float64):
    """Rows zero-padded to the longest."""
    n = max((len(r) for r in rows), default=1)
    a = np.zeros((len(rows), max(n, 1)), dtype=dtype)
    for k, r in enumerate(rows):
        a[k, : len(r)] = r
    return a


def _nasa_coeffs(n7, T):
    return n7["low"] if T <= n7["T-range"][1] else n7["high"]


def _nasa_cpR(n7, T):
    a = _nasa_coeffs(n7, T)
    return a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4])))


def _nasa_hRT(n7, T):
    a = _nasa_coeffs(n7, T)
    poly = T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5)))
    return a[0] + poly + a[5] / T


def _nasa_sR(n7, T):
    a = _nasa_coeffs(n7, T)
    poly = T * (a[1] + T * (a[2] / 2 + T * (a[3] / 3 + T * a[4] / 4)))
    return a[0] * np.log(T) + poly + a[6]


def _cp_source(sp):
    """The species' cp/R samples and (h298/R, s298/R), JANAF first."""
    if "janaf" in sp:
        j = sp["janaf"]
        return np.array(j["T"], float), np.array(j["cp"], float) / RU, (j["dHf298"] / RU, j["s298"] / RU)
    n7 = sp["NASA7"]
    T = np.linspace(n7["T-range"][0], n7["T-range"][-1], 200)
    return T, np.array([_nasa_cpR(n7, t) for t in T]), (_nasa_hRT(n7, TREF) * TREF, _nasa_sR(n7, TREF))


def _sample(sp, trange):
    lo, hi = trange
    T, cpR, _ = _cp_source(sp)
    if lo < T[0]:
        # down to 0 K: translation, and rotation where the shape is known
        frozen = 2.5 + ROTDOF[sp["geometry"]] if "geometry" in sp else cpR[0]
        dT = T[1] - T[0]
        Tx = np.arange(T[0] - dT, lo, -dT)
        if Tx.size == 0 or Tx[-1] > lo:
            Tx = np.append(Tx, lo)
        Tx = Tx[::-1]
        ramp = frozen + (cpR[0] - frozen) * Tx / T[0]
        T, cpR = np.concatenate([Tx, T]), np.concatenate([ramp, cpR])
    if hi > T[-1]:
        dT = T[-1] - T[-2]
        Tx = np.arange(T[-1] + dT, hi, dT)
        if Tx.size == 0 or Tx[-1] < hi:
            Tx = np.append(Tx, hi)
        T, cpR = np.concatenate([T, Tx]), np.concatenate([cpR, np.full_like(Tx, cpR[-1])])
    inside = (T >= lo) & (T <= hi)
    return T[inside], cpR[inside]


def _caloric(species, opts):
    """cppoly, hpoly, h298, spoly per species, stored on each in that order."""
    cpg = opts["eos"] == "cpg"
    for sp in species.values():
        if cpg:
            c = sp["cp0"] * sp["MW"] / RU
            sp["cppoly"] = [c]
            sp["hpoly"] = sp["cppoly"]
        else:
            T, cpR = _sample(sp, opts["T-range"])
            sp["cppoly"] = fit(np.log(T), cpR, opts["refit-tol"], opts["refit-max-deg"])[0]
            sp["hpoly"] = expintegral(sp["cppoly"])
    for sp in species.values():
        if cpg:
            sp["h298"] = sp.get("dHf298", 0.0) / RU - TREF * sp["cppoly"][0]
        else:
            h298R, _ = _cp_source(sp)[2]
            sp["h298"] = h298R - TREF * evaluate(sp["hpoly"], np.log(TREF))
    for sp in species.values():
        if cpg:
            c = sp["cppoly"][0]
            sp["spoly"] = [sp.get("s298", 0.0) / RU - c * np.log(TREF), c]
        else:
            _, srefR = _cp_source(sp)[2]
            S = integral(sp["cppoly"])
            S[0] = srefR - evaluate(S, np.log(TREF))
            sp["spoly"] = S


def _collect(species, key):
    v = [sp[key] for sp in species.values()]
    return v if isinstance(v[0], str) else np.array(v, float)


def gpoly(species):
    """g / (Ru T) less h298 / T: the enthalpy's polynomial in ln T less the entropy's."""
    h, s = padded([sp["hpoly"] for sp in species.values()]), padded([sp["spoly"] for sp in species.values()])
    g = np.zeros((len(species), max(h.shape[1], s.shape[1])))
    g[:, : h.shape[1]] += h
    g[:, : s.shape[1]] -= s
    return g


def gibbs(species, T):
    """g / (Ru T) of every species at the temperatures T."""
    u = np.log(T)
    Tinv = 1.0 / np.asarray(T, dtype=np.float64)
    g, h298 = gpoly(species), _collect(species, "h298")
    return np.array([np.polyval(np.flip(row), u) + h * Tinv for row, h in zip(g, h298)])


# -- kinetic theory ----------------------------------------------------------


class CollisionIntegrals:
    """Omega(2,2)* and A* of the Stockmayer potential off Monchick and Mason's
    table: a natural cubic spline in ln T* down each delta* column, then the
    quadratic through the three columns about delta*."""

    def __init__(self, path=None):
        with np.load(path or os.path.join(DATA, "collision_integrals.npz")) as z:
            self.delta = np.array(z["delta"])
            self._omega22 = self._splines(z["tstar22"], z["omega22"])
            self._astar = self._splines(z["tstar"], z["astar"])

    @staticmethod
    def _splines(tstar, table):
        keep = np.array(tstar, dtype=np.float64) > 0.0
        x = np.log(np.array(tstar, dtype=np.float64)[keep])
        y = np.array(table, dtype=np.float64)[keep]
        n = len(x)
        h = np.diff(x)
        A = np.zeros((n, n))
        rhs = np.zeros((n, y.shape[1]))
        A[0, 0] = A[-1, -1] = 1.0
        for i in range(1, n - 1):
            h0, h1 = h[i - 1], h[i]
            A[i, i - 1], A[i, i], A[i, i + 1] = h0, 2.0 * (h0 + h1), h1
            rhs[i] = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0)
        return x, y, np.linalg.solve(A, rhs)

    @staticmethod
    def _spline(col, x, cols):
        knots, y, m = col
        i = np.clip(np.searchsorted(knots, x) - 1, 0, len(knots) - 2)
        h = knots[i + 1] - knots[i]
        a, b = (knots[i + 1] - x) / h, (x - knots[i]) / h
        cubic = (a**3 - a) * m[i, cols] + (b**3 - b) * m[i + 1, cols]
        return a * y[i, cols] + b * y[i + 1, cols] + cubic * h**2 / 6.0

    def _at(self, col, tstar, delta):
        x = np.log(np.asarray(tstar, dtype=np.float64))
        delta = np.asarray(delta, dtype=np.float64)
        d = self.delta
        j = np.clip(np.searchsorted(d, delta) - 1, 0, len(d) - 3)
        d0, d1, d2 = d[j], d[j + 1], d[j + 2]
        f0, f1, f2 = (self._spline(col, x, j + k) for k in range(3))
        t0 = f0 * (delta - d1) * (delta - d2) / ((d0 - d1) * (d0 - d2))
        t1 = f1 * (delta - d0) * (delta - d2) / ((d1 - d0) * (d1 - d2))
        t2 = f2 * (delta - d0) * (delta - d1) / ((d2 - d0) * (d2 - d1))
        return t0 + t1 + t2

    def omega22(self, tstar, delta):
        return self._at(self._omega22, tstar, delta)

    def astar(self, tstar, delta):
        return self._at(self._astar, tstar, delta)


def _ljparams(species, opts):
    """Every pair's reduced mass, diameter, well and dipole, a polar-nonpolar
    pair's well deepened and diameter shrunk by induction."""
    Ts = np.linspace(*opts["T-range"], 50)
    MW, well, diam = _collect(species, "MW"), _collect(species, "well"), _collect(species, "diam")
    dipole, polarize = _collect(species, "dipole"), _collect(species, "polarize")
    rotdof = np.array([ROTDOF[g] for g in _collect(species, "geometry")])
    mass = MW / AVOGADRO
    rmass = np.outer(mass, mass) / np.add.outer(mass, mass)
    rdiam = 0.5 * np.add.outer(diam, diam)
    rwell = np.sqrt(np.outer(well, well))
    rdipole = np.sqrt(np.outer(dipole, dipole))
    rdelta = 0.5 * rdipole**2 / (4 * np.pi * EPS0 * rwell * rdiam**3)
    polar = dipole > 0.0
    mixed = polar[:, None] != polar[None, :]
    idx = np.arange(len(MW))
    ip = np.where(polar[:, None], idx[:, None], idx[None, :])
    inp = np.where(polar[:, None], idx[None, :], idx[:, None])
    dipolep, wellp, diamp = dipole[ip], well[ip], diam[ip]
    welln = well[inp]
    alphastar = polarize[inp] / diam[inp] ** 3
    dipolestar = dipolep / np.sqrt(4 * np.pi * EPS0 * diamp**3 * wellp)
    xi = 1.0 + 0.25 * alphastar * dipolestar**2 * np.sqrt(wellp / welln)
    rwell = np.where(mixed, rwell * xi**2, rwell)
    rdiam = np.where(mixed, rdiam * xi ** (-1 / 6), rdiam)
    return dict(Ts=Ts, ci=CollisionIntegrals(), MW=MW, well=well, diam=diam, mass=mass,
                zrot=_collect(species, "zrot"), rotdof=rotdof, rmass=rmass, rdiam=rdiam, rwell=rwell, rdelta=rdelta)


def _mupoly(species, opts):
    m = _ljparams(species, opts)
    Ts, well, diam, mass = m["Ts"], m["well"], m["diam"], m["mass"]
    Tstar = np.outer(Ts, KB / well)
    delta = np.broadcast_to(m["rdelta"].diagonal(), Tstar.shape)
    xsec = np.pi * diam**2 * m["ci"].omega22(Tstar, delta)
    visc = (5.0 / 16.0) * np.sqrt(np.pi * mass * KB * Ts[:, None]) / xsec
    # the fit is of sqrt(mu) / T^(1/4)
    visc = np.sqrt(visc / np.sqrt(Ts)[:, None])
    return [fit(np.log(Ts), v, opts["refit-tol"], opts["refit-max-deg"])[0] for v in visc.T]


def _kappapoly(species, opts):
    m = _ljparams(species, opts)
    Ts, well, diam, MW = m["Ts"], m["well"], m["diam"], m["MW"]
    zrot, rotdof, rmass = m["zrot"], m["rotdof"], m["rmass"].diagonal()
    lnT = np.log(Ts)
    sps = species.values()
    visc = np.array([evaluate(sp["mupoly"], lnT) for sp in sps]).T
    visc = visc**2 * np.sqrt(Ts)[:, None]
    cpR = np.array([evaluate(sp["cppoly"], lnT) for sp in sps]).T
    T = Ts[:, None]
    Tstar = np.outer(Ts, KB / well)
    delta = np.broadcast_to(m["rdelta"].diagonal(), Tstar.shape)
    omega22 = m["ci"].omega22(Tstar, delta)
    omega11 = omega22 / m["ci"].astar(Tstar, delta)
    kT = KB * T
    xsec = np.pi * diam**2 * omega11
    Dself = (3.0 / 16.0) * np.sqrt(2.0 * np.pi / rmass) * kT**1.5 / xsec

    # Parker's rotational relaxation at T* over its value at 298.15 K
    def fz(t):
        return 1.0 + np.pi**1.5 / np.sqrt(t) * (0.5 + 1.0 / t) + (0.25 * np.pi**2 + 2) / t

    fint = MW / (RU * T) * Dself / visc
    A = 2.5 - fint
    zrotT = zrot * fz(KB * TREF / well) / fz(Tstar)
    B = zrotT + 2.0 / np.pi * (5 / 3 * rotdof + fint)
    c1 = 2.0 / np.pi * A / B
    cvint = cpR - 2.5 - rotdof
    frot = fint * (1.0 + c1)
    ftrans = 2.5 * (1.0 - c1 * rotdof / 1.5)
    cond = visc / MW * RU * (ftrans * 1.5 + frot * rotdof + fint * cvint)
    # the fit is of kappa / sqrt(T)
    cond = cond / np.sqrt(Ts)[:, None]
    return [fit(lnT, c, opts["refit-tol"], opts["refit-max-deg"])[0] for c in cond.T]


def _binary(species, opts):
    """The binary diffusion's pair fits of T^1.5 / D at unit pressure, and the
    kernel's layout of them."""
    m = _ljparams(species, opts)
    Ts, rmass, rwell, rdiam = m["Ts"], m["rmass"], m["rwell"], m["rdiam"]
    ns = len(rmass)
    k, j = np.triu_indices(ns)
    Tstar = np.outer(Ts, KB / rwell[k, j])
    delta = np.broadcast_to(m["rdelta"][k, j], Tstar.shape)
    omega11 = m["ci"].omega22(Tstar, delta) / m["ci"].astar(Tstar, delta)
    kT = KB * Ts[:, None]
    xsec = np.pi * rdiam[k, j] ** 2 * omega11
    diff = 3.0 / 16.0 * np.sqrt(2.0 * np.pi / rmass[k, j]) * kT**1.5 / xsec
    diffinv = Ts[:, None] ** 1.5 / diff
    dijinv = padded([fit(np.log(Ts), d, opts["refit-tol"], opts["refit-max-deg"])[0] for d in diffinv.T])
    names = list(species)
    chosen = opts.get("bath")
    bath = np.array([names.index(n) for n in (names if chosen is None else chosen)], dtype=np.int32)
    slot = np.zeros((ns, ns), dtype=int)
    slot[np.triu_indices(ns)] = np.arange(ns * (ns + 1) // 2)
    slot = np.maximum(slot, slot.T)
    whole = len(bath) == ns
    rows = [[q for q in range(ns) if q != n] if whole else list(bath) for n in range(ns)]
    pairfit = np.zeros((ns * len(rows[0]), dijinv.shape[1]))
    for n, r in enumerate(rows):
        for kk, q in enumerate(r):
            if q != n:
                pairfit[n * len(r) + kk] = dijinv[slot[n, q]]
    return dict(dijinv=dijinv, bath=bath, pairfit=pairfit, selffit=dijinv[np.diag(slot)])


# -- the cubic real gas ------------------------------------------------------


def _critpoint(species):
    """The critical point, or, for a species without one, Chung's relations
    run backwards from its Lennard-Jones parameters with Pitzer's Zc at w = 0."""
    for sp in species.values():
        if any(k not in sp for k in CRITICAL):
            Tc = 1.2593 * sp["well"] / KB
            Vcmol = (sp["diam"] * 1e10 / 0.809) ** 3 * 1e-3
            got = {"Tcrit": Tc, "pcrit": 0.291 * RU * Tc / Vcmol, "Vcrit": Vcmol / sp["MW"], "acentric": 0.0}
        else:
            got = {k: sp[k] for k in CRITICAL}
        sp.update(got)


def _cubic_tables(species, cubic):
    c = CUBICS[cubic]
    sq = np.sqrt(c["u"] ** 2 - 4.0 * c["w"])
    out = {"cubicu": np.array(c["u"]), "cubicw": np.array(c["w"]), "cubicsigma": np.array(0.5 * (c["u"] + sq)),
           "cubiceps": np.array(0.5 * (c["u"] - sq)),
           "vshift": np.array([sp.get("vshift", 0.0) for sp in species.values()])}
    for key in CRITICAL:
        out[key] = _collect(species, key)
    Tc, pc, w = out["Tcrit"], out["pcrit"], out["acentric"]
    sqrtac = np.sqrt(c["omega_a"] / pc) * RU * Tc
    b = c["omega_b"] * RU * Tc / pc
    m = c["m"][0] + c["m"][1] * w + c["m"][2] * w**2
    invsqrtTc = Tc**-0.5
    out.update(cubicsqrtac=sqrtac, cubicb=b, cubicda=sqrtac * m * invsqrtTc, cubicmTc=m * invsqrtTc,
               cubiconepm=1.0 + m)
    MWinv = 1.0 / _collect(species, "MW")
    for key in ("cubicsqrtac", "cubicb", "vshift", "cubicda"):
        out[("vshiftMW" if key == "vshift" else key + "MW")] = out[key] * MWinv
    out.update(cubic_omega_a=np.array(c["omega_a"]), cubic_omega_b=np.array(c["omega_b"]), cubic_m=np.array(c["m"]))
    return out


# -- finite-rate chemistry ---------------------------------------------------


def lfc(fcent, T):
    """log10 of Troe's centre: a signed log-sum-exp about its largest term,
    Cantera's floor where there are no terms."""
    T = np.asarray(T, dtype=np.float64)
    if not fcent:
        return np.full(T.shape, np.log(np.finfo(np.float64).tiny) * LOG10E)
    e = np.array([c0 + cT * T + cTinv / T for _, c0, cT, cTinv in fcent])
    ref = e.max(axis=0)
    total = sum(sign * np.exp(em - ref) for (sign, *_), em in zip(fcent, e))
    return (ref + np.log(np.maximum(np.finfo(np.float64).tiny, total))) * LOG10E


def _lfcpoly(fcent, uc, uh, degree=12):
    """A Chebyshev least-squares fit of the centre in t = (ln T - uc) / uh,
    in the power basis, coefficients rising."""
    if not fcent:
        return []
    k = np.arange(8 * degree + 64)
    t = np.cos(np.pi * (k + 0.5) / k.size)
    coef = chebyshev.chebfit(t, lfc(fcent, np.exp(uc + uh * t)), degree)
    return [float(c) for c in chebyshev.cheb2poly(coef)]


def _fcent(troe):
    """Troe's centre as (sign, c0, cT, cTinv) terms of sign exp(c0 + cT T +
    cTinv / T); a term underflowing at every gas temperature is dropped, a
    coefficient below rounding zeroed."""
    if troe is None:
        return []
    alpha, T3, T1, T2 = troe
    tmin, tmax = 100.0, 20000.0
    cands = []
    if alpha != 1.0 and T3 != 0:
        cands.append((np.sign(1.0 - alpha), np.log(abs(1.0 - alpha)), -1.0 / T3, 0.0))
    if alpha != 0.0 and T1 != 0:
        cands.append((np.sign(alpha), np.log(abs(alpha)), -1.0 / T1, 0.0))
    if T2:
        cands.append((1.0, 0.0, 0.0, -T2))
    terms = []
    for sign, c0, cT, cTinv in cands:
        if cT * tmin < -745 or cTinv / tmax < -745:
            continue
        cT = 0.0 if abs(cT) * tmax < 1e-14 else cT
        cTinv = 0.0 if abs(cTinv) / tmin < 1e-14 else cTinv
        terms.append((sign, c0, cT, cTinv))
    return terms


# what each kind adds to ln k beyond its Arrhenius rate, concentrations at most e^logcmax
_BOOST = {"elementary": lambda l: 0.0, "three-body": lambda l: l + 2.0, "lindemann": lambda l: 1.0,
          "troe": lambda l: 1.0}


def _product_form(r, T, logT, Tinv, gRT, ns):
    """Whether the reaction's one-way rates go as products of concentrations
    and per-species exponentials: whole reactant orders equal to the
    stoichiometry, every exponential's argument inside the table exp's range
    over the case's temperatures."""
    whole = all(float(v).is_integer() and v > 0 for _, v in r.react + r.prod)
    if not whole or dict(r.fwd) != dict(r.react):
        return False
    sps = [sp for sp, _ in r.react + r.prod]
    if np.abs(gRT[sps]).max() >= EXPBOUND:
        return False
    xk = r.logA + r.b * logT - r.EaR * Tinv - sum(nu * gRT[sp] for sp, nu in r.react)
    low, high = xk.min(), xk.max()
    if r.troe:
        l10 = lfc(r.fcent, T)
        low, high = low + LN10 * min(l10.min(), 0.0), high + LN10 * max(l10.max(), 0.0)
    if r.falloff:
        xpr = r.logprA + r.prb * logT - r.prEaR * Tinv
        if np.abs(xpr).max() >= EXPBOUND - 8.0:
            return False
    if not (low > -EXPBOUND and high < EXPBOUND):
        return False
    logc = 12.0
    chain = xk + (logc + np.log(r.defeff * ns + sum(max(dev, 0.0) for _, dev in r.eff))
                  if r.thirdbody and not r.falloff else 0.0)
    for sp, nu in r.react:
        for _ in range(int(nu)):
            chain = chain + gRT[sp] + logc
            if chain.max() >= EXPBOUND:
                return False
    chain = xk + abs(r.nusum) * 6.0
    for sp, nu in r.prod:
        for _ in range(int(nu)):
            chain = chain + gRT[sp] + logc
            if chain.max() >= EXPBOUND:
                return False
    return True


def _records(species, reactions, trange):
    """Each reaction with a nonzero A as the kernel's record, and the scalars."""
    names = list(species)
    MW = np.array([species[n]["MW"] for n in names])
    index = {n: k for k, n in enumerate(names)}
    rxns = [r for r in reactions if r["rate"][0] != 0.0]
    for r in rxns:
        if r["rate"][0] < 0 or r.get("lowrate", (1.0,))[0] <= 0:
            raise ValueError(f"{r['equation']}: a rate is evaluated in log space, A is positive")
    uc = 0.5 * (np.log(trange[1]) + np.log(trange[0]))
    uh = 0.5 * (np.log(trange[1]) - np.log(trange[0]))
    records, nets, fwds = [], [], []
    for r in rxns:
        A, b, EaR = r["rate"]
        A0, b0, EaR0 = r.get("lowrate", (1.0, 0.0, 0.0))
        logA = np.log(A)
        nu = {}
        for sp, v in r["reactants"].items():
            nu[sp] = nu.get(sp, 0.0) - v
        for sp, v in r["products"].items():
            nu[sp] = nu.get(sp, 0.0) + v
        net = [(index[sp], v) for sp, v in nu.items() if v != 0]
        fwd = [(index[sp], v) for sp, v in r["fwd"].items() if v != 0]
        kind = r["type"]
        troe = kind == "troe"
        fc = _fcent(r.get("troe"))
        rec = SimpleNamespace(
            name=kind, thirdbody=kind != "elementary", falloff=kind in ("lindemann", "troe"), troe=troe,
            reversible=bool(r["reversible"]), troeidx=sum(1 for x in records if x.troe) if troe else None,
            logA=float(logA), b=float(b), EaR=float(EaR), logprA=float(np.log(A0) - logA), prb=float(b0 - b),
            prEaR=float(EaR0 - EaR), fcent=fc, lfcpoly=_lfcpoly(fc, uc, uh), fwd=fwd,
            react=[(index[sp], v) for sp, v in r["reactants"].items() if v != 0],
            prod=[(index[sp], v) for sp, v in r["products"].items() if v != 0],
            net=[(sp, v, float(v * MW[sp])) for sp, v in net],
            eff=[(index[sp], e - r["defeff"]) for sp, e in r["efficiencies"].items() if e != r["defeff"]],
            nusum=float(sum(v for _, v in net)), defeff=float(r["defeff"]))
        records.append(rec)
        nets.append(net)
        fwds.append(fwd)
    grid = np.geomspace(trange[0], trange[1], 2048)
    logT, Tinv, gRT = np.log(grid), 1.0 / grid, gibbs(species, grid)
    for rec in records:
        rec.product = _product_form(rec, grid, logT, Tinv, gRT, len(species))
    gain = np.zeros(len(species))
    for row in nets:
        for sp, v in row:
            gain[sp] += abs(v)
    maxgain = max(1.0, (gain * MW).max()) if records else 1.0
    logcfloor = _logcfloor(species, rxns, records, nets, fwds, index, trange)
    scalars = {"logprefRu": np.array(np.log(101325.0 / RU)), "prefRu": np.array(101325.0 / RU),
               "Rupref": np.array(RU / 101325.0), "logcfloor": np.array(logcfloor),
               "cfloor": np.array(math.exp(logcfloor)), "maxgain": np.array(maxgain), "troeuc": np.array(uc),
               "troeuhinv": np.array(1.0 / uh)}
    return records, scalars


def _logcfloor(species, rxns, records, nets, fwds, index, trange):
    """The log concentration floor: deep enough that every direction of every
    reaction an absent species joins stays below e^-45 at any state over the
    T-range, with ln c at most 12 for the other factors, and no shallower than
    the smallest normal float."""
    logcmax, margin = 12.0, 45.0
    T = np.geomspace(max(trange[0], 100.0), trange[1], 256)
    logT, gRT = np.log(T), gibbs(species, T)
    required = 90.0
    for r, rec, netrow, fwdrow in zip(rxns, records, nets, fwds):
        A, b, EaR = r["rate"]
        logkf = np.log(A) + b * logT - EaR / T
        aux = _BOOST[rec.name](logcmax)
        top = logkf.max() + aux
        for k, vk in fwdrow:
            if vk <= 0:
                continue
            other = sum(v * logcmax for n, v in fwdrow if n != k and v > 0)
            required = max(required, (top + other + margin) / vk)
        if r["reversible"]:
            affinity = sum(v * gRT[n] for n, v in netrow)
            nusum = sum(v for _, v in netrow)
            logkr = logkf + affinity + nusum * np.log(RU * T / 101325.0)
            rev = [(index[sp], float(v)) for sp, v in r["products"].items() if v > 0]
            top = logkr.max() + aux
            for k, vk in rev:
                other = sum(v * logcmax for n, v in rev if n != k)
                required = max(required, (top + other + margin) / vk)
    return -float(required)


def _thirdbody_sets(records):
    sets, keys = [], []
    for r in records:
        r.tb = None
        if r.thirdbody:
            key = (r.defeff, tuple(r.eff))
            if key not in keys:
                keys.append(key)
                sets.append(SimpleNamespace(defeff=r.defeff, eff=list(r.eff)))
            r.tb = keys.index(key)
    return sets


def _columns(records):
    col = {"nr": np.array(len(records)), "type": np.array([r.name for r in records]),
           "reversible": np.array([int(r.reversible) for r in records], np.int32),
           "nfcent": np.array([len(r.fcent) for r in records], np.int32)}
    for name in ("defeff", "logA", "b", "EaR", "logprA", "prb", "prEaR", "nusum"):
        col[name] = np.array([getattr(r, name) for r in records])
    for k, name in enumerate(("fcentsign", "fcentc0", "fcentcT", "fcentcTinv")):
        col[name] = padded([[t[k] for t in r.fcent] for r in records])
    col["lfcpoly"] = padded([r.lfcpoly for r in records])
    col["fwdsp"] = padded([[sp for sp, _ in r.fwd] for r in records], np.int32)
    col["fwdorder"] = padded([[v for _, v in r.fwd] for r in records])
    col["netsp"] = padded([[sp for sp, _, _ in r.net] for r in records], np.int32)
    col["netnu"] = padded([[nu for _, nu, _ in r.net] for r in records])
    col["netnuMW"] = padded([[m for _, _, m in r.net] for r in records])
    rev = []
    for r in records:
        order = {}
        for sp, v in (r.fwd + [(sp, nu) for sp, nu, _ in r.net]) if r.reversible else []:
            order[sp] = order.get(sp, 0.0) + v
        rev.append([(sp, v) for sp, v in order.items() if v != 0])
    col["revsp"] = padded([[sp for sp, _ in row] for row in rev], np.int32)
    col["revorder"] = padded([[v for _, v in row] for row in rev])
    col["product"] = np.array([int(r.product) for r in records], np.int32)
    col["reactsp"] = padded([[sp for sp, _ in r.react] for r in records], np.int32)
    col["reactnu"] = padded([[v for _, v in r.react] for r in records])
    col["prodsp"] = padded([[sp for sp, _ in r.prod] for r in records], np.int32)
    col["prodnu"] = padded([[v for _, v in r.prod] for r in records])
    col["effsp"] = padded([[sp for sp, _ in r.eff] for r in records], np.int32)
    col["effdev"] = padded([[v for _, v in r.eff] for r in records])
    return col


def _chemistry_tables(species, reactions, trange):
    if not reactions:
        raise ValueError("finite-rate chemistry needs reactions")
    out = {}
    # the constants' own columns
    records, scalars = _records(species, reactions, trange)
    col = _columns(records)
    sets = _thirdbody_sets(records)
    out.update(scalars)
    out.update(rxnlogA=col["logA"], rxnb=col["b"], rxnEaR=col["EaR"], rxnlogprA=col["logprA"], rxnprb=col["prb"],
               rxnprEaR=col["prEaR"], rxnnusum=col["nusum"],
               rxnlfcpoly=padded([r.lfcpoly for r in records if r.troe]), rxnfwdorder=col["fwdorder"],
               rxnnetnu=col["netnu"], rxnnetnuMW=col["netnuMW"], rxnreactnu=col["reactnu"],
               tbdefeff=np.array([t.defeff for t in sets]), tbeffdev=padded([[d for _, d in t.eff] for t in sets]))
    # the reaction columns as the kernels' mechanism struct reads them
    records, scalars = _records(species, reactions, trange)
    col = {**_columns(records), **scalars}
    for k, v in col.items():
        if k == "type":
            out["rxn_kind"] = np.array([KINDS[t] for t in v], dtype=np.int32)
        else:
            out["rxn_" + k] = np.asarray(v)
    records, _ = _records(species, reactions, trange)
    sets = _thirdbody_sets(records)
    out["rxn_tb"] = np.array([-1 if r.tb is None else r.tb for r in records], dtype=np.int32)
    out["rxn_troeidx"] = np.array([-1 if r.troeidx is None else r.troeidx for r in records], dtype=np.int32)
    out["tb_effsp"] = padded([[sp for sp, _ in t.eff] for t in sets], np.int32)
    out["tb_neff"] = np.array([len(t.eff) for t in sets], dtype=np.int32)
    out["chemistry"] = np.array("finite-rate")
    return out


# -- the whole set -----------------------------------------------------------


def make_tables(mechanism=None, species=None, library=None, eos="tpg", trans=None, diffusion="lewis",
                mixing_rule="wilke", chemistry=None, trange=(300.0, 3500.0), refit_tol=1e-3, refit_max_deg=6,
                bath=None, cubic="srk"):
    """Every table the kernels read, by the names peregrine_b200.mixture
    loads: from a Cantera-format mechanism file (its phase's species unless
    species names them), or from species alone (a list of names the library
    holds, or a dict of name to data), each supplemented from the library (a
    dict of name to data, or a YAML file of one)."""
    if isinstance(library, str):
        library = _load_yaml(library)
    reactions = []
    if mechanism is not None:
        sp, reactions = read_mechanism(mechanism, species)
    elif isinstance(species, dict):
        sp = {k: dict(v) for k, v in species.items()}
    else:
        sp = {name: {} for name in species}
    sp = supplement(sp, library)
    opts = {"eos": "cpg" if eos == "cpg" else eos, "T-range": tuple(trange), "refit-tol": refit_tol,
            "refit-max-deg": refit_max_deg, "bath": bath}
    realgas = eos in ("real-gas", "real-gas-df")
    if eos not in ("cpg", "tpg") and not realgas:
        raise ValueError(f"eos {eos!r}: cpg, tpg or real-gas")
    names = list(sp)
    for name, d in sp.items():
        if "MW" not in d:
            raise ValueError(f"species {name}: no MW or composition")
    _caloric(sp, opts)
    if realgas:
        _critpoint(sp)
    if trans == "kinetic-theory":
        if eos == "cpg":
            raise ValueError("the kinetic theory's conductivity needs the thermally perfect cp")
        for d, v in zip(sp.values(), _mupoly(sp, opts)):
            d["mupoly"] = v
        for d, v in zip(sp.values(), _kappapoly(sp, opts)):
            d["kappapoly"] = v
    elif trans not in (None, "constant"):
        raise ValueError(f"trans {trans!r}: kinetic-theory or constant")

    MW = _collect(sp, "MW")
    Rsp = RU / MW
    cppoly, hpoly = padded([d["cppoly"] for d in sp.values()]), padded([d["hpoly"] for d in sp.values()])
    h298, spoly = _collect(sp, "h298"), padded([d["spoly"] for d in sp.values()])
    out = dict(Ru=np.array(RU), MW=MW, MWinv=1.0 / MW, Rsp=Rsp, cppoly=cppoly, hpoly=hpoly, h298=h298,
               spoly=spoly, gpoly=gpoly(sp), cppolyR=cppoly * Rsp[:, None], hpolyR=hpoly * Rsp[:, None],
               h298R=h298 * Rsp)
    if eos == "cpg":
        out["cp0"] = _collect(sp, "cp0")
    if realgas:
        out.update(_cubic_tables(sp, cubic))
    if trans == "kinetic-theory":
        out.update(mupoly=padded([d["mupoly"] for d in sp.values()]),
                   kappapoly=padded([d["kappapoly"] for d in sp.values()]))
    elif trans == "constant":
        out.update(mu0=_collect(sp, "mu0"), kappa0=_collect(sp, "kappa0"))
    if trans is not None:
        if diffusion == "lewis":
            out["lewis"] = np.array([d.get("lewis", 1.0) for d in sp.values()])
        elif diffusion == "binary":
            out.update(_binary(sp, opts))
        else:
            raise ValueError(f"diffusion {diffusion!r}: lewis or binary")
        if mixing_rule == "wilke":
            out.update(MWqinv=MW**-0.25, wilkepair=1.0 / np.sqrt(8.0 * (1.0 + MW[:, None] / MW[None, :])))
        elif mixing_rule == "herning":
            out.update(sqrtMW=np.sqrt(MW))
        else:
            raise ValueError(f"mixing-rule {mixing_rule!r}: wilke or herning")
    if chemistry == "finite-rate":
        out.update(_chemistry_tables(sp, reactions, trange))
    elif chemistry is not None:
        raise ValueError(f"chemistry {chemistry!r}: finite-rate")
    out["spnames"] = np.array(names)
    out["eos"] = np.array(eos)
    out["trans"] = np.array(trans if trans is not None else "")
    out["ns"] = np.array(len(names))
    out["diffusion"] = np.array(diffusion if trans is not None else "lewis")
    return out
