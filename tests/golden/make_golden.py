"""Generates the golden fixtures of tests/golden from the reference itself.

    python tests/golden/make_golden.py REFERENCE [FIXTURE ...]

REFERENCE is the path of a checkout of the reference; with FIXTURE names
(the file names below without their extension) only those are rewritten.

Run here, where the reference's Python can be imported; the fixtures it
writes (*.npz, *.json) are committed, and nothing at test time reads the
reference.  The reference's package imports mako, mpi4py, h5py and lxml at
module level for its code generation, MPI and files; none of those run on the
paths used here, so stub modules stand in for them.

What it records, each from the reference's own code:
  faces_kepaec.npz   tests/simulator/oracle.py's cpg sides (cpg) and kepaec
                     flux on random faces, for air and a binary N2/O2 gas;
  metrics.npz        peregrine/multiblock/block/grid.py's cell centres, face
                     centres, area vectors, detJinv and Jinv of a jostled block;
  constants.npz      peregrine/simulator/mixture's constants for the
                     Taylor-Green air and a binary gas with constant transport;
  rk_tables.json     peregrine/integrators/rungekutta.py's combine kernels per
                     stage (registers, weights, dt placement) for every scheme;
  faces_riemann.npz  tests/simulator/oracle.py's hllc, rusanov and ausmup
                     fluxes on the two cells as they are, and on muscl's sides
                     under each of the five limiters, for four cells LL, L, R,
                     RR around random faces of the binary gas;
  mathfns.npz        peregrine/backend/base/mathfns.py's tables for the table
                     log and exp, and tests/mixture/rates.py's numpy twins of
                     the kernels' tlog and texp on sample arguments;
  rates_<mech>.npz   tests/mixture/rates.py's production rates (the kernels'
                     form) on random states of the 9-species H2/O2/N2 subset of
                     GRI-Mech 3.0 and of CH4_O2_FFCMY, with the reference's
                     Gibbs functions, and the species' cp and h by the
                     reference's own polynomial evaluation;
  rates_h2o2_gri30_oneway.npz  the same for the H2/O2/N2 subset with every
                     reaction irreversible (the reference's one-way twin,
                     tests/mixture/rates.py:195-202, as a mechanism file), where
                     no reverse rate cancels a forward one;

  binary_h2o2.npz    peregrine/simulator/mixture/diffusion/binary.py's pair
                     coefficients T^(3/2) / D at unit pressure for the
                     9-species H2/O2/N2 gas, at its fit's sample temperatures,
                     unfitted (the model's fit step replaced by the identity);

  realgas_<cubic>.npz tests/eos/support.py's textbook density of the cubic
                     (numpy's roots and the least Gibbs energy phase) for O2/H2
                     at random (p, T, Y), the reference's Soave-Redlich-Kwong
                     and, with its constants set on the numpy twin, Peng-Robinson.

The mixtures' constant tables themselves are written by
peregrine_b200/data/export_mixture.py from the same reference code.
"""

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = None


def stub(name, **attrs):
    m = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(m, k, v)
    sys.modules[name] = m
    return m


class _Any:
    def __init__(self, *a, **k):
        pass


class _Comm:
    rank, size = 0, 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def bcast(self, x, root=0):
        return x

    def Allreduce(self, *a, **k):
        pass

    def Barrier(self):
        pass


def install_stubs():
    if "cantera" not in sys.modules:
        stub("cantera", add_directory=lambda *a, **k: None)
    mako = stub("mako")
    mako.runtime = stub("mako.runtime", capture=lambda *a, **k: "", supports_caller=lambda f: f)
    mako.lookup = stub("mako.lookup", TemplateLookup=_Any)
    mako.template = stub("mako.template", Template=_Any)
    MPI = types.SimpleNamespace(COMM_WORLD=_Comm(), IN_PLACE=None, MAX=None, SUM=None, Prequest=_Any,
                                Request=_Any, Comm=_Comm)
    m4 = stub("mpi4py", MPI=MPI)
    stub("mpi4py.MPI", **vars(MPI))
    m4.util = stub("mpi4py.util")
    m4.util.dtlib = stub("mpi4py.util.dtlib", from_numpy_dtype=lambda d: d)
    h5 = stub("h5py", File=_Any)
    for s in ("h5fd", "h5p", "h5s"):
        setattr(h5, s, stub("h5py." + s))
    lx = stub("lxml")
    lx.etree = stub("lxml.etree")


def air_tgv():
    sys.path.insert(0, os.path.dirname(HERE))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from peregrine_b200.cases import tgv_gas

    return tgv_gas()[0]


BINARY = {"N2": {"MW": 28.0134, "cp0": 1040.0, "mu0": 1.8e-5, "kappa0": 0.026},
          "O2": {"MW": 31.9988, "cp0": 918.0, "mu0": 2.0e-5, "kappa0": 0.027, "lewis": 1.3}}


def faces(orc, gas, n, rng):
    ns = len(gas)

    def side():
        p = rng.uniform(5e4, 2e5, n)
        T = rng.uniform(200.0, 600.0, n)
        Y = rng.uniform(0.1, 0.9, (n, ns - 1))
        s = orc.cpg(gas, p, T, Y)
        u = rng.uniform(-100.0, 100.0, (n, 3))
        s["u"], s["v"], s["w"] = u[:, 0], u[:, 1], u[:, 2]
        s["Y"] = Y
        rho = s["rho"]
        Q = np.concatenate([rho[:, None], rho[:, None] * u,
                            (rho * (s["e"] + 0.5 * (u * u).sum(axis=1)))[:, None], rho[:, None] * Y], axis=1)
        return s, Q

    L, QL = side()
    R, QR = side()
    S = rng.uniform(-1.0, 1.0, (n, 3))
    F = orc.kepaec(L, R, S)
    return dict(QL=QL, QR=QR, S=S, F=F)


def faces4(orc, gas, n, rng):
    """Four cells around each face: a smooth profile plus noise, so the slope
    ratios take every sign and size the limiters distinguish; a quarter of the
    faces carry a supersonic stream along the normal each way, so HLLC's
    outer cases come up besides the two star cases."""
    ns = len(gas)
    S = rng.uniform(-1.0, 1.0, (n, 3))
    stream = rng.choice([0.0, 0.0, 900.0, -900.0], n)[:, None] * S / np.linalg.norm(S, axis=1, keepdims=True)
    base = dict(p=rng.uniform(5e4, 2e5, n), T=rng.uniform(200.0, 600.0, n), Y=rng.uniform(0.2, 0.8, (n, ns - 1)),
                u=rng.uniform(-200.0, 200.0, (n, 3)))
    slope = dict(p=rng.uniform(-2e4, 2e4, n), T=rng.uniform(-50.0, 50.0, n), Y=rng.uniform(-0.05, 0.05, (n, ns - 1)),
                 u=rng.uniform(-60.0, 60.0, (n, 3)))
    fields = ("p", "T", "rhoinv", "rho", "e", "cp", "gamma", "c")
    Q, state = [], []
    for o in (-2, -1, 0, 1):
        x = o + 0.5
        v = {k: base[k] + slope[k] * (x if base[k].ndim == 1 else x) for k in base}
        noise = dict(p=2e3, T=5.0, Y=0.01, u=8.0)
        v = {k: v[k] + rng.normal(0.0, noise[k], v[k].shape) for k in v}
        v["u"] = v["u"] + stream
        s = orc.cpg(gas, v["p"], v["T"], v["Y"])
        s["rhoinv"] = 1.0 / s["rho"]
        rho, u = s["rho"], v["u"]
        Q.append(np.concatenate([rho[:, None], rho[:, None] * u, (rho * (s["e"] + 0.5 * (u * u).sum(axis=1)))[:, None],
                                 rho[:, None] * v["Y"]], axis=1))
        state.append(np.stack([s[f] for f in fields], axis=-1))
    Q, state = np.stack(Q), np.stack(state)
    # the numpy oracle indexes its cells by offset from the face: -2, -1, 0, 1
    byoff = {o: Q[o + 2] for o in (-2, -1, 0, 1)}
    stbyoff = {o: state[o + 2] for o in (-2, -1, 0, 1)}
    out = dict(Q4=Q, S=S)
    for fn in ("hllc", "rusanov", "ausmup"):
        flux = orc.functions[fn]
        out[f"{fn}_constant"] = flux(orc.cell(Q[1], state[1]), orc.cell(Q[2], state[2]), S)
        for name, lim in orc.limiters.items():
            L, R = orc.muscl(gas, byoff, stbyoff, lim)
            out[f"{fn}_muscl_{name}"] = flux(L, R, S)
    return out


def mathfns():
    from peregrine.backend.base import mathfns as mf
    from tests.mixture import rates

    rng = np.random.default_rng(20261205)
    xl = np.concatenate([np.exp(rng.uniform(-700.0, 700.0, 4000)), rng.uniform(0.5, 2.0, 1000),
                         [1.0, 2.0, 0.5, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308]])
    xe = np.concatenate([rng.uniform(-745.0, 709.0, 4000), rng.uniform(-1.0, 1.0, 1000), [0.0, -708.4, 709.0]])
    return dict(LOGTAB=np.array(mf.LOGTAB), RCPTAB=np.array(mf.RCPTAB), EXPTAB=np.array(mf.EXPTAB),
                scalars=np.array([mf.LN2, mf.EXPK, mf.LN2BINS_HI, mf.LN2BINS_LO]), xlog=xl, tlog=rates.tlog(xl),
                xexp=xe, texp=rates.texp(xe))


def rates_of(reference, mech, keep, n, rng, oneway=False):
    from peregrine_b200.data.export_mixture import reference_mixture, subset
    from tests.mixture import rates
    import tempfile

    path = os.path.join(reference, "peregrine", "simulator", "mixture", "database", "mechanisms", mech)
    with tempfile.TemporaryDirectory() as tmp:
        if keep or oneway:
            path = subset(path, keep, tmp, oneway=oneway)
        mix = reference_mixture(reference, path, "tpg", "kinetic-theory", "finite-rate")
    ns = mix.ns
    rho, T, Y, omega, gRT = [], [], [], [], []
    for trial in range(n):
        y = rng.random(ns)
        if trial % 4 == 3:
            # trace and absent species: the log floor and the product form's zero concentrations
            y[rng.random(ns) < 0.4] = 0.0
            y[0] = max(y[0], 0.1)
        y = y / y.sum()
        p, t = rng.uniform(1e5, 30e5), rng.uniform(600.0, 2800.0)
        r = rates.density(mix, y, t, p)
        rho.append(r), T.append(t), Y.append(y)
        omega.append(rates.production(mix, r, y, t))
        gRT.append(mix.eos.gibbs(mix.species, [t], u=[rates.tlog(t)])[:, 0])
    Ts = np.geomspace(300.0, 3500.0, 64)
    ev = mix.eos.caloric.evaluate
    sps = list(mix.species.values())
    cpR = np.array([ev(sp["cppoly"], np.log(Ts)) for sp in sps]).T
    hR = np.array([ev(sp["hpoly"], np.log(Ts)) * Ts + sp["h298"] for sp in sps]).T
    return dict(rho=np.array(rho), T=np.array(T), Y=np.array(Y), omega=np.array(omega), gRT=np.array(gRT),
                Ts=Ts, cpR=cpR, hR=hR)


def binary_pairs(reference):
    from peregrine_b200.data.export_mixture import reference_mixture, subset
    from peregrine.simulator.mixture.diffusion.binary import BinaryModel
    from peregrine.simulator.mixture.transport.kinetic import KineticTheoryModel
    import tempfile

    path = os.path.join(reference, "peregrine", "simulator", "mixture", "database", "mechanisms", "GRI30.yaml")
    keep = ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "H2O2", "N2"]
    with tempfile.TemporaryDirectory() as tmp:
        mix = reference_mixture(reference, subset(path, keep, tmp), "tpg", "kinetic-theory", None, diffusion="binary")
    model = BinaryModel(mix.cfgsect)
    Ts = KineticTheoryModel(mix.cfgsect).ljparams(mix.species)["Ts"]
    # the model's own pair coefficients before its refit
    model.fit = lambda x, y, tol, deg: (np.asarray(y), None)
    raw = np.array(model.dijinv(mix.species))
    return dict(Ts=np.asarray(Ts), diffinv=raw, tol=np.array(mix.cfgsect["refit-tol"]))


def realgas_densities(reference, cubic, n, rng):
    from peregrine_b200.data.export_mixture import CUBICS, reference_mixture
    from tests.eos import support

    mix = reference_mixture(reference, ["O2", "H2"], "real-gas", trange=(100.0, 1000.0), cubic=cubic)
    support.cubic = CUBICS[cubic] or mix.eos.cubic
    sp = [dict(MW=s["MW"], Tcrit=s["Tcrit"], pcrit=s["pcrit"], acentric=s["acentric"]) for s in mix.species.values()]
    p = rng.uniform(1e6, 8e7, n)
    T = rng.uniform(100.0, 600.0, n)
    Y0 = rng.uniform(0.0, 1.0, n)
    # dense and liquid-like oxygen at the mixing layer's cold side
    p[:8], T[:8], Y0[:8] = 6e6, np.linspace(100.0, 160.0, 8), 1.0
    rho = np.array([support.textbookdensity(sp, p[k], T[k], np.array([Y0[k], 1.0 - Y0[k]])) for k in range(n)])
    return dict(p=p, T=T, Y=Y0[:, None], rho=rho)


def metrics(GridBlock, rng):
    ng = 2
    shape = (7 + 2 * ng, 6 + 2 * ng, 5 + 2 * ng)
    axes = [np.linspace(0.0, 1.0, n) for n in shape]
    nodes = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)
    nodes = nodes + rng.uniform(-1, 1, nodes.shape) * 0.15 / 10
    blk = GridBlock.__new__(GridBlock)
    blk.ng, blk.nblki = ng, 0
    out = dict(nodes=nodes, xcc=blk._cellcenters(nodes), detJinv=blk._detJinv(nodes), Jinv=blk._Jinv(nodes))
    for a, d in enumerate("ijk"):
        out[f"{d}S"] = blk._areavecs(nodes, a)
        out[f"{d}xc"] = blk._facecenters(nodes, a)
    return out


def constants(pg, get_mixture, gas):
    cfg = pg.Config()
    cfg["mixture"]["species"] = gas
    cfg["mixture"]["trans"] = "constant"
    mix = get_mixture(cfg)
    return {k: np.asarray(v, dtype=np.float64) for k, v in mix.constants().items()}


def rk_tables(integrators):
    import peregrine.integrators.base as base

    recorded = []

    class Recorder:
        def __init__(self, provider, template, options=None, **arguments):
            recorded.append(dict(options=options, arguments=arguments))

    base.Kernel = Recorder
    out = {}
    for cls in (integrators.RK1, integrators.RK2, integrators.RK3, integrators.RK34, integrators.RK4):
        integ = cls.__new__(cls)
        integ.provider = None
        regs = [f"R{n}" for n in range(cls.nregs)]
        stages = []
        for n in range(len(cls.stages)):
            recorded.clear()
            integ.stagekerns(n, regs)
            q = integ.stageregs(regs)[n].Q
            combines = []
            for r in recorded:
                a, o = r["arguments"], r["options"]
                terms = [(a[f"X{m}"], a[f"w{m}"]) for m in range(o["terms"])]
                combines.append(dict(out=a["out"], own=a.get("wout") if o["own"] else None, terms=terms, step=o["step"]))
            stages.append(dict(q=q, combines=combines))
        out[cls.name] = dict(nregs=cls.nregs, stages=stages)
    return out


def main():
    global REF
    if len(sys.argv) < 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_golden.py REFERENCE [FIXTURE ...]  (REFERENCE: a checkout of the reference)")
    REF = sys.argv[1]
    only = set(sys.argv[2:])
    install_stubs()
    sys.path.insert(0, REF)
    import peregrine as pg
    from peregrine import integrators
    from peregrine.multiblock.block.grid import GridBlock
    from peregrine.simulator.mixture import get_mixture
    from tests.simulator import oracle as orc

    h2o2 = ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "H2O2", "N2"]
    if only:
        air_tgv()  # puts this package on the path, as the full run does
        # fixtures that draw from their own seeds, one at a time
        single = {"rates_h2o2_gri30_oneway": lambda: rates_of(REF, "GRI30.yaml", h2o2, 96,
                                                              np.random.default_rng(20261209), oneway=True)}
        for name in only:
            if name not in single:
                sys.exit(f"{name}: not a fixture written alone ({sorted(single)})")
            np.savez(os.path.join(HERE, name + ".npz"), **single[name]())
            print("wrote", name)
        return
    rng = np.random.default_rng(20261203)
    air = air_tgv()
    np.savez(os.path.join(HERE, "faces_kepaec.npz"),
             **{f"air_{k}": v for k, v in faces(orc, {"Air": {"MW": air["Air"]["MW"], "cp0": air["Air"]["cp0"]}}, 64, rng).items()},
             **{f"binary_{k}": v for k, v in faces(orc, {k: dict(MW=v["MW"], cp0=v["cp0"]) for k, v in BINARY.items()}, 64, rng).items()})
    np.savez(os.path.join(HERE, "metrics.npz"), **metrics(GridBlock, rng))
    consts = {f"air_{k}": v for k, v in constants(pg, get_mixture, air).items()}
    consts.update({f"binary_{k}": v for k, v in constants(pg, get_mixture, BINARY).items()})
    np.savez(os.path.join(HERE, "constants.npz"), **consts)
    with open(os.path.join(HERE, "rk_tables.json"), "w") as f:
        json.dump(rk_tables(integrators), f, indent=1)
    binary = {k: dict(MW=v["MW"], cp0=v["cp0"]) for k, v in BINARY.items()}
    np.savez(os.path.join(HERE, "faces_riemann.npz"), **faces4(orc, binary, 256, np.random.default_rng(20261204)))
    np.savez(os.path.join(HERE, "mathfns.npz"), **mathfns())
    np.savez(os.path.join(HERE, "rates_h2o2_gri30.npz"),
             **rates_of(REF, "GRI30.yaml", h2o2, 96, np.random.default_rng(20261206)))
    np.savez(os.path.join(HERE, "rates_ch4_o2_ffcmy.npz"),
             **rates_of(REF, "CH4_O2_FFCMY.yaml", None, 96, np.random.default_rng(20261207)))
    np.savez(os.path.join(HERE, "rates_h2o2_gri30_oneway.npz"),
             **rates_of(REF, "GRI30.yaml", h2o2, 96, np.random.default_rng(20261209), oneway=True))
    np.savez(os.path.join(HERE, "binary_h2o2.npz"), **binary_pairs(REF))
    for cubic in ("srk", "pr"):
        np.savez(os.path.join(HERE, f"realgas_{cubic}.npz"),
                 **realgas_densities(REF, cubic, 128, np.random.default_rng(20261208)))
    with open(os.path.join(HERE, "gases.json"), "w") as f:
        json.dump(dict(air=air, binary=BINARY), f, indent=1)
    print("wrote", sorted(p for p in os.listdir(HERE) if not p.endswith(".py")))


if __name__ == "__main__":
    main()
