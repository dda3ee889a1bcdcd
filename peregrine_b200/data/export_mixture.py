"""Writes a mixture's constant tables, as the reference's own mixture computes
them, to an .npz that peregrine_b200 loads.

    python -m peregrine_b200.data.export_mixture REFERENCE OUT.npz MECHANISM \\
        [--keep H2,H,O,...] [--eos tpg] [--trans kinetic-theory] \\
        [--chemistry finite-rate] [--trange 300 3500] [--cubic srk|pr] \\
        [--diffusion lewis|binary] [--oneway]
    python -m peregrine_b200.data.export_mixture --integrals REFERENCE OUT.npz

MECHANISM is a mechanism file, or species of the reference's library
separated by commas.

The thermally perfect fits (cp, h and s in ln T), the kinetic-theory fits of
mu and kappa, the reaction columns and the third-body sets are all worked out
by the reference's Python (peregrine/simulator/mixture/mixture.py:54-58 and
each model's ``constants``); this script runs that code once, offline, on a
checkout of the reference, and stores the numbers.  The kernels then read the
same doubles the reference would have written into its rendered kernels.
``--keep`` restricts a Cantera-format mechanism to a species subset: its
reactions among those species only, and third-body efficiencies of absent
species dropped (the parser refuses them,
peregrine/simulator/mixture/parser/base.py:46-51).

The reference's package imports mako, mpi4py, h5py and lxml at module level
for its code generation, MPI and files; none of those run on this path, so
stub modules stand in for them.
"""

import argparse
import os
import re
import sys
import tempfile
import types

import numpy as np

# reaction kinds, shared with include/pgb200.h
KINDS = {"elementary": 0, "three-body": 1, "lindemann": 2, "troe": 3}

# The reference ships the Soave-Redlich-Kwong cubic
# (peregrine/simulator/mixture/eos/realgas/model.py:26-29); its kernels are
# generic in the form's u and w and the species' a, b and m.  Peng-Robinson is
# these constants (Peng and Robinson, 1976): v^2 + 2 b v - b^2 in the
# attraction's denominator, Omega_a 0.45724, Omega_b 0.07780 and
# m = 0.37464 + 1.54226 w - 0.26992 w^2.  Set on the reference's model class
# here, on the export's side; the reference is not edited.
CUBICS = {
    "srk": None,
    "pr": dict(u=2.0, w=-1.0, omega_a=0.45724, omega_b=0.07780, m=(0.37464, 1.54226, -0.26992)),
}


def _stub(name, **attrs):
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
    """Stand-ins for the modules the reference imports but this path never calls."""
    mako = _stub("mako")
    mako.runtime = _stub("mako.runtime", capture=lambda *a, **k: "", supports_caller=lambda f: f)
    mako.lookup = _stub("mako.lookup", TemplateLookup=_Any)
    mako.template = _stub("mako.template", Template=_Any)
    MPI = types.SimpleNamespace(COMM_WORLD=_Comm(), IN_PLACE=None, MAX=None, SUM=None, Prequest=_Any,
                                Request=_Any, Comm=_Comm)
    m4 = _stub("mpi4py", MPI=MPI)
    _stub("mpi4py.MPI", **vars(MPI))
    m4.util = _stub("mpi4py.util")
    m4.util.dtlib = _stub("mpi4py.util.dtlib", from_numpy_dtype=lambda d: d)
    h5 = _stub("h5py", File=_Any)
    for s in ("h5fd", "h5p", "h5s"):
        setattr(h5, s, _stub("h5py." + s))
    lx = _stub("lxml")
    lx.etree = _stub("lxml.etree")
    if "cantera" not in sys.modules:
        _stub("cantera", add_directory=lambda *a, **k: None)


def _species_of(equation):
    out = []
    for side in re.split(r"<=>|=>", equation.replace("(+M)", "")):
        for term in side.split("+"):
            t = re.sub(r"^[0-9.]+\s*", "", term.strip())
            if t and t != "M":
                out.append(t)
    return out


def subset(mechanism, keep, where, oneway=False):
    """A Cantera-format mechanism cut to the species in keep (every species
    when keep is None), written under where; with oneway every reaction
    irreversible, "<=>" written "=>" (the parser's irreversible arrow,
    peregrine/simulator/mixture/parser/base.py:90-95)."""
    import yaml

    with open(mechanism) as f:
        src = yaml.safe_load(f)
    keep = list(keep) if keep is not None else [s["name"] for s in src["species"]]
    phase = dict(src["phases"][0], species=keep)
    reactions = []
    for r in src["reactions"]:
        if all(s in keep for s in _species_of(r["equation"])):
            r = dict(r)
            if "efficiencies" in r:
                r["efficiencies"] = {k: v for k, v in r["efficiencies"].items() if k in keep}
            if oneway:
                r["equation"] = r["equation"].replace("<=>", "=>")
            reactions.append(r)
    out = dict(units=src["units"], phases=[phase], species=[s for s in src["species"] if s["name"] in keep],
               reactions=reactions)
    path = os.path.join(where, os.path.basename(mechanism))
    with open(path, "w") as f:
        yaml.safe_dump(out, f, sort_keys=False)
    return path


def reference_mixture(reference, species, eos="tpg", trans=None, chemistry=None, trange=(300.0, 3500.0),
                      cubic="srk", diffusion="lewis"):
    """The reference's Mixture for a config, from a checkout at reference."""
    install_stubs()
    if reference not in sys.path:
        sys.path.insert(0, reference)
    import peregrine as pg
    from peregrine.simulator.mixture import get_mixture
    from peregrine.simulator.mixture.eos.realgas.model import RealGasModel

    if not hasattr(RealGasModel, "_shipped_cubic"):
        RealGasModel._shipped_cubic = dict(RealGasModel.cubic)
    RealGasModel.cubic = CUBICS[cubic] or RealGasModel._shipped_cubic

    cfg = pg.Config()
    m = cfg["mixture"]
    m["species"], m["eos"], m["trans"], m["chemistry"] = species, eos, trans, chemistry
    m["T-range"] = tuple(trange)
    m["diffusion"] = diffusion
    return get_mixture(cfg)


def tables(mix):
    """Every table the kernels read, by the reference's names."""
    out = {k: np.asarray(v, dtype=np.float64) for k, v in mix.constants().items()}
    out["spnames"] = np.array(mix.spnames)
    out["eos"] = np.array(mix.eos.name)
    if hasattr(mix.eos, "cubic"):
        c = mix.eos.cubic
        out["cubic_omega_a"], out["cubic_omega_b"] = np.array(c["omega_a"]), np.array(c["omega_b"])
        out["cubic_m"] = np.array(c["m"])
    out["trans"] = np.array(mix.trans.name if mix.trans is not None else "")
    out["ns"] = np.array(mix.ns)
    out["diffusion"] = np.array(mix.diffusion.name if getattr(mix, "diffusion", None) is not None else "lewis")
    if mix.chemistry is not None:
        cols = mix.chemistry.rxnconsts(mix.species)
        terms = mix.chemistry.terms(mix.species)
        for k, v in cols.items():
            if k == "type":
                out["rxn_kind"] = np.array([KINDS[t] for t in v], dtype=np.int32)
            else:
                out["rxn_" + k] = np.asarray(v)
        out["rxn_tb"] = np.array([-1 if r.tb is None else r.tb for r in terms.reactions], dtype=np.int32)
        out["rxn_troeidx"] = np.array([-1 if r.troeidx is None else r.troeidx for r in terms.reactions],
                                      dtype=np.int32)
        out["tb_effsp"] = mix.chemistry.padded([[sp for sp, _ in t.eff] for t in terms.thirdbodies], np.int32)
        out["tb_neff"] = np.array([len(t.eff) for t in terms.thirdbodies], dtype=np.int32)
        out["chemistry"] = np.array(mix.chemistry.name)
    return out


def integrals(reference):
    """The collision-integral table the kinetic theory reads (Monchick and
    Mason's Stockmayer Omega(2,2)* and A* against T* and delta*, as the
    reference's database carries it), for peregrine_b200.mixgen."""
    import yaml

    path = os.path.join(reference, "peregrine", "simulator", "mixture", "database", "integrals.yaml")
    with open(path) as f:
        ci = yaml.safe_load(f)
    return {k: np.array(ci[k], dtype=np.float64) for k in ("delta", "tstar22", "omega22", "tstar", "astar")}


def main(argv=None):
    if argv is None:
        argv = sys.argv[1:]
    if argv and argv[0] == "--integrals":
        # python -m peregrine_b200.data.export_mixture --integrals REFERENCE OUT.npz
        np.savez(argv[2], **integrals(argv[1]))
        print(argv[2])
        return
    ap = argparse.ArgumentParser()
    ap.add_argument("reference")
    ap.add_argument("out")
    ap.add_argument("mechanism")
    ap.add_argument("--keep", default=None)
    ap.add_argument("--eos", default="tpg")
    ap.add_argument("--trans", default=None)
    ap.add_argument("--chemistry", default=None)
    ap.add_argument("--trange", nargs=2, type=float, default=(300.0, 3500.0))
    ap.add_argument("--cubic", default="srk", choices=sorted(CUBICS))
    ap.add_argument("--diffusion", default="lewis", choices=("lewis", "binary"))
    ap.add_argument("--oneway", action="store_true", help="every reaction irreversible")
    a = ap.parse_args(argv)
    mech = a.mechanism
    if "," in mech:
        # species from the reference's library by name
        mech = mech.split(",")
    elif not os.path.isfile(mech):
        mech = os.path.join(a.reference, "peregrine", "simulator", "mixture", "database", "mechanisms", mech)
    with tempfile.TemporaryDirectory() as tmp:
        if (a.keep or a.oneway) and isinstance(mech, str):
            mech = subset(mech, a.keep.split(",") if a.keep else None, tmp, oneway=a.oneway)
        mix = reference_mixture(a.reference, mech, a.eos, a.trans, a.chemistry, a.trange, a.cubic, a.diffusion)
        np.savez(a.out, **tables(mix))
    print(a.out, mix)


if __name__ == "__main__":
    main()
