"""The gas: per-species constants the kernels read.

Each table below is the reference's, computed with the same floating-point
operations so the kernels see the same doubles the reference writes into
its kernels as hex literals (peregrine/codegen/constants.py:13-20):

* mixture basics ``MW``, ``MWinv``, ``Rsp`` (simulator/mixture/mixture.py:54-58);
* calorically perfect gas: ``cppoly`` = cp0 MW / Ru, ``h298`` = dHf298 / Ru -
  Tref cppoly (simulator/mixture/caloric/constcp.py:12-21), and the moments
  ``cp0``, ``h298R`` = h298 Rsp (simulator/mixture/eos/base.py:48-64,
  simulator/mixture/eos/cpg/__init__.py);
* constant transport ``mu0``, ``kappa0`` (simulator/mixture/transport/constant.py);
* Wilke's rule ``MWqinv`` = MW^-1/4, ``wilkepair`` = 1 / sqrt(8 (1 + MW_n / MW_m))
  (simulator/mixture/mixrule/wilke.py:8-14);
* Lewis diffusion ``lewis``, one unless a species states its own
  (simulator/mixture/diffusion/lewis.py).

A thermally perfect gas, kinetic-theory transport, finite-rate chemistry and
the cubic real gas take tables worked out from a mechanism's species and
reactions (polynomial refits in ln T, collision-integral fits, reaction
columns).  Name as ``mixture.species`` either a Cantera-format mechanism file
(``.yaml``/``.yml``), whose tables peregrine_b200.mixgen works out here as the
reference's mixture models do (the case states its ``T-range``), or a table
set: a file under peregrine_b200/data, or a path to an .npz, as
peregrine_b200/data/export_mixture.py or mixgen writes one.
"""

import os

import numpy as np

Ru = 8314.46261815324
Tref = 298.15

# the kernels' table ids, shared with include/pgb200.h
TABLES = ("MW", "MWinv", "Rsp", "cp0", "h298R", "hpolyR0", "h298", "mu0", "kappa0",
          "MWqinv", "wilkepair", "lewis")


DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def load_tables(name):
    """A mixture's tables as the reference's mixture wrote them: a file under
    peregrine_b200/data by its stem, or a path to an .npz."""
    path = name if os.path.isfile(name) else os.path.join(DATA, f"{name}.npz")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"no mixture tables {name!r} (tried {path})")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def mechanism_tables(cfgsect):
    """The tables of the mechanism file cfgsect names, for its eos,
    transport, diffusion, mixing rule and chemistry, fitted over its T-range."""
    from peregrine_b200 import mixgen

    path = cfgsect["species"]
    if not os.path.isfile(path):
        raise FileNotFoundError(f"mixture.species: no mechanism file {path!r}")
    eos = cfgsect["eos"]
    trange = cfgsect.get("T-range")
    if trange is None and eos != "cpg":
        raise ValueError(f"mixture.T-range: the {eos} fits are made over the case's temperatures; state them")
    # the double flux's real gas is the real gas's, same tables
    tables = mixgen.make_tables(
        mechanism=path, eos="real-gas" if eos == "real-gas-df" else eos, trans=cfgsect.get("trans"),
        diffusion=cfgsect.get("diffusion") or "lewis", mixing_rule=cfgsect.get("mixing-rule") or "wilke",
        chemistry=cfgsect.get("chemistry"), trange=tuple(trange) if trange is not None else (300.0, 3500.0),
        refit_tol=cfgsect.get("refit-tol", 1e-3), refit_max_deg=cfgsect.get("refit-max-deg", 6),
        bath=cfgsect.get("bath"))
    return tables


class Mixture:
    def __init__(self, cfgsect):
        species = cfgsect["species"]
        self.tables = None
        if isinstance(species, str) and species.lower().endswith((".yaml", ".yml")):
            self._from_tables(cfgsect, mechanism_tables(cfgsect))
            return
        if isinstance(species, str):
            self._from_tables(cfgsect, load_tables(species))
            return
        if not isinstance(species, dict) or not species:
            raise ValueError("mixture.species: a dict of name to data, or the name of a table set")
        self.cfgsect = cfgsect
        self.species = {k: dict(v) for k, v in species.items()}
        self.spnames = list(self.species)
        self.ns = len(self.spnames)
        self.eos = cfgsect["eos"]
        self.trans = cfgsect["trans"]
        self.diffusion = cfgsect.get("diffusion", "lewis") or "lewis"
        if self.diffusion != "lewis":
            raise ValueError(f"mixture.diffusion {self.diffusion!r}: binary diffusion reads the pair fits a table "
                             "set carries (its species' collision parameters)")
        if self.eos != "cpg":
            raise ValueError(f"mixture.eos {self.eos!r}: this gas model is not built yet")
        for name, sp in self.species.items():
            for need in ("MW", "cp0"):
                if need not in sp:
                    raise ValueError(f"cpg needs {need} for {name}")
            if self.trans == "constant":
                for need in ("mu0", "kappa0"):
                    if need not in sp:
                        raise ValueError(f"constant needs {need} for {name}")

    def _from_tables(self, cfgsect, tables):
        self.cfgsect = cfgsect
        self.tables = tables
        self.spnames = [str(n) for n in tables["spnames"]]
        self.ns = len(self.spnames)
        self.species = {n: {"MW": float(m)} for n, m in zip(self.spnames, tables["MW"])}
        self.eos, self.trans = cfgsect["eos"], cfgsect["trans"]
        self.chemistry = cfgsect.get("chemistry")
        made = str(tables["eos"])
        # the double flux's real gas is the real gas's, same tables
        same = {"real-gas-df": "real-gas"}
        if same.get(self.eos, self.eos) != same.get(made, made):
            raise ValueError(f"mixture.eos {self.eos!r}: the tables were made for {made!r}")
        if self.trans is not None and self.trans != str(tables["trans"]):
            raise ValueError(f"mixture.trans {self.trans!r}: the tables were made for {str(tables['trans'])!r}")
        if self.chemistry is not None and "rxn_nr" not in tables:
            raise ValueError("mixture.chemistry: the tables carry no reactions")
        # species diffusion: Lewis numbers, or binary diffusion's pair fits
        # (peregrine/simulator/mixture/diffusion/{lewis,binary}.py)
        self.diffusion = cfgsect.get("diffusion", "lewis") or "lewis"
        made = str(tables["diffusion"]) if "diffusion" in tables else "lewis"
        if self.trans is not None and self.diffusion != made:
            raise ValueError(f"mixture.diffusion {self.diffusion!r}: the tables were made for {made!r}")

    def collect(self, key, default=None):
        values = [sp.get(key, default) for sp in self.species.values()]
        return np.array(values, dtype=np.float64)

    def constants(self):
        if self.tables is not None:
            return dict(self.tables)
        MW = self.collect("MW")
        out = dict(Ru=np.array(Ru), MW=MW, MWinv=1.0 / MW, Rsp=Ru / MW)
        # calorically perfect: a constant cp is its own fit, exactly
        cp0 = self.collect("cp0")
        cppoly = np.array([[sp["cp0"] * sp["MW"] / Ru] for sp in self.species.values()])
        h298 = np.array([sp.get("dHf298", 0.0) / Ru - Tref * c[0]
                         for sp, c in zip(self.species.values(), cppoly)])
        Rsp = out["Rsp"]
        out.update(cppoly=cppoly, hpoly=cppoly.copy(), h298=h298, cp0=cp0,
                   cppolyR=cppoly * Rsp[:, None], hpolyR=cppoly * Rsp[:, None],
                   h298R=h298 * Rsp)
        if self.trans == "constant":
            out.update(mu0=self.collect("mu0"), kappa0=self.collect("kappa0"))
        if self.trans is not None:
            out.update(MWqinv=MW ** -0.25,
                       wilkepair=1.0 / np.sqrt(8.0 * (1.0 + MW[:, None] / MW[None, :])))
            out.update(lewis=self.collect("lewis", 1.0))
        return out
