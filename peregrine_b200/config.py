"""The case description: sections of keys that refuse a misspelled key.

Mirrors the reference's ``Config`` (peregrine/config.py:12-106): the same
sections and defaults, a ``ConfigError(setting, msg)`` for a refused value
(peregrine/config.py:6-9), and ``from_dict`` / ``to_dict``.  The only added
section is ``backend-b200``, the knobs of this build's device path.
"""

import copy


class ConfigError(Exception):
    def __init__(self, setting, msg):
        self.setting = setting
        text = f"Invalid setting {setting}: {msg}"
        super().__init__(text)


class Section(dict):
    """A dict whose key set is fixed once frozen (reference misc/frozendict.py:1-25)."""

    _frozen = False

    def __setitem__(self, key, value):
        if self._frozen and key not in self:
            raise KeyError(f"{key} is not a valid input for this section, check spelling and case")
        super().__setitem__(key, value)

    def update(self, *args, **kwargs):
        for key, value in dict(*args, **kwargs).items():
            self[key] = value

    def freeze(self):
        self._frozen = True
        return self


_DEFAULTS = {
    "simulation": {
        "simulator": "navier-stokes",
        "precision": "double",
        "niter": 1,
        "controller": "fixed",
        "dt": 1e-3,
        "dt-max": 1e-3,
        "cfl": 0.1,
    },
    "mixture": {
        "species": None,
        "eos": "cpg",
        "trans": None,
        "diffusion": "lewis",
        "mixing-rule": "wilke",
        "chemistry": None,
        "bath": None,
        "T-range": None,
        "refit-tol": 1e-3,
        "refit-max-deg": 6,
    },
    "chem-integration": {
        "kind": None,
        "max-substeps": 200,
        "bulk-substeps": 1,
        "stiff-bins": 8,
        "equilibrium-tolerance": 1e-7,
    },
    "ics": {"p": 101325.0, "u": 0.0, "v": 0.0, "w": 0.0, "T": 300.0, "Y": {}},
    "time-integration": {"integrator": "tvd-rk3"},
    "adv-flux": {
        "formulation": "single",
        "primary": "kepaec",
        "recon": "constant",
        "limiter": None,
        "secondary": None,
        "correction": None,
        "switch": None,
        "values": {},
    },
    "diff-flux": {"formula": "alpha-damping", "values": {}},
    # this build's device path: "batched" is the fused persistent kernel over
    # every block, "per-block" the unfused launches per block and kernel;
    # "metrics" picks the uniform-block form where a block's metrics allow it
    "backend-b200": {"launch": "batched", "metrics": "auto", "graph": True, "chemistry-kernel": "generated"},
    "halo-exchange": {"kind": "device"},
}

SIMULATORS = ("euler", "navier-stokes", "euler-df", "navier-stokes-df")
VISCOUS = ("navier-stokes", "navier-stokes-df")
DOUBLE_FLUX = ("euler-df", "navier-stokes-df")
INTEGRATORS = ("rk1", "rk2", "tvd-rk3", "rk34", "rk4")
EOSES = ("cpg", "tpg", "real-gas", "real-gas-df")
TRANS = (None, "constant", "kinetic-theory")
PRIMARIES = ("kepaec", "hllc", "rusanov", "ausmup")
RECONS = ("constant", "muscl")
LIMITERS = (None, "koren", "minmod", "mc", "superbee", "vanleer")


class Config(dict):
    def __init__(self):
        super().__init__()
        for name, entries in _DEFAULTS.items():
            super().__setitem__(name, Section(copy.deepcopy(entries)).freeze())
        self["bcvals"] = {}
        self["plugins"] = {}

    def __setitem__(self, key, value):
        if key not in self and key not in ("bcvals", "plugins"):
            raise KeyError(f"{key} is not a section of the config")
        super().__setitem__(key, value)

    @classmethod
    def from_dict(cls, given):
        config = cls()
        for section, entries in (given or {}).items():
            for key, value in (entries or {}).items():
                config[section][key] = value
        config.validate()
        return config

    def to_dict(self):
        return {s: dict(e) if isinstance(e, dict) else e for s, e in self.items()}

    def validate(self):
        sim = self["simulation"]
        sim["dt"] = float(sim["dt"])
        checks = [
            ("simulation.simulator", sim["simulator"], SIMULATORS),
            ("time-integration.integrator", self["time-integration"]["integrator"], INTEGRATORS),
            ("mixture.eos", self["mixture"]["eos"], EOSES),
            ("mixture.trans", self["mixture"]["trans"], TRANS),
            ("adv-flux.primary", self["adv-flux"]["primary"], PRIMARIES),
            ("adv-flux.recon", self["adv-flux"]["recon"], RECONS),
            ("adv-flux.limiter", self["adv-flux"]["limiter"], LIMITERS),
        ]
        for setting, value, allowed in checks:
            if value not in allowed:
                raise ConfigError(setting, f"{value!r} is not one of {allowed}")
        if sim["precision"] != "double":
            raise ConfigError("simulation.precision", "this build computes in double only")
        adv = self["adv-flux"]
        if adv["formulation"] != "single":
            raise ConfigError("adv-flux.formulation", "only 'single' is built")
        if adv["recon"] == "muscl" and adv["limiter"] is None:
            raise ConfigError("adv-flux.limiter", "muscl names a limiter")
        if adv["primary"] == "kepaec" and adv["recon"] != "constant":
            raise ConfigError("adv-flux.recon", "kepaec takes the constant reconstruction only")
        if sim["simulator"] in VISCOUS and self["mixture"]["trans"] is None:
            raise ConfigError("mixture.trans", "a viscous case names a transport model")
        # the double flux freezes the real gas's tangent plane (peregrine/simulator/eulerdf/simulator.py:15-20),
        # with the flux functions it has a form of (peregrine/simulator/eulerdf/kernels/flux/function/)
        if (sim["simulator"] in DOUBLE_FLUX) != (self["mixture"]["eos"] == "real-gas-df"):
            raise ConfigError("mixture.eos", f"{sim['simulator']}: euler-df and navier-stokes-df take real-gas-df, "
                                             "and that eos one of them")
        if sim["simulator"] in DOUBLE_FLUX and adv["primary"] == "hllc":
            raise ConfigError("adv-flux.primary", "the double flux has kepaec, rusanov and ausmup")
        if self["mixture"]["mixing-rule"] not in ("wilke", "herning"):
            raise ConfigError("mixture.mixing-rule", f"{self['mixture']['mixing-rule']!r} is not one of ('wilke', 'herning')")
        if self["mixture"]["diffusion"] not in ("lewis", "binary"):
            raise ConfigError("mixture.diffusion", f"{self['mixture']['diffusion']!r} is not one of ('lewis', 'binary')")
        if self["diff-flux"]["formula"] != "alpha-damping":
            raise ConfigError("diff-flux.formula", "only 'alpha-damping' is built")
        if self["mixture"]["chemistry"] not in (None, "finite-rate"):
            raise ConfigError("mixture.chemistry", "null or finite-rate")
        chem = self["chem-integration"]
        kind = chem["kind"]
        if kind not in (None, "coupled", "sub-stepped"):
            raise ConfigError("chem-integration.kind", "null, coupled or sub-stepped")
        if kind is not None and self["mixture"]["chemistry"] is None:
            raise ConfigError("chem-integration.kind", f"{kind} needs mixture.chemistry")
        if kind == "sub-stepped":
            # peregrine/simulator/chemint/substepped.py:21-33
            cap, bulk, bins, tol = (chem[k] for k in ("max-substeps", "bulk-substeps", "stiff-bins",
                                                       "equilibrium-tolerance"))
            if not isinstance(cap, int) or isinstance(cap, bool) or cap < 1:
                raise ConfigError("chem-integration.max-substeps", f"{cap!r} is not a count of one or more")
            if not isinstance(bulk, int) or isinstance(bulk, bool) or not 1 <= bulk <= cap:
                raise ConfigError("chem-integration.bulk-substeps", f"{bulk!r} is not a count from one to max-substeps")
            if not isinstance(bins, int) or isinstance(bins, bool) or not 1 <= bins <= 16:
                raise ConfigError("chem-integration.stiff-bins", f"{bins!r} is not a count from one to sixteen")
            if not isinstance(tol, (int, float)) or isinstance(tol, bool) or not 0.0 <= tol < 1.0:
                raise ConfigError("chem-integration.equilibrium-tolerance",
                                  f"{tol!r} is not a mass fraction below one, zero for no exit")
        if sim["controller"] not in ("fixed", "cfl"):
            raise ConfigError("simulation.controller", f"{sim['controller']!r} is not one of ('fixed', 'cfl')")
        for key in ("cfl", "dt-max"):
            sim[key] = float(sim[key])
            if not sim[key] > 0.0:
                raise ConfigError(f"simulation.{key}", "a positive number")
        launch = self["backend-b200"]["launch"]
        if launch not in ("batched", "per-block", "packed"):
            raise ConfigError("backend-b200.launch", "batched, per-block or packed")
        if self["backend-b200"]["chemistry-kernel"] not in ("generated", "tables"):
            raise ConfigError("backend-b200.chemistry-kernel", "generated or tables")
        return self
