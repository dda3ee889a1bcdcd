"""The solver's named variables and the physics that derives them, as a
script reads them through ``mb.sim.iovars.data(blk, names)``
(peregrine/simulator/iovars.py:1-30, peregrine/simulator/euler/simulator.py:51-90).

The primitives are p, u, v, w, T and every species but the last; the
exported names add rho and the last species.  ``data`` derives them from a
block's register Q and its eos state: p and T from the state the last
right-hand side formed, rho from Q, the velocity and the carried species as
Q over rho, the last species as what the others leave.  The batched path
forms its state in registers and keeps no state array; there (the
calorically perfect single gas it takes) p and T are fromQ's closed form of
Q.
"""

import ctypes

import numpy as np

from peregrine_b200 import native

# the eos state's fields in the order the device keeps them
STATEFIELDS = ("p", "T", "rhoinv", "rho", "e", "cp", "gamma", "c", "Z")


class IoVars:
    def __init__(self, solver):
        self.solver = solver
        species = solver.mixture.spnames
        self.primitives = dict.fromkeys(("p", "u", "v", "w", "T"))
        self.primitives.update({s: 0.0 for s in species[:-1]})
        self.exported = ["rho", *self.primitives, species[-1]]
        self.vectors = {"Velocity": ("u", "v", "w")}

    @property
    def privars(self):
        return list(self.primitives)

    def _field(self, nblk, name):
        s = self.solver
        b = s.mesh_blocks[nblk]
        out = np.empty(tuple(n + 4 for n in b.cells), order="F")
        ptr = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        try:
            native.call("pgb_eos_get", s.case, nblk, STATEFIELDS.index(name), ptr, out.size)
        except native.PgbStateError:
            return None
        return np.ascontiguousarray(out)

    def _closed_form(self, Q):
        """p and T of the calorically perfect single gas from Q (fromQ.mako:5-19
        with the cpg eos, mixture/eos/cpg/kernels/eos.mako:5-15)."""
        t = self.solver.mixture.constants()
        R, cp, h298 = float(t["Rsp"][0]), float(np.ravel(t["cp0"])[0]), float(t["h298R"][0])
        rho = Q[..., 0]
        e = (Q[..., 4] - 0.5 * (Q[..., 1] ** 2 + Q[..., 2] ** 2 + Q[..., 3] ** 2) / rho) / rho
        T = (e - h298) / (cp - R)
        return {"p": rho * R * T, "T": T}

    def data(self, blk, names):
        s = self.solver
        nblk = blk.mesh.nblki if hasattr(blk, "mesh") else int(blk)
        Q = s.blocks[nblk].Q.get()
        species = s.mixture.spnames
        with np.errstate(divide="ignore", invalid="ignore"):
            rhoinv = 1.0 / Q[..., 0]
            values = {}
            for n in ("p", "T"):
                if n in names:
                    values[n] = self._field(nblk, n)
            if any(v is None for v in values.values()):
                values.update({k: v for k, v in self._closed_form(Q).items() if k in values})
            values["rho"] = Q[..., 0]
            for n, name in enumerate("uvw"):
                values[name] = Q[..., 1 + n] * rhoinv
            for n, name in enumerate(species[:-1]):
                values[name] = Q[..., 5 + n] * rhoinv
            others = sum((values[name] for name in species[:-1]), np.zeros_like(Q[..., 0]))
            values[species[-1]] = np.ones_like(Q[..., 0]) - others
        unknown = [n for n in names if n not in values]
        if unknown:
            raise KeyError(f"{unknown}: the variables are {self.exported}")
        return {name: values[name] for name in names}


class Simulator:
    """What a script reads of the physics: its name, mixture, state fields and
    named variables (peregrine/simulator/base.py, euler/simulator.py)."""

    def __init__(self, solver):
        self.name = solver.cfg["simulation"]["simulator"]
        self.mixture = solver.mixture
        self.iovars = IoVars(solver)
        ns = solver.ns
        plane = ("theta", "eps", "kappa", *(f"zeta{n}" for n in range(ns - 1)))
        self.statefields = STATEFIELDS + (plane if self.name.endswith("-df") else ())
