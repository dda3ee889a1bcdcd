"""The Runge-Kutta integrators as stage tables the library runs.

The reference's integrators (peregrine/integrators/rungekutta.py:4-92) name
their registers ``start, stage[, total], dQ`` and turn each stage into
``combine`` kernels by merging repeated registers and dropping zero weights
(peregrine/integrators/base.py:122-137).  The same bookkeeping here yields
``pgb_stage`` records: the register the stage's right-hand side reads and
each combine's output, its own weight and its terms, dQ last with dt on it.
"""

from peregrine_b200 import native

# (fraction of dt, wQ0, wQ, wdQ) per stage: Qout = wQ Q + wQ0 Qstart + wdQ dt dQ
TABLES = {
    "rk1": ((0.0, 0.0, 1.0, 1.0),),
    "rk2": ((0.0, 0.0, 1.0, 1.0), (1.0, 0.5, 0.5, 0.5)),
    "tvd-rk3": ((0.0, 0.0, 1.0, 1.0), (1.0, 0.75, 0.25, 0.25), (0.5, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)),
    "rk34": ((0.0, 0.0, 1.0, 0.5), (0.5, 0.0, 1.0, 0.5), (1.0, 2.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0),
             (0.5, 0.0, 1.0, 0.5)),
}
# rk4: (fraction of dt, wdQ, wsum); the last stage has no wdQ of its own
RK4 = ((0.0, 0.5, 1.0 / 6.0), (0.5, 0.5, 1.0 / 3.0), (0.5, 1.0, 1.0 / 3.0), (1.0, None, 1.0 / 6.0))
NREGS = {"rk1": 2, "rk2": 3, "tvd-rk3": 3, "rk34": 3, "rk4": 4}


def _combine(out, pairs, step=True):
    weights = {}
    for reg, w in pairs:
        weights[reg] = weights.get(reg, 0.0) + w
    own = weights.pop(out, 0.0)
    reads = [(r, w) for r, w in weights.items() if w != 0.0]
    return dict(out=out, own=own, reads=reads, step=step)


def stages(name):
    """[(register read, [combines])], dQ's register, the stage times' fractions."""
    nregs = NREGS[name]
    if name == "rk4":
        start, stage, total, dQ = range(4)
        out = []
        for n, (_, wdQ, wsum) in enumerate(RK4):
            own = 0.0 if n == 0 else 1.0
            share = _combine(total, [(total, own), (dQ, wsum)])
            q = start if n == 0 else stage
            if wdQ is None:
                end = _combine(start, [(start, 1.0), (total, 1.0)], step=False)
                out.append((q, [share, end]))
            else:
                out.append((q, [share, _combine(stage, [(start, 1.0), (dQ, wdQ)])]))
        return out, dQ, nregs
    table = TABLES[name]
    start, stage, dQ = 0, 1, nregs - 1
    last = len(table) - 1
    out = []
    for n, (_, wQ0, wQ, wdQ) in enumerate(table):
        Q = start if n == 0 else stage
        Qout = start if n == last else stage
        out.append((Q, [_combine(Qout, [(Q, wQ), (start, wQ0), (dQ, wdQ)])]))
    return out, dQ, nregs


def stage_fractions(name):
    """The time each stage's right-hand side reads, as a fraction of dt past
    the step's start: the stage table's first column (stage 0 at the start;
    the reference moves its clock to stage n's time before stage n's
    right-hand side, peregrine/integrators/rungekutta.py:28-39)."""
    return [row[0] for row in (RK4 if name == "rk4" else TABLES[name])]


def stage_records(name):
    rows, dQ, nregs = stages(name)
    recs = (native.Stage * len(rows))()
    fracs = stage_fractions(name)
    for s, (q, combines) in enumerate(rows):
        rec = recs[s]
        rec.q, rec.dq, rec.ncombine = q, dQ, len(combines)
        rec.tfrac = fracs[s]
        for m, cb in enumerate(combines):
            c = rec.combine[m]
            c.out = cb["out"]
            c.own = int(cb["own"] != 0.0)
            c.wout = cb["own"]
            c.nterms = len(cb["reads"])
            for n, (r, w) in enumerate(cb["reads"]):
                c.reg[n] = -1 if r == dQ else r
                c.w[n] = w
            c.step = int(cb["step"])
    return recs, nregs


class Fixed:
    """The fixed step: the config's dt (peregrine/integrators/controllers.py:12-17)."""

    name = "fixed"

    def __init__(self, cfg):
        self.cfg = cfg

    def stepsize(self, solver):
        return self.cfg["simulation"]["dt"]


class CFL(Fixed):
    """The CFL target over the combined CFL number per unit step, under
    dt-max (peregrine/integrators/controllers.py:20-30; the reference's
    plugins' output times, which shorten a step, are not built here)."""

    name = "cfl"

    def stepsize(self, solver):
        sim = self.cfg["simulation"]
        return min(sim["cfl"] / solver.cflmax()["combined"], sim["dt-max"])


class StageRegisters(tuple):
    """A stage's registers by name: the one its right-hand side reads, dQ,
    and the one its last combine writes (peregrine/integrators/base.py:4-10)."""

    __slots__ = ()

    def __new__(cls, Q, dQ, Qout):
        return super().__new__(cls, (Q, dQ, Qout))

    Q = property(lambda self: self[0])
    dQ = property(lambda self: self[1])
    Qout = property(lambda self: self[2])


class Integrator:
    """The integrator's name and its step-size controller, as the reference's
    solver carries them (``solver.integ.controller``)."""

    def __init__(self, cfg):
        self.name = cfg["time-integration"]["integrator"]
        self.controller = {"fixed": Fixed, "cfl": CFL}[cfg["simulation"]["controller"]](cfg)

    def stageregs(self, registers):
        """Each stage's registers named from ``registers``, the solver's
        ``regs`` (peregrine/integrators/rungekutta.py:9-14)."""
        rows, dQ, _ = stages(self.name)
        return [StageRegisters(registers[q], registers[dQ], registers[combines[-1]["out"]])
                for q, combines in rows]
