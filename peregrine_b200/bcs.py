"""Boundary entries: the reference's bcvals, compiled for the library.

The reference names each boundary face (a mesher's ``bcnames`` or
``defaultbc``) and says what each name is in the config's ``bcvals``: a kind
and the values the kind reads, each a number or an expression of x, y, z and
t (peregrine/simulator/bcs.py:10-143, peregrine/simulator/euler/bcs.py,
peregrine/simulator/navstokes/bcs.py).  It renders the expressions into its
kernels as C++; here each value becomes a postfix program of the library's
boundary stack machine (include/pgb200.h, PGB_OP_*), evaluated on the device
at every boundary face's centre and the stage's time.  The checks and their
messages follow the reference's: a value the kind reads must be given, a
carried species not given is 0, and an expression may use numbers, x, y, z,
t, + - * / ** and the functions below.
"""

import ast

from peregrine_b200 import native
from peregrine_b200.config import ConfigError

# per kind: the variables an entry gives, in order, and the simulators that
# have it (the no-slip and moving walls are the viscous simulator's)
KINDS = {
    "slp-adia-wall": ((), ("euler", "navier-stokes")),
    "slp-isot-wall": (("T",), ("euler", "navier-stokes")),
    "no-slp-adia-wall": ((), ("navier-stokes",)),
    "mov-adia-wall": (("u", "v", "w"), ("navier-stokes",)),
    "no-slp-isot-wall": (("T",), ("navier-stokes",)),
    "mov-isot-wall": (("u", "v", "w", "T"), ("navier-stokes",)),
    "sub-in-fvt": (("u", "v", "w", "T"), ("euler", "navier-stokes")),
    "sup-in-fa": (("p", "u", "v", "w", "T"), ("euler", "navier-stokes")),
    "sub-in-ftptt": (("pt", "Tt"), ("euler", "navier-stokes")),
    "sub-in-fmt": (("mflux", "T"), ("euler", "navier-stokes")),
    "sub-out-fp": (("p",), ("euler", "navier-stokes")),
    "sup-out-fn": ((), ("euler", "navier-stokes")),
}
# the inflows also give the carried species' mass fractions
# (peregrine/simulator/euler/bcs.py:5-8)
INLETS = ("sub-in-fvt", "sup-in-fa", "sub-in-ftptt", "sub-in-fmt")
WALLS = ("slp-adia-wall", "slp-isot-wall", "no-slp-adia-wall", "mov-adia-wall", "no-slp-isot-wall", "mov-isot-wall")

NAMES = {"x": "x", "y": "y", "z": "z", "t": "t"}
FUNCTIONS = {"sin": 1, "cos": 1, "tan": 1, "exp": 1, "log": 1, "sqrt": 1, "tanh": 1, "abs": 1, "min": 2, "max": 2,
             "pow": 2}
OPERATORS = {ast.Add: "add", ast.Sub: "sub", ast.Mult: "mul", ast.Div: "div", ast.Pow: "pow"}


class Expression:
    """A value's program: postfix operations and their constants, and which of
    x, y, z and t it reads (the reference's Expression,
    peregrine/simulator/bcs.py:101-143)."""

    def __init__(self, value):
        self.text = value
        self.ops, self.args, self.uses = [], [], set()
        if isinstance(value, str):
            self._emit(ast.parse(value, mode="eval").body)
        else:
            self._push("const", float(value))
        depth = top = 0
        for op in self.ops:
            if op <= native.OPS["t"]:
                depth += 1
            elif op in (native.OPS[k] for k in ("add", "sub", "mul", "div", "pow", "min", "max")):
                depth -= 1
            top = max(top, depth)
        if top > native.BC_STACK:
            raise ValueError(f"{self.text!r}: nested deeper than the {native.BC_STACK} a kernel holds")

    def _push(self, op, arg=0.0):
        self.ops.append(native.OPS[op])
        self.args.append(float(arg))

    def _emit(self, node):
        if isinstance(node, ast.Constant) and type(node.value) in (int, float):
            self._push("const", float(node.value))
        elif isinstance(node, ast.Name):
            self._known(node.id, NAMES)
            self.uses.add(node.id)
            self._push(node.id)
        elif isinstance(node, ast.UnaryOp) and type(node.op) in (ast.USub, ast.UAdd):
            self._emit(node.operand)
            if isinstance(node.op, ast.USub):
                self._push("neg")
        elif isinstance(node, ast.BinOp):
            name = self._known(type(node.op), OPERATORS)
            self._emit(node.left)
            self._emit(node.right)
            self._push(name)
        elif isinstance(node, ast.Call) and isinstance(node.func, ast.Name):
            arity = self._known(node.func.id, FUNCTIONS)
            if len(node.args) != arity or node.keywords:
                raise ValueError(f"{self.text!r}: {node.func.id} takes {arity} argument{'s' if arity > 1 else ''}")
            for a in node.args:
                self._emit(a)
            self._push(node.func.id)
        else:
            what = type(node).__name__
            raise ValueError(f"{self.text!r}: {what} is no part of an expression a kernel evaluates")

    def _known(self, key, table):
        try:
            return table[key]
        except KeyError:
            known = ", ".join(getattr(k, "__name__", k) for k in table)
            name = getattr(key, "__name__", key)
            raise ValueError(f"{self.text!r}: {name!r}; a kernel knows {known}") from None


class Entry:
    """One bcvals entry: its kind, the values it gives in the kind's order (the
    carried species after an inflow's variables), and their programs."""

    def __init__(self, name, given, simulator, species):
        self.name = name
        kind = given.get("kind")
        if kind not in KINDS:
            raise ConfigError(f"bcvals.{name}.kind", f"{kind!r} is not a boundary kind; the kinds are {sorted(KINDS)}")
        variables, simulators = KINDS[kind]
        # the double flux's simulators take their plain twins' kinds
        # (peregrine/simulator/eulerdf/simulator.py:10, navstokesdf/bcs.py)
        simulator = {"euler-df": "euler", "navier-stokes-df": "navier-stokes"}.get(simulator, simulator)
        if simulator not in simulators:
            raise ConfigError(f"bcvals.{name}.kind", f"{kind} is not a boundary of the {simulator} simulator")
        self.kind = kind
        self.variables = variables
        names = list(variables) + (list(species[:-1]) if kind in INLETS else [])
        values = []
        for v in names:
            if v in given:
                values.append(Expression(given[v]))
            elif v in variables:
                raise ConfigError(f"bcvals.{name}", f"{kind} reads {v}, which the entry does not give")
            else:
                values.append(Expression(0.0))
        self.names, self.values = names, values

    @property
    def wall(self):
        return self.kind in WALLS

    @property
    def uses(self):
        return set().union(*(v.uses for v in self.values)) if self.values else set()

    def program(self):
        """(kind id, ops, args, starts): the arrays pgb_case_add_bc takes."""
        ops, args, starts = [], [], [0]
        for v in self.values:
            ops += v.ops
            args += v.args
            starts.append(len(ops))
        return native.BC_KINDS[self.kind], ops, args, starts


def entries(bcvals, simulator, species):
    """Every entry of bcvals, each checked, in name order (the reference makes
    every kind, those no face names too, so a bad entry is refused at once:
    peregrine/multiblock/solver.py:200-207)."""
    return {name: Entry(name, given, simulator, species) for name, given in sorted(bcvals.items())}


def check_faces(blocks, bcvals):
    """Every boundary face is named and its name is an entry of bcvals
    (peregrine/multiblock/solver.py:157-173)."""
    for blk in blocks:
        for face in blk.intfaces:
            # a face joined to another rank's block is traded, not a boundary
            if face.nbr is not None or getattr(face, "remote", None) is not None:
                continue
            where = f"block {blk.nblki} interface {face.nface}"
            if face.bcname is None:
                raise ValueError(f"{where} is a boundary the grid did not name; name it -- a mesher's bcnames or "
                                 "defaultbc -- and say what it is in bcvals")
            if face.bcname not in bcvals:
                raise ValueError(f"{where} is named {face.bcname!r}, which bcvals does not have; it has "
                                 f"{sorted(bcvals)}")
