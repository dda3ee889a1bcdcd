"""TEST INFRASTRUCTURE ONLY: the CPU oracle's Python side.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, as the checker of the device path; the product never
does.  It loads ``oracle/liboracle.so`` (the C restatement in
``pg_oracle.cpp``, built by ``oracle/build.sh``) and drives it the way the
reference's solver drives its kernels:

* the halo windows of every interface, as the reference's exchange lays them
  out (peregrine/multiblock/collections/exchange/collection.py:63-96,
  peregrine/launch/ranges.py:32-40): the interface plane proper, never the
  halo's edges or corners;
* the Runge-Kutta stages as the reference's integrators make them
  (peregrine/integrators/rungekutta.py:9-92, peregrine/integrators/base.py:122-137):
  one right-hand side, then each stage's combine kernels in order.
"""

import ast
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_halo_dtype = np.dtype([(n, np.int32) for n in ("dblk", "di", "dj", "dk", "sblk", "si", "sj", "sk", "layer", "rot")])


class OBc(ctypes.Structure):
    _fields_ = [("blk", ctypes.c_int), ("nface", ctypes.c_int), ("kind", ctypes.c_int), ("nval", ctypes.c_int),
                ("vals", ctypes.POINTER(ctypes.c_double))]


class OCase(ctypes.Structure):
    _fields_ = [("simulator", ctypes.c_int), ("primary", ctypes.c_int), ("ns", ctypes.c_int),
                ("alpha", ctypes.c_double)] + \
               [(n, ctypes.POINTER(ctypes.c_double)) for n in
                ("Rsp", "cp0", "h298R", "MWinv", "hpoly0", "h298", "mu0", "kappa0", "MWqinv", "wilkepair", "lewis")] + \
               [("Ru", ctypes.c_double), ("skip_adv", ctypes.c_int), ("recon", ctypes.c_int), ("limiter", ctypes.c_int),
                ("eos", ctypes.c_int), ("ncp", ctypes.c_int), ("cppolyR", ctypes.POINTER(ctypes.c_double)),
                ("nh", ctypes.c_int), ("hpoly", ctypes.POINTER(ctypes.c_double)), ("trans", ctypes.c_int),
                ("nmu", ctypes.c_int), ("nkappa", ctypes.c_int), ("mupoly", ctypes.POINTER(ctypes.c_double)),
                ("kappapoly", ctypes.POINTER(ctypes.c_double)), ("mech", ctypes.c_void_p),
                ("realgas", ctypes.c_int), ("df", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in ("cu", "cw", "csigma", "ceps")] + \
               [(n, ctypes.POINTER(ctypes.c_double)) for n in
                ("csqrtac", "cb", "cda", "cmTc", "conepm", "vshift", "csqrtacMW", "cbMW", "cdaMW", "vshiftMW")] + \
               [("nbc", ctypes.c_int), ("bc", ctypes.POINTER(OBc)), ("substepped", ctypes.c_int), ("cap", ctypes.c_int),
                ("eqtol", ctypes.c_double), ("dt", ctypes.c_double), ("ncppoly", ctypes.c_int),
                ("cppoly", ctypes.POINTER(ctypes.c_double)), ("MW", ctypes.POINTER(ctypes.c_double)),
                ("cfloor", ctypes.c_double), ("binary", ctypes.c_int), ("bwidth", ctypes.c_int),
                ("nfit", ctypes.c_int), ("bpartial", ctypes.c_int), ("pairfit", ctypes.POINTER(ctypes.c_double)),
                ("selffit", ctypes.POINTER(ctypes.c_double)), ("bath", ctypes.POINTER(ctypes.c_int)),
                ("rots", ctypes.POINTER(ctypes.c_double)), ("herning", ctypes.c_int),
                ("sqrtMW", ctypes.POINTER(ctypes.c_double))]

# the boundary kinds (peregrine/simulator/euler/bcs.py, navstokes/bcs.py): the
# oracle's number for each and the variables an entry gives, in order; the
# inflows' carried species follow them
BC_KINDS = {"slp-adia-wall": (1, ()), "slp-isot-wall": (2, ("T",)), "no-slp-adia-wall": (3, ()),
            "mov-adia-wall": (4, ("u", "v", "w")), "no-slp-isot-wall": (5, ("T",)),
            "mov-isot-wall": (6, ("u", "v", "w", "T")), "sub-in-fvt": (7, ("u", "v", "w", "T")),
            "sup-in-fa": (8, ("p", "u", "v", "w", "T")), "sub-in-ftptt": (9, ("pt", "Tt")),
            "sub-in-fmt": (10, ("mflux", "T")), "sub-out-fp": (11, ("p",)), "sup-out-fn": (12, ())}
BC_INLETS = ("sub-in-fvt", "sup-in-fa", "sub-in-ftptt", "sub-in-fmt")

_NP_FUNCS = dict(sin=np.sin, cos=np.cos, tan=np.tan, exp=np.exp, log=np.log, sqrt=np.sqrt, tanh=np.tanh,
                 abs=np.abs, min=np.minimum, max=np.maximum, pow=np.power)


def bc_value(value, x, y, z, t):
    """A bcvals value at face centres x, y, z and time t: a number, or an
    expression of x, y, z and t (peregrine/simulator/bcs.py:101-143) evaluated
    here by numpy, on its own, as the reference's compiled C++ would."""
    if not isinstance(value, str):
        return np.full(x.shape, float(value))
    names = dict(x=x, y=y, z=z, t=t)

    def ev(node):
        if isinstance(node, ast.Constant):
            return float(node.value)
        if isinstance(node, ast.Name):
            return names[node.id]
        if isinstance(node, ast.UnaryOp):
            return -ev(node.operand) if isinstance(node.op, ast.USub) else ev(node.operand)
        if isinstance(node, ast.BinOp):
            a, b = ev(node.left), ev(node.right)
            if isinstance(node.op, ast.Pow):
                return np.power(a, b)
            return {ast.Add: np.add, ast.Sub: np.subtract, ast.Mult: np.multiply, ast.Div: np.divide}[type(node.op)](a, b)
        if isinstance(node, ast.Call):
            return _NP_FUNCS[node.func.id](*[ev(a) for a in node.args])
        raise ValueError(f"{value!r}: {type(node).__name__}")

    return np.broadcast_to(np.asarray(ev(ast.parse(value, mode="eval").body), dtype=np.float64), x.shape)


def stage_fractions(integrator):
    """Each stage's time as a fraction of dt past the step's start
    (peregrine/integrators/rungekutta.py:28-39: stage n's right-hand side runs
    at the n-th stage table row's fraction)."""
    return {"rk1": (0.0,), "rk2": (0.0, 1.0), "tvd-rk3": (0.0, 1.0, 0.5), "rk34": (0.0, 0.5, 1.0, 0.5),
            "rk4": (0.0, 0.5, 0.5, 1.0)}[integrator]

NSTATE = 24  # the oracle's per-cell record: EosState, Z, the double flux's plane


MAXSIDE = 8


class ORxn(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("kind", "reversible", "product", "tb", "troe", "nfcent", "nfwd", "nreact",
                                            "nprod", "nnet")] + \
               [(n, ctypes.c_int * MAXSIDE) for n in ("fwdsp", "reactsp", "prodsp", "netsp")] + \
               [(n, ctypes.c_double * MAXSIDE) for n in ("fwdorder", "reactnu", "prodnu", "netnu", "netnuMW")] + \
               [(n, ctypes.c_double) for n in ("logA", "b", "EaR", "logprA", "prb", "prEaR", "nusum")]


class OTb(ctypes.Structure):
    _fields_ = [("defeff", ctypes.c_double), ("neff", ctypes.c_int), ("effsp", ctypes.c_int * 16),
                ("effdev", ctypes.c_double * 16)]


class OMech(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nr", "ntb", "nlfc", "ng")] + \
               [("rxn", ctypes.POINTER(ORxn)), ("tb", ctypes.POINTER(OTb)),
                ("lfcpoly", ctypes.POINTER(ctypes.c_double)), ("gpoly", ctypes.POINTER(ctypes.c_double)),
                ("h298", ctypes.POINTER(ctypes.c_double)), ("logform", ctypes.c_int), ("product", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in ("logprefRu", "prefRu", "Rupref", "logcfloor", "maxgain", "troeuc",
                                               "troeuhinv", "expclamp", "lfcfloor")]


class OBlock(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("ng", ctypes.c_int),
                ("Q", ctypes.POINTER(ctypes.c_double)),
                ("xcc", ctypes.POINTER(ctypes.c_double)), ("detJinv", ctypes.POINTER(ctypes.c_double)),
                ("Jinv", ctypes.POINTER(ctypes.c_double)),
                ("S", ctypes.POINTER(ctypes.c_double) * 3), ("xf", ctypes.POINTER(ctypes.c_double) * 3),
                ("Tg", ctypes.POINTER(ctypes.c_double)), ("pst", ctypes.POINTER(ctypes.c_double)),
                ("subs", ctypes.POINTER(ctypes.c_int))]


def _side(sp, val):
    """A padded row's real entries: those with a nonzero value (the padding is (0, 0))."""
    return [(int(a), float(b)) for a, b in zip(sp, val) if b != 0.0]


def build_mech(consts):
    """The finite-rate tables of a mixture's constants as the oracle's structs
    (the columns of FiniteRateModel.rxnconsts and its third-body sets)."""
    import math

    nr = int(consts["rxn_nr"])
    rxns = (ORxn * max(nr, 1))()
    for k in range(nr):
        r = rxns[k]
        r.kind, r.reversible, r.product = (int(consts["rxn_kind"][k]), int(consts["rxn_reversible"][k]),
                                           int(consts["rxn_product"][k]))
        r.tb, r.troe, r.nfcent = int(consts["rxn_tb"][k]), int(consts["rxn_troeidx"][k]), int(consts["rxn_nfcent"][k])
        for name, sp, val in (("fwd", "rxn_fwdsp", "rxn_fwdorder"), ("react", "rxn_reactsp", "rxn_reactnu"),
                              ("prod", "rxn_prodsp", "rxn_prodnu")):
            row = _side(consts[sp][k], consts[val][k])
            setattr(r, "n" + name, len(row))
            for j, (a, b) in enumerate(row):
                getattr(r, name + "sp")[j] = a
                getattr(r, {"fwd": "fwdorder", "react": "reactnu", "prod": "prodnu"}[name])[j] = b
        net = [(int(a), float(b), float(c)) for a, b, c in
               zip(consts["rxn_netsp"][k], consts["rxn_netnu"][k], consts["rxn_netnuMW"][k]) if b != 0.0]
        r.nnet = len(net)
        for j, (a, b, c) in enumerate(net):
            r.netsp[j], r.netnu[j], r.netnuMW[j] = a, b, c
        for name in ("logA", "b", "EaR", "logprA", "prb", "prEaR", "nusum"):
            setattr(r, name, float(consts["rxn_" + name][k]))
    ntb = len(consts["tbdefeff"])
    tbs = (OTb * max(ntb, 1))()
    for j in range(ntb):
        tbs[j].defeff = float(consts["tbdefeff"][j])
        n = int(consts["tb_neff"][j])
        tbs[j].neff = n
        for i in range(n):
            tbs[j].effsp[i] = int(consts["tb_effsp"][j][i])
            tbs[j].effdev[i] = float(consts["tbeffdev"][j][i])
    keep = dict(rxns=rxns, tbs=tbs, lfc=np.ascontiguousarray(consts["rxnlfcpoly"], dtype=np.float64).reshape(-1),
                gpoly=np.ascontiguousarray(consts["gpoly"], dtype=np.float64),
                h298=np.ascontiguousarray(consts["h298"], dtype=np.float64))
    m = OMech()
    m.nr, m.ntb = nr, ntb
    m.nlfc = int(np.asarray(consts["rxnlfcpoly"]).shape[-1]) if np.asarray(consts["rxnlfcpoly"]).size else 0
    m.ng = int(keep["gpoly"].shape[1])
    m.rxn, m.tb = ctypes.cast(rxns, ctypes.POINTER(ORxn)), ctypes.cast(tbs, ctypes.POINTER(OTb))
    m.lfcpoly, m.gpoly, m.h298 = _ptr(keep["lfc"]), _ptr(keep["gpoly"]), _ptr(keep["h298"])
    product = consts["rxn_product"][:nr]
    m.logform, m.product = int(not np.all(product == 1)), int(np.any(product == 1))
    for name in ("logprefRu", "prefRu", "Rupref", "logcfloor", "maxgain", "troeuc", "troeuhinv"):
        setattr(m, name, float(consts[name]))
    m.expclamp = math.log(float(np.finfo(np.float64).max)) - math.log(2.0 * float(consts["maxgain"]))
    m.lfcfloor = math.log(float(np.finfo(np.float64).tiny)) * 0.4342944819032518
    keep["mech"] = m
    return keep


# the case size from which the oracle's loops share the host's cores
SMALL = 1 << 16


def _lib():
    if not os.path.exists(LIB):
        raise RuntimeError(f"{LIB} is not built; run oracle/build.sh")
    lib = ctypes.CDLL(LIB)
    lib.oracle_rhs.restype = ctypes.c_int
    lib.oracle_fromprims.restype = ctypes.c_int
    lib.oracle_combine.restype = ctypes.c_int
    lib.oracle_kepaec_faces.restype = ctypes.c_int
    lib.oracle_advective_faces.restype = ctypes.c_int
    for name in ("oracle_production", "oracle_gibbs", "oracle_tlog", "oracle_texp", "oracle_mathtables",
                 "oracle_species_cph", "oracle_fromQ", "oracle_prestep", "oracle_realgas_frompT",
                 "oracle_realgas_fromQ", "oracle_freeze", "oracle_bc_grads", "oracle_cflmax", "oracle_transport",
                 "oracle_exchange"):
        getattr(lib, name).restype = ctypes.c_int
    return lib


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def halo_map(blocks, rots=None):
    """Every face-halo cell of every block and the neighbour cell it copies.

    A face's halo layer l is the neighbour's l-th cell in from the face it
    meets, the neighbour's cells laid out along this block's axes by the
    face's orientation digits (peregrine/multiblock/interface/base.py:96-160).
    rots, a list, gathers the rotational periodics' rotations: an entry's rot
    is 1 + its index there, 0 for none.
    """
    rows = []
    for blk in blocks:
        g = blk.ng
        n = blk.cells
        for face in blk.intfaces:
            if face.nbr is None:
                continue
            a = face.axis
            nbr = blocks[face.nbr]
            # the neighbour's own cell indices, halo included (as wide on every
            # side), laid out along this block's axes
            idx = np.stack(np.meshgrid(*[np.arange(c + 2 * g) for c in nbr.cells], indexing="ij"), axis=-1)
            view = face.inframe(idx)
            assert all(view.shape[d] == n[d] + 2 * g for d in range(3) if d != a), "the faces do not match"
            rot = 0
            if getattr(face, "rotperiodic", False) and rots is not None:
                rots.append(np.asarray(face.rot, np.float64))
                rot = len(rots)
            other = [d for d in range(3) if d != a]
            grid = np.meshgrid(*[np.arange(g, g + n[d]) for d in other], indexing="ij")
            for layer in range(g):
                dst = [None] * 3
                for d, gd in zip(other, grid):
                    dst[d] = gd.ravel()
                cnt = dst[other[0]].size
                sel = [slice(g, g + n[d]) for d in range(3)]
                if face.is_low:
                    dst[a] = np.full(cnt, g - 1 - layer)
                    sel[a] = view.shape[a] - g - 1 - layer
                else:
                    dst[a] = np.full(cnt, g + n[a] + layer)
                    sel[a] = g + layer
                src = view[tuple(sel)].reshape(-1, 3)
                r = np.zeros(cnt, _halo_dtype)
                r["dblk"], r["sblk"], r["layer"], r["rot"] = blk.nblki, face.nbr, layer, rot
                r["di"], r["dj"], r["dk"] = dst
                r["si"], r["sj"], r["sk"] = src[:, 0], src[:, 1], src[:, 2]
                rows.append(r)
    return np.concatenate(rows) if rows else np.zeros(0, _halo_dtype)


def stage_combines(integrator, nregs_names):
    """Each stage's combines as (out, own weight or None, [(register, weight)], step).

    The reference's combine bookkeeping (peregrine/integrators/base.py:122-137)
    on its stage tables (peregrine/integrators/rungekutta.py:42-92).
    """
    def combine(out, pairs, step=True):
        weights = {}
        for reg, w in pairs:
            weights[reg] = weights.get(reg, 0.0) + w
        own = weights.pop(out, 0.0)
        reads = [(r, w) for r, w in weights.items() if w != 0.0]
        return (out, own if own != 0.0 else None, reads, step)

    R = nregs_names
    if integrator == "rk4":
        start, stage, total, dQ = R
        rows = ((0.0, 0.5, 1.0 / 6.0), (0.5, 0.5, 1.0 / 3.0), (0.5, 1.0, 1.0 / 3.0), (1.0, None, 1.0 / 6.0))
        out = []
        for n, (_, wdQ, wsum) in enumerate(rows):
            q = start if n == 0 else stage
            share = combine(total, [(total, 0.0 if n == 0 else 1.0), (dQ, wsum)])
            if wdQ is None:
                last = combine(start, [(start, 1.0), (total, 1.0)], step=False)
            else:
                last = combine(stage, [(start, 1.0), (dQ, wdQ)])
            out.append((q, [share, last]))
        return out, dQ
    tables = {
        "rk1": ((0.0, 0.0, 1.0, 1.0),),
        "rk2": ((0.0, 0.0, 1.0, 1.0), (1.0, 0.5, 0.5, 0.5)),
        "tvd-rk3": ((0.0, 0.0, 1.0, 1.0), (1.0, 0.75, 0.25, 0.25), (0.5, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)),
        "rk34": ((0.0, 0.0, 1.0, 0.5), (0.5, 0.0, 1.0, 0.5), (1.0, 2.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0), (0.5, 0.0, 1.0, 0.5)),
    }
    stages = tables[integrator]
    start, stage, dQ = R[0], R[1], R[-1]
    last = len(stages) - 1
    out = []
    for n, (_, wQ0, wQ, wdQ) in enumerate(stages):
        Q = start if n == 0 else stage
        Qout = start if n == last else stage
        out.append((Q, [combine(Qout, [(Q, wQ), (start, wQ0), (dQ, wdQ)])]))
    return out, dQ


NREGS = {"rk1": 2, "rk2": 3, "tvd-rk3": 3, "rk34": 3, "rk4": 4}


class Oracle:
    """The reference's right-hand side and stepping, on host arrays.

    ``blocks`` are mesher blocks (nodes and connectivity); ``metrics`` one dict
    per block of the arrays ``peregrine_b200.grid.metrics`` makes.
    """

    PRIMARY = {"kepaec": 0, "hllc": 1, "rusanov": 2, "ausmup": 3}
    LIMITERS = {None: 0, "koren": 1, "minmod": 2, "mc": 3, "superbee": 4, "vanleer": 5}

    def __init__(self, constants, ns, simulator, blocks, metrics, integrator="rk4", alpha=1.0, primary="kepaec",
                 recon="constant", limiter=None, eos="cpg", trans="constant", chemistry=None, bcvals=None,
                 species=None, chemint="coupled", max_substeps=200, eqtol=1e-7, mixrule="wilke"):
        """constants: the mixture's tables; blocks/metrics may be empty for face-only use.
        eos "cpg" or "tpg", trans "constant" or "kinetic-theory", chemistry
        None or "finite-rate" (coupled: the source begins dQ).  bcvals: the
        config's boundary entries, by the name each boundary face carries
        (face.bcname); species: the mixture's species names, for the
        inflows' mass fractions.  A boundary face without a name keeps its
        halo as set."""
        self.lib = _lib()
        self.ns, self.ne = ns, 4 + ns
        self.blocks = blocks
        self.metrics = [{k: np.ascontiguousarray(v, dtype=np.float64) for k, v in m.items()} for m in metrics]
        self.integrator = integrator
        self._tables = {}
        c = OCase()
        c.simulator = 1 if simulator in ("navier-stokes", "navier-stokes-df") else 0
        c.primary = self.PRIMARY[primary]
        c.recon = 1 if recon == "muscl" else 0
        c.limiter = self.LIMITERS[limiter]
        c.ns = ns
        c.alpha = alpha
        c.Ru = float(constants["Ru"])
        names = dict(Rsp="Rsp", cp0="cp0", h298R="h298R", MWinv="MWinv", h298="h298",
                     mu0="mu0", kappa0="kappa0", MWqinv="MWqinv", wilkepair="wilkepair", lewis="lewis")
        for field, key in names.items():
            arr = np.ascontiguousarray(constants.get(key, np.ones(ns)), dtype=np.float64).ravel()
            self._tables[field] = arr
            setattr(c, field, _ptr(arr))
        hp = np.ascontiguousarray(np.asarray(constants["hpoly"])[:, 0], dtype=np.float64)
        self._tables["hpoly0"] = hp
        c.hpoly0 = _ptr(hp)
        if eos in ("real-gas", "real-gas-df"):
            c.realgas, c.df = 1, int(eos == "real-gas-df")
            for name in ("cu", "cw", "csigma", "ceps"):
                setattr(c, name, float(constants["cubic" + name[1:]]))
            keys = dict(csqrtac="cubicsqrtac", cb="cubicb", cda="cubicda", cmTc="cubicmTc", conepm="cubiconepm",
                        vshift="vshift", csqrtacMW="cubicsqrtacMW", cbMW="cubicbMW", cdaMW="cubicdaMW",
                        vshiftMW="vshiftMW")
            for field, key in keys.items():
                arr = np.ascontiguousarray(constants[key], dtype=np.float64).ravel()
                self._tables[field] = arr
                setattr(c, field, _ptr(arr))
        if eos != "cpg":
            c.eos = 1
            cpr = np.ascontiguousarray(constants["cppolyR"], dtype=np.float64)
            hpoly = np.ascontiguousarray(constants["hpoly"], dtype=np.float64)
            self._tables["cppolyR"], self._tables["hpoly"] = cpr, hpoly
            c.ncp, c.cppolyR = cpr.shape[1], _ptr(cpr)
            c.nh, c.hpoly = hpoly.shape[1], _ptr(hpoly)
        if "pairfit" in constants and trans is not None:
            # binary diffusion, the mixture's pair fits (a table set made for it)
            ns_ = ns
            self_ = np.ascontiguousarray(constants["selffit"], dtype=np.float64)
            pair = np.ascontiguousarray(constants["pairfit"], dtype=np.float64)
            bath = np.ascontiguousarray(np.asarray(constants["bath"]).astype(np.int32))
            mw = np.ascontiguousarray(constants["MW"], dtype=np.float64)
            self._tables.update(selffit=self_, pairfit=pair, MWb=mw)
            self._bath = bath
            c.binary, c.nfit = 1, self_.shape[1]
            c.bpartial = int(len(bath) < ns_)
            c.bwidth = len(bath) if c.bpartial else ns_ - 1
            c.pairfit, c.selffit, c.MW = _ptr(pair), _ptr(self_), _ptr(mw)
            c.bath = bath.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        if mixrule == "herning":
            # Herning's viscosity mixing rule (peregrine/simulator/mixture/mixrule/herning.py)
            sq = np.ascontiguousarray(np.sqrt(1.0 / np.asarray(constants["MWinv"], dtype=np.float64)))
            self._tables["sqrtMW"] = sq
            c.herning, c.sqrtMW = 1, _ptr(sq)
        if trans == "kinetic-theory":
            c.trans = 1
            mu = np.ascontiguousarray(constants["mupoly"], dtype=np.float64)
            ka = np.ascontiguousarray(constants["kappapoly"], dtype=np.float64)
            self._tables["mupoly"], self._tables["kappapoly"] = mu, ka
            c.nmu, c.mupoly, c.nkappa, c.kappapoly = mu.shape[1], _ptr(mu), ka.shape[1], _ptr(ka)
        self._mech = None
        if chemistry == "finite-rate":
            self._mech = build_mech(constants)
            c.mech = ctypes.cast(ctypes.pointer(self._mech["mech"]), ctypes.c_void_p)
        # the sub-stepped integration (chemint "sub-stepped"): the one-pass form
        # with max_substeps and the exit's tolerance eqtol, over the step dt
        self.substepped = chemistry == "finite-rate" and chemint == "sub-stepped"
        self.dt = 0.0
        if self.substepped:
            c.substepped, c.cap, c.eqtol = 1, int(max_substeps), float(eqtol)
            cpp = np.ascontiguousarray(constants["cppoly"], dtype=np.float64)
            mw = np.ascontiguousarray(constants["MW"], dtype=np.float64)
            self._tables["cppoly"], self._tables["MW"] = cpp, mw
            c.ncppoly, c.cppoly, c.MW = cpp.shape[1], _ptr(cpp), _ptr(mw)
            c.cfloor = float(np.exp(float(constants["logcfloor"])))
        self.case = c
        # one thread below SMALL cells in all (a test's case), every core above
        cells = sum(int(np.prod([n + 2 * b.ng for n in b.cells])) for b in blocks)
        self.threads = 1 if cells < SMALL else (os.cpu_count() or 1)
        self._rots = []
        self.map = halo_map(blocks, self._rots)
        if self._rots:
            self._tables["rots"] = np.ascontiguousarray(np.stack(self._rots), dtype=np.float64)
            c.rots = _ptr(self._tables["rots"])
        self.nregs = NREGS[integrator]
        self.regs = [[np.zeros(self._shape(b)) for b in blocks] for _ in range(self.nregs)]
        # each cell's last temperature, the iterative eos's starting guess
        self.Tg = [np.zeros(self._shape(b)[:3]) for b in blocks]
        # the double flux's kept records (state and frozen plane), and whether
        # the planes are yet to be frozen for the state set
        self.df = eos == "real-gas-df"
        self.pst = [np.zeros(self._shape(b)[:3] + (NSTATE,)) for b in blocks] if self.df else None
        self.df_fresh = True
        self.tme = 0.0
        self.subs = [np.zeros(self._shape(b)[:3], dtype=np.int32) for b in blocks] if self.substepped else None
        self.bcvals = dict(bcvals or {})
        self.species = list(species or [])
        self.bcfaces = []
        for blk in blocks:
            for face in blk.intfaces:
                if face.nbr is None and face.bcname is not None:
                    if face.bcname not in self.bcvals:
                        raise ValueError(f"block {blk.nblki} face {face.nface}: {face.bcname!r} is not in bcvals")
                    self.bcfaces.append((blk, face))

    def _bcs(self, t):
        """The boundary faces with their values at the face centres and time t."""
        rows = (OBc * max(1, len(self.bcfaces)))()
        keep = []
        for m, (blk, face) in enumerate(self.bcfaces):
            given = self.bcvals[face.bcname]
            kind, variables = BC_KINDS[given["kind"]]
            names = list(variables)
            if given["kind"] in BC_INLETS:
                names += self.species[:self.ns - 1]
            a, g, n = face.axis, blk.ng, blk.cells
            xc = self.metrics[blk.nblki]["ijk"[a] + "xc"]
            at = [slice(g, g + n[d]) for d in range(3)]
            at[a] = g if face.is_low else g + n[a]
            plane = xc[tuple(at)]
            x, y, z = plane[..., 0], plane[..., 1], plane[..., 2]
            cols = [bc_value(given.get(v, 0.0) if v not in variables else given[v], x, y, z, t) for v in names]
            vals = np.ascontiguousarray(np.stack(cols, -1) if cols else np.zeros(x.shape + (1,)), dtype=np.float64)
            keep.append(vals)
            r = rows[m]
            r.blk, r.nface, r.kind, r.nval = blk.nblki, face.nface, kind, max(1, len(names))
            r.vals = _ptr(vals)
        return rows, keep

    def _shape(self, blk):
        return tuple(n + 2 * blk.ng for n in blk.cells) + (self.ne,)

    def _oblocks(self, Q):
        self.lib.oracle_set_threads(self.threads)
        obs = (OBlock * len(self.blocks))()
        keep = []
        for n, (blk, m) in enumerate(zip(self.blocks, self.metrics)):
            o = obs[n]
            o.nx, o.ny, o.nz = blk.cells
            o.ng = blk.ng
            o.Q = _ptr(Q[n])
            o.xcc, o.detJinv, o.Jinv = _ptr(m["xcc"]), _ptr(m["detJinv"]), _ptr(m["Jinv"])
            for a, d in enumerate("ijk"):
                o.S[a] = _ptr(m[f"{d}S"])
                o.xf[a] = _ptr(m[f"{d}xc"])
            o.Tg = _ptr(self.Tg[n])
            if self.pst is not None:
                o.pst = _ptr(self.pst[n])
            if self.subs is not None:
                o.subs = self.subs[n].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            keep.append(o)
        return obs

    def set_prims(self, prims):
        for n, (q, Q) in enumerate(zip(prims, self.regs[0])):
            q = np.ascontiguousarray(q, dtype=np.float64)
            assert q.shape == Q.shape
            self.lib.oracle_fromprims(ctypes.byref(self.case), _ptr(q), _ptr(Q), ctypes.c_long(Q.size // self.ne),
                                      _ptr(self.Tg[n]))
        self.df_fresh = True
        # a halo cell's first Newton starts from the stored T of the cell it
        # copies, as the device's set_prims leaves it
        m = self.map
        for r in m:
            self.Tg[r["dblk"]][r["di"], r["dj"], r["dk"]] = self.Tg[r["sblk"]][r["si"], r["sj"], r["sk"]]

    def production(self, rho, Y, T):
        """omega[n, ns] of independent states, rho[n], Y[n, ns] every species, T[n]."""
        rho, Y, T = (np.ascontiguousarray(x, dtype=np.float64) for x in (rho, Y, T))
        out = np.zeros_like(Y)
        self.lib.oracle_production(ctypes.byref(self.case), ctypes.c_long(len(T)), _ptr(rho), _ptr(Y), _ptr(T),
                                   _ptr(out))
        return out

    def gibbs(self, T):
        T = np.ascontiguousarray(T, dtype=np.float64)
        out = np.zeros((len(T), self.ns))
        self.lib.oracle_gibbs(ctypes.byref(self.case), ctypes.c_long(len(T)), _ptr(T), _ptr(out))
        return out

    def species_cph(self, sp, T):
        T = np.ascontiguousarray(T, dtype=np.float64)
        cp, h = np.zeros_like(T), np.zeros_like(T)
        self.lib.oracle_species_cph(ctypes.byref(self.case), sp, ctypes.c_long(len(T)), _ptr(T), _ptr(cp), _ptr(h))
        return cp, h

    def fromQ(self, Q, Tguess):
        """the state (p, T, rhoinv, rho, e, cp, gamma, c) of Q rows, each from its guess."""
        Q, Tg = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, Tguess))
        out = np.zeros((len(Tg), 8))
        self.lib.oracle_fromQ(ctypes.byref(self.case), ctypes.c_long(len(Tg)), _ptr(Q), _ptr(Tg), _ptr(out))
        return out

    def rhs(self, Q, dQ, faces=False, diffusive_only=False, t=None):
        """dQ of every block from Q; with faces, each block's [iF, jF, kF] too.
        t: the time the boundary values read (the oracle's clock if None)."""
        # the double flux's first freeze before this pass's boundary rows are
        # set: the freeze sets (and lets go of) its own
        if self.df and self.df_fresh:
            self.prestep(Q)
        obs = self._oblocks(Q)
        bcs, keep = self._bcs(self.tme if t is None else t)
        self.case.nbc, self.case.bc = len(self.bcfaces), bcs
        self.case.dt = self.dt
        m = np.ascontiguousarray(self.map)
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(dQ))(*[_ptr(d) for d in dQ])
        fl, fptr = None, None
        if faces:
            fl = []
            nf = self.ne + (1 if self.df else 0)
            for blk in self.blocks:
                for a in range(3):
                    shape = [n + 2 * blk.ng for n in blk.cells]
                    shape[a] += 1
                    fl.append(np.zeros(tuple(shape) + (nf,)))
            fptr = (ctypes.POINTER(ctypes.c_double) * len(fl))(*[_ptr(f) for f in fl])
        self.case.skip_adv = int(diffusive_only)
        rc = self.lib.oracle_rhs(ctypes.byref(self.case), obs, len(self.blocks),
                                 m.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(m.size), ptrs, fptr)
        self.case.skip_adv = 0
        if rc:
            raise RuntimeError(f"oracle_rhs: {rc}")
        if faces:
            return [fl[3 * b:3 * b + 3] for b in range(len(self.blocks))]

    def cflmax(self, Q=None):
        """(acoustic, convective, combined): the largest CFL number per unit
        step of each over every block's interior of register Q (regs[0])."""
        obs = self._oblocks(self.regs[0] if Q is None else Q)
        out = np.zeros(3)
        self.lib.oracle_cflmax(ctypes.byref(self.case), obs, len(self.blocks), _ptr(out))
        return dict(zip(("acoustic", "convective", "combined"), out))

    def transport(self, Q, state):
        """(mu, kappa, D[ns]) rows of Q rows at their states (8-wide EosState rows)."""
        Q, st = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, state))
        out = np.zeros((len(Q), 2 + self.ns))
        self.lib.oracle_transport(ctypes.byref(self.case), ctypes.c_long(len(Q)), _ptr(Q), _ptr(st), _ptr(out))
        return out

    def bc_grads(self, grads, t=None):
        """The boundaries' gradient hook alone on grads[b] ([X][Y][Z][ngrad][3]
        per block), in place."""
        bcs, keep = self._bcs(self.tme if t is None else t)
        self.case.nbc, self.case.bc = len(self.bcfaces), bcs
        obs = self._oblocks(self.regs[0])
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(grads))(*[_ptr(g) for g in grads])
        self.lib.oracle_bc_grads(ctypes.byref(self.case), obs, ptrs)

    def advective_faces(self, QLL, QL, QR, QRR, S):
        """The advective flux on independent faces from their four cells' Q."""
        Q4 = np.ascontiguousarray(np.stack([QLL, QL, QR, QRR]), dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.float64)
        F = np.zeros_like(Q4[0])
        self.lib.oracle_advective_faces(ctypes.byref(self.case), ctypes.c_long(S.shape[0]), _ptr(Q4), _ptr(S), _ptr(F))
        return F


    def kepaec_faces(self, QL, QR, S):
        """kepaec on independent faces, each side's state from its Q."""
        QL, QR, S = (np.ascontiguousarray(x, dtype=np.float64) for x in (QL, QR, S))
        F = np.zeros_like(QL)
        self.lib.oracle_kepaec_faces(ctypes.byref(self.case), ctypes.c_long(QL.shape[0]), _ptr(QL), _ptr(QR), _ptr(S), _ptr(F))
        return F

    def exchange(self, Q=None):
        """Register Q's halo filled across every interface, a rotational
        periodic's vectors turned (the reference's exchange of a bank)."""
        Q = self.regs[0] if Q is None else Q
        obs = self._oblocks(Q)
        m = np.ascontiguousarray(self.map)
        self.lib.oracle_exchange(ctypes.byref(self.case), obs, len(self.blocks), m.ctypes.data_as(ctypes.c_void_p),
                                 ctypes.c_long(m.size))

    def prestep(self, Q):
        """The double flux's freeze on register Q: off the eos once after the
        state was set, off the frozen planes at every step's start."""
        obs = self._oblocks(Q)
        m = np.ascontiguousarray(self.map)
        # the boundaries' halo cells at the step's start, frozen with the rest
        bcs, keep = self._bcs(self.tme)
        self.case.nbc, self.case.bc = len(self.bcfaces), bcs
        self.lib.oracle_prestep(ctypes.byref(self.case), obs, len(self.blocks), m.ctypes.data_as(ctypes.c_void_p),
                                ctypes.c_long(m.size), int(self.df_fresh))
        self.df_fresh = False

    def realgas_frompT(self, p, T, Y):
        """Records [n, NSTATE] of the real gas at (p, T, Y carried) points."""
        p, T, Y = (np.ascontiguousarray(x, dtype=np.float64) for x in (p, T, Y))
        out = np.zeros((len(p), NSTATE))
        self.lib.oracle_realgas_frompT(ctypes.byref(self.case), ctypes.c_long(len(p)), _ptr(p), _ptr(T), _ptr(Y),
                                       _ptr(out))
        return out

    def realgas_fromQ(self, Q, Tguess):
        Q, Tg = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, Tguess))
        out = np.zeros((len(Tg), NSTATE))
        self.lib.oracle_realgas_fromQ(ctypes.byref(self.case), ctypes.c_long(len(Tg)), _ptr(Q), _ptr(Tg), _ptr(out))
        return out

    def freeze(self, Q, rec):
        """Freeze at independent cells: Q's energy and rec's planes in place."""
        assert Q.flags["C_CONTIGUOUS"] and rec.flags["C_CONTIGUOUS"]
        self.lib.oracle_freeze(ctypes.byref(self.case), ctypes.c_long(len(Q)), _ptr(Q), _ptr(rec))

    def step(self, dt, before_stage=None):
        """One step; before_stage(register), when given, runs before each
        stage's right-hand side on the register it reads (a shard's halo
        trade, tests/test_shard_cpu.py)."""
        names = list(range(self.nregs))
        stages, dQ = stage_combines(self.integrator, names)
        start = self.tme
        fracs = stage_fractions(self.integrator)
        self.dt = dt
        if self.df:
            if self.df_fresh:
                self.prestep(self.regs[stages[0][0]])
            self.prestep(self.regs[stages[0][0]])
        for n, (Q, combines) in enumerate(stages):
            if before_stage is not None:
                before_stage(self.regs[Q])
            self.rhs(self.regs[Q], self.regs[dQ], t=start + fracs[n] * dt)
            for out, own, reads, step in combines:
                for b, blk in enumerate(self.blocks):
                    X = (ctypes.POINTER(ctypes.c_double) * len(reads))(*[_ptr(self.regs[r][b]) for r, _ in reads])
                    w = (ctypes.c_double * len(reads))(*[wt for _, wt in reads])
                    self.lib.oracle_combine(*blk.cells, blk.ng, self.ne, _ptr(self.regs[out][b]),
                                            int(own is not None), ctypes.c_double(own or 0.0),
                                            len(reads), X, w, int(step), ctypes.c_double(dt))
        self.tme = start + dt


def tlog(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    _lib().oracle_tlog(ctypes.c_long(x.size), _ptr(x), _ptr(y))
    return y


def texp(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    _lib().oracle_texp(ctypes.c_long(x.size), _ptr(x), _ptr(y))
    return y


def mathtables():
    lt, rt, et, sc = np.zeros(128), np.zeros(128), np.zeros(64), np.zeros(4)
    _lib().oracle_mathtables(_ptr(lt), _ptr(rt), _ptr(et), _ptr(sc))
    return lt, rt, et, sc
