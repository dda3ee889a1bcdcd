"""Boundary conditions on the CPU: the bcvals compiler and the oracle's halos.

The oracle's boundary kinds are checked against the rules the reference's own
boundary tests hold each kind to (tests/bcs/test_walls.py, test_inlets.py,
test_exits.py, test_expressions.py): on a jostled box whose every face
carries one entry, each halo layer is the entry's value where the kind
imposes it, the first cell's where it copies, 2 first - deeper where it
extrapolates, the image reflected where it mirrors.  The expression compiler
is checked by running its programs on a model of the device's stack machine
against numpy's evaluation of the same text.
"""

import numpy as np
import pytest

from oracle.oracle import Oracle, bc_value
from peregrine_b200 import bcs as bcmod
from peregrine_b200 import cases, native
from peregrine_b200.config import ConfigError
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mixture import Mixture


def box(kind, ns=1, simulator="euler", primary="kepaec", recon="constant", limiter=None, entry=None, seed=0,
        cells=(7, 5, 3)):
    cfg = cases.bc_box_config(kind, ns=ns, simulator=simulator, primary=primary, recon=recon, limiter=limiter,
                              seed=seed, entry=entry)
    mix = Mixture(cfg["mixture"])
    blocks = cases.bc_box_mesh(cells=cells).make_blocks(2)
    mets = [make_metrics(b.nodes, b.ng) for b in blocks]
    orc = Oracle(mix.constants(), mix.ns, simulator, blocks, mets, "rk4", primary=primary, recon=recon,
                 limiter=limiter, trans="constant" if simulator == "navier-stokes" else "constant",
                 bcvals=cfg["bcvals"], species=mix.spnames)
    orc.set_prims(cases.bc_box_prims(mets, mix.ns, seed=seed))
    return cfg, mix, blocks, mets, orc


def run(orc, faces=False, t=0.0):
    dQ = [np.zeros_like(q) for q in orc.regs[0]]
    return orc.rhs(orc.regs[0], dQ, faces=faces, t=t)


class View:
    """The halo layers and interior planes of one face of a block's arrays."""

    def __init__(self, blk, mets, face, orc):
        self.blk, self.face, self.g = blk, face, blk.ng
        Q = orc.regs[0][blk.nblki]
        st = orc.fromQ(Q.reshape(-1, Q.shape[-1]), np.zeros(Q[..., 0].size)).reshape(Q.shape[:3] + (8,))
        self.Q, self.st = Q, st
        a, g, n = face.axis, blk.ng, blk.cells[face.axis]
        S = np.moveaxis(mets[blk.nblki]["ijk"[a] + "S"], a, 0)[g if face.is_low else g + n][g:-g, g:-g]
        self.S = S
        self.n = S / np.linalg.norm(S, axis=-1, keepdims=True)
        self.sign = -1.0 if face.is_low else 1.0

    def _plane(self, arr, k):
        return np.moveaxis(arr, self.face.axis, 0)[k][self.g:-self.g, self.g:-self.g]

    def halo(self, arr, layer):
        n = self.blk.cells[self.face.axis]
        return self._plane(arr, self.g - 1 - layer if self.face.is_low else self.g + n + layer)

    def inner(self, arr, depth):
        n = self.blk.cells[self.face.axis]
        depth = min(depth, n - 1)
        return self._plane(arr, self.g + depth if self.face.is_low else self.g + n - 1 - depth)

    def prim(self, where, name, depth):
        arr = self.halo if where == "halo" else self.inner
        Q, st = arr(self.Q, depth), arr(self.st, depth)
        if name == "p":
            return st[..., 0]
        if name == "T":
            return st[..., 1]
        if name in "uvw":
            return Q[..., 1 + "uvw".index(name)] / Q[..., 0]
        if name == "velo":
            return Q[..., 1:4] / Q[..., :1]
        return Q[..., 5 + int(name[1:])] / Q[..., 0]


def close(got, want, where=None, rtol=1e-10):
    got, want = np.broadcast_arrays(np.asarray(got, float), np.asarray(want, float))
    if where is not None:
        got, want = got[where], want[where]
    assert np.allclose(got, want, rtol=rtol, atol=rtol * max(1.0, np.abs(want).max(initial=0.0)))


def faces_of(blocks, orc, mets):
    return [View(b, mets, f, orc) for b in blocks for f in b.intfaces if f.nbr is None]


WALLS = {
    "slp-adia-wall": dict(sticks=False, moving=False, isothermal=False),
    "slp-isot-wall": dict(sticks=False, moving=False, isothermal=True),
    "no-slp-adia-wall": dict(sticks=True, moving=False, isothermal=False),
    "mov-adia-wall": dict(sticks=True, moving=True, isothermal=False),
    "no-slp-isot-wall": dict(sticks=True, moving=False, isothermal=True),
    "mov-isot-wall": dict(sticks=True, moving=True, isothermal=True),
}


@pytest.mark.parametrize("ns", [1, 3])
@pytest.mark.parametrize("kind", list(WALLS))
def test_wall_halos(kind, ns):
    sim = "euler" if kind in ("slp-adia-wall", "slp-isot-wall") else "navier-stokes"
    cfg, mix, blocks, mets, orc = box(kind, ns=ns, simulator=sim)
    run(orc)
    entry, rule = cfg["bcvals"]["outer"], WALLS[kind]
    wall = np.array([entry[c] for c in "uvw"]) if rule["moving"] else 0.0
    for v in faces_of(blocks, orc, mets):
        for l in range(2):
            uh, ui = v.prim("halo", "velo", l), v.prim("inner", "velo", l)
            if rule["sticks"]:
                close(uh, 2.0 * wall - ui)
            else:
                un = np.sum(ui * v.n, axis=-1, keepdims=True)
                close(uh, ui - 2.0 * un * v.n)
            for n in range(ns - 1):
                close(v.prim("halo", f"Y{n}", l), v.prim("inner", f"Y{n}", l))
            Qh, Qi = v.halo(v.Q, l), v.inner(v.Q, l)
            if not rule["isothermal"]:
                # the adiabatic reflection keeps the density and the internal energy
                assert np.array_equal(Qh[..., 0], Qi[..., 0])
                close(Qh[..., 4] - 0.5 * Qh[..., 0] * np.sum(uh * uh, -1), Qi[..., 4] - 0.5 * Qi[..., 0] * np.sum(ui * ui, -1))
            close(v.prim("halo", "p", l), v.prim("inner", "p", l))
            close(v.prim("halo", "T", l), entry["T"] if rule["isothermal"] else v.prim("inner", "T", l))


def imposed(v, entry, name, spnames=None):
    value = entry[spnames[int(name[1:])]] if name.startswith("Y") else entry[name]
    for l in range(2):
        close(v.prim("halo", name, l), value)


def extrapolated(v, name, lo=None, hi=None, where=None):
    first = v.prim("inner", name, 0)
    for l in range(2):
        want = 2.0 * first - v.prim("inner", name, l + 1)
        if lo is not None or hi is not None:
            want = np.clip(want, -np.inf if lo is None else lo, np.inf if hi is None else hi)
        close(v.prim("halo", name, l), want, where=where)


@pytest.mark.parametrize("ns", [1, 3])
@pytest.mark.parametrize("kind", ["sup-in-fa", "sub-in-fvt", "sub-in-fmt", "sub-in-ftptt"])
def test_inlet_halos(kind, ns):
    cfg, mix, blocks, mets, orc = box(kind, ns=ns)
    run(orc)
    entry = cfg["bcvals"]["outer"]
    for v in faces_of(blocks, orc, mets):
        for n in range(ns - 1):
            imposed(v, entry, f"Y{n}", mix.spnames)
        if kind == "sup-in-fa":
            for c in "puvwT":
                imposed(v, entry, c)
        elif kind == "sub-in-fvt":
            extrapolated(v, "p")
            for c in "uvwT":
                imposed(v, entry, c)
        elif kind == "sub-in-fmt":
            extrapolated(v, "p")
            imposed(v, entry, "T")
        else:
            # along the inward normal, at the isentropic state of the entry's
            # totals from the first cell's outgoing invariant (cpg: h = cp T
            # less a constant that cancels)
            inward = -v.sign * v.n
            st0 = v.inner(v.st, 0)
            gamma, c, T0 = st0[..., 6], st0[..., 7], st0[..., 1]
            u0 = v.prim("inner", "velo", 0)
            carried = np.array([entry[s] for s in mix.spnames[:-1]])
            Y = np.concatenate([carried, [1.0 - carried.sum()]])
            cp = Y @ np.atleast_1d(mix.constants()["cp0"])
            gm1 = gamma - 1.0
            Ht = c * c / gm1 + cp * entry["Tt"] - cp * T0
            Jm = -np.sum(u0 * inward, -1) + 2.0 * c / gm1
            aq, bq, cq = 1.0 + 2.0 / gm1, -2.0 * Jm, gm1 * (0.5 * Jm * Jm - Ht)
            t1, t2 = -bq / (2.0 * aq), np.sqrt(np.maximum(bq * bq - 4.0 * aq * cq, 0.0)) / (2.0 * aq)
            cb = np.maximum(t1 + t2, t1 - t2)
            Vb = 2.0 * cb / gm1 - Jm
            isen = 1.0 + 0.5 * gm1 * (Vb / cb) ** 2
            for l in range(2):
                uh = v.prim("halo", "velo", l)
                close(uh, np.sum(uh * inward, -1, keepdims=True) * inward, rtol=1e-9)
                close(np.sum(uh * inward, -1), Vb, rtol=1e-9)
                close(v.prim("halo", "p", l), entry["pt"] * isen ** (-gamma / gm1), rtol=1e-9)
                close(v.prim("halo", "T", l), entry["Tt"] / isen, rtol=1e-9)


def test_a_mass_flux_inlet_carries_its_mass_flux():
    # kepaec on the constant reconstruction carries exactly the face averages
    # the kind wrote: the mass through each inlet face is mflux |S|
    cfg, mix, blocks, mets, orc = box("sub-in-fmt", ns=3)
    F = run(orc, faces=True)[0]
    mflux = cfg["bcvals"]["outer"]["mflux"]
    blk = blocks[0]
    for face in blk.intfaces:
        v = View(blk, mets, face, orc)
        a, g, n = face.axis, blk.ng, blk.cells[face.axis]
        Fa = np.moveaxis(F[a][..., 0], a, 0)[g if face.is_low else g + n][g:-g, g:-g]
        inward = 1.0 if face.is_low else -1.0
        assert abs(inward * Fa.sum() - mflux * np.linalg.norm(v.S, axis=-1).sum()) < 1e-12 * mflux * np.linalg.norm(v.S, axis=-1).sum()


@pytest.mark.parametrize("ns", [1, 3])
@pytest.mark.parametrize("kind", ["sub-out-fp", "sup-out-fn"])
def test_exit_halos(kind, ns):
    cfg, mix, blocks, mets, orc = box(kind, ns=ns)
    run(orc)
    entry = cfg["bcvals"]["outer"]
    for v in faces_of(blocks, orc, mets):
        un = np.sum(v.prim("inner", "velo", 0) * v.n, -1) * v.sign
        out, back = un > 0.0, un <= 0.0
        assert out.any() and back.any()
        for c in "uvw":
            extrapolated(v, c, where=out)
        for l in range(2):
            ui = v.prim("inner", "velo", l)
            proj = np.sum(ui * v.n, -1, keepdims=True)
            close(v.prim("halo", "velo", l), ui - 2.0 * proj * v.n, where=back)
        if kind == "sub-out-fp":
            imposed(v, entry, "p")
            for l in range(2):
                close(v.prim("halo", "T", l), v.prim("inner", "T", 0))
                for n in range(ns - 1):
                    close(v.prim("halo", f"Y{n}", l), v.prim("inner", f"Y{n}", 0))
        else:
            p, T = v.prim("inner", "p", 0), v.prim("inner", "T", 0)
            extrapolated(v, "p", lo=0.01 * p, hi=p)
            extrapolated(v, "T", lo=0.01 * T)
            for n in range(ns - 1):
                extrapolated(v, f"Y{n}", lo=0.0, hi=1.0)


@pytest.mark.parametrize("kind", ["sub-in-fvt", "sup-in-fa", "sub-in-ftptt", "sub-in-fmt", "sub-out-fp", "sup-out-fn",
                                  "no-slp-adia-wall"])
def test_the_halo_gradients_are_the_images_and_a_walls_untouched(kind):
    # tests/bcs/test_nshooks.py and test_walls.py's gradient hooks: an inflow's
    # or outflow's halo gradients become its images', a wall leaves them (the
    # flux through a wall face is the wall's own)
    cfg, mix, blocks, mets, orc = box(kind, ns=3, simulator="navier-stokes")
    rng = np.random.default_rng(5)
    blk = blocks[0]
    grads = rng.uniform(-1.0, 1.0, orc.regs[0][0].shape[:3] + (mix.ns + 3, 3))
    before = grads.copy()
    orc.bc_grads([grads])
    if kind in WALLS:
        assert np.array_equal(grads, before)
        return
    for face in blk.intfaces:
        v = View(blk, mets, face, orc)
        for l in range(2):
            assert np.array_equal(v.halo(grads, l), v.inner(grads, l))


# -- the clock --------------------------------------------------------------


def test_the_clock_an_expression_reads_is_the_stage_time():
    cfg, mix, blocks, mets, orc = box("sub-in-fvt", entry={"w": "2.0 * t"})
    for t in (0.0, 1.5e-3):
        run(orc, t=t)
        for v in faces_of(blocks, orc, mets):
            for l in range(2):
                close(v.prim("halo", "w", l), 2.0 * t)


def test_a_step_reads_the_stage_times_and_ends_at_start_plus_dt():
    cfg, mix, blocks, mets, orc = box("sub-in-fvt", entry={"w": "2.0 * t"})
    seen = []
    rhs = orc.rhs

    def spy(Q, dQ, faces=False, diffusive_only=False, t=None):
        seen.append(t)
        return rhs(Q, dQ, faces, diffusive_only, t)

    orc.rhs = spy
    orc.tme = 1.0
    orc.step(0.25)
    assert seen == [1.0, 1.125, 1.125, 1.25]
    assert orc.tme == 1.25


# -- the expression compiler ------------------------------------------------


def run_program(ops, args, x, y, z, t):
    """The device's stack machine (include/pgb200.h PGB_OP_*), on numpy arrays."""
    names = {v: k for k, v in native.OPS.items()}
    fn1 = dict(neg=np.negative, sin=np.sin, cos=np.cos, tan=np.tan, exp=np.exp, log=np.log, sqrt=np.sqrt,
               tanh=np.tanh, abs=np.abs)
    fn2 = dict(add=np.add, sub=np.subtract, mul=np.multiply, div=np.divide, pow=np.power, min=np.fmin, max=np.fmax)
    st = []
    for op, arg in zip(ops, args):
        name = names[op]
        if name == "const":
            st.append(np.full(x.shape, arg))
        elif name in "xyzt":
            st.append(np.broadcast_to(dict(x=x, y=y, z=z, t=t)[name], x.shape))
        elif name in fn1:
            st.append(fn1[name](st.pop()))
        else:
            b, a = st.pop(), st.pop()
            st.append(fn2[name](a, b))
    assert len(st) == 1
    return st[0]


EXPRESSIONS = ["101325.0 + 2000.0 * x - 500.0 * z", "sin(3.0 * x) - 2.0 * x * z", "2.0 * t",
               "300.0 + 40.0 * z**2 + max(x, 0.5)", "-x + +y", "pow(x, 2) / (1 + exp(-y)) - log(2 + z) * sqrt(3)",
               "tanh(x) * cos(y) + tan(0.1 * z) - abs(y - x) + min(x, y)", "7", 3.25, "x - y - z", "x / y / 2"]


@pytest.mark.parametrize("text", EXPRESSIONS)
def test_an_expression_compiles_to_its_value(text):
    rng = np.random.default_rng(3)
    x, y, z = (rng.uniform(0.1, 1.0, 40) for _ in range(3))
    e = bcmod.Expression(text)
    got = run_program(e.ops, e.args, x, y, z, 1.5e-3)
    want = bc_value(text, x, y, z, 1.5e-3)
    assert np.allclose(got, want, rtol=1e-15, atol=0.0)


@pytest.mark.parametrize("text", ["q + 1.0", "foo(x)", "x if y else z", "[x, y]", "x @ y", "sin(x, y)", "x % 2"])
def test_what_a_kernel_cannot_evaluate_is_refused(text):
    with pytest.raises(ValueError):
        bcmod.Expression(text)


def test_a_program_deeper_than_the_stack_is_refused():
    deep = "x" + "".join(f" + (x * (y" for _ in range(9)) + ")" * 18
    with pytest.raises(ValueError):
        bcmod.Expression(deep)


# -- the entries and the faces ----------------------------------------------


def test_an_entry_missing_a_value_its_kind_reads_is_refused():
    with pytest.raises(ConfigError):
        bcmod.Entry("inlet", {"kind": "sub-in-fvt", "u": 1.0, "v": 0.0, "w": 0.0}, "euler", ["N2"])


def test_a_viscous_wall_kind_is_refused_on_the_euler_simulator():
    with pytest.raises(ConfigError):
        bcmod.Entry("wall", {"kind": "no-slp-adia-wall"}, "euler", ["N2"])
    with pytest.raises(ConfigError):
        bcmod.Entry("wall", {"kind": "sub-in-sem", "T": 300.0}, "navier-stokes", ["N2"])


def test_an_inlets_species_not_given_are_zero_and_given_ones_in_order():
    e = bcmod.Entry("in", {"kind": "sup-in-fa", "p": 1.0, "u": 2.0, "v": 3.0, "w": 4.0, "T": 5.0, "B": 0.25},
                    "euler", ["A", "B", "C"])
    assert e.names == ["p", "u", "v", "w", "T", "A", "B"]
    kind, ops, args, starts = e.program()
    assert kind == native.BC_KINDS["sup-in-fa"]
    assert starts == list(range(8))
    assert args == [1.0, 2.0, 3.0, 4.0, 5.0, 0.0, 0.25]


def test_an_unnamed_or_unknown_boundary_is_refused():
    blocks = cases.bc_box_mesh(defaultbc=None, bcnames={1: "inlet"}).make_blocks(2)
    with pytest.raises(ValueError, match="did not name"):
        bcmod.check_faces(blocks, {"inlet": {}})
    blocks = cases.bc_box_mesh(defaultbc="wall").make_blocks(2)
    with pytest.raises(ValueError, match="bcvals does not have"):
        bcmod.check_faces(blocks, {"inlet": {}})


# -- the viscous walls' known answers (tests/bcs/test_viscwalls.py) ----------

N, H = 16, 1e-3
DY = H / N
CP, MW = 1005.0, 28.96
# a diffusivity half of a cell's acoustic reach per unit time, at Prandtl one
MU0 = 0.5 * DY * 347.0 * 1.17
KAPPA0 = MU0 * CP
T0, U = 300.0, 100.0


def column(low, high, u0=0.0, integrator="tvd-rk3"):
    """A column of N cells between two walls (the j faces), periodic along i and k."""
    gas = {"Air": {"MW": MW, "cp0": CP, "mu0": MU0, "kappa0": KAPPA0}}
    mix = Mixture({"species": gas, "eos": "cpg", "trans": "constant"})
    mesh = cases.CubeMesher(cells=[[1], [N], [1]], lengths=[DY, H, DY], periodic=[True, False, True],
                            bcnames={3: "low", 4: "high"})
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    orc = Oracle(mix.constants(), 1, "navier-stokes", blocks, mets, integrator, bcvals={"low": low, "high": high},
                 species=mix.spnames)
    q = np.zeros(mets[0]["xcc"].shape[:3] + (5,))
    q[..., 0], q[..., 1], q[..., 4] = 101325.0, u0, T0
    orc.set_prims([q])
    return orc, blocks[0], mets[0]


# the column's fundamental acoustic wave, which only viscosity damps, decays
# twenty-six fold per thousand steps, so eight thousand reach roundoff
def settle(orc, blk, steps=8000):
    g = blk.ng
    Q = orc.regs[0][0]
    st = orc.fromQ(Q[blk.interior].reshape(-1, 5), np.zeros(N))
    dt = 0.3 * DY / st[:, 7].max()
    for _ in range(steps):
        orc.step(dt)
    Q = orc.regs[0][0][g, g:-g, g]
    st = orc.fromQ(np.ascontiguousarray(Q), np.zeros(N))
    return Q, st


def wallflux(orc, blk, mets, row):
    dQ = [np.zeros_like(orc.regs[0][0])]
    F = orc.rhs(orc.regs[0], dQ, faces=True)[0][1]
    g = blk.ng
    S = np.linalg.norm(mets["jS"][g, [g, g + N], g], axis=-1)
    return F[g, g, g, row], F[g, g + N, g, row], S


def test_couette_flow_is_linear_and_heats_the_fluid():
    orc, blk, mets = column({"kind": "no-slp-isot-wall", "T": T0},
                            {"kind": "mov-isot-wall", "u": U, "v": 0.0, "w": 0.0, "T": T0}, u0=0.5 * U)
    Q, st = settle(orc, blk)
    y = mets["xcc"][2, 2:-2, 2, 1]
    u = Q[:, 1:4] / Q[:, :1]
    # linear profiles are exact to roundoff: the alpha-damping gradients are
    # exact on them and the wall halos are their linear extrapolation
    assert np.allclose(u[:, 0], U * y / H, rtol=0.0, atol=1e-12 * U)
    assert np.allclose(u[:, 1:], 0.0, atol=1e-12 * U)
    low, high, S = wallflux(orc, blk, mets, 1)
    assert np.allclose([low, high], -MU0 * U / H * S, rtol=1e-12)
    # the dissipation mu U^2 / h leaves half through each wall; the profile
    # within the two-point wall flux's shift of 1/N^2 of the peak
    peak = MU0 * U * U / (8.0 * KAPPA0)
    want = T0 + MU0 * U * U / (2.0 * KAPPA0) * (y / H) * (1.0 - y / H)
    assert np.abs(st[:, 1] - want).max() <= 2.0 / N ** 2 * peak
    low, high, S = wallflux(orc, blk, mets, 4)
    assert np.allclose([low, high], -MU0 * U * U / (2.0 * H) * S, rtol=1e-10)


def test_conduction_is_linear():
    T1, T2 = 300.0, 400.0
    orc, blk, mets = column({"kind": "no-slp-isot-wall", "T": T1}, {"kind": "no-slp-isot-wall", "T": T2})
    Q, st = settle(orc, blk)
    want = T1 + (T2 - T1) * (np.arange(N) + 0.5) / N
    assert np.allclose(st[:, 1], want, rtol=0.0, atol=1e-12 * (T2 - T1))
    assert np.allclose(Q[:, 1:4] / Q[:, :1], 0.0, atol=1e-11)
    low, high, S = wallflux(orc, blk, mets, 4)
    assert np.allclose([low, high], -KAPPA0 * (T2 - T1) / H * S, rtol=1e-12)
