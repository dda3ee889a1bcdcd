"""The sub-stepped chemistry on the device: the reference's own checks of it
(tests/chemint/test_integration.py, test_equilibrium.py, test_compaction.py)
run through the library, and the device against the CPU oracle.

The checks within the device hold to the bit where the reference's do: one
substep within the bound is the coupled source, the exit leaves an igniting
or unsettled cell alone.  The compacted passes (bulk pass, stiff list,
stiff pass) give the one-pass form to the bit where the stiff pass takes a
cell to a lane (a long list); a short list goes a cell to a warp, its lanes
over the reactions, whose terms then sum in another order: the one-pass
form within the reference's own device bar (tests/gases.py:50-55, rtol 1e-6).  Against the oracle (pinned in
tests/test_substep_cpu.py) the species source is within 1e-9 of the largest
rate and the state after steps within 1e-9 (the species as mass fractions): the
integrator's substep sizes follow the rates, so the device's contracted
arithmetic moves it off the oracle's by more than a rounding but far less
than a substep's truncation.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAS = "ch4_o2_ffcmy"
# the hot half of the duct runs to the cap over this step; over 1e-6 s one substep covers it
STIFF = 1e-5


def config(kind, cap=200, bulk=1, bins=8, eqtol=1e-7, simulator="euler"):
    from peregrine_b200.config import Config

    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"].update(species=GAS, eos="tpg", chemistry="finite-rate",
                          trans="kinetic-theory" if simulator == "navier-stokes" else None)
    cfg["chem-integration"]["kind"] = kind
    cfg["chem-integration"].update({"max-substeps": cap, "bulk-substeps": bulk, "stiff-bins": bins,
                                    "equilibrium-tolerance": eqtol})
    cfg["backend-b200"]["launch"] = "per-block"
    # the substeps' fold walks the mechanism's tables; the coupled source held
    # to it bit for bit walks them too
    cfg["backend-b200"]["chemistry-kernel"] = "tables"
    cfg["bcvals"]["walls"] = {"kind": "slp-adia-wall"}
    return cfg.validate()


def stoichiometric(mix):
    X = np.zeros(mix.ns)
    X[mix.spnames.index("CH4")], X[mix.spnames.index("O2")] = 1.0, 2.0
    Y = X * np.asarray(mix.constants()["MW"])
    return Y / Y.sum()


def solver(cfg, cells, lengths):
    import peregrine_b200 as pg
    from peregrine_b200.mesher import CubeMesher

    mesh = CubeMesher(cells=[[c] for c in cells], lengths=list(lengths), defaultbc="walls")
    return pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))


def cell(kind, p, T, Y, dt=1e-9, stepset=True, **kw):
    mb = solver(config(kind, **kw), (1, 1, 1), (0.01,) * 3)
    q = np.zeros((5, 5, 5, mb.ne))
    q[..., 0], q[..., 4], q[..., 5:] = p, T, np.asarray(Y)[:-1]
    mb.set_prims([q])
    if stepset:
        mb.set_dt(dt)
    mb.rhs()
    return mb


def at_cell(mb, reg="Q"):
    return getattr(mb.blocks[0], reg).get()[2, 2, 2]


def dQ(mb):
    return at_cell(mb, mb.regs[-1])


def mixture():
    from peregrine_b200.mixture import Mixture

    return Mixture({"species": GAS, "eos": "tpg", "trans": None})


def test_one_substep_within_the_bound_is_the_finite_rate_source():
    rng = np.random.default_rng(5)
    mix = mixture()
    Y = rng.random(mix.ns)
    Y /= Y.sum()
    explicit = cell("coupled", 10e5, 1800.0, Y)
    rho = at_cell(explicit)[0]
    omega = np.append(dQ(explicit)[5:], 0.0)
    omega[-1] = -omega[:-1].sum()
    headroom = np.where(omega < 0, Y, 1.0 - Y)
    dt = 0.5 * (rho * headroom / np.maximum(np.abs(omega), 1e-300)).min()
    explicit = cell("coupled", 10e5, 1800.0, Y, dt=dt)
    substepped = cell("sub-stepped", 10e5, 1800.0, Y, dt=dt, cap=1)
    assert np.array_equal(dQ(explicit)[5:], dQ(substepped)[5:])


@pytest.mark.parametrize("cap", [1, 10, 50])
def test_substeps_keep_the_state_in_bounds(cap):
    mix = mixture()
    Y, dt = stoichiometric(mix), 1e-5
    explicit = cell("coupled", 10e5, 2500.0, Y, dt=dt)
    Q, r = at_cell(explicit), dQ(explicit)
    after = (Q[5:] + r[5:] * dt) / Q[0]
    assert after.min() < -0.1 or after.max() > 1.1
    sub = cell("sub-stepped", 10e5, 2500.0, Y, dt=dt, cap=cap, bulk=1)
    Q, r = at_cell(sub), dQ(sub)
    after = (Q[5:] + r[5:] * dt) / Q[0]
    assert np.isfinite(r).all()
    assert after.min() > -1e-12 and after.sum() < 1.0 + 1e-12


def reactants(kind, tolerance, dt=1e-6, **kw):
    return cell(kind, 10e5, 400.0, stoichiometric(mixture()), dt=dt, cap=200, eqtol=tolerance, **kw)


def test_a_settled_cell_finishes_in_one_relaxed_move():
    explicit = dQ(reactants("coupled", 0.0))[5:]
    withexit = reactants("sub-stepped", 1e-7)
    assert int(withexit.substeps()[0, 0, 0]) == 1
    source = dQ(withexit)[5:]
    assert np.abs(source - explicit).max() < 1e-6 * np.abs(explicit).max()
    assert not np.array_equal(source, explicit)
    assert np.array_equal(dQ(reactants("sub-stepped", 0.0))[5:], explicit)


def test_a_right_hand_side_before_any_step_is_the_finite_rate_source():
    explicit = dQ(reactants("coupled", 0.0))[5:]
    assert np.array_equal(dQ(reactants("sub-stepped", 1e-7, stepset=False))[5:], explicit)


def test_an_unsettled_cell_substeps_as_the_one_pass_form():
    runs = []
    for tol in (1e-7, 0.0):
        mb = cell("sub-stepped", 10e5, 2500.0, stoichiometric(mixture()), dt=1e-6, cap=200, eqtol=tol)
        mb.step(1e-6, 3)
        runs.append(mb)
    assert np.array_equal(runs[0].substeps(), runs[1].substeps()) and runs[0].substeps()[0, 0, 0] > 1
    assert np.array_equal(at_cell(runs[0]), at_cell(runs[1]))


def duct(nx=8, dt=1e-6, hot=2500.0, cold=400.0, simulator="euler", cap=200, bulk=1, bins=8, ny=2):
    """The reference's duct (tests/chemint/cases.py:67-82): nx x ny x ny cells
    5 cm wide, its first half hot, the rest cold, stoichiometric CH4/O2 at 10 bar."""
    # wide cells (5 cm) keep the acoustic CFL small at a step the chemistry is stiff over
    mb = solver(config("sub-stepped", cap=cap, bulk=bulk, bins=bins, simulator=simulator), (nx, ny, ny),
                (0.05 * nx, 0.05 * ny, 0.05 * ny))
    q = np.zeros((nx + 4, ny + 4, ny + 4, mb.ne))
    T = np.full(nx + 4, cold)
    T[: 2 + nx // 2] = np.max(hot)
    T[2: 2 + nx // 2] = hot
    q[..., 0], q[..., 4] = 10e5, T[:, None, None]
    q[..., 5:] = stoichiometric(mb.mixture)[:-1]
    mb.set_prims([q])
    mb.set_dt(dt)
    mb.rhs()
    return mb, q


def same(a, b):
    """The reference's device bar for one form against another (tests/gases.py:50-55)."""
    return np.allclose(a, b, rtol=1e-6, atol=1e-6 * np.abs(b).max())


def rhs_of(mb):
    return getattr(mb.blocks[0], mb.regs[-1]).get()[mb.mesh_blocks[0].interior]


def Q_of(mb):
    return mb.blocks[0].Q.get()[mb.mesh_blocks[0].interior]


@pytest.mark.parametrize("bulk", [1, 2])
def test_the_compaction_is_the_one_pass_form(bulk):
    # a short list: a warp per stiff cell
    plain, _ = duct(dt=STIFF, bulk=200)
    compact, _ = duct(dt=STIFF, bulk=bulk)
    assert compact.stiff_head()[0] > 0 and plain.stiff_head()[0] == 0
    assert same(rhs_of(compact), rhs_of(plain))
    assert np.array_equal(compact.substeps(), plain.substeps())
    # and through steps, the list emptied and refilled each stage
    for mb in (plain, compact):
        mb.step(STIFF, 2)
    assert same(Q_of(compact), Q_of(plain))
    assert np.isfinite(Q_of(compact)).all()


def test_a_long_list_is_the_one_pass_form_to_the_bit():
    # 4096 hot cells, more than two a warp of the stiff pass: a lane per cell
    plain, _ = duct(nx=128, ny=8, dt=STIFF, bulk=200)
    compact, _ = duct(nx=128, ny=8, dt=STIFF, bulk=1)
    assert compact.stiff_head()[0] == 64 * 64
    assert np.array_equal(rhs_of(compact), rhs_of(plain))
    # the later stages start near the hot cells' equilibrium, their lists
    # short: a warp per cell there
    for mb in (plain, compact):
        mb.step(STIFF, 2)
    assert same(Q_of(compact), Q_of(plain))


def test_the_list_holds_the_stiff_cells_alone():
    nx = 8
    mb, _ = duct(nx=nx, dt=STIFF, bulk=1, bins=1)
    head = mb.stiff_head()
    hot = (nx // 2) * 2 * 2
    assert head[0] == hot == head[1]
    subs = mb.substeps()
    assert (subs[nx // 2:] == 1).all() and (subs[: nx // 2] == 200).all()
    source = rhs_of(mb)[..., 5:]
    assert np.abs(source[nx // 2:]).max() < 1e-6 * np.abs(source[: nx // 2]).max()
    # the count is reset before each right-hand side, not carried on
    mb.rhs()
    assert mb.stiff_head()[0] == hot


def test_nothing_is_listed_where_one_substep_covers_the_step():
    mb, _ = duct(dt=1e-6, bulk=1, bins=1)
    assert mb.stiff_head()[0] == 0
    assert (mb.substeps() == 1).all()


def binof(count, bulk, cap, bins):
    if bins == 1:
        return 0
    b = int(np.log(max(count, bulk) / bulk) * bins / np.log(cap / bulk))
    return min(max(b, 0), bins - 1)


def test_the_bins_hold_the_cells_of_their_count():
    # thirty short steps leave the hot cells part way into ignition at two to
    # a few dozen substeps; a second right-hand side of the same state bins
    # each by the count it took the time before, so its bin is exact
    nx, bulk, cap, bins, dt = 16, 1, 200, 8, 2e-8
    hot = np.linspace(1200.0, 2800.0, nx // 2)
    mb, _ = duct(nx=nx, dt=dt, hot=hot, bulk=bulk, cap=cap, bins=bins)
    mb.step(dt, 30)
    mb.rhs()
    subs = mb.substeps()
    mb.rhs()
    head = np.array(mb.stiff_head())
    total, counts = head[0], head[1:]
    assert total == counts.sum() > 0 and (counts > 0).sum() > 1
    assert (subs > bulk).sum() == total
    want = np.zeros(bins, int)
    for s in subs[subs > bulk]:
        want[binof(s, bulk, cap, bins)] += 1
    assert np.array_equal(counts, want)
    # the one-pass form through the same calls: every right-hand side's tpg
    # Newton starts from the T the one before left
    # the one-pass form's right-hand side of the same state (thirty steps
    # through ignition would carry the two forms' rounding apart)
    plain, _ = duct(nx=nx, dt=dt, hot=hot, bulk=cap, cap=cap)
    plain.blocks[0].Q.set(mb.blocks[0].Q.get())
    plain.rhs()
    plain.rhs()
    assert same(rhs_of(mb), rhs_of(plain))


def test_the_viscous_fluid_compacts_alike():
    euler, _ = duct(dt=STIFF, bulk=1)
    viscous, _ = duct(dt=STIFF, bulk=1, simulator="navier-stokes")
    species = rhs_of(euler)[..., 5:]
    assert np.allclose(rhs_of(viscous)[..., 5:], species, rtol=0.0, atol=1e-14 * np.abs(species).max())
    onepass, _ = duct(dt=STIFF, bulk=200, simulator="navier-stokes")
    assert same(rhs_of(viscous), rhs_of(onepass))
    viscous.step(STIFF)
    assert np.isfinite(Q_of(viscous)).all()


@pytest.mark.parametrize("dt", [1e-6, STIFF])
def test_the_duct_matches_the_oracle(dt):
    from oracle.oracle import Oracle

    mb, q = duct(nx=16, dt=dt, bulk=1)
    orc = Oracle(mb.mixture.constants(), mb.ns, "euler", mb.mesh_blocks, mb.metrics, "tvd-rk3", eos="tpg",
                 trans="constant", chemistry="finite-rate", chemint="sub-stepped", max_substeps=200, eqtol=1e-7,
                 bcvals=mb.cfg["bcvals"], species=mb.mixture.spnames)
    orc.set_prims([q])
    orc.dt = dt
    want = [np.zeros_like(orc.regs[0][0])]
    orc.rhs(orc.regs[0], want)
    g = mb.mesh_blocks[0].interior
    got, w = rhs_of(mb), want[0][g]
    scale = np.abs(w[..., 5:]).max()
    assert np.abs(got[..., 5:] - w[..., 5:]).max() < 1e-9 * scale
    assert np.array_equal(mb.substeps(), orc.subs[0][g])
    mb.step(dt, 3)
    for _ in range(3):
        orc.step(dt)
    got, w = Q_of(mb), orc.regs[0][0][g]
    # the density and energy within 1e-9 of their largest, each species'
    # density within 1e-9 of the largest density (a mass fraction's error; a
    # trace radical's own largest is no scale), and the momentum, which only
    # the hot half's pressure raises over these three steps and which carries
    # the heat release's rounding, within 5e-8 of its own small largest
    scale = np.abs(w).reshape(-1, w.shape[-1]).max(axis=0)
    scale[5:] = scale[0]
    scale[scale == 0.0] = 1.0
    err = np.abs(got - w).reshape(-1, w.shape[-1]).max(axis=0) / scale
    # at the stiff step the hot cells take the cap, 200 substeps a stage and
    # 1800 over the three steps, and the rounding they gather is 1e-8
    bar = 1e-8 if dt == STIFF else 1e-9
    assert np.delete(err, [1, 2, 3]).max() < bar
    assert err[1:4].max() < 50 * bar
