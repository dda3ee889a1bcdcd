"""The double flux's Riemann forms and its viscous simulator on the device,
held to the reference's own checks of them
(tests/doubleflux/test_doubleflux.py:83-112, 243-265) and to the CPU oracle:
a real-gas contact of CH4 in O2 at 59.8 MPa, advected at 20 m/s through a
periodic line of forty cells, keeps its pressure to 1e-9 under the double
flux's Rusanov and AUSM+-up, where the plain fluxes scatter it, with mass
and species kept to 1e-12; a diffusing layer under navier-stokes-df keeps
the plain simulator's temperature within 0.1 K.  The pressure and
temperature are the solver's own, read through ``mb.sim.iovars.data``.

The reference walls the line's one-cell-thick cross-section with slip walls;
a flow along the line alone sees the same halo cells through a periodic
cross-section, which these cases use.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P0, CELLS, DX = 59.8e6, 40, 5e-5


def solver(simulator, primary="kepaec", recon="constant", limiter=None, dx=DX):
    import peregrine_b200 as pg
    from peregrine_b200.config import Config
    from peregrine_b200.mesher import CubeMesher

    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    cfg["mixture"]["species"] = "ch4_o2_srk"
    cfg["mixture"]["eos"] = "real-gas-df" if simulator.endswith("-df") else "real-gas"
    cfg["mixture"]["trans"] = "kinetic-theory" if simulator.startswith("navier-stokes") else None
    cfg["time-integration"]["integrator"] = "tvd-rk3"
    cfg["adv-flux"].update(primary=primary, recon=recon, limiter=limiter)
    cfg["backend-b200"]["launch"] = "per-block"
    cfg.validate()
    mesh = CubeMesher(cells=[[CELLS], [1], [1]], lengths=[CELLS * dx, dx, dx], periodic=[True] * 3)
    return pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))


def slab(mb, u0=20.0, Tin=162.7, Tout=111.7, smear=1.5):
    blk = mb.mesh_blocks[0]
    shape = tuple(n + 4 for n in blk.cells)
    q = np.zeros(shape + (6,))
    i = np.arange(shape[0]) - 2 + 0.5
    f = (0.5 * (np.tanh((i - CELLS // 4) / smear) - np.tanh((i - CELLS // 2) / smear)))[:, None, None]
    q[..., 0], q[..., 1] = P0, u0
    q[..., 4] = Tout + f * (Tin - Tout)
    q[..., 5] = f
    mb.set_prims([q])
    return (slice(2, -2), 2, 2), q


def field(mb, name, where):
    return mb.sim.iovars.data(mb.blocks[0], [name])[name][where]


def sound(mb, where):
    from oracle.oracle import Oracle

    orc = Oracle(mb.mixture.constants(), 2, "euler", [], [], eos="real-gas")
    Q = np.ascontiguousarray(mb.blocks[0].Q.get()[where])
    return orc.realgas_fromQ(Q, field(mb, "T", where))[:, 7]


def advect(mb, cfl, steps, u0=20.0):
    inner, _ = slab(mb, u0=u0)
    dt = cfl * DX / sound(mb, inner).max()
    Q0 = mb.blocks[0].Q.get()[inner]
    totals0 = Q0.sum(axis=0)
    scatter = 0.0
    for _ in range(steps):
        mb.step(dt)
        p = field(mb, "p", inner)
        assert np.all(np.isfinite(p))
        scatter = max(scatter, np.abs(p / P0 - 1.0).max())
    change = mb.blocks[0].Q.get()[inner].sum(axis=0) - totals0
    return scatter, np.divide(change, np.abs(totals0), out=np.zeros_like(change), where=totals0 != 0)


@pytest.mark.parametrize(
    "primary, recon, limiter, plainabove",
    [
        ("rusanov", "constant", None, 1e-3),
        ("ausmup", "constant", None, 1e-4),
        ("rusanov", "muscl", "koren", 1e-5),
        ("ausmup", "muscl", "koren", 1e-5),
    ],
    ids=["rusanov", "ausmup", "muscl-koren-rusanov", "muscl-koren-ausmup"],
)
def test_the_riemann_solvers_keep_the_pressure(primary, recon, limiter, plainabove):
    flux = dict(primary=primary, recon=recon, limiter=limiter)
    plain, _ = advect(solver("euler", **flux), 0.4, 200)
    scatter, drift = advect(solver("euler-df", **flux), 0.4, 200)
    assert plain > plainabove and scatter < 1e-9
    assert abs(drift[0]) < 1e-12 and abs(drift[5]) < 1e-12


def test_the_line_steps_as_the_oracle_does():
    from oracle.oracle import Oracle

    mb = solver("euler-df", "ausmup", "muscl", "koren")
    inner, q = slab(mb)
    orc = Oracle(mb.mixture.constants(), 2, "euler-df", mb.mesh_blocks, mb.metrics, "tvd-rk3", primary="ausmup",
                 recon="muscl", limiter="koren", eos="real-gas-df", trans=None)
    orc.set_prims([q])
    dt = 0.4 * DX / sound(mb, inner).max()
    for _ in range(20):
        mb.step(dt)
        orc.step(dt)
    got, want = mb.blocks[0].Q.get()[inner], orc.regs[0][0][inner]
    scale = np.abs(want).max(axis=0)
    scale[scale == 0.0] = 1.0
    assert (np.abs(got - want).max(axis=0) / scale).max() < 1e-9
    # the state the solver reads back is the last right-hand side's, the oracle's kept record
    assert np.abs(field(mb, "p", inner) / orc.pst[0][inner][:, 0] - 1.0).max() < 1e-9


def diffusing(simulator, dx=1e-7, steps=2000):
    mb = solver(simulator, dx=dx)
    inner, _ = slab(mb, u0=0.0, Tin=140.0, Tout=140.0, smear=3.0)
    dt = 0.4 * dx / sound(mb, inner).max()
    E0 = mb.blocks[0].Q.get()[inner][:, 4].sum()
    mb.step(dt, steps)
    drift = (mb.blocks[0].Q.get()[inner][:, 4].sum() - E0) / abs(E0)
    return field(mb, "T", inner), field(mb, "p", inner), drift


def test_a_diffusing_layer_keeps_its_temperature():
    Tplain, pplain, _ = diffusing("navier-stokes")
    T, p, drift = diffusing("navier-stokes-df")
    assert np.abs(T - Tplain).max() < 0.1
    assert np.abs(p - pplain).max() / P0 < 1e-4
    assert abs(drift) < 1e-4


def test_iovars_derive_the_named_variables():
    # the batched path keeps no state array: its p and T are fromQ's closed
    # form of Q; the per-block path's are the last right-hand side's state
    import peregrine_b200 as pg
    from peregrine_b200 import cases

    for launch in ("batched", "per-block"):
        cfg = cases.tgv_config("navier-stokes", "rk4", launch)
        mb = pg.get_solver(cfg, cases.tgv_mesh(16, (1, 1, 1)), pg.get_backend("cuda", cfg))
        mb.set_prims(cases.tgv_prims(mb.mesh_blocks, mb.metrics))
        mb.step(1e-3, 2)
        if launch == "per-block":
            mb.rhs(Q="Q")
        d = mb.sim.iovars.data(mb.blocks[0], mb.sim.iovars.exported)
        inner = mb.mesh_blocks[0].interior
        Q = mb.blocks[0].Q.get()[inner]
        assert np.allclose(d["rho"][inner], Q[..., 0], rtol=0, atol=0)
        assert np.allclose(d["u"][inner], Q[..., 1] / Q[..., 0], rtol=1e-15)
        R = float(mb.mixture.constants()["Rsp"][0])
        assert np.abs(d["p"][inner] / (Q[..., 0] * R * d["T"][inner]) - 1.0).max() < 1e-13
        assert set(d) == set(mb.sim.iovars.exported)
