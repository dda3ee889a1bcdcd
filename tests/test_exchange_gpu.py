"""The halo exchange across oriented interfaces and rotational periodics on
the device: the library's exchange against the reference's own checks
(tests/communication/test_orientation.py, test_xchg.py:130-212), and the
physics through such interfaces against the identity layout and the oracle.

Bars: the exchange to the bit (it copies; a rotation within 1e-15 as the
reference's test holds it); a reoriented pair's steps within 1e-12 of the
identity pair's (the face sums run in another order); the annulus's steps
within 1e-9 of the oracle's.
"""

import numpy as np
import pytest

from peregrine_b200.mesher import AnnulusMesher, CubeMesher, fill_node_halos, reorient

from tests.test_exchange_cpu import SPECIES, laid, orientations

pytestmark = pytest.mark.gpu


class Reoriented:
    """A mesher's blocks with one laid out along other axes."""

    def __init__(self, mesher, n, S):
        self.mesher, self.n, self.S = mesher, n, S

    def make_blocks(self, ng):
        blocks = self.mesher.make_blocks(ng)
        if self.S != "123":
            reorient(blocks, self.n, self.S)
            fill_node_halos(blocks)
        return blocks


def config(simulator="euler", launch="per-block", integrator="tvd-rk3"):
    from peregrine_b200.config import Config

    cfg = Config()
    cfg["simulation"]["simulator"] = simulator
    species = {k: dict(v, mu0=1.8e-5, kappa0=0.026) for k, v in SPECIES.items()}
    cfg["mixture"]["species"] = species
    cfg["mixture"]["trans"] = "constant" if simulator == "navier-stokes" else None
    cfg["ics"]["Y"] = {"N2": 0.77}
    cfg["bcvals"]["wall"] = {"kind": "slp-adia-wall"}
    cfg["time-integration"]["integrator"] = integrator
    cfg["backend-b200"]["launch"] = launch
    return cfg.validate()


def solver(mesh, **kw):
    import peregrine_b200 as pg

    cfg = config(**kw)
    return pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))


def traded(S, seed=20260901):
    mb = solver(Reoriented(CubeMesher(mbdims=[2, 1, 1], blkdims=[6, 3, 2], lengths=[2, 1, 1], defaultbc="wall"),
                           1, S))
    ident = CubeMesher(mbdims=[2, 1, 1], blkdims=[6, 3, 2], lengths=[2, 1, 1], defaultbc="wall").make_blocks(2)
    rng = np.random.default_rng(seed)
    for n, blk in enumerate(mb.blocks):
        values = rng.random(tuple(c + 4 for c in ident[n].cells) + (6,))
        values[..., 0] += 1.0
        blk.Q.set(values if n == 0 else laid(values, S))
    mb.exchange()
    return mb


@pytest.mark.parametrize("S", orientations())
def test_orientation(S):
    ref = traded("123")
    mb = traded(S)
    assert np.array_equal(mb.blocks[0].Q.get(), ref.blocks[0].Q.get())
    assert np.array_equal(mb.blocks[1].Q.get(), laid(ref.blocks[1].Q.get(), S))
    a, b = (blk.Q.get() for blk in ref.blocks)
    for g in range(2):
        assert np.array_equal(a[-2 + g, 2:-2, 2:-2], b[2 + g, 2:-2, 2:-2])


@pytest.mark.parametrize("launch,simulator", [("per-block", "euler"), ("per-block", "navier-stokes"),
                                              ("batched", "navier-stokes")])
@pytest.mark.parametrize("S", ["264", "345", "534"])
def test_a_reoriented_pair_steps_as_the_identity_pair(S, launch, simulator):
    # a periodic box of two blocks, the second laid out along other axes: the
    # batched path takes it too, its halo table carrying the orientation
    from peregrine_b200 import cases

    def run(S):
        mesher = CubeMesher(mbdims=[2, 1, 1], blkdims=[9, 8, 7], lengths=[2.0, 1.0, 0.9], periodic=[True] * 3)
        mb = solver(Reoriented(mesher, 1, S), simulator=simulator, launch=launch, integrator="rk4")
        ident = mesher.make_blocks(2)
        from peregrine_b200.grid import metrics as make_metrics

        prims = cases.tgv_prims(ident, [make_metrics(b.nodes, 2) for b in ident], ne=6, seed=5, noise=1e-3, mach=0.3)
        for q in prims:
            q[..., 5:] = 0.77
        mb.set_prims([prims[0], laid(prims[1], S)])
        mb.step(2e-5, 3)
        return mb

    ref, mb = run("123"), run(S)
    assert mb.path == ref.path
    for n in range(2):
        want = ref.blocks[n].Q.get()[ref.mesh_blocks[n].interior]
        got = mb.blocks[n].Q.get()[mb.mesh_blocks[n].interior]
        if n == 1:
            want = laid(want, S)
        scale = np.abs(want).reshape(-1, 6).max(axis=0)
        scale[1:4] = scale[1:4].max()
        assert (np.abs(got - want).reshape(-1, 6).max(axis=0) / scale).max() < 1e-12


def annulus(**kw):
    mesher = AnnulusMesher(mbdims=[1, 1, 2], blkdims=[5, 5, 6], p1=[0, 0, 0], p2=[1, 0, 0], p3=[0, 0.5, 0],
                           sweep=90, thickness=0.5, periodic=True, defaultbc="wall")
    return solver(mesher, **kw)


def test_a_rotational_periodic_rotates_the_vectors():
    mb = annulus()
    for blk in mb.blocks:
        Q = np.zeros(blk.Q.shape)
        Q[..., 0], Q[..., 1:4], Q[..., 4], Q[..., 5] = 1.0, (1.0, 2.0, 3.0), 5.0, 0.3
        blk.Q.set(Q)
    mb.exchange()
    a, b = (blk.Q.get() for blk in mb.blocks)
    for g in range(2):
        assert np.allclose(a[2, 2, g, 1:4], (1.0, 3.0, -2.0), rtol=1e-15, atol=1e-15)
        assert np.allclose(b[2, 2, -1 - g, 1:4], (1.0, -3.0, 2.0), rtol=1e-15, atol=1e-15)
    assert a[2, 2, 0, 0] == 1.0 and a[2, 2, 0, 4] == 5.0 and a[2, 2, 0, 5] == 0.3


@pytest.mark.parametrize("simulator", ["euler", "navier-stokes"])
def test_the_annulus_steps_as_the_oracle(simulator):
    # the momentum turned across the ends, and with viscosity the gradients' tensor
    from oracle.oracle import Oracle

    mb = annulus(simulator=simulator, integrator="rk4")
    rng = np.random.default_rng(3)
    prims = []
    for m in mb.metrics:
        x = m["xcc"]
        q = np.zeros(x.shape[:3] + (6,))
        q[..., 0] = 101325.0 * (1.0 + 0.05 * np.sin(4.0 * x[..., 0]))
        y, z = x[..., 1], x[..., 2]
        r = np.hypot(y, z)
        q[..., 2], q[..., 3] = -60.0 * z / r, 60.0 * y / r
        q[..., 1] = 10.0 + rng.uniform(-1, 1, y.shape)
        q[..., 4] = 300.0 + 20.0 * np.cos(3.0 * r)
        q[..., 5] = 0.77
        prims.append(q)
    mb.set_prims(prims)
    orc = Oracle(mb.mixture.constants(), 2, simulator, mb.mesh_blocks, mb.metrics, "rk4",
                 trans="constant", bcvals=mb.cfg["bcvals"], species=mb.mixture.spnames)
    orc.set_prims(prims)
    dt = 2e-6
    mb.step(dt, 3)
    for _ in range(3):
        orc.step(dt)
    for b, w in zip(mb.blocks, orc.regs[0]):
        got, want = b.Q.get()[b.mesh.interior], w[b.mesh.interior]
        scale = np.abs(want).reshape(-1, 6).max(axis=0)
        scale[1:4] = scale[1:4].max()
        assert (np.abs(got - want).reshape(-1, 6).max(axis=0) / scale).max() < 1e-9
