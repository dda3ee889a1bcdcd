"""The coupled source generated for the case's mechanism against the
table-driven kernel, on the device.

Both evaluate the same arithmetic in the same order (the generated source
makes every species index and constant a literal); the two compilations
contract a few multiply-adds differently, so their right-hand sides agree to
rounding: within 1e-13 of each component's largest, on the per-block path
and on the batched path's fused passes, for the H2/O2/N2 subset of GRI-Mech
3.0, its one-way twin and CH4/O2 FFCM-Y (three-body, Lindemann and Troe
reactions in the product and log forms).  Steps carry those roundings into
the thermally perfect temperature, which its Newton fixes only to about
1e-11 relative (the rounding band of the reacting tests), so three steps are
held within 1e-10 of each component's largest.
"""

import numpy as np
import pytest

from peregrine_b200 import cases

pytestmark = pytest.mark.gpu

MECHS = ["h2o2_gri30", "h2o2_gri30_oneway", "ch4_o2_ffcmy"]


def pair(mechanism, launch, cells=10):
    import peregrine_b200 as pg

    out = []
    for kernel in ("generated", "tables"):
        cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, tables=mechanism,
                                    launch=launch)
        cfg["backend-b200"]["chemistry-kernel"] = kernel
        mesh = cases.reacting_mesh(cells, (2, 1, 1))
        mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
        consts = mb.mixture.constants()
        spnames = mb.mixture.spnames
        if "H2" in spnames and "O2" in spnames and "N2" in spnames:
            prims = cases.reacting_prims(mb.metrics, spnames, consts["MW"], cells, seed=3, width=2.0, dT=700.0,
                                         radicals=2e-3)
        else:
            prims = methane(mb.metrics, spnames)
        mb.set_prims(prims)
        out.append(mb)
    return out


@pytest.mark.parametrize("mechanism", MECHS)
@pytest.mark.parametrize("launch", ["per-block", "batched"])
def test_the_generated_source_equals_the_tables_to_rounding(mechanism, launch):
    gen, tab = pair(mechanism, launch)
    on, why = gen.generated_chemistry()
    assert on, why
    assert not tab.generated_chemistry()[0]
    for mb in (gen, tab):
        mb.rhs(Q="Q", dQ="Q1")
    for a, b in zip(gen.blocks, tab.blocks):
        x, y = a.Q1.get()[a.mesh.interior], b.Q1.get()[b.mesh.interior]
        assert np.isfinite(x).all()
        assert rowrel(x, y).max() <= 1e-13, rowrel(x, y)
    for mb in (gen, tab):
        mb.step(1e-9, 3)
    for a, b in zip(gen.blocks, tab.blocks):
        x, y = a.Q.get()[a.mesh.interior], b.Q.get()[b.mesh.interior]
        assert np.isfinite(y).all() and np.isfinite(x).all()
        assert rowrel(x, y).max() <= 1e-10, rowrel(x, y)


def methane(metrics, spnames, seed=5):
    """CH4/O2 at 10 bar, 1200 to 1800 K, a trace of every other species."""
    rng = np.random.default_rng(seed)
    out = []
    for m in metrics:
        shape = m["xcc"].shape[:3]
        Y = np.full(len(spnames), 1e-3)
        Y[spnames.index("CH4")], Y[spnames.index("O2")] = 0.2, 0.7
        Y /= Y.sum()
        q = np.zeros(shape + (4 + len(spnames),))
        q[..., 0] = 1e6
        q[..., 1:4] = 5.0 * rng.standard_normal(shape + (3,))
        q[..., 4] = 1200.0 + 600.0 * rng.random(shape)
        q[..., 5:] = Y[:-1]
        out.append(q)
    return out


def rowrel(x, y):
    """Each component's largest difference over its largest magnitude."""
    ne = y.shape[-1]
    scale = np.abs(y).reshape(-1, ne).max(axis=0)
    scale[scale == 0.0] = 1.0
    return np.abs(x - y).reshape(-1, ne).max(axis=0) / scale
