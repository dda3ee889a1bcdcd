"""The CPU oracle and the host logic against fixtures made by the reference itself.

tests/golden/make_golden.py produced the fixtures from the reference's own
code (its numpy test oracle, its grid metrics, its mixture constants and its
integrators); no test reads the reference.
"""

import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, stage_combines
from peregrine_b200 import grid, integrators
from peregrine_b200.mixture import Mixture

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


def gases():
    with open(os.path.join(GOLD, "gases.json")) as f:
        return json.load(f)


def mixture(species, trans="constant"):
    return Mixture({"species": species, "eos": "cpg", "trans": trans})


def close_rows(got, want, within):
    """The reference's measure: each component within `within` of its largest magnitude
    (tests/simulator/test_facefluxes.py:53-56)."""
    scale = np.abs(want).reshape(-1, want.shape[-1]).max(axis=0)
    return np.all(np.abs(got - want) <= within * scale)


@pytest.mark.parametrize("gas", ["air", "binary"])
def test_kepaec_matches_the_reference_numpy_oracle(gas):
    f = gold("faces_kepaec.npz")
    species = gases()[gas]
    consts = mixture(species).constants()
    ns = len(species)
    orc = Oracle(consts, ns, "euler", [], [])
    got = orc.kepaec_faces(f[f"{gas}_QL"], f[f"{gas}_QR"], f[f"{gas}_S"])
    # the reference's own bar for a face flux against this oracle
    assert close_rows(got, f[f"{gas}_F"], 1e-13)


LIMITERS = ["koren", "minmod", "mc", "superbee", "vanleer"]


@pytest.mark.parametrize("recon", ["constant"] + [f"muscl_{name}" for name in LIMITERS])
@pytest.mark.parametrize("primary", ["hllc", "rusanov", "ausmup"])
def test_riemann_fluxes_match_the_reference_numpy_oracle(primary, recon):
    f = gold("faces_riemann.npz")
    species = gases()["binary"]
    consts = mixture(species).constants()
    muscl = recon != "constant"
    orc = Oracle(consts, len(species), "euler", [], [], primary=primary, recon="muscl" if muscl else "constant",
                 limiter=recon[6:] if muscl else None)
    Q4 = f["Q4"]
    got = orc.advective_faces(Q4[0], Q4[1], Q4[2], Q4[3], f["S"])
    # the reference's bar for its kernels' face fluxes against this oracle
    # (tests/simulator/test_facefluxes.py:53-63); the limiters here take the
    # two differences, the numpy oracle their ratio, so the two agree to rounding
    assert close_rows(got, f[f"{primary}_{recon}"], 1e-13)


def test_the_fixture_exercises_every_hllc_wave_case():
    f = gold("faces_riemann.npz")
    Q4, S = f["Q4"], f["S"]
    consts = mixture(gases()["binary"]).constants()
    area = np.linalg.norm(S, axis=1)

    def side(Q):
        rho = Q[:, 0]
        u = Q[:, 1:4] / rho[:, None]
        Y = np.c_[Q[:, 5:] / rho[:, None], 1.0 - Q[:, 5:].sum(1) / rho]
        R, cp = Y @ consts["Rsp"], Y @ consts["cp0"]
        T = (Q[:, 4] / rho - 0.5 * (u * u).sum(1) - Y @ consts["h298R"]) / (cp - R)
        return (u * S).sum(1) / area, np.sqrt(cp / (cp - R) * R * T)

    (unL, cL), (unR, cR) = side(Q4[1]), side(Q4[2])
    SL, SR = unL - cL, unR + cR
    # the left and right outer cases, and subsonic faces whose star state is either side
    assert (SL >= 0).sum() > 8 and (SR < 0).sum() > 8
    sub = (SL < 0) & (SR >= 0)
    assert (sub & (unL + unR > 0)).sum() > 8 and (sub & (unL + unR < 0)).sum() > 8
    assert not np.array_equal(f["hllc_constant"], f["hllc_muscl_koren"])


def test_metrics_match_the_reference_grid_bit_for_bit():
    g = gold("metrics.npz")
    mine = grid.metrics(g["nodes"], 2)
    for name in ("xcc", "detJinv", "Jinv", "iS", "jS", "kS", "ixc", "jxc", "kxc"):
        assert np.array_equal(mine[name], g[name], equal_nan=True), name


@pytest.mark.parametrize("gas", ["air", "binary"])
def test_mixture_constants_match_the_reference_bit_for_bit(gas):
    c = gold("constants.npz")
    mine = mixture(gases()[gas]).constants()
    keys = [k[len(gas) + 1:] for k in c.files if k.startswith(gas + "_")]
    needed = ("MW", "MWinv", "Rsp", "cppoly", "hpoly", "h298", "cp0", "h298R", "mu0", "kappa0", "MWqinv",
              "wilkepair", "lewis")
    for k in needed:
        assert k in keys, k
        assert np.array_equal(np.asarray(mine[k], dtype=np.float64), c[f"{gas}_{k}"]), k


def reference_tables():
    with open(os.path.join(GOLD, "rk_tables.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["rk1", "rk2", "tvd-rk3", "rk34", "rk4"])
def test_stage_tables_match_the_reference_integrators(name):
    ref = reference_tables()[name]
    regs = [f"R{n}" for n in range(ref["nregs"])]
    rows, dq, nregs = integrators.stages(name)
    assert nregs == ref["nregs"]
    assert len(rows) == len(ref["stages"])
    ones, _ = stage_combines(name, regs)
    for (q, combines), (oq, ocombines), want in zip(rows, ones, ref["stages"]):
        assert regs[q] == want["q"] == oq
        assert len(combines) == len(want["combines"]) == len(ocombines)
        for cb, ocb, w in zip(combines, ocombines, want["combines"]):
            assert regs[cb["out"]] == w["out"] == ocb[0]
            own = cb["own"] if cb["own"] != 0.0 else None
            assert own == w["own"] == ocb[1]
            assert [(regs[r], x) for r, x in cb["reads"]] == [tuple(t) for t in w["terms"]] == ocb[2]
            assert cb["step"] == w["step"] == ocb[3]
