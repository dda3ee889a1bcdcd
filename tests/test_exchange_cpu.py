"""The halo exchange across oriented interfaces and rotational periodics on
the CPU oracle, pinned to the reference's own exchange checks
(tests/communication/test_orientation.py, test_xchg.py:130-212).

* a pair of blocks whose second is laid out along each of the 24 proper
  orientations trades Q and the nodes as the identity pair does, the second
  block's arrays the identity's laid out alike, to the bit;
* an annulus swept through 90 degrees, its ends a rotational periodic,
  turns the vectors arriving in each end's halo by that face's rotation,
  carries the scalars as they are, and lands a radial and an azimuthal
  field at the halo's own centres.
"""

import itertools

import numpy as np
import pytest

from oracle.oracle import Oracle
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import AnnulusMesher, CubeMesher, fill_node_halos, reorient, signedaxis
from peregrine_b200.mixture import Mixture

SPECIES = {"N2": {"MW": 28.0134, "cp0": 1040.0}, "O2": {"MW": 31.9988, "cp0": 918.0}}


def orientations():
    """The 24 signed permutations of determinant one, as digits."""
    valid = []
    for axes in itertools.permutations((0, 1, 2)):
        for signs in itertools.product((1, -1), repeat=3):
            P = np.zeros((3, 3))
            for m, (a, s) in enumerate(zip(axes, signs)):
                P[m, a] = s
            if np.linalg.det(P) > 0:
                valid.append("".join(str(a + 1 + (3 if s < 0 else 0)) for a, s in zip(axes, signs)))
    assert len(valid) == 24
    return valid


def laid(a, S):
    """An array of a block's cells (three index axes first) as the block laid
    out along S holds it."""
    out = a
    for m, c in enumerate(S):
        if signedaxis(c)[1]:
            out = np.flip(out, axis=m)
    return np.moveaxis(out, (0, 1, 2), [signedaxis(c)[0] for c in S])


def pair(S):
    blocks = CubeMesher(mbdims=[2, 1, 1], blkdims=[6, 3, 2], lengths=[2, 1, 1], defaultbc="wall").make_blocks(2)
    if S != "123":
        reorient(blocks, 1, S)
        fill_node_halos(blocks)
    return blocks


def oracle_of(blocks):
    mix = Mixture({"species": SPECIES, "eos": "cpg", "trans": None})
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    return Oracle(mix.constants(), 2, "euler", blocks, mets, "tvd-rk3", bcvals={"wall": {"kind": "slp-adia-wall"}},
                  species=list(SPECIES))


def traded(S, seed=20260901):
    blocks = pair(S)
    orc = oracle_of(blocks)
    rng = np.random.default_rng(seed)
    # drawn in the identity layout, so block 1 holds the same field however it is stored
    for n, blk in enumerate(blocks):
        values = rng.random(tuple(c + 4 for c in pair("123")[n].cells) + (6,))
        orc.regs[0][n][...] = values if n == 0 else laid(values, S)
    orc.exchange()
    return blocks, orc


@pytest.mark.parametrize("S", orientations())
def test_orientation(S):
    ref_blocks, ref = traded("123")
    blocks, orc = traded(S)
    assert np.array_equal(orc.regs[0][0], ref.regs[0][0])
    assert np.array_equal(orc.regs[0][1], laid(ref.regs[0][1], S))
    assert np.array_equal(blocks[0].nodes, ref_blocks[0].nodes)
    assert np.array_equal(blocks[1].nodes, laid(ref_blocks[1].nodes, S))


def test_the_identity_pair_lands_the_neighbours_cells():
    # a trade that wrote nothing would pass the comparison above
    _, ref = traded("123")
    a, b = ref.regs[0]
    for g in range(2):
        assert np.array_equal(a[-2 + g, 2:-2, 2:-2], b[2 + g, 2:-2, 2:-2])


def annulus():
    mesher = AnnulusMesher(mbdims=[1, 1, 2], blkdims=[4, 4, 4], p1=[0, 0, 0], p2=[1, 0, 0], p3=[0, 0.5, 0],
                           sweep=90, thickness=0.5, periodic=True, defaultbc="wall")
    blocks = mesher.make_blocks(2)
    return blocks, oracle_of(blocks)


def test_a_rotational_periodic_rotates_the_vectors():
    blocks, orc = annulus()
    for Q in orc.regs[0]:
        Q[..., 0], Q[..., 1:4], Q[..., 4], Q[..., 5] = 1.0, (1.0, 2.0, 3.0), 5.0, 0.3
    orc.exchange()
    low, high = blocks[0].get_intface(5), blocks[1].get_intface(6)
    assert low.rotperiodic and high.rotperiodic
    a, b = orc.regs[0]
    # block 0's far end comes back through its low face turned by -90 about +x,
    # (y, z) -> (z, -y); block 1's through its high face by +90
    for g in range(2):
        assert np.allclose(a[2, 2, g, 1:4], (1.0, 3.0, -2.0), rtol=1e-15, atol=1e-15)
        assert np.allclose(b[2, 2, -1 - g, 1:4], (1.0, -3.0, 2.0), rtol=1e-15, atol=1e-15)
    assert np.allclose(a[2, 2, 0, 1:4], low.rot @ np.array([1.0, 2.0, 3.0]), rtol=1e-15, atol=1e-15)
    # the scalars are carried as they are
    assert a[2, 2, 0, 0] == 1.0 and a[2, 2, 0, 4] == 5.0 and a[2, 2, 0, 5] == 0.3


def radial(x):
    y, z = x[..., 1], x[..., 2]
    return np.stack([np.zeros_like(y), y, z], axis=-1) / np.hypot(y, z)[..., None]


def azimuthal(x):
    y, z = x[..., 1], x[..., 2]
    return np.stack([np.zeros_like(y), -z, y], axis=-1) / np.hypot(y, z)[..., None]


@pytest.mark.parametrize("field", [radial, azimuthal])
def test_a_rotational_periodic_lands_a_field_at_the_halos_centers(field):
    # a wrong sign or angle would land the field somewhere other than the halo's own centres
    blocks, orc = annulus()
    mets = [make_metrics(b.nodes, 2) for b in blocks]
    for Q, m in zip(orc.regs[0], mets):
        Q[..., 0], Q[..., 4] = 1.0, 5.0
        Q[..., 1:4] = field(m["xcc"])
    orc.exchange()
    checked = 0
    for blk, Q, m in zip(blocks, orc.regs[0], mets):
        for face in blk.intfaces:
            if not face.rotperiodic:
                continue
            # the halo's nodes were turned into place, so its own centres are the reference
            sl = [slice(2, -2)] * 3
            sl[face.axis] = slice(0, 2) if face.is_low else slice(-2, None)
            halo, centers = Q[tuple(sl)], m["xcc"][tuple(sl)]
            assert np.allclose(halo[..., 1:4], field(centers), rtol=0, atol=1e-14)
            checked += 1
    assert checked == 2


def test_a_rotational_periodics_halo_continues_the_sweep():
    # the centres step by 15 degrees through halo and interior alike
    blocks, _ = annulus()
    x = make_metrics(blocks[0].nodes, 2)["xcc"][2, 2]
    angles = np.degrees(np.arctan2(x[:, 2], x[:, 1]))
    assert np.allclose(angles, -7.5 - 15 * 1 + 15 * np.arange(3 + 4), atol=1e-12)
