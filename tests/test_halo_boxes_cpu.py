"""The halo as boxes (pgb_case_halo_boxes), on the CPU.

The fill launches over boxes of halo cells whose sources one block holds at
an affine index, and lists the other cells one by one.  Expanded, the boxes
and that list are exactly the cells pgb_case_halo_entries lists, each with
the same source: on the 27 uneven blocks of the 128^3 Taylor-Green grid, on
a pair of blocks in each of the 24 orientations, across a rotational
periodic, and on blocks thinner than the halo, whose cells reach through
two blocks and take no box.
"""

import ctypes

import numpy as np
import pytest

from peregrine_b200 import cases, native
from peregrine_b200.mesher import AnnulusMesher

from tests.test_exchange_cpu import orientations, pair

LL = ctypes.POINTER(ctypes.c_longlong)


def scratch(blocks):
    """A case of the blocks' extents and interfaces, never finalized."""
    phys = native.Physics(simulator=native.EULER, eos=native.EOS_CPG, primary=native.FLUX_KEPAEC,
                          recon=native.RECON_CONSTANT, limiter=0, trans=native.TRANS_NONE, ns=1, nregs=2, alpha=1.0)
    h = ctypes.c_void_p()
    native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(h))
    for b in blocks:
        out = ctypes.c_int()
        native.call("pgb_case_add_block", h, *b.cells, ctypes.byref(out))
    for b in blocks:
        for face in b.intfaces:
            if face.nbr is None:
                continue
            rot = getattr(face, "rot", None)
            if face.orient != "123" or rot is not None:
                r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64).ravel()
                rp = None if r is None else r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                native.call("pgb_case_connect_oriented", h, b.nblki, face.nface, face.nbr, face.orient.encode(), rp)
            else:
                native.call("pgb_case_connect", h, b.nblki, face.nface, face.nbr, face.nbrface or 0)
    return h


def entries_and_boxes(blocks):
    h = scratch(blocks)
    try:
        n = ctypes.c_longlong()
        native.call("pgb_case_halo_entries", h, 0, None, ctypes.byref(n))
        ent = np.zeros((n.value, 6), dtype=np.int64)
        native.call("pgb_case_halo_entries", h, n.value, ent.ctypes.data_as(LL), ctypes.byref(n))
        nb, rest = ctypes.c_longlong(), ctypes.c_longlong()
        native.call("pgb_case_halo_boxes", h, 0, None, ctypes.byref(nb), ctypes.byref(rest))
        box = np.zeros((nb.value, 14), dtype=np.int64)
        native.call("pgb_case_halo_boxes", h, nb.value, box.ctypes.data_as(LL), ctypes.byref(nb), ctypes.byref(rest))
    finally:
        native.call("pgb_case_destroy", h)
    return ent, box, rest.value


def expand(box):
    """Every cell of every box: (dst block, dst index, src block, src index, rotated)."""
    rows = []
    for db, d0, d1, d2, d3, n0, n1, n2, sb, s0, t1, t2, t3, rot in box:
        x0, x1, x2 = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2), indexing="ij")
        d = d0 + x0 * d1 + x1 * d2 + x2 * d3
        s = s0 + x0 * t1 + x1 * t2 + x2 * t3
        for a, b in zip(d.ravel(), s.ravel()):
            rows.append((int(db), int(a), int(sb), int(b), rot != 0))
    return rows


def check(blocks):
    ent, box, rest = entries_and_boxes(blocks)
    listed = [(int(r[0]), int(r[1]), int(r[2]), int(r[3]), r[4] != 0) for r in ent]
    assert len(set(listed)) == len(listed)
    cells = expand(box)
    # no cell twice, every box cell a listed one, and the rest the cells left over
    assert len(set(cells)) == len(cells)
    assert set(cells) <= set(listed)
    assert len(cells) + rest == len(listed)
    return ent, box, rest


def test_the_uneven_blocks_are_all_boxes():
    mesh = cases.tgv_mesh(128, (3, 3, 3), seed=0, low=30, high=56)
    ent, box, rest = check(mesh.make_blocks(2))
    # six faces and twelve edges a block, every one a box
    assert rest == 0 and len(box) == 27 * 18
    # a box runs i fastest: its first step is one cell wherever it is wider than one
    assert np.all((box[:, 2] == 1) | (box[:, 5] == 1))


@pytest.mark.parametrize("S", orientations())
def test_each_orientation(S):
    ent, box, rest = check(pair(S))
    assert rest == 0 and len(ent) > 0


def test_a_rotational_periodic():
    mesher = AnnulusMesher(mbdims=[1, 1, 2], blkdims=[4, 4, 4], p1=[0, 0, 0], p2=[1, 0, 0], p3=[0, 0.5, 0],
                           sweep=90, thickness=0.5, periodic=True, defaultbc="wall")
    ent, box, rest = check(mesher.make_blocks(2))
    assert np.any(box[:, 13] != 0)


def test_blocks_thinner_than_the_halo():
    # cuts of one to two cells: a face halo two deep reaches through the
    # thin neighbour into the next block, which no one box holds
    mesh = cases.tgv_mesh(8, (4, 3, 1), seed=1, low=1, high=4)
    ent, box, rest = check(mesh.make_blocks(2))
    assert rest > 0 and len(box) > 0


def pull_allowed(blocks, want=True):
    h = scratch(blocks)
    try:
        native.call("pgb_case_set_halo_pull", h, 1 if want else 0)
        on = ctypes.c_int(-1)
        native.call("pgb_case_halo_pull", h, ctypes.byref(on))
        return on.value
    finally:
        native.call("pgb_case_destroy", h)


def test_reading_across_faces_is_allowed_only_where_every_face_joins_unrotated():
    # the uniform stage reads past a face from the neighbour's own cells only
    # where every face of every block is joined low face to high face in the
    # identity orientation, unrotated, both blocks two cells thick or more
    from peregrine_b200.mesher import CubeMesher, fill_node_halos, reorient

    tgv = cases.tgv_mesh(128, (3, 3, 3), seed=0, low=30, high=56).make_blocks(2)
    assert pull_allowed(tgv) == 1
    assert pull_allowed(tgv, want=False) == 0
    thin = cases.tgv_mesh(8, (4, 3, 1), seed=1, low=1, high=4).make_blocks(2)
    assert min(b.cells[0] for b in thin) < 2
    assert pull_allowed(thin) == 0
    # a periodic pair: in the identity orientation, then with the second
    # block laid out along other axes
    for S, want in (("123", 1), ("213", 0), ("456", 0)):
        blocks = CubeMesher(mbdims=[2, 1, 1], blkdims=[6, 4, 4], lengths=[2, 1, 1],
                            periodic=[True] * 3).make_blocks(2)
        if S != "123":
            reorient(blocks, 1, S)
            fill_node_halos(blocks)
        assert pull_allowed(blocks) == want, S
    # a wall (a face with no neighbour), and a rotational periodic
    assert pull_allowed(pair("123")) == 0
    mesher = AnnulusMesher(mbdims=[1, 1, 2], blkdims=[5, 5, 6], p1=[0, 0, 0], p2=[1, 0, 0], p3=[0, 0.5, 0],
                           sweep=90, thickness=0.5, periodic=True, defaultbc="wall")
    assert pull_allowed(mesher.make_blocks(2)) == 0
