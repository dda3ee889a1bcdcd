"""Block geometry: nodes with halo, and the finite-volume metrics made of them.

The metrics are the reference's (peregrine/multiblock/block/grid.py:90-202),
formed with the same floating-point operations in the same order so the
arrays agree bit for bit with the reference's on the same nodes:

* cell centres, the mean of a cell's eight corner nodes (grid.py:97-108);
* face centres, the mean of a face's four nodes (grid.py:110-114);
* face area vectors, half the cross product of the face diagonals over the
  cyclic axis pair (grid.py:116-121);
* volumes, the body diagonal dotted with the sum of the three high faces,
  over three (grid.py:147-156); ``detJinv`` = 1 / volume (grid.py:158-162);
* ``Jinv``, the adjugate of the cell's edge-mean Jacobian over the volume
  (grid.py:178-202).

All host arrays here are numpy, indexed ``[i, j, k, component...]`` like the
reference's host views.
"""

import numpy as np

METRICS = ("xcc", "detJinv", "Jinv", "iS", "jS", "kS", "ixc", "jxc", "kxc")


def _corner(nodes, axes, highs):
    s = [slice(None)] * 3
    for a, high in zip(axes, highs):
        s[a] = slice(1, None) if high else slice(None, -1)
    return nodes[tuple(s)]


def cell_centres(nodes):
    c = [_corner(nodes, (0, 1, 2), h) for h in
         ((0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1))]
    total = c[0] + c[1]
    for x in c[2:]:
        total = total + x
    return 0.125 * total


def face_centres(nodes, axis):
    inplane = [a for a in range(3) if a != axis]
    c00, c01, c10, c11 = (_corner(nodes, inplane, h) for h in ((0, 0), (0, 1), (1, 0), (1, 1)))
    return 0.25 * (c00 + c01 + c10 + c11)


def area_vectors(nodes, axis):
    pair = [(axis + 1) % 3, (axis + 2) % 3]
    c00, c01, c10, c11 = (_corner(nodes, pair, h) for h in ((0, 0), (0, 1), (1, 0), (1, 1)))
    return 0.5 * np.cross(c10 - c01, c11 - c00)


def volumes(nodes):
    diag = nodes[1:, 1:, 1:] - nodes[:-1, :-1, :-1]
    S = [area_vectors(nodes, a) for a in range(3)]
    high = S[0][1:] + S[1][:, 1:] + S[2][:, :, 1:]
    return sum(diag[..., n] * high[..., n] for n in range(3)) / 3.0


def inverse_jacobian(nodes, vol):
    c1, c2, c3, c4, c5, c6, c7, c8 = (_corner(nodes, (0, 1, 2), h) for h in
                                      ((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0),
                                       (0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)))
    dxi = 0.25 * ((c4 - c1) + (c8 - c5) + (c3 - c2) + (c7 - c6))
    deta = 0.25 * ((c2 - c1) + (c3 - c4) + (c7 - c8) + (c6 - c5))
    dzeta = 0.25 * ((c5 - c1) + (c8 - c4) + (c6 - c2) + (c7 - c3))
    rows = np.cross(deta, dzeta), np.cross(dzeta, dxi), np.cross(dxi, deta)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.stack(rows, axis=-2) / vol[..., None, None]


def metrics(nodes, ng):
    """Every metric of one block from its nodes (halo included)."""
    vol = volumes(nodes)
    interior = (slice(ng, -ng),) * 3 if ng else (slice(None),) * 3
    bad = int((vol[interior] <= 0.0).sum())
    if bad:
        raise ValueError(f"{bad} cells with no volume or a negative one")
    with np.errstate(divide="ignore"):
        detJinv = 1.0 / vol
    out = dict(xcc=cell_centres(nodes), detJinv=detJinv, Jinv=inverse_jacobian(nodes, vol))
    for a, d in enumerate("ijk"):
        out[f"{d}S"] = area_vectors(nodes, a)
        out[f"{d}xc"] = face_centres(nodes, a)
    return out
