"""Structured block lattices: the blocks, their nodes and their connectivity.

``CubeMesher`` follows the reference's (peregrine/mesher/cube.py:6-53,
peregrine/mesher/base.py:65-133): a box cut into an ``mbdims`` lattice of
blocks, numbered ``k * mbj * mbi + j * mbi + i`` (base.py:88-92), faces
numbered 1..6 as i-low, i-high, j-low, j-high, k-low, k-high, orientation
"123", periodic axes joining the last block to the first with a translation
of one box length (cube.py:34-42).  Beyond the reference it takes uneven cuts:
``cells`` gives each axis's per-block cell counts, so a 128-cell axis can be
cut 41 + 30 + 57.  ``blkdims`` (nodes per block, every block alike) is the
reference's form and still accepted.

An interface's orientation is the reference's three digits: for each axis
of the block, the neighbour's axis it runs along, 1-3 forward and 4-6
backward (peregrine/multiblock/interface/base.py:96-160).  ``reorient``
lays a block out along other axes, its neighbours' digits following, as
the reference's partitioner does; ``AnnulusMesher`` sweeps blocks about an
axis, its ends joined as rotational periodics (peregrine/mesher/annulus.py).
"""

import numpy as np


def signedaxis(code):
    """An orientation digit's axis and whether it runs backward."""
    n = int(code)
    return (n - 1) % 3, n > 3


def orientcode(axis, flip):
    return str(axis + 1 + (3 if flip else 0))


def rotabout(axis, deg):
    """The rotation by deg degrees about axis (Rodrigues' formula)."""
    u = np.asarray(axis, np.float64)
    u = u / np.linalg.norm(u)
    th = np.radians(deg)
    ct, st = np.cos(th), np.sin(th)
    x, y, z = u
    cross = np.array([[0.0, -z, y], [z, 0.0, -x], [-y, x, 0.0]])
    return ct * np.eye(3) + st * cross + (1.0 - ct) * np.outer(u, u)


class Interface:
    def __init__(self, nface):
        self.nface = nface
        self.axis = (nface - 1) // 2
        self.is_low = nface % 2 == 1
        self.nbr = None          # neighbour block number, None at a boundary
        self.nbrface = None      # the neighbour's face across
        self.orient = "123"
        self.xlate = np.zeros(3)  # periodic translation of what lands in this halo
        self.rot = None           # a rotational periodic's turn of what lands in this halo
        self.periodic = False
        self.bcname = None

    @property
    def rotperiodic(self):
        return self.rot is not None and not np.allclose(self.rot, np.eye(3))

    def set_nbrface(self):
        """The neighbour's face, from the digit of this face's own axis: a low
        face meets the neighbour's high one unless the axis runs backward."""
        axis, flip = signedaxis(self.orient[self.axis])
        self.nbrface = 2 * axis + (1 if self.is_low == flip else 2)

    def inframe(self, a):
        """An array of the neighbour's cells or nodes (its three index axes
        first) laid out along this block's axes."""
        out = np.moveaxis(a, [signedaxis(c)[0] for c in self.orient], [0, 1, 2])
        for m, c in enumerate(self.orient):
            if signedaxis(c)[1]:
                out = np.flip(out, axis=m)
        return out


class Block:
    def __init__(self, nblki, ni, nj, nk, ng):
        self.nblki = nblki
        self.ni, self.nj, self.nk = ni, nj, nk      # nodes per axis, as the reference's extents
        self.ng = ng
        self.intfaces = [Interface(f) for f in range(1, 7)]
        self.nodes = np.zeros((ni + 2 * ng, nj + 2 * ng, nk + 2 * ng, 3))

    @property
    def extents(self):
        return (self.ni, self.nj, self.nk)

    @property
    def cells(self):
        return (self.ni - 1, self.nj - 1, self.nk - 1)

    @property
    def ncells(self):
        return int(np.prod(self.cells))

    @property
    def interior(self):
        g = self.ng
        return np.s_[g:-g, g:-g, g:-g]

    def get_intface(self, nface):
        return self.intfaces[nface - 1]


class CubeMesher:
    name = "cube"

    def __init__(self, mbdims=(1, 1, 1), blkdims=None, cells=None, lengths=(1.0, 1.0, 1.0),
                 origin=(0.0, 0.0, 0.0), periodic=(False, False, False), bcnames=None, defaultbc=None,
                 jostle=0.0, jostle_seed=7):
        self.mbdims = [int(n) for n in mbdims]
        if cells is None:
            if blkdims is None:
                raise ValueError("a cube takes blkdims (nodes per block) or cells (per-axis cuts)")
            cells = [[int(blkdims[a]) - 1] * self.mbdims[a] for a in range(3)]
        self.cells = [[int(c) for c in axis] for axis in cells]
        for a in range(3):
            if len(self.cells[a]) != self.mbdims[a] or min(self.cells[a]) < 1:
                raise ValueError(f"axis {a}: {self.cells[a]} does not cut {self.mbdims[a]} blocks")
        self.lengths = [float(x) for x in lengths]
        self.origin = [float(x) for x in origin]
        self.periodic = [bool(p) for p in periodic]
        self.bcnames = dict(bcnames or {})
        self.defaultbc = defaultbc
        # moves every node inside a block (not its faces) by up to jostle
        # spacings, so no face normal is an axis (the reference's test
        # JostledCube, tests/simulator/support.py:48-56)
        self.jostle = float(jostle)
        self.jostle_seed = jostle_seed
        # where each block of the lattice starts, in cells and in space
        self.starts = [np.concatenate([[0], np.cumsum(c)]) for c in self.cells]

    @property
    def nblks(self):
        return int(np.prod(self.mbdims))

    def make_blocks(self, ng):
        mbi, mbj, mbk = self.mbdims
        blocks = []
        for k in range(mbk):
            for j in range(mbj):
                for i in range(mbi):
                    nblki = k * mbj * mbi + j * mbi + i
                    dims = [self.cells[a][m] + 1 for a, m in enumerate((i, j, k))]
                    blk = Block(nblki, *dims, ng)
                    self._shape(blk, (i, j, k))
                    self._connect(blk, nblki, (i, j, k))
                    blocks.append(blk)
        fill_node_halos(blocks)
        return blocks

    def _shape(self, blk, ijk):
        axes = []
        for a, m in enumerate(ijk):
            total = self.starts[a][-1]
            lo = self.origin[a] + self.lengths[a] * self.starts[a][m] / total
            hi = self.origin[a] + self.lengths[a] * self.starts[a][m + 1] / total
            axes.append(np.linspace(lo, hi, self.cells[a][m] + 1))
        grid = np.meshgrid(*axes, indexing="ij")
        blk.nodes[blk.interior] = np.stack(grid, axis=-1)
        if self.jostle:
            g = blk.ng
            inner = np.s_[g + 1:-g - 1, g + 1:-g - 1, g + 1:-g - 1]
            spacing = min(self.lengths[a] / self.starts[a][-1] for a in range(3))
            rng = np.random.default_rng(self.jostle_seed + blk.nblki)
            blk.nodes[inner] += rng.uniform(-1, 1, blk.nodes[inner].shape) * self.jostle * spacing

    def _connect(self, blk, nblki, ijk):
        for axis, (n, index, wraps) in enumerate(zip(self.mbdims, ijk, self.periodic)):
            stride = int(np.prod(self.mbdims[:axis]))
            for nface, end, step in ((2 * axis + 1, 0, -1), (2 * axis + 2, n - 1, 1)):
                face = blk.get_intface(nface)
                if index != end:
                    face.nbr = nblki + step * stride
                elif wraps:
                    face.nbr = nblki - step * stride * (n - 1)
                    face.periodic = True
                    span = -self.lengths[axis] if face.is_low else self.lengths[axis]
                    face.xlate = np.array([span if m == axis else 0.0 for m in range(3)])
                else:
                    face.bcname = self.bcnames.get(nface, self.defaultbc)
                    face.orient = None
                    continue
                face.nbrface = nface + 1 if face.is_low else nface - 1


def fill_node_halos(blocks):
    """The node halo: mirrored through a boundary plane, the neighbour's nodes across an interface.

    A face halo across an interface is the neighbour's node planes one in from
    the shared plane (the reference's node exchange starts one plane in,
    peregrine/launch/ranges.py:122-124), moved by the periodic translation
    (peregrine/multiblock/block/grid.py:279-288).  At a boundary each halo layer
    is the mirror image through the boundary plane (grid.py:225-234).  Edge
    and corner halo nodes, which the reference leaves as extrapolations no
    kernel reads, are linear extrapolations here.
    """
    for blk in blocks:
        x, g = blk.nodes, blk.ng
        for axis in range(3):
            planes = np.moveaxis(x, axis, 0)
            n = planes.shape[0]
            for layer in range(g):
                lo, hi = g - 1 - layer, n - g + layer
                planes[lo] = 2.0 * planes[lo + 1] - planes[lo + 2]
                planes[hi] = 2.0 * planes[hi - 1] - planes[hi - 2]
    # the interface planes proper (no edges), mirrored or exchanged
    for blk in blocks:
        g = blk.ng
        for face in blk.intfaces:
            a = face.axis
            inplane = [slice(g, g + blk.extents[m]) if m != a else None for m in range(3)]
            for layer in range(g):
                dst = list(inplane)
                dst[a] = g - 1 - layer if face.is_low else g + blk.extents[a] + layer
                if face.nbr is None:
                    src = list(inplane)
                    # the mirror: 2 x(plane) - x(plane + layer + 1 inward)
                    edge = g if face.is_low else g + blk.extents[a] - 1
                    step = 1 if face.is_low else -1
                    near, far = list(inplane), list(inplane)
                    near[a], far[a] = edge, edge + step * (layer + 1)
                    blk.nodes[tuple(dst)] = 2.0 * blk.nodes[tuple(near)] - blk.nodes[tuple(far)]
                    continue
                # the neighbour's nodes (its halo as wide on every side) along
                # this block's axes, then its plane one in from the shared
                # plane, deeper by layer (past a thin neighbour, into its halo)
                nbr = face.inframe(blocks[face.nbr].nodes)
                src = list(inplane)
                src[a] = nbr.shape[a] - g - 2 - layer if face.is_low else g + 1 + layer
                x = nbr[tuple(src)]
                if face.rot is not None:
                    x = x @ np.asarray(face.rot).T
                blk.nodes[tuple(dst)] = x + face.xlate


def reorient(blocks, n, S):
    """Block n laid out along other axes: its old axis m becomes axis
    axes[m] of the new layout, running backward where flips[m] (S the
    reference's digits; tests/communication/test_orientation.py:39-46), its
    faces and its neighbours' orientation digits following."""
    axes = [signedaxis(c)[0] for c in S]
    flips = [signedaxis(c)[1] for c in S]
    blk = blocks[n]
    # the digits of every face across into block n: its axis t is now axes[t]
    for other in blocks:
        for face in other.intfaces:
            if face.nbr == n:
                codes = [signedaxis(c) for c in face.orient]
                face.orient = "".join(orientcode(axes[t], f != flips[t]) for t, f in codes)
    # block n's own faces move with its axes, and their digits with them
    old = list(blk.intfaces)
    new = [None] * 6
    for face in old:
        m = face.axis
        low = face.is_low != flips[m]
        nface = 2 * axes[m] + (1 if low else 2)
        if face.nbr is not None:
            codes = [None] * 3
            for d, c in enumerate(face.orient):
                t, f = signedaxis(c)
                codes[axes[d]] = orientcode(t, f != flips[d])
            face.orient = "".join(codes)
        face.nface, face.axis, face.is_low = nface, (nface - 1) // 2, nface % 2 == 1
        new[nface - 1] = face
    blk.intfaces = new
    out = blk.nodes
    for m, f in enumerate(flips):
        if f:
            out = np.flip(out, axis=m)
    blk.nodes = np.ascontiguousarray(np.moveaxis(out, (0, 1, 2), axes))
    ext = [None] * 3
    for m in range(3):
        ext[axes[m]] = blk.extents[m]
    blk.ni, blk.nj, blk.nk = ext
    for other in blocks:
        for face in other.intfaces:
            if face.nbr is not None:
                face.set_nbrface()


class AnnulusMesher:
    """Blocks swept about the axis p1 -> p2 (peregrine/mesher/annulus.py):
    i along the axis, j out from it from the radius of p3 by thickness, k
    round it through sweep degrees; periodic joins the sweep's ends, as a
    rotational periodic whose low face takes its halo turned back by the
    sweep and whose high face turned on by it (annulus.py:82-94)."""

    name = "annulus"

    def __init__(self, mbdims=(1, 1, 1), blkdims=(5, 5, 5), p1=(0, 0, 0), p2=(1, 0, 0), p3=(0, 1, 0), sweep=45.0,
                 thickness=0.1, periodic=False, bcnames=None, defaultbc=None):
        self.mbdims = [int(n) for n in mbdims]
        self.blkdims = [int(n) for n in blkdims]
        self.p1, self.p2, self.p3 = (np.asarray(p, np.float64) for p in (p1, p2, p3))
        self.sweep, self.thickness, self.periodic = float(sweep), float(thickness), bool(periodic)
        self.bcnames = dict(bcnames or {})
        self.defaultbc = defaultbc
        length = np.linalg.norm(self.p2 - self.p1)
        rin = np.linalg.norm(self.p3 - self.p1)
        if length == 0.0 or rin == 0.0:
            raise ValueError("p1 -> p2 is the axis and p3 off it")
        self.axis = (self.p2 - self.p1) / length
        self.radial = (self.p3 - self.p1) / rin
        if abs(np.dot(self.axis, self.radial)) > 1e-7:
            raise ValueError("the line (p1, p3) is not orthogonal to (p1, p2)")
        if not 0.0 < self.sweep <= 360.0:
            raise ValueError("the sweep is more than 0 and at most 360 degrees")
        self.edges = [np.linspace(0.0, length, self.mbdims[0] + 1),
                      np.linspace(rin, rin + self.thickness, self.mbdims[1] + 1),
                      np.linspace(0.0, self.sweep, self.mbdims[2] + 1)]

    def _turn(self, p, theta):
        n = self.axis
        ct, st = np.cos(theta)[:, None], np.sin(theta)[:, None]
        return ct * p + st * np.cross(n, p) + (1.0 - ct) * np.dot(n, p) * n

    def make_blocks(self, ng):
        mbi, mbj, mbk = self.mbdims
        blocks = []
        for k in range(mbk):
            for j in range(mbj):
                for i in range(mbi):
                    nblki = k * mbj * mbi + j * mbi + i
                    blk = Block(nblki, *self.blkdims, ng)
                    x, r, theta = (np.linspace(e[m], e[m + 1], nn)
                                   for e, m, nn in zip(self.edges, (i, j, k), self.blkdims))
                    radial = self._turn(self.radial, np.radians(theta))
                    pts = (self.p1 + x[:, None, None, None] * self.axis +
                           r[None, :, None, None] * radial[None, None, :, :])
                    blk.nodes[blk.interior] = pts
                    for axis, (nb, index) in enumerate(zip(self.mbdims, (i, j, k))):
                        stride = int(np.prod(self.mbdims[:axis]))
                        for nface, end, step in ((2 * axis + 1, 0, -1), (2 * axis + 2, nb - 1, 1)):
                            face = blk.get_intface(nface)
                            if index != end:
                                face.nbr = nblki + step * stride
                            elif axis == 2 and self.periodic:
                                face.nbr = nblki - step * stride * (nb - 1)
                                face.periodic = True
                                if self.sweep != 360.0:
                                    face.rot = rotabout(self.axis, -self.sweep if face.is_low else self.sweep)
                            else:
                                face.bcname = self.bcnames.get(nface, self.defaultbc)
                                continue
                            face.set_nbrface()
                    blocks.append(blk)
        fill_node_halos(blocks)
        return blocks


def uneven_cuts(total, pieces, low, high, rng):
    """Per-axis block sizes in [low, high] cells that sum to total, drawn from rng."""
    for _ in range(100000):
        cuts = rng.integers(low, high + 1, size=pieces - 1)
        last = total - int(cuts.sum())
        if low <= last <= high:
            return [int(c) for c in cuts] + [last]
    raise ValueError(f"no cut of {total} into {pieces} pieces of {low}..{high}")
