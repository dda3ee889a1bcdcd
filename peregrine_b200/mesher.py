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
"""

import numpy as np


class Interface:
    def __init__(self, nface):
        self.nface = nface
        self.axis = (nface - 1) // 2
        self.is_low = nface % 2 == 1
        self.nbr = None          # neighbour block number, None at a boundary
        self.nbrface = None      # the neighbour's face across
        self.orient = "123"
        self.xlate = np.zeros(3)  # periodic translation of what lands in this halo
        self.periodic = False
        self.bcname = None


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
                nbr = blocks[face.nbr]
                src = list(inplane)
                # the neighbour's plane one in from the shared plane, then deeper by layer
                if face.is_low:
                    src[a] = g + nbr.extents[a] - 2 - layer
                else:
                    src[a] = g + 1 + layer
                blk.nodes[tuple(dst)] = nbr.nodes[tuple(src)] + face.xlate


def uneven_cuts(total, pieces, low, high, rng):
    """Per-axis block sizes in [low, high] cells that sum to total, drawn from rng."""
    for _ in range(100000):
        cuts = rng.integers(low, high + 1, size=pieces - 1)
        last = total - int(cuts.sum())
        if low <= last <= high:
            return [int(c) for c in cuts] + [last]
    raise ValueError(f"no cut of {total} into {pieces} pieces of {low}..{high}")
