"""Blocks over GPUs: a grid's blocks partitioned to ranks, each rank's halo
cells traded with the others once per stage, and a solver that steps its
rank's blocks a stage at a time so the trades fall between stages.

The reference places whole blocks on MPI ranks by weight
(peregrine/partition/base.py:30-72, docs/files.md:72-80) and trades each
exchanged array's halo planes through persistent per-neighbour messages,
staged through pinned host memory by default or direct on device pointers
(peregrine/multiblock/collections/exchange/message/{buffer,hoststaged,device}.py,
exchange/pool.py:9-71).  Here:

* ``partition`` weighs a block as the reference does (its interior cells,
  plus 0.25 an interior cell for every halo cell behind each interface and
  0.06 more for a traded one) and places the heaviest block first on the
  rank it shares the most interface with among those with room, else the
  least loaded;
* ``ExchangePlan`` lists, for each pair of ranks, the halo cells one fills
  from the other's blocks, in one order both sides agree on (the global
  halo entries' order, which the library lists on the host,
  ``pgb_case_halo_entries``); a halo cell the rank's own fill cannot reach
  (an edge cell whose first hop crosses to another rank) is traded too, with
  the rank itself when its source is local;
* ``trade`` moves the values through torch.distributed point-to-point
  sends: host tensors (gloo, the reference's host-staged default) or
  device tensors (NCCL over NVLink, its device mode);
* ``ShardedSolver`` holds the rank's blocks as its own case, packs the send
  cells on the device (``pgb_exchange_pack``), trades, unpacks into the halo
  (``pgb_exchange_unpack``) and runs the stage (``pgb_step_stage``).

Only the conserved register Q is traded, once per stage.  The batched
path's fused stage kernel forms each tile's gradients from Q's two-deep
halo, so a viscous shard steps there; the per-block kernels and the fused
passes exchange the gradients' first halo layer inside a stage, which a
trade between stages does not give them, so they take inviscid shards and
refuse viscous ones.  Rotationally periodic interfaces across ranks are not
traded.
"""

import ctypes

import numpy as np

from peregrine_b200 import native

NG = 2
HALOCOST, TRADECOST = 0.25, 0.06


def _plane(blk, face):
    cells = list(blk.cells)
    del cells[face.axis]
    return cells[0] * cells[1]


def block_weights(blocks, ng=NG, halocost=HALOCOST, tradecost=TRADECOST):
    """Each block's work in interior cells: its cells, plus every halo cell
    behind its interfaces at halocost and, behind a traded one, tradecost
    more (the reference's weights, peregrine/partition/base.py:56-62)."""
    w = np.array([float(b.ncells) for b in blocks])
    for b in blocks:
        for face in b.intfaces:
            trade = tradecost if face.nbr is not None else 0.0
            w[b.nblki] += (halocost + trade) * ng * _plane(b, face)
    return w


def partition(blocks, nranks, tol=0.05, **costs):
    """The rank of each block: heaviest first, onto the rank with room
    (within tol of an even share) it shares the most interface cells with,
    else onto the least loaded rank."""
    nb = len(blocks)
    if nranks < 1:
        raise ValueError("at least one rank")
    w = block_weights(blocks, **costs)
    cap = w.sum() / nranks * (1.0 + tol)
    owner = np.full(nb, -1, dtype=np.int64)
    load = np.zeros(nranks)
    for b in np.argsort(-w, kind="stable"):
        aff = np.zeros(nranks)
        for face in blocks[b].intfaces:
            if face.nbr is not None and owner[face.nbr] >= 0:
                aff[owner[face.nbr]] += _plane(blocks[b], face)
        room = load + w[b] <= cap
        if room.any() and aff[room].max() > 0.0:
            cand = np.flatnonzero(room)
            r = int(cand[np.argmax(aff[cand])])
        else:
            r = int(np.argmin(load))
        owner[b] = r
        load[r] += w[b]
    return owner


def _scratch_case(blocks, connect=None):
    """A case holding the blocks' extents and connectivity alone (never
    finalized: no device memory), to list its halo entries.  connect(blk,
    face) gives the neighbour to join, None for a face left unfilled."""
    phys = native.Physics(simulator=native.EULER, eos=native.EOS_CPG, primary=native.FLUX_KEPAEC,
                          recon=native.RECON_CONSTANT, limiter=0, trans=native.TRANS_NONE, ns=1, nregs=2, alpha=1.0)
    h = ctypes.c_void_p()
    native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(h))
    try:
        for b in blocks:
            out = ctypes.c_int()
            native.call("pgb_case_add_block", h, *b.cells, ctypes.byref(out))
        for b in blocks:
            for face in b.intfaces:
                nbr = face.nbr if connect is None else connect(b, face)
                if nbr is None:
                    continue
                if getattr(face, "rotperiodic", False):
                    raise NotImplementedError("a rotationally periodic interface across ranks is not traded")
                if face.orient != "123":
                    native.call("pgb_case_connect_oriented", h, b.nblki, face.nface, nbr, face.orient.encode(), None)
                else:
                    native.call("pgb_case_connect", h, b.nblki, face.nface, nbr, face.nbrface or 0)
        n = ctypes.c_longlong()
        native.call("pgb_case_halo_entries", h, 0, None, ctypes.byref(n))
        out = np.zeros((n.value, 6), dtype=np.int64)
        native.call("pgb_case_halo_entries", h, n.value, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                    ctypes.byref(n))
        return out
    finally:
        native.call("pgb_case_destroy", h)


def halo_entries(blocks):
    """Every halo cell the grid's interfaces fill: rows (dst block, dst cell
    index, src block, src cell index, rotation, layer flag), full layouts."""
    return _scratch_case(blocks)


class ExchangePlan:
    """Who trades which halo cells with whom.  For rank r: ``send[q]`` the
    (local block, cell index) pairs it packs for rank q, ``recv[q]`` the halo
    cells it fills from q's pack, both in the global entries' order."""

    def __init__(self, blocks, owner, rank):
        owner = np.asarray(owner)
        self.owner, self.rank = owner, rank
        self.nranks = int(owner.max()) + 1
        self.local = [int(b) for b in np.flatnonzero(owner == rank)]
        glob = halo_entries(blocks)
        if np.any(glob[:, 4] != 0):
            raise NotImplementedError("a rotationally periodic interface across ranks is not traded")
        # each rank's own fill: its blocks' entries with the other ranks' faces unjoined
        own = {}
        for r in range(self.nranks):
            mine = set(int(b) for b in np.flatnonzero(owner == r))
            order = sorted(mine)
            lid = {g: n for n, g in enumerate(order)}
            sub = [blocks[g] for g in order]

            def join(b, face, lid=lid, order=order):
                return lid.get(face.nbr) if face.nbr is not None else None

            loc = _scratch_case(_Renumbered(sub), join) if sub else np.zeros((0, 6), np.int64)
            own[r] = set(zip((order[int(d)] for d in loc[:, 0]), loc[:, 1].tolist()))
        # a global entry is traded when its destination's rank cannot fill it
        dst_rank = owner[glob[:, 0]]
        src_rank = owner[glob[:, 2]]
        traded = np.array([(int(d), int(i)) not in own[int(r)] for d, i, r in zip(glob[:, 0], glob[:, 1], dst_rank)],
                          dtype=bool)
        lid = {g: n for n, g in enumerate(self.local)}
        self.send, self.recv = {}, {}
        for q in range(self.nranks):
            s = glob[traded & (src_rank == rank) & (dst_rank == q)]
            self.send[q] = np.array([(lid[int(b)], int(i)) for b, i in s[:, 2:4]], dtype=np.int64).reshape(-1, 2)
            r = glob[traded & (dst_rank == rank) & (src_rank == q)]
            self.recv[q] = np.array([(lid[int(b)], int(i)) for b, i in r[:, 0:2]], dtype=np.int64).reshape(-1, 2)

    def counts(self):
        return ([len(self.send[q]) for q in range(self.nranks)], [len(self.recv[q]) for q in range(self.nranks)])

    def flat(self, which):
        """The lists of every peer end to end, in rank order."""
        d = self.send if which == "send" else self.recv
        rows = [d[q] for q in range(self.nranks)]
        return np.concatenate(rows) if rows else np.zeros((0, 2), np.int64)


class _Renumbered:
    """A subset of mesher blocks read with local numbers, 0 .. n-1."""

    def __init__(self, blocks):
        self.blocks = blocks

    def __iter__(self):
        for n, b in enumerate(self.blocks):
            yield _View(b, n)

    def __len__(self):
        return len(self.blocks)


class _View:
    def __init__(self, blk, n):
        self._blk, self.nblki = blk, n

    def __getattr__(self, name):
        return getattr(self._blk, name)


def trade(plan, packed, group=None):
    """One trade: packed[q] the values this rank sends q (ne x n_q tensors,
    host or device); returns the values each peer sent, by rank.  A rank's
    trade with itself is a copy; the others are point-to-point sends and
    receives, posted together (torch.distributed: gloo for host tensors,
    NCCL for device ones)."""
    import torch
    import torch.distributed as dist

    out, reqs = {}, []
    for q in range(plan.nranks):
        if q == plan.rank:
            continue
        n = len(plan.recv[q])
        ref = packed[plan.rank] if plan.rank in packed else next(iter(packed.values()))
        out[q] = torch.empty((ref.shape[0], n), dtype=ref.dtype, device=ref.device)
    for q in range(plan.nranks):
        if q == plan.rank:
            continue
        if len(plan.recv[q]):
            reqs.append(dist.irecv(out[q], src=q, group=group))
        if len(plan.send[q]):
            reqs.append(dist.isend(packed[q].contiguous(), dst=q, group=group))
    for r in reqs:
        r.wait()
    out[plan.rank] = packed[plan.rank]
    return out


CFL_KEYS = ("acoustic", "convective", "combined")


def reduce_cfl(local, group=None, device=None):
    """The CFL numbers over every rank's blocks: each rank's own maxima, then
    a MAX over the ranks (the reference's Allreduce of its cflmax speeds,
    peregrine/multiblock/solver.py:292-296).  device: a CUDA device for the
    tensor (NCCL), None for a host tensor (gloo)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(local[k]) for k in CFL_KEYS], dtype=torch.float64)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return dict(zip(CFL_KEYS, t.cpu().tolist()))


def cfl_stepsize(cfl, dtmax, cflmax):
    """The cfl controller's step (peregrine/integrators/controllers.py:21-26)."""
    return min(cfl / cflmax["combined"], dtmax)


class LocalMesh:
    """A rank's blocks of a mesh, numbered 0 .. n-1 in global order; a face
    joined to another rank's block is left unjoined (its halo is traded)."""

    def __init__(self, mesh, owner, rank):
        self.mesh, self.owner, self.rank = mesh, np.asarray(owner), rank

    def make_blocks(self, ng):
        every = self.mesh.make_blocks(ng)
        order = [b for b in range(len(every)) if self.owner[b] == self.rank]
        lid = {g: n for n, g in enumerate(order)}
        out = []
        for g in order:
            b = every[g]
            b.global_nblki = g
            b.nblki = lid[g]
            for face in b.intfaces:
                if face.nbr is None:
                    continue
                if face.nbr in lid:
                    face.nbr = lid[face.nbr]
                else:
                    face.remote = face.nbr
                    face.nbr = None
            out.append(b)
        return out


class ShardedSolver:
    """A rank's share of a case: its blocks as a case of their own, stepped a
    stage at a time, the halo traded between stages.  ``exchange`` is
    "host" (device -> host tensors, gloo or any backend) or "device" (device
    tensors, NCCL)."""

    def __init__(self, cfg, mesh, backend, owner, rank, exchange="host", group=None):
        import peregrine_b200 as pg

        self.owner, self.rank, self.group, self.mode = np.asarray(owner), rank, group, exchange
        self.plan = ExchangePlan(mesh.make_blocks(NG), owner, rank)
        self.solver = pg.get_solver(cfg, LocalMesh(mesh, owner, rank), backend)
        if cfg["simulation"]["simulator"] == "navier-stokes" and not (
                self.solver.path == native.PATH_BATCHED and self.solver.batched_form() == 1):
            # the per-block kernels and the fused passes exchange the gradients'
            # first halo layer inside a stage; only the fused stage kernel forms
            # them from Q's two-deep halo, which the trade between stages fills
            raise NotImplementedError("a viscous shard steps on the batched path's fused stage kernel alone")
        s, r = self.plan.flat("send"), self.plan.flat("recv")
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        sb, si, rb, ri = i32(s[:, 0]), i32(s[:, 1]), i32(r[:, 0]), i32(r[:, 1])
        p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        native.call("pgb_case_set_exchange", self.solver.case, len(s), p(sb), p(si), len(r), p(rb), p(ri))
        self.nsend, self.nrecv = self.plan.counts()
        from peregrine_b200.integrators import stages

        self.nstages = len(stages(self.solver.integrator)[0])

    def __getattr__(self, name):
        return getattr(self.solver, name)

    def _trade_stage(self, s):
        import torch

        mb = self.solver
        ne = mb.ne
        dev = torch.device("cuda", torch.cuda.current_device())
        nsend, nrecv = sum(self.nsend), sum(self.nrecv)
        sbuf = torch.empty((ne, max(nsend, 1)), dtype=torch.float64, device=dev)
        stream = torch.cuda.ExternalStream(mb.stream())
        native.call("pgb_exchange_pack", mb.case, s, mb.path, ctypes.c_void_p(sbuf.data_ptr()))
        with torch.cuda.stream(stream):
            packed, off = {}, 0
            for q in range(self.plan.nranks):
                chunk = sbuf[:, off:off + self.nsend[q]]
                packed[q] = chunk.cpu() if self.mode == "host" else chunk.contiguous()
                off += self.nsend[q]
            stream.synchronize()
            got = trade(self.plan, packed, self.group)
            rbuf = torch.empty((ne, max(nrecv, 1)), dtype=torch.float64, device=dev)
            off = 0
            for q in range(self.plan.nranks):
                if self.nrecv[q]:
                    rbuf[:, off:off + self.nrecv[q]].copy_(got[q].to(dev))
                off += self.nrecv[q]
            stream.synchronize()
        native.call("pgb_exchange_unpack", mb.case, s, mb.path, ctypes.c_void_p(rbuf.data_ptr()))

    def cflmax(self):
        """The CFL numbers over every rank's blocks."""
        import torch

        dev = torch.device("cuda", torch.cuda.current_device()) if self.mode == "device" else None
        return reduce_cfl(self.solver.cflmax(), self.group, dev)

    def step_cfl(self, cfl, dtmax, nsteps=1):
        """nsteps steps under the cfl controller, each step's size from the
        CFL numbers over every rank's blocks; returns the last step's size."""
        dt = None
        for _ in range(nsteps):
            dt = cfl_stepsize(cfl, dtmax, self.cflmax())
            self.step(dt, 1)
        return dt

    def step(self, dt, nsteps=1):
        mb = self.solver
        native.call("pgb_set_dt", mb.case, float(dt))
        for _ in range(nsteps):
            for s in range(self.nstages):
                self._trade_stage(s)
                native.call("pgb_step_stage", mb.case, s, mb.path)
        mb.nrt += nsteps
        mb.tme += dt * nsteps
