"""Serving: independent reacting cases admitted while others run.

A request is one small case, a single block periodic onto itself: a
uniform 2 x 2 x 2 box (a closed constant-volume reactor, as the reference's
auto-ignition example builds one, examples/autoIgnition.py:33-56) or an
N x 2 x 2 periodic 1-D domain.  The ``Pool`` keeps every admitted case's
state on the device (pgb_pool_* in include/pgb200.h); each step advances
every running case in the same launches, at one shared dt.  A closed
reactor's box is uniform and has no flux divergence, so the pool holds it
as one cell of a reactor table, stepped by its eos, its source and the
stage's combines (pgb_pool_admit_reactor); a 1-D domain is a block of the
arena, stepped by the fused passes.  The
``Server`` loop admits arrivals in order whenever the arena has room,
steps, and reads each case out when its step count is done, so requests
that arrive while others are on the GPU join them at the next step
(continuous batching).  Time to result is measured from a request's arrival
to the moment its result is on the host.
"""

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from peregrine_b200 import native
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.mesher import CubeMesher

NG = 2
ATM = 101325.0


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class Request:
    """One case: its block's cells, lengths (m), interior primitives
    (p, u, v, w, T, Y...; shape cells + (ne,)) and RK step count."""
    rid: int
    arrival: float
    cells: tuple
    lengths: tuple
    prims: np.ndarray
    steps: int
    kind: str = "0d"
    # filled by the server
    admitted: float = None
    finished: float = None
    result: np.ndarray = field(default=None, repr=False)


_METRICS = {}


def box_metrics(cells, lengths):
    """The grid metrics of a periodic box (cached by shape and size), from
    the same mesher and metric code every case uses."""
    key = (tuple(cells), tuple(float(x) for x in lengths))
    if key not in _METRICS:
        mesh = CubeMesher(cells=[[c] for c in cells], lengths=list(lengths), periodic=[True] * 3)
        blk = mesh.make_blocks(NG)[0]
        _METRICS[key] = make_metrics(blk.nodes, NG)
    return _METRICS[key]


class Pool:
    """The device arena of a prototype solver's physics (pgb_pool_*)."""

    def __init__(self, proto, max_cells, max_blocks=4096):
        h = ctypes.c_void_p()
        native.call("pgb_pool_create", proto.case, int(max_cells), int(max_blocks), ctypes.byref(h))
        self.handle, self.ne, self.max_blocks = h, proto.ne, max_blocks

    def close(self):
        if self.handle:
            native.call("pgb_pool_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, req):
        """The request's slot, or None when the arena has no room for it now."""
        slot = ctypes.c_int()
        if req.kind == "0d":
            q = np.asarray(req.prims, dtype=np.float64).reshape(-1, self.ne)
            if np.any(q != q[:1]):
                raise ValueError(f"request {req.rid}: a closed reactor's box is uniform")
            rc = native.load().pgb_pool_admit_reactor(self.handle, ctypes.byref(slot))
            if rc == native.ERR_NOMEM:
                return None
            native.check(rc)
            q0 = np.ascontiguousarray(q[0])
            native.call("pgb_pool_set_prims", self.handle, slot.value, _fptr(q0), q0.size)
            native.call("pgb_pool_start", self.handle, slot.value, int(req.steps))
            return slot.value
        rc = native.load().pgb_pool_admit(self.handle, *req.cells, ctypes.byref(slot))
        if rc == native.ERR_NOMEM:
            return None
        native.check(rc)
        s = slot.value
        for name, arr in box_metrics(req.cells, req.lengths).items():
            a = np.asfortranarray(np.asarray(arr, dtype=np.float64).reshape(arr.shape[:3] + (-1,)))
            native.call("pgb_pool_metric_set", self.handle, s, native.METRIC_IDS[name], _fptr(a), a.size)
        q = np.asfortranarray(np.asarray(req.prims, dtype=np.float64))
        native.call("pgb_pool_set_prims", self.handle, s, _fptr(q), q.size)
        native.call("pgb_pool_start", self.handle, s, int(req.steps))
        return s

    def step(self, dt, n=1):
        native.call("pgb_pool_step", self.handle, float(dt), int(n))
        ms, launches = ctypes.c_float(), ctypes.c_int()
        native.call("pgb_pool_last", self.handle, ctypes.byref(ms), ctypes.byref(launches))
        return ms.value, launches.value

    def done(self):
        cap = self.max_blocks
        buf = (ctypes.c_int * cap)()
        n = ctypes.c_int()
        native.call("pgb_pool_done", self.handle, buf, cap, ctypes.byref(n))
        return list(buf[: min(n.value, cap)])

    def take(self, slot, cells, kind="1d"):
        """The slot's Q over its interior (a reactor's over its box), then the
        slot is free."""
        if kind == "0d":
            one = np.zeros(self.ne)
            native.call("pgb_pool_get", self.handle, slot, 0, _fptr(one), one.size)
            native.call("pgb_pool_release", self.handle, slot)
            return np.asfortranarray(np.broadcast_to(one, tuple(cells) + (self.ne,)))
        out = np.zeros(tuple(cells) + (self.ne,), order="F")
        native.call("pgb_pool_get", self.handle, slot, 0, _fptr(out), out.size)
        native.call("pgb_pool_release", self.handle, slot)
        return out

    def info(self):
        free, run, done = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        native.call("pgb_pool_info", self.handle, ctypes.byref(free), ctypes.byref(run), ctypes.byref(done))
        return free.value, run.value, done.value


class Server:
    """Continuous batching over a Pool: admit in arrival order while there is
    room, step every running case together, read out the finished ones."""

    def __init__(self, pool, dt):
        self.pool, self.dt = pool, dt
        self.device_ms = 0.0
        self.launches = 0
        self.steps = 0
        self.cell_stages = 0
        self.running_sum = 0
        self.admit_s = 0.0
        self.admit_max_s = 0.0

    def run(self, requests, stages_per_step, clock=time.perf_counter, sleep=time.sleep):
        """Serve every request; arrival times are seconds from the start.
        Returns the requests with admitted, finished (seconds from the start)
        and result set."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        running = {}
        t0 = clock()
        q = 0
        left = len(pending)
        while left:
            now = clock() - t0
            # admit every arrival so far, in order, while the arena has room
            while q < len(pending) and pending[q].arrival <= now:
                ta = clock()
                slot = self.pool.admit(pending[q])
                took = clock() - ta
                self.admit_s += took
                self.admit_max_s = max(self.admit_max_s, took)
                if slot is None:
                    break
                pending[q].admitted = clock() - t0
                running[slot] = pending[q]
                q += 1
            if not running:
                if q < len(pending):
                    sleep(max(0.0, min(pending[q].arrival - (clock() - t0), 0.01)))
                continue
            ms, launches = self.pool.step(self.dt, 1)
            self.device_ms += ms
            self.launches += launches
            self.steps += 1
            self.running_sum += len(running)
            # a reactor is one cell
            self.cell_stages += stages_per_step * sum(1 if r.kind == "0d" else int(np.prod(r.cells))
                                                      for r in running.values())
            for slot in self.pool.done():
                req = running.pop(slot)
                req.result = self.pool.take(slot, req.cells, req.kind)
                req.finished = clock() - t0
                left -= 1
        return requests


def latency_stats(requests):
    t = np.array([r.finished - r.arrival for r in requests])
    return {"p50_ms": float(np.percentile(t, 50) * 1e3), "p99_ms": float(np.percentile(t, 99) * 1e3),
            "mean_ms": float(t.mean() * 1e3), "n": len(t)}


def h2_air(spnames, MW, phi):
    """Mass fractions of H2/air at equivalence ratio phi (H2 : O2 : N2 = 2 phi : 1 : 3.76)."""
    X = np.zeros(len(spnames))
    for name, moles in (("H2", 2.0 * phi), ("O2", 1.0), ("N2", 3.76)):
        X[list(spnames).index(name)] = moles
    Y = X * np.asarray(MW)
    return Y / Y.sum()


def requests(n, rate, spnames, MW, seed=0, steps=100, dx=1e-4, frac0d=0.5, nmin=64, nmax=2048):
    """Poisson arrivals (rate per second) of seeded H2/air cases: closed
    reactors (phi ~ U[0.5, 2], T0 ~ U[900, 1400] K, p ~ U[1, 40] atm) and
    periodic 1-D domains of N ~ log-uniform [nmin, nmax] cells of dx with a
    Gaussian hot spot (400 K over 1000 K, 8 cells wide) at phi 1 and 1 atm."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    ns = len(spnames)
    out = []
    for k in range(n):
        if rng.uniform() < frac0d:
            phi, T0, p = rng.uniform(0.5, 2.0), rng.uniform(900.0, 1400.0), rng.uniform(1.0, 40.0) * ATM
            cells = (2, 2, 2)
            q = np.zeros(cells + (4 + ns,))
            q[..., 0], q[..., 4] = p, T0
            q[..., 5:] = h2_air(spnames, MW, phi)[:-1]
            out.append(Request(k, float(t[k]), cells, (2 * dx,) * 3, q, steps, "0d"))
        else:
            N = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
            cells = (N, 2, 2)
            x = (np.arange(N) + 0.5) / N
            T = 1000.0 + 400.0 * np.exp(-0.5 * ((x - 0.5) * N / 8.0) ** 2)
            q = np.zeros(cells + (4 + ns,))
            q[..., 0] = ATM
            q[..., 4] = T[:, None, None]
            q[..., 5:] = h2_air(spnames, MW, 1.0)[:-1]
            out.append(Request(k, float(t[k]), cells, (N * dx, 2 * dx, 2 * dx), q, steps, "1d"))
    return out
