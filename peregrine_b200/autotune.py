"""Picks the fused kernel's launch shape and tiles for a case by timing them.

The batched path's uniform-metric kernel comes in several launch shapes
(threads per CTA x the CTAs per SM its registers are bounded for), and each
block's tile (columns across, rows across, planes per work item) sets how
much of a tile is halo and how evenly the work queue drains.  The tuner
times a few steps of each candidate on the case itself, on the device, and
keeps the fastest; the state it steps is put back afterwards.
"""

import ctypes
import itertools

import numpy as np

from peregrine_b200 import native

KSPLITS = (1, 2, 3, 4)


def shapes():
    """The uniform kernel's instances the library has: (threads, minblocks, width, height)."""
    buf = (ctypes.c_int * 64)()
    n = ctypes.c_int()
    native.call("pgb_fused_shapes", buf, 16, ctypes.byref(n))
    return [tuple(buf[4 * q:4 * q + 4]) for q in range(n.value)]


def _time(mb, dt, steps):
    native.call("pgb_step", mb.case, float(dt), int(steps), native.PATH_BATCHED, 0)
    ms = ctypes.c_float()
    native.call("pgb_last_step_ms", mb.case, ctypes.byref(ms))
    return ms.value / steps


def _tiles(mb, threads, ksplit):
    """Each block's tile for a launch shape: the library's default columns and
    rows for that shape, k in ksplit runs."""
    out = []
    for n, b in enumerate(mb.mesh_blocks):
        native.call("pgb_set_tile", mb.case, n, 0, 0, 1)  # back to the shape's default
        tw, th, _ = mb.get_tile(n)
        out.append((tw, th, -(-b.cells[2] // ksplit)))
    return out


def tune(mb, dt, steps=3, only=None, ksplits=KSPLITS, verbose=False):
    """Times every candidate; leaves the fastest set on the case and returns it."""
    if mb.path != native.PATH_BATCHED:
        return None
    saved = [b.Q.get() for b in mb.blocks]
    results = []
    cands = [s[:3] for s in shapes()]
    if only is not None:
        cands = [c for c in cands if c in only]
    for (threads, minb, width), ksplit in itertools.product(cands, ksplits):
        try:
            native.call("pgb_set_fused_shape", mb.case, threads, minb, width)
            for n, (tw, th, kc) in enumerate(_tiles(mb, threads, ksplit)):
                mb.set_tile(n, tw, th, kc)
            _time(mb, dt, 1)
            ms = _time(mb, dt, steps)
        except native.PgbError as e:
            if verbose:
                print(f"  {threads}x{minb} k/{ksplit}: {e}")
            continue
        results.append((ms, threads, minb, width, ksplit))
        if verbose:
            print(f"  {threads}x{minb} w{width} k/{ksplit}: {ms:.4f} ms/step")
    if not results:
        return None
    ms, threads, minb, width, ksplit = min(results)
    native.call("pgb_set_fused_shape", mb.case, threads, minb, width)
    for n, (tw, th, kc) in enumerate(_tiles(mb, threads, ksplit)):
        mb.set_tile(n, tw, th, kc)
    for b, q in zip(mb.blocks, saved):
        b.Q.set(q)
    return {"threads": threads, "minblocks": minb, "width": width, "ksplit": ksplit, "ms_per_step": ms,
            "candidates": len(results), "all": sorted((round(r[0], 4),) + r[1:] for r in results)}
