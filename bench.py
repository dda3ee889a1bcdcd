#!/usr/bin/env python
"""FP64 cell-stage updates/s of the RHS + Runge-Kutta step, on B200.

Workload (the multiblock Taylor-Green configuration): a periodic 128^3
cube on [0, 2 pi]^3 cut into 3 x 3 x 3 blocks whose per-axis sizes are drawn
from a seed in [30, 56] cells, Navier-Stokes with the kepaec flux and
alpha-damping viscous flux, calorically perfect air, constant transport at
Re 1600, Mach 0.1, RK4, FP64; seeded synthetic initial field.  One step is
one RK4 step (four stages) of every cell; the metric counts cells x stages.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The b200 arm times K steps of the batched fused path replayed as a CUDA
graph (CUDA events on the case's stream), then the same K steps with a
CUDA event after every launch for the fused kernel's own time (the roofline
line), the plain per-block path for comparison, an end-to-end leg with the
state copied in from and out to pinned host memory every step, and the CPU
oracle on a bounded sample.  With N > 1 (torchrun), every rank runs its own
replica of the workload (the cross-GPU halo exchange is not built); the
time is the max over ranks.  The reference arm times the reference CPU
restatement (oracle/, OpenMP on every host core) on the same workload.

A reacting leg (key "reacting") reports the reacting configuration beside
the headline: a single periodic block of 96^3 cells, 1 cm a side, of
stoichiometric H2/air at 1 atm and 1000 K with seeded Gaussian hot spots
(up to 400 K, 8 cells wide) and a seeded divergence-free velocity (u_rms
10 m/s); the 9-species H2/O2/N2 subset of GRI-Mech 3.0 (28 reactions,
thermally perfect, kinetic-theory transport, coupled finite-rate chemistry),
MUSCL with the koren limiter and HLLC, Navier-Stokes, TVD-RK3, on the
batched path (the fused passes), with the per-block and packed paths and
the CPU oracle on one stage of it beside it.

A real-gas leg (key "realgas") times the transcritical mixing layer: 256 x
128 x 4 cells of 20 um in 8 blocks of seeded uneven widths along i, O2 at
120 K in a band between two tanh interfaces in an H2 stream at 300 K, 60
bar, the streams 50 m/s apart with seeded 1 % noise; Peng-Robinson with the
double flux, kepaec, Euler, TVD-RK3, per-block path.

A serving leg (key "serving") plays a seeded Poisson stream of 300 H2/air
requests at 60 per second: closed constant-volume reactors (phi, T0 and p
drawn uniformly) and periodic 1-D domains of 64 to 2048 cells (log-uniform),
100 RK3 steps each at one shared dt, admitted into one device pool while
others run (peregrine_b200/serving.py); it reports throughput and the p50
and p99 time from a request's arrival to its result on the host.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CELLS = 128
BLOCKS = (3, 3, 3)
CUT_LOW, CUT_HIGH = 30, 56
SEED = 0
NE = 5
STAGES = 4
# RK4 register traffic per cell and stage, 8 ne (reads + writes): stage 0
# reads start, writes total and stage (3); stages 1, 2 read stage, total and
# start, write total and stage (5); stage 3 reads stage, total and start,
# writes start (4); the mean is 4.25 registers, 170 bytes
STAGE_REGS = (3, 5, 5, 4)
METRIC = "FP64 cell-stage updates/s, batched vs per-block, % HBM roofline; p50/p99 latency"
WORKLOAD = "tgv-128^3-27-uneven-blocks-ns-kepaec-alpha-damping-cpg-rk4"


def set_cells(n):
    global CELLS
    CELLS = n


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: the region opens once it
            # samples (within 5 s), so a short region is not left unsampled
            t0 = time.monotonic()
            while not self.samples and self.proc.poll() is None and time.monotonic() - t0 < 5.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and s[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_case(launch, device=0):
    import peregrine_b200 as pg
    from peregrine_b200 import cases

    cfg = cases.tgv_config("navier-stokes", "rk4", launch)
    mesh = cases.tgv_mesh(CELLS, BLOCKS, seed=SEED, low=CUT_LOW, high=CUT_HIGH)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg, device=device))
    prims = cases.tgv_prims(mb.mesh_blocks, mb.metrics, seed=SEED)
    mb.set_prims(prims)
    return mb, mesh, prims


def stable_dt():
    from peregrine_b200 import cases

    _, g = cases.tgv_gas()
    h = 2 * np.pi / CELLS
    return 0.3 * h / (g["U0"] + np.sqrt(g["gamma"] * g["R"] * cases.T0))


def time_graph(mb, dt, steps):
    mb.step(dt, steps)
    return mb.last_step_ms()


def fused_kernel_times(mb, dt, steps):
    import ctypes

    from peregrine_b200 import native

    cap = 64 * steps
    ms = (ctypes.c_float * cap)()
    kind = (ctypes.c_int * cap)()
    n = ctypes.c_int()
    native.call("pgb_step_timed", mb.case, float(dt), int(steps), mb.path, ms, kind, cap, ctypes.byref(n))
    rows = [(ms[q], kind[q]) for q in range(min(n.value, cap))]
    return rows


def e2e_leg(mb, dt, steps):
    import ctypes

    from peregrine_b200 import native

    n = mb.ncells * NE
    host = np.zeros(n)
    native.call("pgb_host_register", host.ctypes.data_as(ctypes.c_void_p), host.nbytes)
    ptr = host.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    try:
        native.call("pgb_state_get", mb.case, 0, ptr, n)
        # warm
        native.call("pgb_state_set", mb.case, 0, ptr, n)
        mb.step(dt)
        native.call("pgb_state_get", mb.case, 0, ptr, n)
        t0 = time.perf_counter()
        for _ in range(steps):
            native.call("pgb_state_set", mb.case, 0, ptr, n)
            mb.step(dt)
            native.call("pgb_state_get", mb.case, 0, ptr, n)
        wall = time.perf_counter() - t0
    finally:
        native.call("pgb_host_unregister", host.ctypes.data_as(ctypes.c_void_p))
    return wall, host.nbytes


def cpu_baseline(mesh_blocks, metrics, prims, constants, budget_s=15.0):
    """The oracle (reference CPU restatement, OpenMP on every core) on stages of the same grid."""
    from oracle.oracle import Oracle

    orc = Oracle(constants, 1, "navier-stokes", mesh_blocks, metrics, "rk4")
    orc.set_prims(prims)
    orc.threads = os.cpu_count() or 1
    dQ = [np.zeros_like(r) for r in orc.regs[0]]
    ncells = sum(b.ncells for b in mesh_blocks)
    stages = 0
    t0 = time.perf_counter()
    while True:
        orc.rhs(orc.regs[0], dQ)
        stages += 1
        if time.perf_counter() - t0 > budget_s or stages >= 8:
            break
    wall = time.perf_counter() - t0
    return ncells * stages / wall, stages, wall


REACT_CELLS = 96
REACT_STAGES = 3
# TVD-RK3 register traffic per cell and stage (reads + writes): stage 0 reads
# Q and writes Q1 (2), stages 1 and 2 read Q1 and Q and write one (3); 8/3
# registers of 13 doubles, 277 bytes
REACT_BYTES = 8 * 13 * 8 / 3


def reacting_leg(steps, cpu=True):
    """Cell-stage/s of the reacting configuration: the batched path (the fused
    passes), with the per-block and packed paths beside it."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases, native

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="batched")
    mesh = cases.reacting_mesh(REACT_CELLS, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], REACT_CELLS, seed=SEED)
    ncells = mb.ncells
    dt = 2e-8
    legs = {}
    for path, name in ((native.PATH_PER_BLOCK, "per_block"), (native.PATH_PACKED, "packed"),
                       (native.PATH_BATCHED, "batched")):
        mb.set_prims(prims)
        mb.path = path
        mb.step(dt, 3)
        mb.backend.sync()
        ms = time_graph(mb, dt, steps)
        legs[name] = {"value": ncells * REACT_STAGES * steps / (ms / 1e3), "ms_per_step": ms / steps,
                      "launches_per_step": mb.launches_per_step()}
    # the batched path's launches by kind, timed by events between launches
    kinds = {0: "halo fill", 1: "divergence and combines", 2: "face, gradient and source passes",
             8: "cell pass (fromQ and transport)"}
    rows = fused_kernel_times(mb, dt, 2)
    share = {}
    for k, label in kinds.items():
        t = [m for m, kk in rows if kk == k]
        if t:
            share[label] = {"launches_per_step": len(t) // 2, "ms_per_step": float(np.sum(t)) / 2}
    b = legs["batched"]
    gen_on, gen_why = mb.generated_chemistry()
    # the same batched step with the table-driven source kernel in place of
    # the one generated for the mechanism
    cfg_t = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="batched")
    cfg_t["backend-b200"]["chemistry-kernel"] = "tables"
    mbt = pg.get_solver(cfg_t, mesh, pg.get_backend("cuda", cfg_t))
    mbt.set_prims(prims)
    mbt.step(dt, 3)
    mbt.backend.sync()
    ms_t = time_graph(mbt, dt, steps)
    del mbt
    peak, peak_kind = peaks()
    achieved = b["value"] * REACT_BYTES / 1e9
    out = {"value": b["value"], "unit": "cell-stage/s", "steps": steps, "ms_per_step": b["ms_per_step"],
           "launches_per_step": b["launches_per_step"], "dt": dt,
           "workload": "h2-air-96^3-9sp-28rxn-tpg-kinetic-coupled-chem-muscl-koren-hllc-ns-tvd-rk3",
           "path": "batched: the fused passes (cell pass, source, gradients, a face pass per axis with the "
                   "advective and diffusive flux in one thread, divergence and combines in one pass)",
           "per_block": legs["per_block"], "packed": legs["packed"],
           "speedup_vs_per_block": legs["per_block"]["ms_per_step"] / b["ms_per_step"],
           "batched_launch_kinds": share,
           "source_kernel": {"generated": gen_on, "why_not": gen_why or None,
                             "tables_ms_per_step": ms_t / steps},
           "roofline": {"bound": "fp64 (see profiles); hbm fraction of the algorithmic bytes", "achieved": achieved,
                        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                        "algorithmic_bytes_per_cell_stage": REACT_BYTES}}
    if cpu:
        from oracle.oracle import Oracle

        orc = Oracle(consts, mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3", primary="hllc",
                     recon="muscl", limiter="koren", eos="tpg", trans="kinetic-theory", chemistry="finite-rate")
        orc.set_prims(prims)
        orc.threads = os.cpu_count() or 1
        dQ = [np.zeros_like(r) for r in orc.regs[0]]
        t0 = time.perf_counter()
        orc.rhs(orc.regs[0], dQ)
        wall = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": ncells / wall, "unit": "cell-stage/s", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"one stage (RHS) of the 96^3 reacting field, {wall:.1f} s"}
    del mb
    return out


def reacting_profile(kernel):
    """The reacting case's batched step twice (a warm-up and one more), its
    launches plain (no graph), so a profiler sees each pass on its own: the
    stage's seven launches after a halo fill (cell pass, source, gradients,
    gradient halo, three face passes, divergence and combines)."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="batched")
    cfg["backend-b200"]["chemistry-kernel"] = kernel
    mesh = cases.reacting_mesh(REACT_CELLS, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    mb.set_prims(cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], REACT_CELLS, seed=SEED))
    mb.graph = False
    mb.step(2e-8, 1)
    mb.step(2e-8, 1)
    mb.backend.sync()
    print(json.dumps({"reacting_profile": kernel, "generated": mb.generated_chemistry()[0]}), flush=True)


def realgas_profile():
    """The mixing layer's batched step three times (two warm-ups and one
    more), its launches plain (no graph), so a profiler sees each pass on its
    own: the step start's two passes and halo pass, then per stage the
    interior's state, the halo pass and the faces, divergence and combines."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases, native

    cfg = cases.mixing_layer_config("pr", "euler-df", "tvd-rk3", launch="batched")
    mesh = cases.mixing_layer_mesh(256, 128, 4, 8, seed=SEED)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    mb.set_prims(cases.mixing_layer_prims(mb.metrics, 128, seed=SEED))
    mb.path = native.PATH_BATCHED
    mb.graph = False
    for _ in range(3):
        mb.step(2e-9, 1)
    mb.backend.sync()
    print(json.dumps({"realgas_profile": "batched", "launches_per_step": mb.launches_per_step()}), flush=True)


# the sub-stepped leg's timed steps, fixed: the hot spots burn through in a
# few microseconds, so the stiff cells a step lists depend on how far the
# field has run (three warm-up steps, then these)
SUBSTEP_STEPS = 5


def substep_leg(steps, dt=1e-7, dT=1500.0):
    """The reacting field with burnt-hot spots (up to 2500 K) and the
    sub-stepped chemistry (the reference's defaults: a 200-substep cap, one
    bulk substep, 8 bins, the 1e-7 exit) at five times the coupled leg's step:
    cell-stage/s, the bulk and stiff passes' shares of a step and the share of
    cells the stiff pass takes."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True, launch="per-block")
    cfg["chem-integration"]["kind"] = "sub-stepped"
    cfg.validate()
    mesh = cases.reacting_mesh(REACT_CELLS, (1, 1, 1))
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    consts = mb.mixture.constants()
    prims = cases.reacting_prims(mb.metrics, mb.mixture.spnames, consts["MW"], REACT_CELLS, seed=SEED, dT=dT)
    mb.set_prims(prims)
    mb.step(dt, 3)
    mb.backend.sync()
    ms = time_graph(mb, dt, steps)
    rows = fused_kernel_times(mb, dt, 1)
    total = sum(m for m, _ in rows)
    bulk = sum(m for m, k in rows if k == 6)
    stiff = sum(m for m, k in rows if k == 7)
    per_stage_stiff = [m for m, k in rows if k == 7]
    # the listing of a step's first stage (the later stages start from states
    # the first stage's mean rates carried near the hot cells' equilibrium)
    mb.rhs()
    head = mb.stiff_head()
    subs = mb.substeps()
    ncells = mb.ncells
    value = ncells * REACT_STAGES * steps / (ms / 1e3)
    out = {"value": value, "unit": "cell-stage/s", "steps": steps, "ms_per_step": ms / steps, "dt": dt,
           "launches_per_step": mb.launches_per_step(),
           "bulk_share_of_step": bulk / total if total else None,
           "stiff_share_of_step": stiff / total if total else None,
           "stiff_ms_per_stage": per_stage_stiff,
           "first_stage_listed_fraction": head[0] / ncells, "first_stage_bin_counts": head[1:],
           "first_stage_mean_substeps": float(subs.mean()), "first_stage_max_substeps": int(subs.max()),
           "first_stage_listed_mean_substeps": float(subs[subs > 1].mean()) if (subs > 1).any() else None,
           "workload": f"h2-air-96^3-9sp-28rxn hot spots of {dT:g} K over 1000 K, sub-stepped chemistry (cap 200, "
                       "bulk 1, 8 bins, exit 1e-7), muscl-koren-hllc-ns-tvd-rk3",
           "path": "per-block kernels; chemistry: bulk pass over every cell, one persistent stiff pass over the list"}
    del mb
    return out


def packed_leg(mb, dt, steps, ncells, stages):
    """The same steps on the packed path: the per-block kernels, each pass one
    launch over every block."""
    from peregrine_b200 import native

    path = mb.path
    mb.path = native.PATH_PACKED
    mb.step(dt, 2)
    mb.backend.sync()
    ms = time_graph(mb, dt, steps)
    out = {"value": ncells * stages * steps / (ms / 1e3), "ms_per_step": ms / steps,
           "launches_per_step": mb.launches_per_step()}
    mb.path = path
    return out


def realgas_leg(steps, cpu=True):
    """Cell-stage/s of the transcritical mixing layer: the batched path (the
    double flux's fused stage), with the per-block and packed paths beside it."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases, native

    cfg = cases.mixing_layer_config("pr", "euler-df", "tvd-rk3", launch="batched")
    mesh = cases.mixing_layer_mesh(256, 128, 4, 8, seed=SEED)
    mb = pg.get_solver(cfg, mesh, pg.get_backend("cuda", cfg))
    prims = cases.mixing_layer_prims(mb.metrics, 128, seed=SEED)
    dt = 2e-9
    ncells = mb.ncells
    legs = {}
    for path, name in ((native.PATH_PER_BLOCK, "per_block"), (native.PATH_PACKED, "packed"),
                       (native.PATH_BATCHED, "batched")):
        mb.set_prims(prims)
        mb.path = path
        mb.step(dt, 3)
        mb.backend.sync()
        ms = time_graph(mb, dt, steps)
        legs[name] = {"value": ncells * 3 * steps / (ms / 1e3), "ms_per_step": ms / steps,
                      "launches_per_step": mb.launches_per_step()}
    b = legs["batched"]
    # RK3 registers (8/3 of 6 doubles) and the frozen plane's 4 doubles read
    nbytes = 8 * 6 * 8 / 3 + 8 * 4
    peak, peak_kind = peaks()
    achieved = b["value"] * nbytes / 1e9
    out = {"value": b["value"], "unit": "cell-stage/s", "steps": steps, "ms_per_step": b["ms_per_step"],
           "launches_per_step": b["launches_per_step"], "dt": dt,
           "workload": "mixing-layer-256x128x4-8-uneven-blocks-o2-h2-60bar-peng-robinson-double-flux-kepaec-euler-rk3",
           "path": "batched: the planes frozen each step (a launch a pass over every block), then per stage the "
                   "interior's state off the planes, Q's halo with the state's copy in one pass, and one kernel "
                   "of each cell's six faces, divergence and combines",
           "blocks": [b_.cells[0] for b_ in mb.mesh_blocks], "per_block": legs["per_block"], "packed": legs["packed"],
           "speedup_vs_per_block": legs["per_block"]["ms_per_step"] / b["ms_per_step"],
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": peak_kind, "algorithmic_bytes_per_cell_stage": nbytes}}
    if cpu:
        from oracle.oracle import Oracle

        orc = Oracle(mb.mixture.constants(), mb.ns, "euler", mb.mesh_blocks, mb.metrics, "tvd-rk3",
                     eos="real-gas-df", trans="constant")
        orc.set_prims(prims)
        orc.threads = os.cpu_count() or 1
        dQ = [np.zeros_like(r) for r in orc.regs[0]]
        orc.rhs(orc.regs[0], dQ)  # the planes' settle
        t0 = time.perf_counter()
        orc.rhs(orc.regs[0], dQ)
        wall = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": ncells / wall, "unit": "cell-stage/s", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"one stage (RHS) of the mixing layer, {wall:.2f} s"}
    del mb
    return out


def boundary_leg(steps, cpu=True):
    """Cell-stage/s of the bounded channel on the per-block path, under the
    device-side cfl controller, and the boundary passes' share of a step."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases

    cfg = cases.channel_config()
    mb = pg.get_solver(cfg, cases.channel_mesh(), pg.get_backend("cuda", cfg))
    sim = cfg["simulation"]
    mb.step_cfl(sim["cfl"], sim["dt-max"], 3)
    mb.backend.sync()
    mb.step_cfl(sim["cfl"], sim["dt-max"], steps)
    ms = mb.last_step_ms()
    dt = mb.last_dt()
    # the same steps at the controller's last size: what the controller's
    # reduction and step-size kernel cost per step
    mb.step(dt, steps)
    ms_fixed = mb.last_step_ms()
    rows = fused_kernel_times(mb, dt, 2)
    total = sum(m for m, _ in rows)
    boundary = sum(m for m, k in rows if k == 4)
    ncells = mb.ncells
    value = ncells * 3 * steps / (ms / 1e3)
    out = {"value": value, "unit": "cell-stage/s", "steps": steps, "ms_per_step": ms / steps,
           "ms_per_step_fixed_dt": ms_fixed / steps, "controller_overhead": ms / ms_fixed - 1.0,
           "last_dt": dt, "launches_per_step": mb.launches_per_step(),
           "boundary_share_of_step": boundary / total if total else None,
           "boundary_ms_per_step": boundary / 2,
           "workload": "channel-192x96x96-8-blocks-2sp-ns-muscl-koren-hllc-rk3-cfl-0.8: velocity inflow "
                       "(expressions of y, z, t), pressure exit, isothermal no-slip floor, moving lid, periodic across",
           "path": "per-block kernels, boundary passes one launch each over every boundary face"}
    out["packed"] = packed_leg(mb, dt, steps, ncells, 3)
    if cpu:
        from oracle.oracle import Oracle

        orc = Oracle(mb.mixture.constants(), mb.ns, "navier-stokes", mb.mesh_blocks, mb.metrics, "tvd-rk3",
                     primary="hllc", recon="muscl", limiter="koren", bcvals=cfg["bcvals"], species=mb.mixture.spnames)
        ic = cfg["ics"]
        prims = []
        for b in mb.mesh_blocks:
            q = np.empty(tuple(n + 4 for n in b.cells) + (mb.ne,))
            q[...] = [ic["p"], ic["u"], ic["v"], ic["w"], ic["T"], ic["Y"]["A"]]
            prims.append(q)
        orc.set_prims(prims)
        orc.threads = os.cpu_count() or 1
        dQ = [np.zeros_like(r) for r in orc.regs[0]]
        t0 = time.perf_counter()
        orc.rhs(orc.regs[0], dQ)
        wall = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": ncells / wall, "unit": "cell-stage/s", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"one stage (RHS) of the channel, {wall:.2f} s"}
    del mb
    return out


def serving_leg(n=300, rate=60.0, steps=100, sweep=(30.0, 120.0, 480.0, 1920.0), nsweep=200):
    """The serving stream: Poisson arrivals of H2/air closed reactors and
    periodic 1-D domains, admitted into one pool while others run; then the
    same mix at other arrival rates (nsweep requests each), for the latency
    against the load."""
    import ctypes

    import peregrine_b200 as pg
    from peregrine_b200 import cases, native, serving

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True)
    proto = pg.get_solver(cfg, cases.reacting_mesh(4), pg.get_backend("cuda", cfg))
    consts = proto.mixture.constants()
    reqs = serving.requests(n, rate, proto.mixture.spnames, consts["MW"], seed=SEED, steps=steps)
    # the client side: each case arrives with its mesh's metrics made
    for r in reqs:
        serving.box_metrics(r.cells, r.lengths)
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    native.call("pgb_mem_info", ctypes.byref(free), ctypes.byref(total))
    ns, ne = proto.ns, proto.ne
    per_cell = 8 * (proto.nregs * ne + 31 + 8 + (2 + ns) + ns + 3 * (ne - 1) + 3 * ne)
    cap = int(min(free.value * 0.5 / per_cell, 20_000_000))
    pool = serving.Pool(proto, cap, 4096)
    dt = 2e-8
    # warm the kernels on one case
    warm = serving.requests(1, 0.0, proto.mixture.spnames, consts["MW"], seed=SEED + 1, steps=3)
    serving.Server(pool, dt).run(warm, 3)
    srv = serving.Server(pool, dt)
    t0 = time.perf_counter()
    srv.run(reqs, 3)
    wall = time.perf_counter() - t0
    st = serving.latency_stats(reqs)
    zero = [r for r in reqs if r.kind == "0d"]
    one = [r for r in reqs if r.kind == "1d"]
    loads = []
    for k, lam in enumerate(sweep):
        more = serving.requests(nsweep, lam, proto.mixture.spnames, consts["MW"], seed=SEED + 2 + k, steps=steps)
        for r in more:
            serving.box_metrics(r.cells, r.lengths)
        sv = serving.Server(pool, dt)
        ta = time.perf_counter()
        sv.run(more, 3)
        w = time.perf_counter() - ta
        ls = serving.latency_stats(more)
        loads.append({"arrival_rate_per_s": lam, "requests": nsweep, "requests_per_s": nsweep / w,
                      "p50_ms": ls["p50_ms"], "p99_ms": ls["p99_ms"],
                      "mean_running": sv.running_sum / max(sv.steps, 1), "pool_steps": sv.steps,
                      "device_ms": sv.device_ms, "admit_s": sv.admit_s, "admit_max_ms": sv.admit_max_s * 1e3})
    pool.close()
    return {"requests": n, "arrival_rate_per_s": rate, "steps_per_request": steps, "dt": dt, "sweep": loads,
            "cell_stages_per_s": srv.cell_stages / wall, "requests_per_s": n / wall, "wall_s": wall,
            "device_ms": srv.device_ms, "pool_steps": srv.steps, "launches": srv.launches,
            "mean_running": srv.running_sum / max(srv.steps, 1), "admit_s": srv.admit_s,
            "admit_max_ms": srv.admit_max_s * 1e3,
            "latency_ms": st, "latency_0d_ms": serving.latency_stats(zero) if zero else None,
            "latency_1d_ms": serving.latency_stats(one) if one else None,
            "arena_cells": cap, "per_cell_bytes": per_cell,
            "workload": "h2-air-serving: closed reactors (phi U[0.5,2], T0 U[900,1400] K, p U[1,40] atm) and "
                        "periodic 1-D domains of 64-2048 cells, Poisson arrivals, one pool, continuous batching"}


def serving_profile(n=200):
    """A saturated pool: n seeded requests (closed reactors and 1-D domains)
    admitted at once, then a step (its graph captured) and two more."""
    import peregrine_b200 as pg
    from peregrine_b200 import cases, serving

    cfg = cases.reacting_config("navier-stokes", "tvd-rk3", "hllc", "muscl", "koren", True)
    proto = pg.get_solver(cfg, cases.reacting_mesh(4), pg.get_backend("cuda", cfg))
    consts = proto.mixture.constants()
    reqs = serving.requests(n, 0.0, proto.mixture.spnames, consts["MW"], seed=SEED + 7, steps=100)
    pool = serving.Pool(proto, 8_000_000, 4096)
    slots = [pool.admit(r) for r in reqs]
    assert None not in slots
    pool.step(2e-8, 1)
    ms, launches = pool.step(2e-8, 2)
    free, run, done = pool.info()
    cells = sum(1 if r.kind == "0d" else int(np.prod(r.cells)) for r in reqs)
    print(json.dumps({"serving_profile": {"requests": n, "running": run, "reactors": sum(r.kind == "0d" for r in reqs),
                                          "cells": cells, "ms_per_step": ms / 2, "launches_per_step": launches / 2}}),
          flush=True)
    pool.close()


def reference_arm(args):
    """The reference CPU restatement's throughput on the same workload; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from peregrine_b200 import cases
    from peregrine_b200.grid import metrics as make_metrics
    from peregrine_b200.mixture import Mixture
    from oracle.oracle import Oracle

    cfg = cases.tgv_config("navier-stokes", "rk4")
    mesh = cases.tgv_mesh(CELLS, BLOCKS, seed=SEED, low=CUT_LOW, high=CUT_HIGH)
    blocks = mesh.make_blocks(2)
    mets = [make_metrics(b.nodes, b.ng) for b in blocks]
    prims = cases.tgv_prims(blocks, mets, seed=SEED)
    mix = Mixture(cfg["mixture"])
    orc = Oracle(mix.constants(), 1, "navier-stokes", blocks, mets, "rk4")
    orc.set_prims(prims)
    orc.threads = os.cpu_count() or 1
    dQ = [np.zeros_like(r) for r in orc.regs[0]]
    ncells = sum(b.ncells for b in blocks)
    for _ in range(args.warmup):
        orc.rhs(orc.regs[0], dQ)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.rhs(orc.regs[0], dQ)
    wall = time.perf_counter() - t0
    value = ncells * args.steps / wall
    cores = os.cpu_count()
    sample = f"one RK stage (RHS) of every cell of the workload per step, {args.steps} steps"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cell-stage/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD if CELLS == 128 else f"{WORKLOAD} at {CELLS}^3", "cells": ncells, "blocks": len(blocks), "parallelism": "openmp"},
            "cpu_baseline": {"value": value, "unit": "cell-stage/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def shard_leg(args, dist, rank, world, local):
    """The workload's blocks over the ranks (peregrine_b200/shard.py), Q's halo
    traded between stages on the device (NCCL), timed by CUDA events on every
    rank, the max taken; strong scaling of the one grid."""
    import torch

    import peregrine_b200 as pg
    from peregrine_b200 import cases, shard
    from peregrine_b200.replicas import max_over_ranks

    cfg = cases.tgv_config("navier-stokes", "rk4", "batched")
    mesh = cases.tgv_mesh(CELLS, BLOCKS, seed=SEED, low=CUT_LOW, high=CUT_HIGH)
    blocks = mesh.make_blocks(2)
    owner = shard.partition(blocks, world)
    sh = shard.ShardedSolver(cfg, mesh, pg.get_backend("cuda", cfg, device=local), owner, rank, exchange="device")
    every = cases.tgv_prims(*_every_field(mesh))
    sh.solver.set_prims([every[g] for g in sh.plan.local])
    dt = stable_dt()
    sh.step(dt, args.warmup)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sh.step(dt, args.steps)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, device=f"cuda:{local}")
    ncells = sum(b.ncells for b in blocks)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": ncells * STAGES * args.steps / (ms / 1e3), "unit": "cell-stage/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": ncells, "blocks": len(blocks),
                       "parallelism": f"blocks over {world} ranks, Q halo traded each stage (NCCL)",
                       "blocks_per_rank": np.bincount(owner, minlength=world).tolist()}}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def _every_field(mesh):
    from peregrine_b200.grid import metrics as make_metrics

    blocks = mesh.make_blocks(2)
    return blocks, [make_metrics(b.nodes, 2) for b in blocks]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-extra", action="store_true", help="skip the per-block and end-to-end legs")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape and tiles")
    ap.add_argument("--halo-fill", action="store_true",
                    help="fill each stage's halo before it instead of reading across the blocks' faces")
    ap.add_argument("--shape", default=None, help="force the fused kernel's THREADSxMINBLOCKSxWIDTH (no tuning)")
    ap.add_argument("--ksplit", type=int, default=3, help="k runs per block with --shape")
    ap.add_argument("--cells", type=int, default=CELLS, help="cells per axis of the cube (a smaller case for profiling)")
    ap.add_argument("--no-reacting", action="store_true", help="skip the reacting leg")
    ap.add_argument("--reacting-only", action="store_true", help="the reacting leg alone (profiling)")
    ap.add_argument("--realgas-profile", action="store_true",
                    help="three plain batched steps of the mixing layer (for a profiler)")
    ap.add_argument("--reacting-profile", default=None, choices=("generated", "tables"),
                    help="one warm-up and one RK3 step of the 96^3 reacting case on the batched path, no graph, "
                         "with the named source kernel: the command an ncu capture of its passes runs")
    ap.add_argument("--serving-only", action="store_true", help="the serving leg alone")
    ap.add_argument("--serving-profile", type=int, default=0, metavar="N",
                    help="N seeded requests admitted into one pool at once, then three pool steps: the command an "
                         "ncu launch list of a pool step runs (200: saturated)")
    ap.add_argument("--realgas-only", action="store_true", help="the real-gas leg alone")
    ap.add_argument("--no-realgas", action="store_true", help="skip the real-gas leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--boundary-only", action="store_true", help="the bounded channel leg alone")
    ap.add_argument("--substep-only", action="store_true", help="the sub-stepped chemistry leg alone")
    ap.add_argument("--no-substep", action="store_true", help="skip the sub-stepped chemistry leg")
    ap.add_argument("--no-boundary", action="store_true", help="skip the bounded channel leg")
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1 ranks: the workload's blocks over the ranks, halos traded each stage (strong "
                         "scaling) instead of a replica per rank")
    args = ap.parse_args()
    set_cells(args.cells)
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.realgas_only:
        print(json.dumps({"realgas": realgas_leg(max(1, min(args.steps, 20)), cpu=not args.no_cpu)}), flush=True)
        return
    if args.substep_only:
        print(json.dumps({"substepped": substep_leg(SUBSTEP_STEPS)}), flush=True)
        return
    if args.boundary_only:
        print(json.dumps({"boundary": boundary_leg(max(1, min(args.steps, 20)), cpu=not args.no_cpu)}), flush=True)
        return
    if args.serving_only:
        print(json.dumps({"serving": serving_leg()}), flush=True)
        return
    if args.serving_profile:
        serving_profile(args.serving_profile)
        return
    if args.reacting_only:
        print(json.dumps({"reacting": reacting_leg(max(1, min(args.steps, 20)), cpu=not args.no_cpu)}), flush=True)
        return
    if args.reacting_profile:
        reacting_profile(args.reacting_profile)
        return
    if args.realgas_profile:
        realgas_profile()
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.shard and world > 1:
        shard_leg(args, dist, rank, world, local)
        return

    mb, mesh, prims = build_case("batched", device=local)
    if args.halo_fill:
        from peregrine_b200 import native

        native.call("pgb_case_set_halo_pull", mb.case, 0)
    dt = stable_dt()
    ncells = mb.ncells
    mb.step(dt, 1)
    # the launch shape and tiles, picked by timing them on this case
    from peregrine_b200 import autotune

    if args.shape:
        shape = tuple(int(x) for x in args.shape.split("x"))
        tuned = autotune.tune(mb, dt, only=(shape,), ksplits=(args.ksplit,))
    else:
        tuned = None if args.no_tune else autotune.tune(mb, dt)
    # warm-up (the first call captures the graph)
    mb.step(dt, args.warmup)
    mb.backend.sync()

    def barrier():
        if dist is not None:
            dist.barrier()

    barrier()
    with Clocks(local) as clk:
        ms = time_graph(mb, dt, args.steps)
    barrier()
    from peregrine_b200.replicas import max_over_ranks, weak_throughput

    ms = max_over_ranks(ms, dist, device=f"cuda:{local}")
    value = weak_throughput(ncells, STAGES, args.steps, ms, world)
    launches = mb.launches_per_step()

    # the fused kernel's own launches, timed by events between launches
    rows = fused_kernel_times(mb, dt, min(args.steps, 20))
    fused = [m for m, k in rows if k == 1]
    halo = [m for m, k in rows if k == 0]
    per_stage = [float(np.mean(fused[s::STAGES])) for s in range(STAGES)]
    bytes_per_launch = [ncells * 8 * NE * r for r in STAGE_REGS]
    achieved = float(np.mean([b / (t / 1e3) / 1e9 for b, t in zip(bytes_per_launch, per_stage)]))
    peak, peak_kind = peaks()
    # the ncu-measured DRAM bytes per cell-stage of the fused kernel (profiles/),
    # as bytes per launch of this workload
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "fused_traffic.txt")
    if os.path.exists(tpath) and CELLS == 128:
        with open(tpath) as f:
            for line in f:
                if line.startswith("bytes_per_cell_stage"):
                    traffic = float(line.split()[1]) * ncells

    from peregrine_b200 import native

    # the cfl controller on the headline: the same steps with the device's
    # reduction and step-size kernel ahead of each (dt-max the fixed dt, so
    # the steps are the same size)
    cfl_cost = None
    if not args.no_extra:
        cfl_steps = max(3, min(args.steps // 4, 50))
        mb.step_cfl(1e6, dt, 2)
        mb.step_cfl(1e6, dt, cfl_steps)
        ms_c = mb.last_step_ms()
        mb.step(dt, cfl_steps)
        ms_f = mb.last_step_ms()
        cfl_cost = {"ms_per_step": ms_c / cfl_steps, "ms_per_step_fixed": ms_f / cfl_steps,
                    "overhead": ms_c / ms_f - 1.0, "cflmax": mb.cflmax()}

    per_block, e2e = None, None
    if not args.no_extra:
        # the plain per-block path
        mb.path = native.PATH_PER_BLOCK
        mb.step(dt, 2)
        mb.backend.sync()
        pb_steps = max(2, min(args.steps // 4, 20))
        ms_pb = time_graph(mb, dt, pb_steps)
        pb_launches = mb.launches_per_step()
        mb.path = native.PATH_BATCHED
        value_pb = ncells * STAGES * pb_steps / (ms_pb / 1e3)
        # the same kernels packed, each pass one launch over every block: the
        # un-fused device baseline without the per-block launch count
        mb.path = native.PATH_PACKED
        mb.step(dt, 2)
        mb.backend.sync()
        ms_pk = time_graph(mb, dt, pb_steps)
        pk_launches = mb.launches_per_step()
        mb.path = native.PATH_BATCHED
        value_pk = ncells * STAGES * pb_steps / (ms_pk / 1e3)
        per_block = {"value": value_pb, "ms_per_step": ms_pb / pb_steps, "launches_per_step": pb_launches,
                     "speedup_batched": value / world / value_pb,
                     "packed": {"value": value_pk, "ms_per_step": ms_pk / pb_steps, "launches_per_step": pk_launches,
                                "speedup_batched": value / world / value_pk}}
        # end to end: state in from pinned host, a step, state out, every step
        e2e_steps = max(3, min(args.steps // 4, 20))
        wall, nbytes = e2e_leg(mb, dt, e2e_steps)
        e2e = {"value": ncells * STAGES * e2e_steps / wall * world, "unit": "cell-stage/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}

    cpu = None
    if rank == 0 and not args.no_cpu:
        v, stages, cwall = cpu_baseline(mb.mesh_blocks, mb.metrics, prims, mb.mixture.constants())
        cpu = {"value": v, "unit": "cell-stage/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{stages} RK stages (RHS) of the full workload, {cwall:.1f} s, OpenMP"}

    reacting = None
    if rank == 0 and not args.no_reacting and not args.no_extra:
        reacting = reacting_leg(max(2, min(args.steps // 30, 20)), cpu=not args.no_cpu)
    served = None
    if rank == 0 and not args.no_serving and not args.no_extra:
        served = serving_leg()
    realgas = None
    if rank == 0 and not args.no_realgas and not args.no_extra:
        realgas = realgas_leg(max(2, min(args.steps // 30, 20)), cpu=not args.no_cpu)
    substepped = None
    if rank == 0 and not args.no_substep and not args.no_extra:
        substepped = substep_leg(SUBSTEP_STEPS)
    boundary = None
    if rank == 0 and not args.no_boundary and not args.no_extra:
        boundary = boundary_leg(max(2, min(args.steps // 30, 20)), cpu=not args.no_cpu)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-stage/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": ncells, "blocks": len(mb.blocks), "stages_per_step": STAGES,
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "l2": "inputs larger than L2 (four registers of 2.4M cells x 5 doubles, 0.38 GB)",
                       "path": "batched fused persistent kernel, CUDA graph per RK4 step",
                       "tuned": tuned},
            "per_block": per_block,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_fused2 (fused RK stage, uniform metrics)" if all(mb.uniform(n) for n in range(len(mb.blocks)))
                         else "k_fused1 (fused RK stage, metric arrays)", "kernel_ms_per_stage": per_stage,
                         "halo_ms_per_stage": float(np.mean(halo)) if halo else None,
                         "algorithmic_bytes_per_cell_stage": 170,
                         # the whole step's: the same algorithmic bytes over the
                         # step's own time (any halo fill included)
                         "step_achieved": ncells * STAGES * 170 / (ms / args.steps / 1e3) / 1e9,
                         "step_frac": ncells * STAGES * 170 / (ms / args.steps / 1e3) / 1e9 / peak},
            "cpu_baseline": cpu,
            "reacting": reacting,
            "serving": served,
            "realgas": realgas,
            "boundary": boundary,
            "substepped": substepped,
            "cfl": cfl_cost,
            "e2e": e2e,
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
