#!/usr/bin/env python3
"""Benchmark of the narrow-band level-set advection step on B200.

Prints ONE JSON line on rank 0.  Metric: active voxels per second per step.

Default workload ``large8192``: one grid, the union of 8,000 seeded random
spheres with radii U(6, 40) voxels and centres uniform in an 8192^3 index
extent, half-width 3 (2.5 M leaves, 384 M active voxels), divergence-free
curl-noise velocity (3 octaves, 1 voxel/step), SSP-RK3 backtrace, two Godunov
reinitialisation iterations and band re-tracking per step.  ``value`` is the
FP16-leaf step (f32 arithmetic); the plain FP32 step is under ``fp32``.
Beside it: ``e2e`` (the host-resident step through vlr_ls_step_host, pinned
buffers, copies inside the wall-clock timed region), ``ref_step`` (the
crate's own advect_level_set + rebuild_narrow_band on the GPU over the same
grid), ``data_path`` (constant velocity, Euler, no reinitialisation
iteration), ``batched256`` and ``deformation512`` sections, the full-period
accuracy runs, the level-set adjoint and volume_to_mesh.  ``cpu_baseline`` is
the FP64 method oracle on a box of the grid on all host threads.

Other workloads: ``deformation512`` (unit cube at 512^3, sphere r = 0.15,
vortex T = 3, RK2 at CFL 0.5), ``batched256`` (256 uneven grids in one pool),
``adjoint256``, ``reference-sphere128`` (sphere r = 32 in 128^3,
v = (1, 0.5, 0.25), dt = 1, hw = 3; the crate's step, bit-exact), ``mesh96``
and ``tools160``.

Timing: W warm-up steps, then exactly K timed steps, each bracketed by CUDA
events on the library's stream; a 256 MiB write flushes the L2 between
steps, outside the events.  ``--impl reference`` times the crate's own step
(a C++ restatement of advect_level_set + rebuild_narrow_band with its data
structure, one thread as the crate runs it) on the host CPU, for large8192 on
a box of the same grid with the whole-grid rate extrapolated (see
RefLargeSample).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0
METRIC = "active voxels/s per advection step"

DEFORM = dict(radius=0.15, center=(0.35, 0.35, 0.35), voxel_size=1.0 / 512.0, half_width=3.0, period=3.0)
REF_SPHERE = dict(radius=32.0, center=(64.0, 64.0, 64.0), voxel_size=1.0, half_width=3.0)
REF_VEL = (1.0, 0.5, 0.25)
BATCH = dict(grids=256, seed=3)
LARGE = dict(spheres=8000, extent=8192.0, radius=(6.0, 40.0), seed=7)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the GPU is timed.

    The sampler starts before the warm-up and waits for its first sample; the
    timed regions are marked with ``mark()``; ``summary()`` keeps the samples
    whose timestamps fall inside a marked region widened by the sampling
    period (a timed region of a few milliseconds is shorter than one period).
    """

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 50

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.windows = []
        self.path = Path(tempfile.gettempdir()) / f"vlr_clocks_{os.getpid()}_{device}.csv"

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.PERIOD_MS)], stdout=self.out, stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 10.0 and self.path.stat().st_size == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(2.0 * self.PERIOD_MS / 1000.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.out.close()
        except Exception:
            pass

    def mark(self):
        """Context manager around one timed region."""
        sampler = self

        class _W:
            def __enter__(self):
                self.t0 = time.time()

            def __exit__(self, *a):
                sampler.windows.append((self.t0, time.time()))

        return _W()

    def summary(self):
        import datetime
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 10:
                    try:
                        ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    except ValueError:
                        continue
                    rows.append((ts, parts[1:]))
        except Exception:
            pass
        pad = 1.5 * self.PERIOD_MS / 1000.0
        sel = [r for ts, r in rows if any(a - pad <= ts <= b + pad for a, b in self.windows)]
        timed_s = sum(b - a for a, b in self.windows)
        if not sel:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "samples_total": len(rows), "timed_s": timed_s}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in sel) if v is not None]
        mx = [v for v in (num(r[2]) for r in sel) if v is not None]
        pw = [v for v in (num(r[3]) for r in sel) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in sel for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(sel),
                "period_ms": self.PERIOD_MS, "timed_s": timed_s}


# ---------------------------------------------------------------- CPU legs

def cpu_method_oracle(steps: int = 2, threads: int | None = None):
    """FP64 oracle of the same narrow-band method on all host threads, bounded sample."""
    import numpy as np
    from oracle import pyoracle
    threads = threads or os.cpu_count() or 1
    vs = DEFORM["voxel_size"]
    vel = {"kind": "vortex", "vs": vs, "period": DEFORM["period"]}
    dt = 0.5 * vs / 2.0
    g = pyoracle.MOGrid.sphere(DEFORM["radius"], DEFORM["center"], vs, DEFORM["half_width"])
    act = []
    t0 = time.perf_counter()
    for s in range(steps):
        g.step(vel, 2, 2, s * dt, dt, threads)
        o, m, v = g.arrays()
        act.append(int(np.unpackbits(m.view(np.uint8)).sum()))
    t = time.perf_counter() - t0
    return (sum(act) / t, threads,
            f"FP64 method oracle (same RK2 + 2x Godunov + re-track step), {steps} steps of the deformation "
            f"config on {threads} host threads")


def cpu_reference_algorithm(sphere: dict, velocity_world, dt: float, sample_voxels: int = 1500):
    """The crate's own step (advect_level_set + rebuild_narrow_band) restated in
    C++ with its data structure, one thread as the crate runs it.  The O(N x M)
    distance loop of rebuild_narrow_band runs on `sample_voxels` voxels and is
    extrapolated linearly.  Returns (voxels/s, description)."""
    import ctypes as C
    from oracle import pyoracle
    lib = pyoracle.load()
    g = pyoracle.OGrid.sphere(sphere["radius"], sphere["center"], sphere["voxel_size"], sphere["half_width"])
    n_active = g.active_voxel_count()
    vel = pyoracle.uniform_velocity(sphere["voxel_size"], velocity_world)
    h = C.c_void_p(g.h)
    ta, tr, nr = C.c_double(), C.c_double(), C.c_size_t()
    lib.vo_time_ref_step(C.byref(h), vel[0].h, vel[1].h, vel[2].h, dt, C.c_float(sphere["half_width"]),
                         sample_voxels, C.byref(ta), C.byref(tr), C.byref(nr))
    g.h = h.value
    t_step = ta.value + tr.value * (n_active / max(nr.value, 1))
    return n_active / t_step, (f"reference algorithm (advect_level_set over all {n_active} active voxels with a "
                               f"three-grid VelocityField + rebuild_narrow_band's distance loop on {sample_voxels} "
                               f"voxels, extrapolated), 1 thread")


LARGE_ORACLE_BOX = 1536   # FP64 method oracle sample: spheres near this box at the grid's centre
LARGE_REF_BOX = 1024      # the crate's step sample: spheres near this box at the grid's centre


def _large_box_spheres(args, box):
    import numpy as np
    from sharc.volrus_b200.method import large_sphere_grid, spheres_near_box
    sph, vel = large_sphere_grid(args.large_spheres, LARGE["seed"])
    lo = np.full(3, LARGE["extent"] / 2 - box / 2)
    return sph, spheres_near_box(sph, lo, lo + box, 3.0), vel


def cpu_method_oracle_large(args, threads: int | None = None):
    """FP64 method oracle (the same RK3 + 2x Godunov + re-track step) on the
    spheres of the large grid whose band reaches a 1536^3 box at its centre,
    one step on all host threads; the rate per active voxel is that of the
    whole grid, whose spheres are alike."""
    import numpy as np
    from oracle import pyoracle
    threads = threads or os.cpu_count() or 1
    _, sub, vel = _large_box_spheres(args, LARGE_ORACLE_BOX)
    g = pyoracle.MOGrid.spheres(sub, 3.0)
    n_act = int(np.unpackbits(g.arrays()[1].view(np.uint8)).sum())
    t0 = time.perf_counter()
    g.step(vel, 3, 2, 0.0, 1.0, threads)
    t = time.perf_counter() - t0
    return (n_act / t, threads,
            f"FP64 method oracle, one SSP-RK3 + 2x Godunov + re-track step of the {len(sub)} spheres of the large "
            f"grid near a {LARGE_ORACLE_BOX}^3 box at its centre ({n_act} active voxels) on {threads} host threads; "
            f"rate per active voxel")


class RefLargeSample:
    """The crate's step (advect_level_set + rebuild_narrow_band, restated in C++
    with its data structure, one thread as the crate runs it) on the spheres of
    the large grid near a 1024^3 box at its centre, with the curl-noise
    velocity sampled at every voxel of the band into three grids (the crate's
    VelocityField).

    The crate's rebuild_narrow_band (src/tools/level_set_track.rs:80-114)
    loops, for every active voxel, over every zero crossing of the grid, so a
    step of the whole grid costs advect + crossing search per voxel plus
    (active voxels x crossings of the whole grid) distance evaluations.  Each
    sample times advect and the crossing search over the box's grid and the
    distance loop over `sample_voxels` voxels; the whole-grid rate is
    1 / (t_advect/voxel + t_cross/voxel + t_pair x M), with M the box's
    crossings scaled by the ratio of the whole grid's sphere area to the
    box's."""

    def __init__(self, args, sample_voxels: int = 200):
        import numpy as np
        from oracle import pyoracle
        self.lib = pyoracle.load()
        self.pyoracle = pyoracle
        sph, sub, vel = _large_box_spheres(args, LARGE_REF_BOX)
        o, m, p = pyoracle.MOGrid.spheres(sub, 3.0).arrays()
        self.arrays = (o, m, p.astype(np.float32))
        off = np.arange(512)
        q = o[:, None, :].astype(np.float64) + np.stack([off >> 6, (off >> 3) & 7, off & 7], axis=1)[None]
        u = curl_velocity(vel, q[..., 0], q[..., 1], q[..., 2], np)
        self.vel = [pyoracle.OGrid.from_arrays(o, m, c.astype(np.float32), 0.0, 1.0) for c in u]
        self.n_active = int(np.unpackbits(m.view(np.uint8)).sum())
        self.area_ratio = float((sph[:, 3] ** 2).sum() / (sub[:, 3] ** 2).sum())
        self.n_spheres = len(sub)
        self.sample_voxels = sample_voxels

    def step(self):
        import ctypes as C
        g = self.pyoracle.OGrid.from_arrays(*self.arrays, 3.0, 1.0)
        h = C.c_void_p(g.h)
        ta, tr, tc = C.c_double(), C.c_double(), C.c_double()
        nr, nc = C.c_size_t(), C.c_size_t()
        self.lib.vo_time_ref_step(C.byref(h), self.vel[0].h, self.vel[1].h, self.vel[2].h, 1.0, C.c_float(3.0),
                                  self.sample_voxels, C.byref(ta), C.byref(tr), C.byref(nr), C.byref(tc),
                                  C.byref(nc))
        g.h = h.value
        t_pair = max(tr.value - tc.value, 0.0) / max(nr.value * nc.value, 1)
        per_voxel = (ta.value + tc.value) / self.n_active + t_pair * nc.value * self.area_ratio
        box_per_voxel = (ta.value + tc.value) / self.n_active + t_pair * nc.value
        return {"value": 1.0 / per_voxel, "box_value": 1.0 / box_per_voxel,
                "advect_only_value": self.n_active / ta.value, "t_advect_s": ta.value, "t_cross_s": tc.value,
                "t_pair_ns": t_pair * 1e9, "box_crossings": nc.value,
                "grid_crossings_est": nc.value * self.area_ratio}

    def describe(self):
        return (f"the crate's step (C++ restatement of advect_level_set + rebuild_narrow_band with its tree, 1 thread) "
                f"on the {self.n_spheres} spheres near a {LARGE_REF_BOX}^3 box at the grid's centre "
                f"({self.n_active} active voxels, curl noise sampled into three grids); the distance loop on "
                f"{self.sample_voxels} voxels; whole-grid rate from the per-voxel times and the box's crossings "
                f"x {self.area_ratio:.1f} (sphere area of the grid / of the box's spheres)")


# ---------------------------------------------------------------- GPU legs

STEP_KERNELS = ("k_m_advect", "k_m_reinit", "k_t_scanalloc", "k_t_finalize", "k_t_nbr")


# DRAM bytes (read + write) per leaf of one launch of the stencil kernels,
# dram__bytes_read.sum + dram__bytes_write.sum over the launch's leaves, from
# ncu captures of these bench commands (one GPU, --clock-control none,
# -k 'regex:k_m_(advect|reinit)' -c 2, the fixed launch shape
# 128,1184,0,128,1184,0 so no tuning launch precedes the captured step);
# keyed by (workload, kernel, value bytes):
#   large8192: the same generator with 1,500 spheres (466k leaves; traffic per
#     leaf does not depend on the sphere count), `bench.py --large-spheres 1500
#     --steps 1 --warmup 3 --no-...`, FP16 at -s 6, FP32 at -s 6 of the
#     float kernels (--kernel-name-base mangled -k 'regex:k_m_(advect|reinit)If');
#   batched256: its first 48 grids (151k leaves), `bench.py --workload
#     batched256 --grids 48 --steps 1 --warmup 3`, -s 6;
#   deformation512: `bench.py --workload deformation512 --steps 1 --warmup 3`,
#     -s 6 (2,858 leaves, L2-resident).
TRAFFIC_PER_LEAF: dict = {
    ("large8192", "k_m_advect", 2): 2548.8,
    ("large8192", "k_m_reinit", 2): 2342.5,
    ("large8192", "k_m_advect", 4): 4864.1,
    ("large8192", "k_m_reinit", 4): 4509.9,
    ("batched256", "k_m_advect", 2): 2327.1,
    ("batched256", "k_m_reinit", 2): 2081.1,
    ("deformation512", "k_m_advect", 2): 1238.0,
    ("deformation512", "k_m_reinit", 2): 1224.9,
}


# Warp instructions per leaf of one launch (smsp__inst_executed.sum over the
# launch's leaves) from the same captures, FP16, 128-thread CTAs.
INST_PER_LEAF: dict = {
    ("large8192", "k_m_advect"): 4452.5,
    ("large8192", "k_m_reinit"): 4198.8,
    ("batched256", "k_m_advect"): 4768.3,
    ("batched256", "k_m_reinit"): 4194.8,
    ("deformation512", "k_m_advect"): 3003.1,
    ("deformation512", "k_m_reinit"): 4440.2,
}
SM_COUNT = 148
ISSUE_PER_SM_PER_CYCLE = 4  # one warp instruction per scheduler per cycle


def issue_roofline(r, workload, sm_mhz):
    """Instruction-issue roofline of the dominant stencil kernel: warp
    instructions per launch (ncu count per leaf x leaves) / launch time, against
    148 SMs x 4 schedulers x the sampled SM clock."""
    dom = max(("k_m_advect", "k_m_reinit"), key=lambda k: r["kernels"][k])
    ipl = INST_PER_LEAF.get((workload, dom))
    if ipl is None or not sm_mhz:
        return None
    achieved = ipl * r["leaves"] / (r["kernels"][dom] * 1e-3)
    peak = SM_COUNT * ISSUE_PER_SM_PER_CYCLE * sm_mhz * 1e6
    return {"kernel": dom, "achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "inst_per_leaf_ncu": ipl, "sm_mhz": sm_mhz}


def method_bytes_per_leaf(value_bytes: int):
    """Algorithmic bytes per leaf and launch.
    advect: read values 512*s, mask 64, origin 16, neighbour row 108; write values 512*s, dilated mask 64.
    reinit (2 fused iterations + trim): read values 512*s, dilated mask 64, origin 16, neighbour row 108;
            write values 512*s, mask 64, spill 4, flag 4."""
    s = value_bytes
    return {"k_m_advect": 1024 * s + 64 + 16 + 108 + 64, "k_m_reinit": 1024 * s + 64 + 16 + 108 + 64 + 8}


def time_steps(args, ctx, ls, flush, stream, clock=None, steps=None, warmup=None):
    """Warm up, then time `steps` graph replays of a method level set, each
    bracketed by CUDA events on the library stream with the L2 flushed before
    it (outside the events); then per-kernel durations from the same steps
    enqueued without the graph (events around each kernel, L2 flushed between
    steps)."""
    import torch

    steps = steps or args.steps
    warmup = args.warmup if warmup is None else warmup
    if args.launch_shape:
        v = [int(x) for x in args.launch_shape.split(",")]
        if len(v) == 4:
            ls.set_launch_shape((v[0], v[1]), (v[2], v[3]))
        else:
            ls.set_launch_shape(tuple(v[0:3]), tuple(v[3:6]))
    ls.step(warmup)
    n0, a0, _ = ls.info()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize(args.device)
    with (clock.mark() if clock is not None else _Null()):
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                ev[k][0].record(stream)
            ls.enqueue(1)
            with torch.cuda.stream(stream):
                ev[k][1].record(stream)
        ctx.check_device()
    times = [x.elapsed_time(y) for x, y in ev]
    n1, a1, _ = ls.info()
    ms = sum(times) / len(times)
    active = 0.5 * (a0 + a1)
    leaves = 0.5 * (n0 + n1)
    ctx.profile(True)
    with (clock.mark() if clock is not None else _Null()):
        for k in range(max(3, min(steps, 10))):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            ls.step(1)
    kern = {k: ctx.kernel_time(k) for k in STEP_KERNELS}
    ctx.profile(False)
    return {"ms_per_step": ms, "value": active / (ms * 1e-3), "leaves": leaves, "active": active,
            "kernels": {k: v[0] / max(v[1], 1) for k, v in kern.items()}, "ls": ls, "launch": ls.launch_shape()}


def run_method(args, ctx, precision, flush, stream, clock=None, steps=None):
    from sharc.volrus_b200.method import LevelSet

    vs = DEFORM["voxel_size"]
    vel = {"kind": "vortex", "vs": vs, "period": DEFORM["period"]}
    dt = 0.5 * vs / 2.0
    ls = LevelSet.sphere(DEFORM["radius"], DEFORM["center"], vs, vel, dt, half_width=DEFORM["half_width"],
                         precision=precision, integrator=2, reinit_iters=2, ctx=ctx)
    return time_steps(args, ctx, ls, flush, stream, clock, steps=steps)


def run_batched(args, ctx, precision, flush, stream, clock=None, steps=None):
    """256 uneven grids (unions of 1-64 random spheres, extents 64^3-1024^3
    log-uniform, curl-noise velocity, RK3), one persistent launch per kernel.
    With N ranks each rank runs its LPT share of the grids (no data-path
    collective); the whole-job rate is the summed active voxels over the
    slowest rank's step time."""
    from sharc.volrus_b200.method import LevelSet, random_sphere_grids
    from sharc.volrus_b200.shard import reduce_totals, shard_of

    gr = random_sphere_grids(args.grids, seed=BATCH["seed"])
    gr, idx = shard_of(gr, args.rank, args.world)
    ls = LevelSet.spheres([(sph, vel) for sph, vel, _ in gr], 1.0, half_width=3.0, precision=precision,
                          integrator=3, reinit_iters=2, ctx=ctx)
    r = time_steps(args, ctx, ls, flush, stream, clock, steps=steps)
    r["grids_this_rank"] = len(idx)
    r["active_this_rank"] = r["active"]
    if args.world > 1:
        import torch
        total, ms = reduce_totals(r["active"], r["ms_per_step"], torch.device("cuda", args.device))
        r["active"], r["ms_per_step"], r["value"] = total, ms, total / (ms * 1e-3)
    return r


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


def e2e_method(args, ctx, ls, precision, steps=None):
    """Host-resident step through the C ABI (vlr_ls_step_host): upload of the
    leaves from pinned host memory, one step, download of the result into
    pinned host memory, all inside the wall-clock timed region."""
    import ctypes as C

    import numpy as np
    import torch

    from sharc.volrus_b200._lib import ptr
    steps = steps or args.steps
    o, m, v = ls.arrays()
    n = len(o)
    cap = n + n // 16 + 4096  # the band may gain leaves during the step

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    pin_o, pin_m, pin_v = pinned((n, 3), torch.int32), pinned((n, 8), torch.int64).view(np.uint64), \
        pinned((n, 512), torch.float32)
    pin_o[:], pin_m[:], pin_v[:] = o, m, v
    del o, m, v
    out_o, out_m, out_v = pinned((cap, 3), torch.int32), pinned((cap, 8), torch.int64).view(np.uint64), \
        pinned((cap, 512), torch.float32)
    h2d = d2h = 0

    def call():
        nonlocal h2d, d2h
        nn = C.c_size_t()
        ctx.check(ctx.lib.vlr_ls_step_host(ctx.handle, ls.handle, ptr(pin_o, C.c_int32), ptr(pin_m, C.c_uint64),
                                           ptr(pin_v, C.c_float), n, 1, ptr(out_o, C.c_int32),
                                           ptr(out_m, C.c_uint64), ptr(out_v, C.c_float), cap, C.byref(nn)),
                  "vlr_ls_step_host")
        h2d = n * (12 + 64 + 2048)
        d2h = nn.value * (12 + 64 + 2048)
        return nn.value

    def timed(slabs):
        ls.set_host_slabs(slabs)
        call()
        t0 = time.perf_counter()
        for _ in range(steps):
            call()
        return (time.perf_counter() - t0) / steps

    _, a, _ = ls.info()
    one_pass_s = timed(1)
    e2e_s = timed(0)
    return {"value": a / e2e_s, "unit": "voxels/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "seconds_per_step": e2e_s, "steps": steps, "slabs": min(16, n >> 17) if n >= 1 << 18 else 1,
            "one_pass_seconds_per_step": one_pass_s,
            "path": "vlr_ls_step_host (upload, one step, sorted download), pinned host buffers, f32 values on the "
                    "host; states of 2^18 leaves or more step as a pipeline of x-slabs whose copies overlap"}


def roofline_of(r, value_bytes, peak, peak_kind, workload):
    """Roofline of the dominant stencil kernel of a timed level set."""
    per = method_bytes_per_leaf(value_bytes)
    dom = max(("k_m_advect", "k_m_reinit"), key=lambda k: r["kernels"][k])
    dom_ms = r["kernels"][dom]
    achieved = per[dom] * r["leaves"] / (dom_ms * 1e-3) / 1e9
    tr = TRAFFIC_PER_LEAF.get((workload, dom, value_bytes))
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": None if tr is None else tr * r["leaves"],
            "traffic_per_leaf_ncu": tr,
            "algorithmic_bytes": per[dom] * r["leaves"], "algorithmic_bytes_per_leaf": per[dom],
            "launch_ms": dom_ms}


def bench_batched(args, ctx, peak, peak_kind, flush, stream, clk, steps=None):
    from sharc.volrus_b200.method import F16, F32
    out = {}
    for prec, name, nb in ((F16, "f16", 2), (F32, "f32", 4)):
        r = run_batched(args, ctx, prec, flush, stream, clk, steps=steps)
        out[name] = {"_r": {"kernels": r["kernels"], "leaves": r["leaves"]},
                     "value": r["value"], "ms_per_step": r["ms_per_step"], "leaves_this_rank": r["leaves"],
                     "active_voxels": r["active"], "grids_this_rank": r["grids_this_rank"], "kernels_ms_per_launch": r["kernels"],
                     "roofline": roofline_of(r, nb, peak, peak_kind, "batched256")}
        r["ls"].close()
    out["fp16_over_fp32"] = out["f16"]["value"] / out["f32"]["value"]
    out["scaling"] = "strong"
    out["n_gpus"] = args.world
    out["config"] = {"workload": "batched256", "grids": args.grids, "seed": BATCH["seed"],
                     "sharding": "whole grids per rank, greedy LPT on estimated band voxels; no data-path collective",
                     "extent": "2^U(6,10) voxels per axis", "spheres": "1-64 per grid, r~U(4,24)",
                     "velocity": "curl noise, 3 octaves, 1 voxel/step", "integrator": "SSP-RK3", "dt": 1.0,
                     "half_width": 3, "reinit_iters": 2, "l2": "inputs larger than L2 and flushed between steps"}
    return out


def bench_batched_line(args, ctx, peak, peak_kind):
    """The batched workload on its own: FP16 line with FP32 beside it."""
    import torch
    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    with ClockSampler(args.device) as clk:
        b = bench_batched(args, ctx, peak, peak_kind, flush, stream, clk)
    f = b["f16"]
    ck = clk.summary()
    f["issue_roofline"] = issue_roofline(f.pop("_r"), "batched256", ck.get("sm_mhz"))
    b["f32"].pop("_r", None)
    return {"metric": METRIC, "value": f["value"], "unit": "voxels/s", "ms_per_step": f["ms_per_step"],
            "dtype": "f16 storage, f32 arithmetic", "config": dict(b["config"], active_voxels=f["active_voxels"],
                                                                  leaves_this_rank=f["leaves_this_rank"]),
            "fp32": b["f32"], "fp16_over_fp32": b["fp16_over_fp32"], "roofline": f["roofline"],
            "issue_roofline": f["issue_roofline"],
            "kernels_ms_per_launch": f["kernels_ms_per_launch"], "e2e": None, "clocks": ck,
            "gpu_launches": len(STEP_KERNELS) * args.steps}


def leaf_voxel_coords(origins, masks):
    """Index coordinates (n_active, 3) and (leaf, offset) of the active voxels."""
    import numpy as np
    off = np.arange(512)
    rel = np.stack([off >> 6, (off >> 3) & 7, off & 7], axis=1)
    bits = np.unpackbits(masks.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    li, vi = np.nonzero(bits)
    return origins[li].astype(np.int64) + rel[vi], li, vi


def full_period(args, ctx, precision, reinit_mode=0):
    """One full period of the deformation test (T = 3, dt = vs / 4: 6,144 steps
    at 512^3): the shape returns to the start sphere, so the error of phi on the
    interface (active voxels with |phi_exact| <= 1 voxel) against the exact
    signed distance, and the relative change of the FP64 enclosed volume, measure
    the method's accuracy at this resolution."""
    import numpy as np
    from sharc.volrus_b200.method import LevelSet
    vs, T = DEFORM["voxel_size"], DEFORM["period"]
    dt = 0.5 * vs / 2.0
    steps = int(round(T / dt))
    # the stretched sheet at t = T/2 holds many times the sphere's leaves
    ls = LevelSet.sphere(DEFORM["radius"], DEFORM["center"], vs, {"kind": "vortex", "vs": vs, "period": T}, dt,
                         half_width=DEFORM["half_width"], precision=precision, integrator=2, reinit_iters=2,
                         capacity=200_000, reinit_mode=reinit_mode, ctx=ctx)
    v0 = ls.volume()
    n0 = ls.leaf_count()
    peak = n0
    for _ in range(16):
        ls.step(steps // 16)
        peak = max(peak, ls.leaf_count())
    ls.step(steps - 16 * (steps // 16))
    v1 = ls.volume()
    o, m, p = ls.arrays()
    ls.close()
    xyz, li, vi = leaf_voxel_coords(o, m)
    c = np.asarray(DEFORM["center"]) / vs
    exact = np.sqrt(((xyz - c) ** 2).sum(axis=1)) - DEFORM["radius"] / vs
    sel = np.abs(exact) <= 1.0
    err = p[li, vi][sel] - exact[sel]
    exact_vol = 4.0 / 3.0 * math.pi * (DEFORM["radius"] / vs) ** 3
    far = int((np.abs(exact) > 2.0 * DEFORM["half_width"]).sum())
    return {"steps": steps, "reinit_mode": reinit_mode, "leaves_start": n0, "leaves_peak_sampled": peak, "leaves_end": int(len(o)),
            "active_far_from_start_shape": far,
            "interface_voxels": int(sel.sum()), "max_err_vox": float(np.abs(err).max()),
            "rms_err_vox": float(np.sqrt(np.mean(err ** 2))), "volume_change_rel": (v1 - v0) / v0,
            "volume_start_vs_exact_rel": (v0 - exact_vol) / exact_vol,
            "against": "exact signed distance of the start sphere (the flow returns to it after one period)"}


# Algorithmic bytes per band voxel of one launch of the adjoint's kernels,
# each array counted once per launch (the trilinear corners and the
# candidates' feet are read through the cache by up to 27 neighbours):
#   k_adj_forward: band index 4 + displacement 12 + phi_k 4 + phi_k+1 4
#   k_adj_pack:    band index 4 + displacement 12 + lambda 4 + foot word 4 + weights and lambda 16
#   k_adj_lambda:  band index 4 + own foot 20 + phi_k 4 + G read and written 24 + lambda out 4
ADJ_BYTES_PER_BAND_VOXEL = {"k_adj_forward": 24, "k_adj_pack": 40, "k_adj_lambda": 56}


def adjoint_roofline(kern, nb, peak, peak_kind):
    """HBM roofline of the adjoint's dominant kernel from a profiled pass:
    kern = {name: (total ms, launches)}."""
    timed = {k: v for k, v in kern.items() if k in ADJ_BYTES_PER_BAND_VOXEL and v[1] > 0}
    if not timed:
        return None
    dom = max(timed, key=lambda k: timed[k][0])
    ms = timed[dom][0] / timed[dom][1]
    per = ADJ_BYTES_PER_BAND_VOXEL[dom]
    achieved = per * nb / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes_per_band_voxel": per,
            "algorithmic_bytes": per * nb, "launch_ms": ms}


def bench_adjoint(args, ctx):
    """The adjoint configuration: sphere r = 32 centred in 256^3, FP32, K = 64
    steps of the deformation field (T = 2), checkpoints every 8 steps, a 128^3
    staggered velocity; forward then backward, timed with CUDA events on the
    library stream.  Rate = band voxels x K / (forward + backward)."""
    import numpy as np
    import torch
    from sharc.volrus_b200.adjoint import AdvectionFunction, sphere_band, staggered_vortex
    domain, radius, n, steps, chk = 256, 32.0, 128, 64, 8
    cell, vs = domain / n, 1.0 / domain
    dt = 0.5 / (2.0 / vs)
    o, m, p = sphere_band(radius, (128.0, 128.0, 128.0), domain, ctx=ctx)
    V = staggered_vortex(n, cell, vs)
    fn = AdvectionFunction(o, m, p, V, cell, dt, 2.0, steps, chk, ctx=ctx)
    band = fn.band()
    target = (np.sqrt(((band - np.array([136.0, 128.0, 128.0])) ** 2).sum(axis=1)) - radius).astype(np.float32)
    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    # device-resident passes (buffers in HBM; what a GPU training loop calls)
    d_phik = torch.empty(fn.n_band, dtype=torch.float32, device=dev)
    d_lam = torch.empty(fn.n_band, dtype=torch.float32, device=dev)
    d_g0 = torch.empty(fn.n_band, dtype=torch.float32, device=dev)
    d_gv = torch.empty(3 * n ** 3, dtype=torch.float32, device=dev)
    d_target = torch.from_numpy(target).to(dev)
    fw, bw = [], []
    for k in range(args.warmup + max(3, min(args.steps, 10))):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        with torch.cuda.stream(stream):
            e[0].record(stream)
            fn.forward_device(d_phik.data_ptr())
            e[1].record(stream)
            torch.sub(d_phik, d_target, out=d_lam)
            d_lam.mul_(2.0)
            fn.backward_device(d_lam.data_ptr(), d_g0.data_ptr(), d_gv.data_ptr())
            e[2].record(stream)
        ctx.check_device()
        if k >= args.warmup:
            fw.append(e[0].elapsed_time(e[1]))
            bw.append(e[1].elapsed_time(e[2]))
    # host-resident passes through the C ABI: inputs and outputs in pinned host
    # buffers allocated once (phi_K out, dL/dphi_K in, dL/dphi_0 and dL/dV out)
    import ctypes as C
    from sharc.volrus_b200._lib import ptr
    h_phik = torch.empty(fn.n_band, dtype=torch.float32).pin_memory().numpy()
    h_lam = torch.empty(fn.n_band, dtype=torch.float32).pin_memory().numpy()
    h_g0 = torch.empty(fn.n_band, dtype=torch.float32).pin_memory().numpy()
    h_gv = torch.empty(3 * n ** 3, dtype=torch.float32).pin_memory().numpy()
    hw_ = []
    for k in range(1 + 5):
        t0 = time.perf_counter()
        ctx.check(ctx.lib.vlr_adj_forward(ctx.handle, fn.handle, ptr(h_phik, C.c_float)), "vlr_adj_forward")
        np.subtract(h_phik, target, out=h_lam)
        h_lam *= 2.0
        ctx.check(ctx.lib.vlr_adj_backward(ctx.handle, fn.handle, ptr(h_lam, C.c_float), ptr(h_g0, C.c_float),
                                           ptr(h_gv, C.c_float)), "vlr_adj_backward")
        if k >= 1:
            hw_.append(time.perf_counter() - t0)
    ctx.profile(True)
    phik = fn.forward()
    fn.backward(2.0 * (phik - target))
    kern = {k: ctx.kernel_time(k) for k in ("k_adj_forward", "k_adj_pack", "k_adj_lambda", "k_adj_emit_vel")}
    ctx.profile(False)
    nb = fn.n_band
    fn.close()
    f, b = statistics.median(fw), statistics.median(bw)
    he = statistics.median(hw_)
    return {"workload": "adjoint256: sphere r=32 in 256^3, K=64, checkpoint 8, 128^3 staggered velocity, FP32",
            "band_voxels": nb, "forward_ms": f, "backward_ms": b,
            "value": nb * steps / ((f + b) * 1e-3), "unit": "band voxel-steps/s (forward + backward)",
            "timing": "device buffers, CUDA events on the library stream (forward_device + backward_device)",
            "e2e": {"value": nb * steps / he, "unit": "band voxel-steps/s",
                    "path": "vlr_adj_forward + vlr_adj_backward with pinned host buffers (dL/dV: 25 MB to the "
                            "host)",
                    "h2d_bytes_per_step": nb * 4, "d2h_bytes_per_step": nb * 8 + 3 * n ** 3 * 4},
            "forward_voxels_per_s": nb * steps / (f * 1e-3),
            "kernels_ms_total_per_pass": {k: v[0] for k, v in kern.items()},
            "kernels_launches_per_pass": {k: v[1] for k, v in kern.items()},
            "roofline": adjoint_roofline(kern, nb, *measured_peaks())}


def bench_level_set_adjoint(args, ctx, ls, steps=32, chk=6, shift=(4, 0, 0)):
    """Frozen-band adjoint of a level set's own step (vlr_adj_create_level_set):
    K = steps, checkpoints every chk (~sqrt K), L = sum over the band of
    (phi_K - phi_0(x - shift))^2; forward_device + backward_device timed with
    CUDA events on the library stream.  Rate = band voxels x K / (forward +
    backward)."""
    import torch
    from sharc.volrus_b200.adjoint import AdvectionFunction
    free0 = torch.cuda.mem_get_info()[0]
    t0 = time.perf_counter()
    fn = AdvectionFunction.from_level_set(ls, steps, chk)
    create_s = time.perf_counter() - t0
    nb = fn.n_band
    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    d_phik, d_lam, d_g0, d_target = (torch.empty(nb, dtype=torch.float32, device=dev) for _ in range(4))
    held = (free0 - torch.cuda.mem_get_info()[0]) / 2**30
    with torch.cuda.stream(stream):
        fn.shifted_phi0_device(shift, d_target.data_ptr())
    fw, bw = [], []
    for k in range(1 + 2):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        with torch.cuda.stream(stream):
            e[0].record(stream)
            fn.forward_device(d_phik.data_ptr())
            e[1].record(stream)
            torch.sub(d_phik, d_target, out=d_lam)
            d_lam.mul_(2.0)
            fn.backward_device(d_lam.data_ptr(), d_g0.data_ptr(), 0)
            e[2].record(stream)
        ctx.check_device()
        if k >= 1:
            fw.append(e[0].elapsed_time(e[1]))
            bw.append(e[1].elapsed_time(e[2]))
    loss = float(((d_phik - d_target) ** 2).sum().item())
    gnorm = float(d_g0.norm().item())
    ctx.profile(True)  # kernel times from a separate pass (the events would perturb the timed passes)
    with torch.cuda.stream(stream):
        fn.forward_device(d_phik.data_ptr())
        torch.sub(d_phik, d_target, out=d_lam)
        d_lam.mul_(2.0)
        fn.backward_device(d_lam.data_ptr(), d_g0.data_ptr(), 0)
    ctx.check_device()
    kern = {k: ctx.kernel_time(k) for k in ("k_adj_forward", "k_adj_pack", "k_adj_lambda")}
    ctx.profile(False)
    fn.close()
    f, b = statistics.median(fw), statistics.median(bw)
    return {"workload": f"level-set adjoint, K={steps}, checkpoint every {chk}, L2 loss against phi_0 shifted by "
                        f"{list(shift)} voxels, FP32 band values",
            "band_voxels": nb, "forward_ms": f, "backward_ms": b, "create_s": create_s,
            "device_gib_held": held, "loss": loss, "grad_norm": gnorm,
            "value": nb * steps / ((f + b) * 1e-3), "unit": "band voxel-steps/s (forward + backward)",
            "forward_voxels_per_s": nb * steps / (f * 1e-3),
            "kernels_ms_per_launch": {k: v[0] / max(v[1], 1) for k, v in kern.items()},
            "roofline": adjoint_roofline(kern, nb, *measured_peaks()),
            "timing": "device buffers, CUDA events on the library stream (forward_device + backward_device)"}


def large_config(args) -> dict:
    """The large single grid's configuration (both arms print this dict)."""
    return {"workload": "large8192", "spheres": args.large_spheres, "seed": LARGE["seed"], "extent": "8192^3",
            "radius": "U(6, 40)", "velocity": "curl noise, 3 octaves, 1 voxel/step", "integrator": "SSP-RK3",
            "dt": 1.0, "half_width": 3, "reinit_iters": 2,
            "l2": "inputs larger than L2 (126 MB) and flushed between steps"}


def curl_velocity(vel: dict, x, y, z, xp):
    """Curl-noise velocity (voxels per unit time) at index points, the field of
    the method's curl velocity: v = sum_o grad f_o x e_o with
    f_o = A_o prod_a sin(k_o p_a + ph_{o,a}); `xp` is numpy or torch."""
    u = [0.0 * x, 0.0 * x, 0.0 * x]
    for A, k, ph, e in vel["octaves"]:
        s = [xp.sin(k * q + f) for q, f in zip((x, y, z), ph)]
        c = [xp.cos(k * q + f) for q, f in zip((x, y, z), ph)]
        g = [A * k * c[0] * s[1] * s[2], A * k * s[0] * c[1] * s[2], A * k * s[0] * s[1] * c[2]]
        u[0] = u[0] + g[1] * e[2] - g[2] * e[1]
        u[1] = u[1] + g[2] * e[0] - g[0] * e[2]
        u[2] = u[2] + g[0] * e[1] - g[1] * e[0]
    return u


def data_path(args, ctx, flush, stream, clk, sph, peak, peak_kind):
    """The same grid with the lightest arithmetic the step allows: constant
    velocity (0.6, -0.4, 0.3) voxels/step, Euler backtrace, no reinitialisation
    iteration (trim and re-track only).  Shows what the staging and the
    topology kernels reach on their own, and what FP16 storage buys there."""
    from sharc.volrus_b200.method import F16, F32, LevelSet
    out = {"velocity": "constant (0.6, -0.4, 0.3) voxels/step", "integrator": "Euler", "reinit_iters": 0}
    steps = min(args.steps, 5)
    for prec, name, nb in ((F16, "f16", 2), (F32, "f32", 4)):
        # without reinitialisation the band widens every step: room for 3.2x the start's leaves
        ls = LevelSet.spheres([(sph, {"kind": "constant", "c": (0.6, -0.4, 0.3)})], 1.0, half_width=3.0,
                              precision=prec, integrator=1, reinit_iters=0, capacity=8_000_000, ctx=ctx)
        r = time_steps(args, ctx, ls, flush, stream, clk, steps=steps)
        out[name] = {"value": r["value"], "ms_per_step": r["ms_per_step"], "steps": steps,
                     "kernels_ms_per_launch": r["kernels"],
                     "roofline": roofline_of(r, nb, peak, peak_kind, "large8192-data-path")}
        ls.close()
    out["fp16_over_fp32"] = out["f16"]["value"] / out["f32"]["value"]
    return out


def ref_step_leg(args, ctx, ls, flush, stream, clk):
    """The crate's own step on the GPU, vlr_advect_level_set +
    vlr_rebuild_narrow_band (src/tools/advection.rs:32-56,
    src/tools/level_set_track.rs:80-114), over the same grid: the FP32 level
    set's leaves as a world-unit grid (voxel size 1, background 3) and the
    curl-noise velocity sampled at every voxel of those leaves into three grids
    (the crate's VelocityField; the crate samples it at voxel positions, where
    trilinear interpolation returns the voxel's own value).  Each timed step
    advects the same input grid."""
    import torch
    from sharc.volrus_b200 import VelocityField
    from sharc.volrus_b200.method import large_sphere_grid
    from sharc.volrus_b200.tools import DeviceGrid, advect_level_set, rebuild_narrow_band
    dev = torch.device("cuda", args.device)
    n = ls.leaf_count()
    o = torch.empty((n, 3), dtype=torch.int32, device=dev)
    m = torch.empty((n, 8), dtype=torch.int64, device=dev)
    p = torch.empty((n, 512), dtype=torch.float32, device=dev)
    k = ls.download_device(o.data_ptr(), m.data_ptr(), p.data_ptr(), n)
    lo = (o[:k] >> 3).long() + (1 << 20)
    order = torch.argsort((lo[:, 0] << 42) | (lo[:, 1] << 21) | lo[:, 2])
    o, m, p = o[:k][order].contiguous(), m[:k][order].contiguous(), p[:k][order].contiguous()
    del lo, order
    g0 = DeviceGrid.from_device(o.data_ptr(), m.data_ptr(), p.data_ptr(), k, 3.0, 1.0, ctx)
    del p
    _, vel = large_sphere_grid(args.large_spheres, LARGE["seed"])
    off = torch.arange(512, device=dev)
    rel = torch.stack([off >> 6, (off >> 3) & 7, off & 7], dim=1).double()
    comps = [torch.empty((k, 512), dtype=torch.float32, device=dev) for _ in range(3)]
    chunk = 1 << 16
    for a in range(0, k, chunk):
        b = min(k, a + chunk)
        q = o[a:b].double()[:, None, :] + rel[None]
        u = curl_velocity(vel, q[..., 0], q[..., 1], q[..., 2], torch)
        for c in range(3):
            comps[c][a:b] = u[c].float()
    vgrids = [DeviceGrid.from_device(o.data_ptr(), m.data_ptr(), c.data_ptr(), k, 0.0, 1.0, ctx) for c in comps]
    del comps, o, m
    dvel = VelocityField(*vgrids)
    n_active = g0.active_voxel_count()

    def step():
        out = advect_level_set(g0, dvel, 1.0, ctx=ctx)
        rebuild_narrow_band(out, 3.0, ctx=ctx)
        return out

    for _ in range(2):
        step().close()
    ctx.synchronize()
    steps = min(args.steps, 10)
    times = []
    ctx.profile(True)
    with clk.mark():
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = step()
            with torch.cuda.stream(stream):
                e1.record(stream)
            ctx.synchronize()
            times.append(e0.elapsed_time(e1))
            out_active = out.active_voxel_count()
            out.close()
    kern = {kk: ctx.kernel_time(kk) for kk in ("k_advect_ref", "k_crossings", "k_rebuild_window")}
    ctx.profile(False)
    ms = sum(times) / len(times)
    for gg in (g0, *vgrids):
        gg.close()
    return {"value": n_active / (ms * 1e-3), "unit": "voxels/s", "ms_per_step": ms, "steps": steps,
            "leaves": k, "active_voxels": n_active, "active_after": out_active,
            "kernels_ms_per_launch": {kk: v[0] / max(v[1], 1) for kk, v in kern.items()},
            "step": "vlr_advect_level_set (three-grid curl-noise VelocityField, dt 1) + vlr_rebuild_narrow_band (hw 3), "
                    "f32 world values: the crate's algorithm, bit-exact to its CPU code",
            "timing": "CUDA events on the library stream, L2 flushed before each step, same input grid every step"}


def bench_large_line(args, ctx, peak, peak_kind):
    """The large single grid: FP16 line with FP32, the data-path diagnostic,
    the crate's own step on the GPU and the end-to-end host step beside it."""
    import torch
    from sharc.volrus_b200.method import F16, F32, LevelSet, large_sphere_grid
    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sph, vel = large_sphere_grid(args.large_spheres, LARGE["seed"])
    out = {}
    with ClockSampler(args.device) as clk:
        for prec, name, nb in ((F16, "f16", 2), (F32, "f32", 4)):
            t0 = time.perf_counter()
            ls = LevelSet.spheres([(sph, vel)], 1.0, half_width=3.0, precision=prec, integrator=3, reinit_iters=2,
                                  ctx=ctx)
            build_s = time.perf_counter() - t0
            r = time_steps(args, ctx, ls, flush, stream, clk)
            out[name] = {"value": r["value"], "ms_per_step": r["ms_per_step"], "leaves": r["leaves"],
                         "active_voxels": r["active"], "kernels_ms_per_launch": r["kernels"],
                         "launch_shape": r["launch"], "create_s": build_s, "_r": r,
                         "roofline": roofline_of(r, nb, peak, peak_kind, "large8192")}
            if prec == F16:
                out["e2e"] = e2e_method(args, ctx, ls, prec, steps=min(args.steps, 3))
                if not args.no_adjoint:
                    out["adjoint"] = bench_level_set_adjoint(args, ctx, ls)
            elif not args.no_ref_step:
                out["ref_step"] = ref_step_leg(args, ctx, ls, flush, stream, clk)
            ls.close()
        if not args.no_data_path:
            out["data_path"] = data_path(args, ctx, flush, stream, clk, sph, peak, peak_kind)
        if not args.no_batched:
            b = bench_batched(args, ctx, peak, peak_kind, flush, stream, clk, steps=min(args.steps, 10))
            for kk in ("f16", "f32"):
                b[kk].pop("_r", None)
            out["batched256"] = b
        if not args.no_deformation:
            d = {}
            for prec, name in ((F16, "f16"), (F32, "f32")):
                r = run_method(args, ctx, prec, flush, stream, clk, steps=min(args.steps, 10))
                d[name] = {"value": r["value"], "ms_per_step": r["ms_per_step"], "leaves": r["leaves"],
                           "active_voxels": r["active"], "kernels_ms_per_launch": r["kernels"]}
                r["ls"].close()
            d["fp16_over_fp32"] = d["f16"]["value"] / d["f32"]["value"]
            d["config"] = {"workload": "deformation512", "domain": "unit cube at 512^3",
                           "sphere": "r=0.15 at (0.35,0.35,0.35)", "velocity": "vortex T=3, analytic",
                           "integrator": "RK2 midpoint", "cfl": 0.5, "half_width": 3, "reinit_iters": 2,
                           "l2": "inputs smaller than L2; flushed between steps"}
            out["deformation512"] = d
    ck = clk.summary()
    f = out["f16"]
    accuracy = None
    if not args.no_accuracy:
        accuracy = {"f16": full_period(args, ctx, F16), "f32": full_period(args, ctx, F32),
                    "f16_subcell_fix": full_period(args, ctx, F16, reinit_mode=1)}
    mesh = None if args.no_mesh else bench_mesh(args, ctx, peak, peak_kind)
    line = {"metric": METRIC, "value": f["value"], "unit": "voxels/s", "ms_per_step": f["ms_per_step"],
            "dtype": "f16 storage, f32 arithmetic", "config": large_config(args),
            "active_voxels": f["active_voxels"], "leaves": f["leaves"], "create_s": f["create_s"],
            "fp32": {k: v for k, v in out["f32"].items() if k != "_r"},
            "fp16_over_fp32": f["value"] / out["f32"]["value"], "roofline": f["roofline"],
            "issue_roofline": issue_roofline(f["_r"], "large8192", ck.get("sm_mhz")),
            "kernels_ms_per_launch": f["kernels_ms_per_launch"], "launch_shape": f["launch_shape"],
            "e2e": out["e2e"], "clocks": ck, "gpu_launches": len(STEP_KERNELS) * args.steps}
    for k in ("ref_step", "data_path", "adjoint", "batched256", "deformation512"):
        if k in out:
            line[k] = out[k]
    if accuracy is not None:
        line["full_period"] = accuracy
    if mesh is not None:
        line["volume_to_mesh"] = mesh
    return line


MESH = dict(radius=96.0, center=(0.5, -0.25, 0.125), voxel_size=1.0, half_width=3.0)


def bench_mesh(args, ctx, peak, peak_kind):
    """volume_to_mesh on a world-unit sphere (r = 96 voxels, half-width 3):
    one C-ABI call per step with host output buffers (device work, sync and
    the vertex / triangle downloads inside the timed region), kernel times
    from the context profiler, and the single-threaded oracle on the same
    grid as the CPU baseline."""
    import ctypes as C

    import numpy as np

    from oracle import pyoracle
    from sharc.volrus_b200 import make_level_set_sphere

    g = make_level_set_sphere(MESH["radius"], MESH["center"], MESH["voxel_size"], MESH["half_width"], ctx=ctx,
                              device=True)
    n_leaves = g.leaf_count()
    nv, nt = C.c_size_t(), C.c_size_t()
    ctx.check(ctx.lib.vlr_volume_to_mesh(ctx.handle, g.handle, C.c_float(0.0), None, 0, None, 0, C.byref(nv),
                                         C.byref(nt)), "vlr_volume_to_mesh")
    verts = np.zeros((nv.value, 3), np.float64)
    tris = np.zeros((nt.value, 3), np.uint32)

    def call():
        ctx.check(ctx.lib.vlr_volume_to_mesh(ctx.handle, g.handle, C.c_float(0.0),
                                             verts.ctypes.data_as(C.POINTER(C.c_double)), nv.value,
                                             tris.ctypes.data_as(C.POINTER(C.c_uint32)), nt.value, C.byref(nv),
                                             C.byref(nt)), "vlr_volume_to_mesh")

    for _ in range(max(3, args.warmup)):
        call()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call()
    call_s = (time.perf_counter() - t0) / args.steps
    ctx.profile(True)  # kernel times from a separate pass (the events would perturb the timed calls)
    for _ in range(args.steps):
        call()
    names = ("k_mc_classify", "k_mc_emit", "k_rs_hist", "k_rs_scatter")
    kern = {k: ctx.kernel_time(k) for k in names}
    ctx.profile(False)
    kms = {k: v[0] / max(args.steps, 1) for k, v in kern.items()}
    # tiles visited: every leaf tile and its face neighbours (counted on the host from the leaf list)
    o, _, _ = g.download().to_arrays()
    tiles = set()
    for x, y, z in (o // 8).tolist():
        for d in ((0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
            tiles.add((x + d[0], y + d[1], z + d[2]))
    cells = 512 * len(tiles)
    dev_ms = kms["k_mc_classify"] + kms["k_mc_emit"]
    # classify + emit bytes: leaf values read twice (each tile reads its own and
    # its +1 neighbours' layers: ~1.4x a leaf), cell words written and read,
    # vertices and triangles written
    algo = 2 * 1.4 * 2048 * len(tiles) + 2 * 4 * cells + 24 * nv.value + 12 * nt.value
    achieved = algo / (dev_ms * 1e-3) / 1e9
    cpu_s, exact = None, None
    if not args.no_cpu_baseline:
        host = g.download()
        ho, hm, hv = host.to_arrays()
        og = pyoracle.OGrid.from_arrays(ho, hm, hv, host.background, host.transform.voxel_size)
        t0 = time.perf_counter()
        ov, ot = og.volume_to_mesh(0.0)
        cpu_s = time.perf_counter() - t0
        exact = bool(np.array_equal(ov.view(np.uint64), verts.view(np.uint64)) and np.array_equal(ot, tris))
    return {
        "workload": f"world-unit sphere r={MESH['radius']:g} voxels, half-width {MESH['half_width']:g}, isovalue 0",
        "leaves": n_leaves, "tiles": len(tiles), "cells": cells, "vertices": nv.value, "triangles": nt.value,
        "value": cells / call_s, "unit": "cells/s (one C-ABI call, host output buffers, downloads included)",
        "call_ms": call_s * 1e3, "kernels_ms_per_call": kms, "device_ms": dev_ms,
        "device_cells_per_s": cells / (dev_ms * 1e-3),
        "roofline": {"bound": "hbm", "kernels": "k_mc_classify + k_mc_emit", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "algorithmic_bytes": algo},
        "d2h_bytes_per_call": int(verts.nbytes + tris.nbytes),
        "cpu_baseline": None if cpu_s is None else {
            "value": cells / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
            "sample": "the oracle restatement of volume_to_mesh on the same grid, one call"},
        "matches_oracle": exact,
    }


def bench_adjoint_line(args, ctx):
    """The adjoint configuration on its own (forward + backward per step)."""
    with ClockSampler(args.device) as clk, clk.mark():
        a = bench_adjoint(args, ctx)
    return {"metric": "band voxel-steps/s of the adjoint (forward + backward)", "value": a["value"],
            "unit": "voxels/s", "ms_per_step": (a["forward_ms"] + a["backward_ms"]) / 64.0, "dtype": "f32",
            "config": {"workload": "adjoint256", "active_voxels": a["band_voxels"], "steps": 64,
                       "checkpoint_every": 8, "velocity": "128^3 staggered, trilinear upsample"},
            "roofline": a["roofline"], "e2e": None, "clocks": clk.summary(), "gpu_launches": None,
            "kernels_ms_per_launch": {k: a["kernels_ms_total_per_pass"][k] / max(a["kernels_launches_per_pass"][k], 1)
                                      for k in a["kernels_ms_total_per_pass"]}, "adjoint": a}


def bench_mesh_line(args, ctx, peak, peak_kind):
    """volume_to_mesh on its own: `value` is the device rate of its two kernels,
    `e2e` the C-ABI call with host output buffers."""
    with ClockSampler(args.device) as clk, clk.mark():
        m = bench_mesh(args, ctx, peak, peak_kind)
    return {"metric": "cells/s of volume_to_mesh", "value": m["device_cells_per_s"], "unit": "cells/s",
            "ms_per_step": m["device_ms"], "dtype": "f32 values, f64 vertices",
            "config": {"workload": "mesh96", "active_voxels": m["cells"], "grid": m["workload"]},
            "roofline": m["roofline"],
            "e2e": {"value": m["value"], "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": m["d2h_bytes_per_call"]},
            "clocks": clk.summary(), "gpu_launches": None, "kernels_ms_per_launch": m["kernels_ms_per_call"],
            "volume_to_mesh": m}


TOOLS = dict(radius=160.0, center=(0.5, -0.25, 0.125), voxel_size=1.0, half_width=3.0, particles=1 << 20)


def bench_tools_line(args, ctx, peak, peak_kind):
    """The crate's other tools on one sphere (radius 160 voxels, half-width 3),
    each call timed on the device (CUDA events on the library stream, L2
    flushed before it, a fresh copy of the input for the in-place tools):
    find_zero_crossings, trim and rebuild_narrow_band, dilate (1 iteration),
    flood_fill_sign, extend_velocity (half-width 3), volume_to_mesh, the .vol
    and NanoGrid writers and readers, and the RK4 particle update (2^20
    particles in the band).  Rates are the input's active voxels (particles
    for the update) per second of device time; `value` is the median over
    the grid tools."""
    import numpy as np
    import torch

    from sharc.volrus_b200 import (DeviceGrid, VelocityField, dilate, extend_velocity, find_zero_crossings,
                                   flood_fill_sign, make_level_set_sphere, make_uniform_velocity, rebuild_narrow_band,
                                   trim_narrow_band, volume_to_mesh)
    from sharc.volrus_b200.io import NanoGrid, read_vol, write_vol
    from sharc.volrus_b200.tools import advect_particles

    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sph = {k: TOOLS[k] for k in ("radius", "center", "voxel_size", "half_width")}
    host = make_level_set_sphere(**sph, ctx=ctx)
    n_active, n_leaves = host.active_voxel_count(), host.leaf_count()
    vel = make_uniform_velocity(1.0, (0.5, -0.25, 1.0))
    dvel = VelocityField(*[DeviceGrid.upload(c, ctx) for c in (vel.vx, vel.vy, vel.vz)])
    vol_bytes = write_vol(host)
    nano = NanoGrid.from_grid(host).as_bytes()
    rng = np.random.default_rng(5)
    o, m, _ = host.to_arrays()
    pts = (o[rng.integers(0, len(o), TOOLS["particles"])] + rng.uniform(0, 8, (TOOLS["particles"], 3))).astype(
        np.float64)

    def timed(fn, fresh=None, reps=None):
        reps = reps or max(3, min(args.steps, 10))
        ts = []
        for r in range(reps + 1):
            arg = fresh() if fresh else None
            ctx.synchronize()
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = fn(arg)
            with torch.cuda.stream(stream):
                e1.record(stream)
            ctx.synchronize()
            if r:  # the first call warms up
                ts.append(e0.elapsed_time(e1))
            for x in (arg, out):
                if isinstance(x, DeviceGrid):
                    x.close()
        return statistics.median(ts)

    fresh = lambda: DeviceGrid.upload(host, ctx)
    res = {}
    with ClockSampler(args.device) as clk, clk.mark():
        res["find_zero_crossings"] = timed(lambda g: find_zero_crossings(g, ctx=ctx), fresh)
        res["trim_narrow_band"] = timed(lambda g: trim_narrow_band(g, 2.0, ctx=ctx), fresh)
        res["rebuild_narrow_band"] = timed(lambda g: rebuild_narrow_band(g, 3.0, ctx=ctx), fresh)
        res["dilate"] = timed(lambda g: dilate(g, 1, ctx=ctx), fresh)
        res["flood_fill_sign"] = timed(lambda g: flood_fill_sign(g, ctx=ctx), fresh)
        ext = lambda: [DeviceGrid.upload(host, ctx) for _ in range(4)]

        def run_ext(gs):
            extend_velocity(*gs, 3.0, ctx=ctx)
            for g in gs:
                g.close()
        res["extend_velocity"] = timed(run_ext, ext)
        res["volume_to_mesh"] = timed(lambda g: volume_to_mesh(g, 0.0, ctx=ctx), fresh)
        res["write_vol"] = timed(lambda g: write_vol(g), fresh)
        res["read_vol"] = timed(lambda _: read_vol(vol_bytes, ctx))
        res["nano_from_grid"] = timed(lambda g: NanoGrid.from_grid(g), fresh)
        res["nano_to_grid"] = timed(lambda _: NanoGrid.from_bytes(nano).to_grid(ctx))
        t_part = timed(lambda _: advect_particles(pts, dvel, 1.0, ctx=ctx))
    grid_rates = {k: n_active / (v * 1e-3) for k, v in res.items()}
    value = statistics.median(grid_rates.values())
    return {"metric": "active voxels/s per tool call (median over the grid tools)", "value": value,
            "unit": "voxels/s", "ms_per_step": statistics.median(res.values()), "dtype": "f32",
            "config": {"workload": "tools160", "leaves": n_leaves, "active_voxels": n_active,
                       "sphere": sph, "particles": TOOLS["particles"],
                       "l2": "flushed before every call (256 MiB write outside the call's events)",
                       "timing": "CUDA events on the library stream around the public call; host copies "
                                 "of the crate-facing calls (crossing list, .vol and NanoGrid bytes, particle "
                                 "positions) are inside the events"},
            "roofline": None, "e2e": None, "clocks": clk.summary(), "gpu_launches": None, "kernels_ms_per_launch": {},
            "tools_ms_per_call": res, "tools_voxels_per_s": grid_rates,
            "advect_particles": {"ms_per_call": t_part, "particles_per_s": TOOLS["particles"] / (t_part * 1e-3),
                                 "integrator": "RK4 through three uniform velocity grids"}}


def bench_deformation(args, ctx, peak, peak_kind):
    import torch
    from sharc.volrus_b200.method import F16, F32

    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    batched = None
    with ClockSampler(args.device) as clk:
        r16 = run_method(args, ctx, F16, flush, stream, clk)
        r32 = run_method(args, ctx, F32, flush, stream, clk)
        if not args.no_batched:
            batched = bench_batched(args, ctx, peak, peak_kind, flush, stream, clk, steps=min(args.steps, 10))
    e2e = e2e_method(args, ctx, r16["ls"], F16)
    accuracy = None if args.no_accuracy else {"f16": full_period(args, ctx, F16), "f32": full_period(args, ctx, F32),
                                              "f16_subcell_fix": full_period(args, ctx, F16, reinit_mode=1)}
    adjoint = None if args.no_adjoint else bench_adjoint(args, ctx)
    mesh = None if args.no_mesh else bench_mesh(args, ctx, peak, peak_kind)
    launches_per_step = len(STEP_KERNELS)  # one CUDA graph per step
    line = {
        "metric": METRIC, "value": r16["value"], "unit": "voxels/s", "ms_per_step": r16["ms_per_step"],
        "dtype": "f16 storage, f32 arithmetic",
        "config": {"workload": "deformation512", "domain": "unit cube at 512^3", "sphere": "r=0.15 at (0.35,0.35,0.35)",
                   "half_width": 3, "velocity": "vortex T=3, analytic", "integrator": "RK2 midpoint",
                   "cfl": 0.5, "reinit_iters": 2, "leaves": r16["leaves"], "active_voxels": r16["active"],
                   "l2": "flushed between steps (256 MiB write outside the step events)",
                   "step": "advect + 2x Godunov reinit + trim + re-track, one CUDA graph"},
        "fp32": {"value": r32["value"], "ms_per_step": r32["ms_per_step"], "kernels_ms": r32["kernels"],
                 "launch_shape": r32["launch"]},
        "launch_shape": r16["launch"],
        "fp16_over_fp32": r16["value"] / r32["value"],
        "roofline": roofline_of(r16, 2, peak, peak_kind, "deformation512"),
        "issue_roofline": None,
        "kernels_ms_per_launch": r16["kernels"],
        "e2e": e2e,
        "clocks": clk.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }
    ck = line["clocks"]
    line["issue_roofline"] = issue_roofline(r16, "deformation512", ck.get("sm_mhz"))
    if batched is not None:
        batched["f16"]["issue_roofline"] = issue_roofline(batched["f16"]["_r"], "batched256", ck.get("sm_mhz"))
        for k in ("f16", "f32"):
            batched[k].pop("_r", None)
        line["batched256"] = batched
    if accuracy is not None:
        line["full_period"] = accuracy
    if adjoint is not None:
        line["adjoint"] = adjoint
    if mesh is not None:
        line["volume_to_mesh"] = mesh
    return line


def bench_ref_sphere(args, ctx, peak, peak_kind):
    import ctypes as C

    import numpy as np
    import torch

    from sharc.volrus_b200 import DeviceGrid, VelocityField, make_level_set_sphere, make_uniform_velocity
    from sharc.volrus_b200._lib import ptr
    from sharc.volrus_b200.tools import advect_level_set, rebuild_narrow_band

    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    g0 = make_level_set_sphere(**REF_SPHERE, ctx=ctx, device=True)
    n_active, n_leaves = g0.active_voxel_count(), g0.leaf_count()
    vel = make_uniform_velocity(1.0, REF_VEL)
    dvel = VelocityField(*[DeviceGrid.upload(c, ctx) for c in (vel.vx, vel.vy, vel.vz)])

    def step():
        out = advect_level_set(g0, dvel, 1.0, ctx=ctx)
        rebuild_narrow_band(out, 3.0, ctx=ctx)
        return out

    for _ in range(args.warmup):
        step().close()
    ctx.synchronize()
    ctx.profile(True)
    times = []
    with ClockSampler(args.device) as clk, clk.mark():
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = step()
            with torch.cuda.stream(stream):
                e1.record(stream)
            ctx.synchronize()
            times.append(e0.elapsed_time(e1))
            out.close()
    kernels = {k: ctx.kernel_time(k) for k in ("k_advect_ref", "k_crossings", "k_rebuild_window")}
    ctx.profile(False)
    ms = sum(times) / len(times)
    per_leaf = {"k_advect_ref": 1024 * 4 + 144, "k_crossings": 512 * 4 + 64 + 16 + 64,
                "k_rebuild_window": 1024 * 4 + 64 * 3}
    dom = max(kernels, key=lambda k: kernels[k][0])
    dom_ms = kernels[dom][0] / max(kernels[dom][1], 1)
    achieved = per_leaf[dom] * n_leaves / (dom_ms * 1e-3) / 1e9
    host = g0.download()
    o, m, v = host.to_arrays()
    cap = len(o) + 1024
    oo, om, ov = np.zeros((cap, 3), np.int32), np.zeros((cap, 8), np.uint64), np.zeros((cap, 512), np.float32)
    nout = C.c_size_t()
    velv = np.array(REF_VEL, np.float32)
    t = host.c_transform()

    def e2e_call():
        ctx.check(ctx.lib.vlr_advect_rebuild_host(ctx.handle, C.byref(t), C.c_float(host.background),
                                                  ptr(o, C.c_int32), ptr(m, C.c_uint64), ptr(v, C.c_float), len(o),
                                                  ptr(velv, C.c_float), 1.0, C.c_float(3.0), ptr(oo, C.c_int32),
                                                  ptr(om, C.c_uint64), ptr(ov, C.c_float), cap, C.byref(nout)),
                  "vlr_advect_rebuild_host")

    for _ in range(max(1, args.warmup)):
        e2e_call()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_call()
    e2e_s = (time.perf_counter() - t0) / args.steps
    return {
        "metric": METRIC, "value": n_active / (ms * 1e-3), "unit": "voxels/s", "ms_per_step": ms, "dtype": "f32",
        "config": {"workload": "reference-sphere128", "leaves": n_leaves, "active_voxels": n_active,
                   "velocity": list(REF_VEL), "dt": 1.0, "half_width": 3.0,
                   "step": "advect_level_set + rebuild_narrow_band (reference semantics, bit-exact)",
                   "l2": "flushed between steps (256 MiB write outside the step events)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_leaf": per_leaf[dom], "launch_ms": dom_ms},
        "kernels_ms_per_launch": {k: (v[0] / max(v[1], 1)) for k, v in kernels.items()},
        "e2e": {"value": n_active / e2e_s, "unit": "voxels/s", "h2d_bytes_per_step": int(o.nbytes + m.nbytes + v.nbytes),
                "d2h_bytes_per_step": int(nout.value * (12 + 64 + 2048))},
        "clocks": clk.summary(),
        "gpu_launches": int(sum(v[1] for v in kernels.values())),
    }


def vortex_velocity_world(p):
    """Deformation field at world point p, t = 0 (for the reference arm's uniform grids)."""
    x, y, z = p
    s = math.sin
    pi = math.pi
    return (2 * s(pi * x) ** 2 * s(2 * pi * y) * s(2 * pi * z), -s(2 * pi * x) * s(pi * y) ** 2 * s(2 * pi * z),
            -s(2 * pi * x) * s(2 * pi * y) * s(pi * z) ** 2)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["deformation512", "batched256", "large8192", "adjoint256",
                                           "reference-sphere128", "mesh96", "tools160"],
                    default="large8192")
    ap.add_argument("--grids", type=int, default=BATCH["grids"], help="grids of the batched workload")
    ap.add_argument("--large-spheres", type=int, default=LARGE["spheres"], help="spheres of the large single grid")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-grid batched measurement")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the full-period accuracy run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint measurement")
    ap.add_argument("--no-mesh", action="store_true", help="skip the volume_to_mesh measurement")
    ap.add_argument("--no-ref-step", action="store_true", help="skip the GPU run of the crate's own step (large8192)")
    ap.add_argument("--no-data-path", action="store_true", help="skip the data-path diagnostic (large8192)")
    ap.add_argument("--no-deformation", action="store_true", help="skip the deformation512 section (large8192)")
    ap.add_argument("--launch-shape", default="",
                    help="threads,CTAs[,staging] of advect then reinit, e.g. 128,1184,0,128,888,0 (default: "
                         "autotuned; 128 threads and staging 0 are the only kernels built)")
    args = ap.parse_args()
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    args.device = local
    args.rank, args.world = rank, world

    if args.workload == "deformation512":
        sphere = dict(radius=DEFORM["radius"], center=DEFORM["center"], voxel_size=DEFORM["voxel_size"],
                      half_width=DEFORM["half_width"])
        vel_world = vortex_velocity_world(DEFORM["center"])
        ref_dt = 0.5 * DEFORM["voxel_size"] / 2.0
    else:
        sphere, vel_world, ref_dt = REF_SPHERE, REF_VEL, 1.0

    if args.impl == "reference" and args.workload == "mesh96":
        if rank != 0:
            return
        # the reference's volume_to_mesh restated on the host (its data structure, one thread)
        from oracle import pyoracle
        og = pyoracle.OGrid.sphere(MESH["radius"], MESH["center"], MESH["voxel_size"], MESH["half_width"])
        tiles = set()
        for x, y, z in (og.arrays()[0] // 8).tolist():
            for d in ((0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
                tiles.add((x + d[0], y + d[1], z + d[2]))
        cells = 512 * len(tiles)
        for _ in range(min(args.warmup, 1)):
            og.volume_to_mesh(0.0)
        vals = []
        for _ in range(min(args.steps, 5)):
            t0 = time.perf_counter()
            og.volume_to_mesh(0.0)
            vals.append(cells / (time.perf_counter() - t0))
        value = statistics.median(vals)
        print(json.dumps({
            "impl": "reference", "metric": "cells/s of volume_to_mesh", "value": value, "unit": "cells/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": len(vals), "warmup": args.warmup,
            "dtype": "f32", "data": "synthetic", "config": {"workload": args.workload},
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": 1, "kind": "port",
                             "sample": "oracle restatement of volume_to_mesh on the full sphere, one call per step"},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return
    if args.impl == "reference" and args.workload == "large8192":
        if rank != 0:
            return
        ref = RefLargeSample(args)
        for _ in range(args.warmup):
            ref.step()
        samples = [ref.step() for _ in range(args.steps)]
        value = statistics.median(x["value"] for x in samples)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": large_config(args),
            "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": 1, "kind": "port", "sample": ref.describe()},
            "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "box": {k: statistics.median(x[k] for x in samples)
                    for k in ("box_value", "advect_only_value", "t_advect_s", "t_cross_s", "t_pair_ns",
                              "box_crossings", "grid_crossings_est")},
        }))
        return
    if args.impl == "reference":
        if rank != 0:
            return
        vals, desc = [], ""
        for _ in range(args.warmup):
            cpu_reference_algorithm(sphere, vel_world, ref_dt, 300)
        for _ in range(args.steps):
            v, desc = cpu_reference_algorithm(sphere, vel_world, ref_dt)
            vals.append(v)
        value = statistics.median(vals)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload},
            "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": 1, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from sharc.volrus_b200 import Context
    ctx = Context.default(local)
    peak, peak_kind = measured_peaks()
    if args.workload == "deformation512":
        res = bench_deformation(args, ctx, peak, peak_kind)
    elif args.workload == "batched256":
        res = bench_batched_line(args, ctx, peak, peak_kind)
    elif args.workload == "adjoint256":
        res = bench_adjoint_line(args, ctx)
    elif args.workload == "large8192":
        res = bench_large_line(args, ctx, peak, peak_kind)
    elif args.workload == "mesh96":
        res = bench_mesh_line(args, ctx, peak, peak_kind)
    elif args.workload == "tools160":
        res = bench_tools_line(args, ctx, peak, peak_kind)
    else:
        res = bench_ref_sphere(args, ctx, peak, peak_kind)
    value = res["value"]
    ms = res["ms_per_step"]
    # batched: ranks hold disjoint grids and the totals are already whole-job;
    # deformation: one replica per rank (a single grid does not shard)
    scaling = "strong" if args.workload == "batched256" else "weak"
    if world > 1:
        import torch.distributed as dist
        if args.workload != "batched256":
            active = res.get("active_voxels", res["config"].get("active_voxels"))
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            value = world * active / (ms * 1e-3)
            if res.get("e2e"):
                e = torch.tensor([res["e2e"]["seconds_per_step"]], device="cuda")
                dist.all_reduce(e, op=dist.ReduceOp.MAX)
                res["e2e"]["value"] = world * active / float(e.item())
        dist.barrier()
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            if args.workload == "deformation512":
                v, cores, desc = cpu_method_oracle()
                cpu = {"value": v, "unit": "voxels/s", "cores": cores, "kind": "port", "sample": desc}
            elif args.workload == "large8192":
                v, cores, desc = cpu_method_oracle_large(args)
                cpu = {"value": v, "unit": "voxels/s", "cores": cores, "kind": "port", "sample": desc}
            elif args.workload == "reference-sphere128":
                v, desc = cpu_reference_algorithm(sphere, vel_world, ref_dt)
                cpu = {"value": v, "unit": "voxels/s", "cores": 1, "kind": "port", "sample": desc}
        line = {"metric": res["metric"], "value": value, "unit": res["unit"], "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": scaling,
                "vs_baseline": None, "dtype": res["dtype"], "data": "synthetic", "config": res["config"],
                "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res["e2e"],
                "gpu_launches": res["gpu_launches"], "clocks": res["clocks"],
                "kernels_ms_per_launch": res["kernels_ms_per_launch"]}
        for k in ("active_voxels", "leaves", "create_s", "issue_roofline", "fp32", "fp16_over_fp32", "launch_shape",
                  "ref_step", "data_path", "batched256", "deformation512", "full_period", "adjoint", "volume_to_mesh",
                  "tools_ms_per_call", "tools_voxels_per_s", "advect_particles"):
            if k in res and res[k] is None:
                continue
            if k in res:
                line[k] = res[k]
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
