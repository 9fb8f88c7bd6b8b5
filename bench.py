#!/usr/bin/env python3
"""Benchmark of the narrow-band level-set advection step on B200.

Prints ONE JSON line on rank 0.  Metric: active voxels per second per step.

Default workload ``deformation512`` (the deformation test): unit cube at
512^3 voxels, sphere of radius 0.15 at (0.35, 0.35, 0.35), half-width 3,
vortex velocity with period T = 3 sampled analytically, RK2 midpoint
backtrace at CFL 0.5 (dt = 0.5 * vs / 2), two Godunov reinitialisation
iterations and band re-tracking per step.  ``value`` is the FP16-leaf step;
the plain FP32 step is reported beside it under ``fp32``.

Other workload: ``reference-sphere128`` (sphere r=32 in 128^3, v=(1,0.5,0.25),
dt=1, hw=3; step = advect_level_set + rebuild_narrow_band, bit-exact with the
reference's CPU code).

Timing: W warm-up steps, then K timed steps, each bracketed by CUDA events on
the library's stream; a 256 MiB write flushes the L2 between steps, outside
the events.  ``e2e`` times the host-resident form of the step through the C
ABI (upload from pinned host memory, one step, download) with a wall clock.
``--impl reference`` times the reference algorithm on the host CPU (the C++
restatement of the crate's advect_level_set + rebuild_narrow_band with its
data structure, one thread as the crate runs it) on the same sphere.
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


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"vlr_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.out.close()
        except Exception:
            pass

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


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


# ---------------------------------------------------------------- GPU legs

def method_bytes_per_leaf(value_bytes: int):
    """Algorithmic bytes per leaf and launch.
    advect: read values 512*s, mask 64, origin 16, neighbour row 108; write values 512*s, dilated mask 64.
    reinit (2 fused iterations + trim): read values 512*s, dilated mask 64, origin 16, neighbour row 108;
            write values 512*s, mask 64, spill 4, flag 4."""
    s = value_bytes
    return {"k_m_advect": 1024 * s + 64 + 16 + 108 + 64, "k_m_reinit": 1024 * s + 64 + 16 + 108 + 64 + 8}


def run_method(args, ctx, precision, flush, stream, clock=None):
    import numpy as np
    import torch

    from sharc.volrus_b200.method import LevelSet

    vs = DEFORM["voxel_size"]
    vel = {"kind": "vortex", "vs": vs, "period": DEFORM["period"]}
    dt = 0.5 * vs / 2.0
    ls = LevelSet.sphere(DEFORM["radius"], DEFORM["center"], vs, vel, dt, half_width=DEFORM["half_width"],
                         precision=precision, integrator=2, reinit_iters=2, ctx=ctx)
    ls.step(args.warmup)
    n0, a0, _ = ls.info()
    times = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = clock or _Null()
    with sampler:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                ev[k][0].record(stream)
            ls.enqueue(1)
            with torch.cuda.stream(stream):
                ev[k][1].record(stream)
        ctx.check_device()
    times = [a.elapsed_time(b) for a, b in ev]
    n1, a1, _ = ls.info()
    ms = sum(times) / len(times)
    active = 0.5 * (a0 + a1)
    leaves = 0.5 * (n0 + n1)
    # per-kernel durations: the same steps enqueued without the graph, with events
    ctx.profile(True)
    ls.step(max(3, min(args.steps, 10)))
    kern = {k: ctx.kernel_time(k) for k in ("k_m_advect", "k_m_reinit", "k_t_propose")}
    ctx.profile(False)
    n2, a2, _ = ls.info()
    res = {"ms_per_step": ms, "value": active / (ms * 1e-3), "leaves": leaves, "active": active,
           "kernels": {k: v[0] / max(v[1], 1) for k, v in kern.items()}, "ls": ls}
    return res


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def summary(self):
        return None


def e2e_method(args, ctx, ls, precision):
    """Host-resident step through the C ABI: upload from pinned host, step, download."""
    import numpy as np
    import torch
    o, m, v = ls.arrays()
    n = len(o)
    cap = n + 4096
    pin_o = torch.empty((cap, 3), dtype=torch.int32).pin_memory().numpy()
    pin_m = torch.empty((cap, 8), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    pin_v = torch.empty((cap, 512), dtype=torch.float32).pin_memory().numpy()
    pin_o[:n], pin_m[:n], pin_v[:n] = o, m, v
    out_o = torch.empty((cap, 3), dtype=torch.int32).pin_memory().numpy()
    out_m = torch.empty((cap, 8), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    out_v = torch.empty((cap, 512), dtype=torch.float32).pin_memory().numpy()
    import ctypes as C
    from sharc.volrus_b200._lib import ptr
    h2d = d2h = 0
    cur = n

    def call():
        nonlocal cur, h2d, d2h
        ctx.check(ctx.lib.vlr_ls_upload(ctx.handle, ls.handle, ptr(pin_o, C.c_int32), ptr(pin_m, C.c_uint64),
                                        ptr(pin_v, C.c_float), cur), "upload")
        h2d = cur * (12 + 64 + 2048)
        ctx.check(ctx.lib.vlr_ls_step(ctx.handle, ls.handle, 1), "step")
        nn = C.c_size_t()
        ctx.check(ctx.lib.vlr_ls_info(ctx.handle, ls.handle, C.byref(nn), None, None), "info")
        ctx.check(ctx.lib.vlr_ls_download(ctx.handle, ls.handle, ptr(out_o, C.c_int32), ptr(out_m, C.c_uint64),
                                          ptr(out_v, C.c_float), cap), "download")
        d2h = nn.value * (12 + 64 + 2048)
        return nn.value

    for _ in range(max(1, args.warmup)):
        call()
    _, a, _ = ls.info()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call()
    e2e_s = (time.perf_counter() - t0) / args.steps
    return {"value": a / e2e_s, "unit": "voxels/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "path": "vlr_ls_upload + vlr_ls_step + vlr_ls_download, pinned host buffers"}


def bench_deformation(args, ctx, peak, peak_kind):
    import torch
    from sharc.volrus_b200.method import F16, F32

    dev = torch.device("cuda", args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    clk = ClockSampler(args.device)
    r16 = run_method(args, ctx, F16, flush, stream, clk)
    r32 = run_method(args, ctx, F32, flush, stream)
    per16 = method_bytes_per_leaf(2)
    dom = max(("k_m_advect", "k_m_reinit"), key=lambda k: r16["kernels"][k])
    dom_ms = r16["kernels"][dom]
    achieved = per16[dom] * r16["leaves"] / (dom_ms * 1e-3) / 1e9
    e2e = e2e_method(args, ctx, r16["ls"], F16)
    launches_per_step = 2 + 17  # stencils + re-track/index kernels (one graph)
    return {
        "metric": METRIC, "value": r16["value"], "unit": "voxels/s", "ms_per_step": r16["ms_per_step"],
        "dtype": "f16 storage, f32 arithmetic",
        "config": {"workload": "deformation512", "domain": "unit cube at 512^3", "sphere": "r=0.15 at (0.35,0.35,0.35)",
                   "half_width": 3, "velocity": "vortex T=3, analytic", "integrator": "RK2 midpoint",
                   "cfl": 0.5, "reinit_iters": 2, "leaves": r16["leaves"], "active_voxels": r16["active"],
                   "l2": "flushed between steps (256 MiB write outside the step events)",
                   "step": "advect + 2x Godunov reinit + trim + re-track, one CUDA graph"},
        "fp32": {"value": r32["value"], "ms_per_step": r32["ms_per_step"], "kernels_ms": r32["kernels"]},
        "fp16_over_fp32": r16["value"] / r32["value"],
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_leaf": per16[dom], "launch_ms": dom_ms},
        "kernels_ms_per_launch": r16["kernels"],
        "e2e": e2e,
        "clocks": clk.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }


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
    clk = ClockSampler(args.device)
    with clk:
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
    ap.add_argument("--workload", choices=["deformation512", "reference-sphere128"], default="deformation512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    args.device = local

    if args.workload == "deformation512":
        sphere = dict(radius=DEFORM["radius"], center=DEFORM["center"], voxel_size=DEFORM["voxel_size"],
                      half_width=DEFORM["half_width"])
        vel_world = vortex_velocity_world(DEFORM["center"])
        ref_dt = 0.5 * DEFORM["voxel_size"] / 2.0
    else:
        sphere, vel_world, ref_dt = REF_SPHERE, REF_VEL, 1.0

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
    res = bench_deformation(args, ctx, peak, peak_kind) if args.workload == "deformation512" else \
        bench_ref_sphere(args, ctx, peak, peak_kind)
    value = res["value"]
    ms = res["ms_per_step"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        value = world * res["config"]["active_voxels"] / (ms * 1e-3)
        dist.barrier()
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            if args.workload == "deformation512":
                v, cores, desc = cpu_method_oracle()
                cpu = {"value": v, "unit": "voxels/s", "cores": cores, "kind": "port", "sample": desc}
            else:
                v, desc = cpu_reference_algorithm(sphere, vel_world, ref_dt)
                cpu = {"value": v, "unit": "voxels/s", "cores": 1, "kind": "port", "sample": desc}
        line = {"metric": res["metric"], "value": value, "unit": res["unit"], "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": res["dtype"], "data": "synthetic", "config": res["config"],
                "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res["e2e"],
                "gpu_launches": res["gpu_launches"], "clocks": res["clocks"],
                "kernels_ms_per_launch": res["kernels_ms_per_launch"]}
        for k in ("fp32", "fp16_over_fp32"):
            if k in res:
                line[k] = res[k]
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
