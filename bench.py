#!/usr/bin/env python3
"""Benchmark of the narrow-band level-set advection step on B200.

Prints ONE JSON line (rank 0).  Metric: active voxels per second per step.

Workloads (``--workload``):
  reference-sphere128   sphere r=32 centred in a 128^3 index domain, voxel 1,
                        half-width 3, constant velocity (1, 0.5, 0.25), dt=1;
                        one step = advect_level_set + rebuild_narrow_band with
                        the reference's semantics (bit-exact path).

``--impl reference`` times the reference algorithm on the host CPU instead
(the C++ restatement with the reference's data structure, one thread, as the
crate runs it) on the same workload and prints the same metric.

Timing: W warm-up steps, then K timed steps.  Each step is bracketed by CUDA
events on the library's stream; the L2 is flushed (a 256 MiB write) between
steps, outside the events.  ``value`` = active voxels processed / device
time.  ``e2e`` times the host-buffer C-ABI entry point (upload + step +
download) with a wall clock.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = open(os.devnull if False else "/tmp/vlr_clocks.csv", "w")
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
        if self.out:
            self.out.close()

    def summary(self):
        rows = []
        try:
            for line in open("/tmp/vlr_clocks.csv"):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# reference-semantics workload (sphere in 128^3)

REF_SPHERE = dict(radius=32.0, center=(64.0, 64.0, 64.0), voxel_size=1.0, half_width=3.0)
REF_VEL = (1.0, 0.5, 0.25)


def cpu_reference_ref_sphere(sample_voxels: int = 1500, reps: int = 1):
    """Reference algorithm on one host thread: advect_level_set over every active
    voxel plus rebuild_narrow_band's O(N x M) loop over `sample_voxels` voxels,
    extrapolated to all voxels.  Returns (voxels/s, description)."""
    import ctypes as C
    from oracle import pyoracle
    lib = pyoracle.load()
    best = None
    n_active = None
    for _ in range(reps):
        g = pyoracle.OGrid.sphere(REF_SPHERE["radius"], REF_SPHERE["center"], REF_SPHERE["voxel_size"],
                                  REF_SPHERE["half_width"])
        n_active = g.active_voxel_count()
        vel = pyoracle.uniform_velocity(1.0, REF_VEL)
        h = C.c_void_p(g.h)
        ta, tr, nr = C.c_double(), C.c_double(), C.c_size_t()
        lib.vo_time_ref_step(C.byref(h), vel[0].h, vel[1].h, vel[2].h, 1.0, C.c_float(3.0), sample_voxels,
                             C.byref(ta), C.byref(tr), C.byref(nr))
        g.h = h.value
        t_step = ta.value + tr.value * (n_active / max(nr.value, 1))
        best = t_step if best is None else min(best, t_step)
    return n_active / best, (f"advect_level_set on all {n_active} active voxels + rebuild_narrow_band "
                             f"distance loop on {sample_voxels} voxels, extrapolated linearly")


def run_ref_sphere(args, ctx, peak, peak_kind):
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
    n_active = g0.active_voxel_count()
    n_leaves = g0.leaf_count()
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
    with ClockSampler(args.device) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = step()
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize(dev)
            ctx.synchronize()
            times.append(e0.elapsed_time(e1))
            out.close()
    kernels = {}
    for name in ("k_advect_ref", "k_crossings", "k_rebuild_window"):
        kernels[name] = ctx.kernel_time(name)
    ctx.profile(False)
    ms = sum(times) / len(times)
    value = n_active / (ms * 1e-3)

    # roofline of the dominant kernel: algorithmic bytes per leaf (f32):
    # advect reads 512*4 + 64 + 16, writes 512*4 + 64; rebuild reads values,
    # mask and crossing mask, writes values and mask.
    per_leaf = {"k_advect_ref": 1024 * 4 + 144, "k_crossings": 512 * 4 + 64 + 16 + 64,
                "k_rebuild_window": 1024 * 4 + 64 * 3}
    dom = max(kernels, key=lambda k: kernels[k][0])
    dom_ms = kernels[dom][0] / max(kernels[dom][1], 1)
    achieved = per_leaf[dom] * n_leaves / (dom_ms * 1e-3) / 1e9

    # e2e through the host-buffer C-ABI entry point
    host = g0.download()
    o, m, v = host.to_arrays()
    cap = len(o) + 1024
    oo = np.zeros((cap, 3), np.int32)
    om = np.zeros((cap, 8), np.uint64)
    ov = np.zeros((cap, 512), np.float32)
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

    result = {
        "metric": "active voxels/s per advection step",
        "value": value,
        "unit": "voxels/s",
        "ms_per_step": ms,
        "dtype": "f32",
        "config": {"workload": "reference-sphere128", "leaves": n_leaves, "active_voxels": n_active,
                   "velocity": list(REF_VEL), "dt": 1.0, "half_width": 3.0,
                   "step": "advect_level_set + rebuild_narrow_band (reference semantics, bit-exact)",
                   "l2": "flushed between steps (256 MiB write outside the step events)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_leaf": per_leaf[dom], "launch_ms": dom_ms},
        "kernels_ms_per_launch": {k: (v[0] / max(v[1], 1)) for k, v in kernels.items()},
        "e2e": {"value": n_active / e2e_s, "unit": "voxels/s",
                "h2d_bytes_per_step": int(o.nbytes + m.nbytes + v.nbytes),
                "d2h_bytes_per_step": int(nout.value * (12 + 64 + 2048))},
        "clocks": clk.summary(),
        "gpu_launches": None,
    }
    # kernel launches of one step, counted from the profiler totals
    launches = sum(v[1] for v in kernels.values()) // max(args.steps, 1)
    result["gpu_launches"] = int(launches * args.steps)
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="reference-sphere128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    args.device = local

    if args.impl == "reference":
        if rank != 0:
            return
        vals = []
        desc = ""
        for _ in range(args.warmup):
            cpu_reference_ref_sphere()
        for _ in range(args.steps):
            v, desc = cpu_reference_ref_sphere()
            vals.append(v)
        value = statistics.median(vals)
        print(json.dumps({
            "impl": "reference", "metric": "active voxels/s per advection step", "value": value,
            "unit": "voxels/s", "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload},
            "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": 1,
                             "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    from sharc.volrus_b200 import Context
    ctx = Context.default(local)
    peak, peak_kind = measured_peaks()
    res = run_ref_sphere(args, ctx, peak, peak_kind)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([res["ms_per_step"]], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        res["ms_per_step"] = float(t.item())
        res["value"] = world * res["config"]["active_voxels"] / (res["ms_per_step"] * 1e-3)
        dist.barrier()
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            v, desc = cpu_reference_ref_sphere()
            cpu = {"value": v, "unit": "voxels/s", "cores": 1, "kind": "port", "sample": desc}
        line = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": res["dtype"],
                "data": "synthetic", "config": res["config"], "roofline": res["roofline"],
                "cpu_baseline": cpu, "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
                "clocks": res["clocks"], "kernels_ms_per_launch": res["kernels_ms_per_launch"]}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
