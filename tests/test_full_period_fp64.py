"""A full period of the deformation test at 512^3 against the FP64 method oracle.

The deformation configuration (sphere r = 0.15 at (0.35, 0.35, 0.35) in the
unit cube at 512^3, half-width 3, the vortex with T = 3, RK2 midpoint, CFL 0.5:
dt = vs / 4, 6,144 steps) run for one full period on the device in FP32 and
in FP16 leaves, and by the FP64 oracle of the same method
(oracle/method_oracle.hpp) from the same start sphere.  Reported per
precision: the largest and RMS difference of phi on the interface (voxels
active in both runs with |phi_FP64| <= 1 voxel), the largest difference on
the whole common band, and the voxels active in one run only.  Measured on
B200 against an 18-minute FP64 run (8 host threads): FP32 5.1e-5 voxel max, 1.8e-5 RMS, same
topology; FP16 0.059 max, 0.017 RMS, 621 voxels active in one run only (at
the band's edge, |phi| near the half-width).

Opt-in: the FP64 oracle takes 10-20 minutes on 8-16 host threads, so the test
runs only with VLR_FULL_PERIOD=1.  VLR_FULL_PERIOD_CACHE=<file.npz> stores the
oracle's final state there on the first run and reads it on later ones (the
oracle's result does not depend on the device).  VLR_FULL_PERIOD_OUT=<file>
writes the statistics as JSON.
"""
import json
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow,
              pytest.mark.skipif(os.environ.get("VLR_FULL_PERIOD") != "1", reason="opt-in: VLR_FULL_PERIOD=1")]

VS = 1.0 / 512.0
R, C, HW, T = 0.15, (0.35, 0.35, 0.35), 3.0, 3.0
DT = 0.5 * VS / 2.0  # CFL 0.5 at the vortex's peak speed of 2
STEPS = int(round(T / DT))
VEL = {"kind": "vortex", "vs": VS, "period": T}


def oracle_full_period(nthreads=None):
    """Final (origins, masks, phi f64) of the FP64 oracle after one period."""
    from oracle import pyoracle
    cache = os.environ.get("VLR_FULL_PERIOD_CACHE")
    if cache and os.path.exists(cache):
        z = np.load(cache)
        return z["o"], z["m"], z["p"]
    nthreads = nthreads or os.cpu_count()
    g = pyoracle.MOGrid.sphere(R, C, VS, HW)
    for s in range(STEPS):
        assert g.step(VEL, 2, 2, s * DT, DT, nthreads=nthreads), s
    o, m, p = g.arrays()
    if cache:
        np.savez(cache, o=o, m=m, p=p)
    return o, m, p


def device_full_period(ctx, precision):
    from sharc.volrus_b200.method import LevelSet
    ls = LevelSet.sphere(R, C, VS, VEL, DT, half_width=HW, precision=precision, integrator=2, reinit_iters=2,
                         capacity=200_000, ctx=ctx)
    for _ in range(16):
        ls.step(STEPS // 16)
    ls.step(STEPS - 16 * (STEPS // 16))
    out = ls.arrays()
    ls.close()
    return out


def _bits(m):
    return np.unpackbits(np.ascontiguousarray(m).view(np.uint8).reshape(-1, 64), axis=1,
                         bitorder="little").astype(bool)


def compare(dev, ref):
    """Interface and band differences of a device state against the FP64 state."""
    (go, gm, gv), (oo, om, ov) = dev, ref
    gi = {tuple(int(v) for v in o): i for i, o in enumerate(go)}
    oi = {tuple(int(v) for v in o): i for i, o in enumerate(oo)}
    gb, ob = _bits(gm), _bits(om)
    iface, band = [], []
    only = 0
    for k in set(gi) | set(oi):
        a, b = gi.get(k), oi.get(k)
        if a is None or b is None:
            only += int(gb[a].sum()) if b is None else int(ob[b].sum())
            continue
        both = gb[a] & ob[b]
        only += int((gb[a] ^ ob[b]).sum())
        d = np.abs(gv[a].astype(np.float64) - ov[b])
        band.append(d[both])
        iface.append(d[both & (np.abs(ov[b]) <= 1.0)])
    i = np.concatenate(iface) if iface else np.zeros(1)
    bd = np.concatenate(band) if band else np.zeros(1)
    return {"interface_voxels": int(i.size), "max_interface_err_vox": float(i.max()),
            "rms_interface_err_vox": float(np.sqrt(np.mean(i ** 2))), "max_band_err_vox": float(bd.max()),
            "voxels_active_in_one_run_only": only, "leaves_device": len(go), "leaves_fp64": len(oo)}


def test_full_period_against_fp64(ctx, oracle):
    ref = oracle_full_period()
    stats = {"steps": STEPS, "dt": DT}
    for name, prec in (("f32", 0), ("f16", 1)):
        stats[name] = compare(device_full_period(ctx, prec), ref)
    out = os.environ.get("VLR_FULL_PERIOD_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(stats, f, indent=1)
    print(json.dumps(stats))
    for name in ("f32", "f16"):
        assert stats[name]["interface_voxels"] > 1000
    # FP32 leaves meet the 0.05-voxel bar with three orders of magnitude to
    # spare, and the topology is the FP64 run's
    assert stats["f32"]["max_interface_err_vox"] <= 1e-3, stats["f32"]
    assert stats["f32"]["voxels_active_in_one_run_only"] == 0, stats["f32"]
    # FP16 leaves miss it (measured 0.059 voxel max, 0.017 RMS): the state is
    # rounded to FP16 once per step (half an ulp, 2^-12 voxel near the
    # interface) and the rounding errors walk over 6,144 steps; rounding the
    # advected field once instead of twice per step changes nothing (0.063 /
    # 0.019 measured), so the bound here is the measured one with margin
    assert stats["f16"]["max_interface_err_vox"] <= 0.1, stats["f16"]
    assert stats["f16"]["rms_interface_err_vox"] <= 0.03, stats["f16"]
