"""A full period of the deformation test at 512^3 against the FP64 method oracle.

The deformation configuration (sphere r = 0.15 at (0.35, 0.35, 0.35) in the
unit cube at 512^3, half-width 3, the vortex with T = 3, RK2 midpoint, CFL 0.5:
dt = vs / 4, 6,144 steps) runs for one full period on the device in FP32 and
in FP16 leaves.  The FP64 method oracle's final state of the same run is the
committed fixture tests/golden/full_period_fp64_512.npz, made by
tests/golden/make_full_period_fp64.py (15-25 minutes on 6-8 host threads).

Reported per precision: the largest and RMS difference of phi on the
interface (voxels active in both runs with |phi_FP64| <= 1 voxel), the
largest difference on the whole common band, the voxels active in one run
only, and the relative change of the enclosed volume over the period beside
the FP64 run's.  FP32 leaves meet the 0.05-voxel interface bar with orders of
magnitude to spare; FP16 leaves miss it (measured 0.059 voxel), recorded as
an expected failure with its number.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

FIXTURE = Path(__file__).resolve().parent / "golden" / "full_period_fp64_512.npz"

VS = 1.0 / 512.0
R, C, HW, T = 0.15, (0.35, 0.35, 0.35), 3.0, 3.0
DT = 0.5 * VS / 2.0  # CFL 0.5 at the vortex's peak speed of 2
STEPS = int(round(T / DT))
VEL = {"kind": "vortex", "vs": VS, "period": T}


def _bits(m):
    return np.unpackbits(np.ascontiguousarray(m).view(np.uint8).reshape(-1, 64), axis=1,
                         bitorder="little").astype(bool)


def load_fixture():
    """(origins, masks, phi (n, 512) f64 with zeros off the mask), volumes."""
    z = np.load(FIXTURE)
    o, m = z["origins"], z["masks"]
    p = np.zeros((len(o), 512), np.float64)
    p[_bits(m)] = z["active_phi"].astype(np.float64)
    return (o, m, p), float(z["volume_start"]), float(z["volume_end"])


def test_fixture_consistent():
    z = np.load(FIXTURE)
    o, m, a = z["origins"], z["masks"], z["active_phi"]
    assert int(z["steps"]) == STEPS and float(z["dt"]) == DT
    assert len(o) > 1000 and int(_bits(m).sum()) == len(a)
    assert np.all(o % 8 == 0)
    key = (o[:, 0].astype(np.int64) << 42) | (o[:, 1].astype(np.int64) << 21) | o[:, 2].astype(np.int64)
    assert np.all(np.diff(key) > 0), "leaves sorted (x, y, z)"
    assert np.abs(a).max() < HW
    # the method loses the thin sheet of the stretched shape (trilinear
    # semi-Lagrangian advection cannot carry it below a voxel): the FP64 run
    # ends with 14.5 % of its start volume
    assert abs(float(z["volume_end"]) / float(z["volume_start"]) - 0.1446) < 2e-3


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


_RUNS = {}


def device_full_period(ctx, precision):
    """Final state and volumes of one full period on the device (cached per precision)."""
    if precision in _RUNS:
        return _RUNS[precision]
    from sharc.volrus_b200.method import LevelSet
    ls = LevelSet.sphere(R, C, VS, VEL, DT, half_width=HW, precision=precision, integrator=2, reinit_iters=2,
                         capacity=200_000, ctx=ctx)
    v0 = ls.volume()
    for _ in range(16):
        ls.step(STEPS // 16)
    ls.step(STEPS - 16 * (STEPS // 16))
    v1 = ls.volume()
    out = ls.arrays()
    ls.close()
    _RUNS[precision] = (out, v0, v1)
    return _RUNS[precision]


def _stats(ctx, precision):
    ref, fv0, fv1 = load_fixture()
    dev, v0, v1 = device_full_period(ctx, precision)
    s = compare(dev, ref)
    s["volume_change_rel"] = (v1 - v0) / v0
    s["volume_change_rel_fp64"] = (fv1 - fv0) / fv0
    s["volume_end_vs_fp64_rel"] = (v1 - fv1) / fv1
    out = os.environ.get("VLR_FULL_PERIOD_OUT")
    if out:
        with open(f"{out}.{'f32' if precision == 0 else 'f16'}.json", "w") as f:
            json.dump(s, f, indent=1)
    print(json.dumps(s))
    return s


@pytest.mark.gpu
def test_full_period_fp32_against_fp64(ctx):
    s = _stats(ctx, 0)
    assert s["interface_voxels"] > 1000
    assert s["max_interface_err_vox"] <= 1e-3, s
    assert s["voxels_active_in_one_run_only"] == 0, s
    # the enclosed volume follows the FP64 run's
    assert abs(s["volume_end_vs_fp64_rel"]) < 1e-4, s


@pytest.mark.gpu
def test_full_period_fp16_bounds(ctx):
    """FP16 leaves: the state is rounded to FP16 once per step (half an ulp,
    2^-12 voxel near the interface) and the rounding errors walk over 6,144
    steps; the bounds are the measured ones (0.059 max, 0.017 RMS) with margin."""
    s = _stats(ctx, 1)
    assert s["interface_voxels"] > 1000
    assert s["max_interface_err_vox"] <= 0.1, s
    assert s["rms_interface_err_vox"] <= 0.03, s
    assert abs(s["volume_end_vs_fp64_rel"]) < 5e-3, s


@pytest.mark.gpu
@pytest.mark.xfail(reason="FP16 leaves miss the 0.05-voxel interface bar after a full period: measured 0.059 voxel "
                          "max (0.017 RMS) against FP64", strict=False)
def test_full_period_fp16_meets_0_05_voxel(ctx):
    s = _stats(ctx, 1)
    assert s["max_interface_err_vox"] <= 0.05, s
