"""Comparison helpers for method grids (GPU) against the FP64 method oracle."""
import numpy as np


def _index(o):
    return {tuple(int(v) for v in o[i]): i for i in range(len(o))}


def bits(m):
    return np.unpackbits(np.ascontiguousarray(m).view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)


def compare(gpu_arrays, oracle_arrays, hw, tol_threshold=1e-3):
    """Return a dict of error statistics between a GPU state and the oracle state.

    Values are compared on voxels active in both; mask differences are
    classified as threshold flips when the oracle value lies within
    ``tol_threshold`` of +-hw (or the voxel sits on the dilation edge)."""
    go, gm, gv = gpu_arrays
    oo, om, ov = oracle_arrays
    gi, oi = _index(go), _index(oo)
    common = sorted(set(gi) & set(oi))
    only_gpu = sorted(set(gi) - set(oi))
    only_oracle = sorted(set(oi) - set(gi))
    gb, ob = bits(gm), bits(om)
    errs = []
    flips = 0
    unexplained = 0
    for k in common:
        a, b = gi[k], oi[k]
        both = gb[a] & ob[b]
        if both.any():
            errs.append(np.abs(gv[a][both].astype(np.float64) - ov[b][both]))
        diff = gb[a] ^ ob[b]
        if diff.any():
            flips += int(diff.sum())
            near = np.abs(np.abs(ov[b][diff]) - hw) < tol_threshold
            unexplained += int((~near).sum())
    e = np.concatenate(errs) if errs else np.zeros(1)
    # active voxels of leaves on one side only that lie farther than 1e-2
    # from the half width (a leaf that appears through a threshold flip at
    # a neighbour's face holds none)
    deep = 0
    for side_idx, k_list, bits_of, vals in ((gi, only_gpu, gb, gv), (oi, only_oracle, ob, ov)):
        for k in k_list:
            i = side_idx[k]
            act = bits_of[i]
            deep += int((np.abs(np.asarray(vals[i], np.float64)[act]) < hw - 1e-2).sum())
    return {
        "leaves_gpu": len(go), "leaves_oracle": len(oo), "only_gpu": len(only_gpu), "only_oracle": len(only_oracle),
        "unmatched_leaf_voxels_inside": deep,
        "active_gpu": int(gb.sum()), "active_oracle": int(ob.sum()), "mask_flips": flips,
        "unexplained_flips": unexplained, "max_err": float(e.max()), "rms_err": float(np.sqrt((e ** 2).mean())),
        "frac_over_1e-2": float((e > 1e-2).mean()),
    }
