"""Generate full_period_fp64_512.npz: the FP64 method oracle's state after one
full period of the deformation test at 512^3.

Configuration: sphere r = 0.15 at (0.35, 0.35, 0.35) in the unit cube at
512^3 (voxel size 1/512), half-width 3, the vortex field with T = 3, RK2
midpoint backtrace, CFL 0.5 (dt = vs / 4, 6,144 steps), two Godunov
reinitialisation iterations and re-tracking per step, run by the FP64 method
oracle (oracle/method_oracle.hpp) from the start sphere.

Stored: leaf origins (int32 (n, 3), sorted (x, y, z)), value masks (uint64
(n, 8)), the values of the active voxels in leaf then mask-bit order as
float32 (voxel units), and the FP64 enclosed volume at the start and at the
end (index units^3, about (0, 0, 0)).  The run takes 15-25 minutes on 6-8
host threads.

Usage: python tests/golden/make_full_period_fp64.py [threads]
"""
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402

VS = 1.0 / 512.0
R, C, HW, T = 0.15, (0.35, 0.35, 0.35), 3.0, 3.0
DT = 0.5 * VS / 2.0
STEPS = int(round(T / DT))
VEL = {"kind": "vortex", "vs": VS, "period": T}
OUT = Path(__file__).resolve().parent / "full_period_fp64_512.npz"


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    g = pyoracle.MOGrid.sphere(R, C, VS, HW)
    v0 = g.volume()
    t0 = time.time()
    for s in range(STEPS):
        assert g.step(VEL, 2, 2, s * DT, DT, nthreads=threads), s
        if s % 512 == 0:
            print(f"step {s}/{STEPS} leaves {g.leaf_count()} {time.time() - t0:.0f} s", flush=True)
    v1 = g.volume()
    o, m, p = g.arrays()
    bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    np.savez_compressed(OUT, origins=o.astype(np.int32), masks=m.astype(np.uint64),
                        active_phi=p[bits].astype(np.float32), volume_start=np.float64(v0),
                        volume_end=np.float64(v1), steps=np.int64(STEPS), dt=np.float64(DT))
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes), {len(o)} leaves, volume change {(v1 - v0) / v0:.3e}")


if __name__ == "__main__":
    main()
