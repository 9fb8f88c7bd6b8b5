"""FP64 method oracle checks that need no GPU.

The narrow-band METHOD (RK backtrace, Godunov reinitialisation, optionally
with the subcell fix, re-tracking) has no counterpart in the reference crate; these
tests check properties of its FP64 definition (oracle/method_oracle.hpp).
"""


def test_subcell_fix_keeps_volume_under_translation(oracle):
    """Method check on the FP64 oracle: 200 steps of a sphere translated at 0.5
    voxel per step lose far less volume with the subcell-fixed reinitialisation
    than with plain Godunov."""
    vel = {"kind": "constant", "c": (0.5, 0.0, 0.0)}
    out = {}
    for mode in (1, 0):
        og = oracle.MOGrid.sphere(0.15, (0.35, 0.35, 0.35), 1 / 128, 3.0)
        v0 = og.volume()
        for s in range(200):
            assert og.step(vel, 1, 2, float(s), 1.0, 8, mode)
        out[mode] = og.volume() / v0
    assert out[1] > 0.85 and out[0] < 0.8 and out[1] - out[0] > 0.1, out
