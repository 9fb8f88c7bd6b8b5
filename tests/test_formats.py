"""Serialised grid formats: .vol (src/io/vol_format.rs) and NanoGrid
(src/nano/layout.rs, src/nano/lookup.rs).

CPU: the byte-level oracle (oracle/pyformats.py) against every assertion the
crate's own tests make on these formats (vol_format.rs:165-300,
lookup.rs:108-363).  GPU: the device readers and writers byte-for-byte against
the oracle, including shuffled, repeated and unaligned .vol records, empty
grids, negative coordinates and the error cases.
"""
import struct

import numpy as np
import pytest

from oracle import pyformats as pf
from sharc.volrus_b200.grid import AffineMap, Grid, GridClass, VoxelTransform


def sphere_grid(oracle, radius=5.0, center=(0.0, 0.0, 0.0), vs=0.5, hw=3.0):
    og = oracle.OGrid.sphere(radius, center, vs, hw)
    o, m, v = og.arrays()
    g = Grid.from_arrays(o, m, v, float(np.float32(hw * vs)), VoxelTransform.uniform(vs))
    g.grid_class = GridClass.LEVEL_SET
    return g


# ---------------------------------------------------------------- oracle KATs

def test_vol_roundtrip_sphere(oracle):  # vol_format.rs:170-193
    g = sphere_grid(oracle)
    loaded = pf.read_vol(pf.write_vol(g))
    assert loaded.grid_class == g.grid_class
    assert loaded.transform.voxel_size == g.transform.voxel_size
    assert loaded.background == g.background
    assert loaded.leaf_count() == g.leaf_count()
    assert loaded.active_voxel_count() == g.active_voxel_count()
    for c, v in list(g.iter_active())[:50]:
        assert loaded.get(c) == v


def test_vol_roundtrip_empty_grid():  # vol_format.rs:195-210
    g = Grid(42.0, 1.0)
    buf = pf.write_vol(g)
    assert len(buf) == pf.VOL_HEADER
    loaded = pf.read_vol(buf)
    assert loaded.leaf_count() == 0 and loaded.active_voxel_count() == 0 and loaded.background == 42.0


def test_vol_roundtrip_specific_voxels():  # vol_format.rs:212-231
    g = Grid(-1.0, 0.25)
    g.grid_class = GridClass.FOG_VOLUME
    g.set((0, 0, 0), 1.0)
    g.set((7, 7, 7), 2.0)
    g.set((100, 200, 50), 3.14)
    loaded = pf.read_vol(pf.write_vol(g))
    assert loaded.grid_class == GridClass.FOG_VOLUME
    assert loaded.get((0, 0, 0)) == 1.0 and loaded.get((7, 7, 7)) == 2.0
    assert abs(loaded.get((100, 200, 50)) - 3.14) < 1e-6
    assert loaded.get((99, 99, 99)) == -1.0


def test_vol_magic_and_version_bytes():  # vol_format.rs:233-241
    buf = pf.write_vol(Grid(0.0, 1.0))
    assert buf[0:4] == b"VOLR" and struct.unpack("<I", buf[4:8])[0] == 1


def test_vol_bad_magic_and_version():  # vol_format.rs:243-264
    with pytest.raises(pf.FormatError, match="bad magic"):
        pf.read_vol(b"NOPE____________________________")
    with pytest.raises(pf.FormatError, match="version"):
        pf.read_vol(b"VOLR" + struct.pack("<I", 99) + bytes(24))


def test_vol_preserves_active_mask():  # vol_format.rs:266-279
    g = Grid(0.0, 1.0)
    g.set((3, 3, 3), 10.0)
    loaded = pf.read_vol(pf.write_vol(g))
    assert loaded.is_active((3, 3, 3)) and not loaded.is_active((4, 4, 4))


def test_nano_round_trip():  # lookup.rs:108-124
    g = Grid(-1.0, 0.5)
    for c, v in (((0, 0, 0), 1.0), ((1, 2, 3), 2.0), ((10, 20, 5), 3.0)):
        g.set(c, v)
    g2 = pf.nano_to_grid(pf.nano_from_grid(g))
    assert g2.get((0, 0, 0)) == 1.0 and g2.get((1, 2, 3)) == 2.0 and g2.get((10, 20, 5)) == 3.0
    assert g2.get((99, 99, 99)) == -1.0 and g2.background == -1.0


def test_nano_header_fields():  # lookup.rs:126-143
    g = Grid(0.5, 0.25)
    g.grid_class = GridClass.LEVEL_SET
    g.set((5, 10, 15), 42.0)
    g.set((-3, -7, 2), -1.0)
    h = pf.nano_header(pf.nano_from_grid(g))
    assert h["magic"] == b"NANO" and h["version"] == 1 and h["grid_class"] == 1
    assert abs(h["voxel_size"] - 0.25) < 1e-10 and h["background"] == 0.5
    assert h["bbox_min"] == [-3, -7, 2] and h["bbox_max"] == [5, 10, 15]


def test_nano_get_and_is_active():  # lookup.rs:145-178
    g = Grid(-7.5, 1.0)
    g.set((1, 2, 3), 42.0)
    g.set((4, 5, 6), 99.0)
    g.set((3, 3, 3), 1.0)
    b = pf.nano_from_grid(g)
    assert pf.nano_get(b, (1, 2, 3)) == 42.0 and pf.nano_get(b, (4, 5, 6)) == 99.0
    assert pf.nano_get(b, (100, 100, 100)) == -7.5
    assert pf.nano_is_active(b, (3, 3, 3)) and not pf.nano_is_active(b, (0, 0, 0))
    assert not pf.nano_is_active(b, (100, 100, 100))


def test_nano_sizes_and_validation():  # lookup.rs:180-228
    g = Grid(0.0, 1.0)
    g.set((0, 0, 0), 1.0)
    g.set((8, 0, 0), 2.0)
    b = pf.nano_from_grid(g)
    assert len(b) == pf.NANO_HEADER + 2 * pf.NANO_LEAF == 320 + 2 * 2128
    with pytest.raises(pf.FormatError, match="Invalid magic"):
        pf.nano_from_bytes(b"XYZW" + bytes(pf.NANO_HEADER - 4))
    with pytest.raises(pf.FormatError):
        pf.nano_from_bytes(bytes(10))
    assert pf.nano_from_bytes(b) == b


def test_nano_leaf_order_negative_and_many():  # lookup.rs:230-345
    g = Grid(0.0, 1.0)
    for c, v in (((100, 0, 0), 1.0), ((0, 0, 0), 2.0), ((50, 50, 50), 3.0), ((-10, -10, -10), 4.0),
                 ((-5, -10, -3), 77.0), ((-100, -200, -300), 88.0)):
        g.set(c, v)
    b = pf.nano_from_grid(g)
    o = pf._nano_origins(b)
    assert all(tuple(o[i - 1]) < tuple(o[i]) for i in range(1, len(o)))
    assert pf.nano_get(b, (-5, -10, -3)) == 77.0 and pf.nano_get(b, (-100, -200, -300)) == 88.0
    g2 = pf.nano_to_grid(b)
    assert g2.get((-5, -10, -3)) == 77.0 and g2.get((-100, -200, -300)) == 88.0
    many = Grid(0.0, 1.0)
    for i in range(20):
        many.set((i * 8, 0, 0), float(i))
    bm = pf.nano_from_grid(many)
    assert pf.nano_header(bm)["leaf_count"] == 20
    assert all(pf.nano_get(bm, (i * 8, 0, 0)) == float(i) for i in range(20))


def test_nano_empty_fog_and_affine():  # lookup.rs:277-363
    e = pf.nano_from_grid(Grid(5.0, 1.0))
    h = pf.nano_header(e)
    assert h["leaf_count"] == 0 and h["background"] == 5.0 and h["magic"] == b"NANO"
    assert pf.nano_get(e, (0, 0, 0)) == 5.0 and not pf.nano_is_active(e, (0, 0, 0))
    assert pf.nano_to_grid(e).active_voxel_count() == 0
    f = Grid(0.0, 1.0)
    f.grid_class = GridClass.FOG_VOLUME
    f.set((0, 0, 0), 1.0)
    fb = pf.nano_from_grid(f)
    assert pf.nano_header(fb)["grid_class"] == 2 and pf.nano_to_grid(fb).grid_class == GridClass.FOG_VOLUME
    a = Grid(0.0, 0.25)
    a.set((1, 1, 1), 1.0)
    ha = pf.nano_header(pf.nano_from_grid(a))
    assert all(abs(ha["affine_mat"][i][i] - 0.25) < 1e-10 for i in range(3))
    assert abs(pf.nano_to_grid(pf.nano_from_grid(a)).affine.voxel_size - 0.25) < 1e-10


# ---------------------------------------------------------------- GPU

def random_grid(seed, n=60, neg=True, bg=-0.75, vs=0.5):
    rng = np.random.default_rng(seed)
    lo = -40 if neg else 0
    origins = set()
    while len(origins) < n:
        origins.add(tuple(int(v) * 8 for v in rng.integers(lo, 40, 3)))
    o = np.array(sorted(origins), np.int32)
    m = rng.integers(0, 2 ** 63, (n, 8), dtype=np.int64).astype(np.uint64)
    m[::7] = 0  # some leaves without active voxels
    v = rng.normal(size=(n, 512)).astype(np.float32)
    g = Grid.from_arrays(o, m, v, bg, VoxelTransform.uniform(vs))
    g.grid_class = GridClass.FOG_VOLUME
    return g


def _same(a: Grid, b: Grid):
    ao, am, av = a.to_arrays()
    bo, bm, bv = b.to_arrays()
    assert np.array_equal(ao, bo) and np.array_equal(am, bm)
    assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))
    assert a.background == b.background


@pytest.mark.gpu
def test_device_vol_write_read_byte_exact(ctx, oracle):
    from sharc.volrus_b200.io import read_vol, write_vol
    from sharc.volrus_b200.tools import DeviceGrid
    for g in (random_grid(1), sphere_grid(oracle, 20.0, (3.0, -2.0, 1.0), 1.0), Grid(42.0, 1.0)):
        want = pf.write_vol(g)
        d = DeviceGrid.upload(g, ctx)
        assert write_vol(d) == want
        back = read_vol(want, ctx)
        assert back.grid_class == g.grid_class
        _same(back.download(), pf.read_vol(want))
        assert write_vol(back) == want


@pytest.mark.gpu
def test_device_vol_read_shuffled_repeated_unaligned(ctx):
    """Records in any order; a repeated leaf keeps its last record; a record's
    origin is aligned down to its leaf (read_vol's set + leaf_mut)."""
    from sharc.volrus_b200.io import read_vol
    g = random_grid(2, n=40)
    rows = list(range(40))
    np.random.default_rng(3).shuffle(rows)
    buf = bytearray(pf.write_vol(g, order=rows + rows[:5]))
    struct.pack_into("<I", buf, 24, 45)
    # unaligned origin in record 3 (same leaf), different values in the repeats
    struct.pack_into("<3i", buf, pf.VOL_HEADER + 3 * pf.VOL_LEAF, *(int(x) + 5 for x in g._o[rows[3]]))
    for k in range(40, 45):
        base = pf.VOL_HEADER + k * pf.VOL_LEAF + 76
        buf[base:base + 2048] = np.full(512, float(k), "<f4").tobytes()
    want = pf.read_vol(bytes(buf))
    got = read_vol(bytes(buf), ctx).download()
    _same(got, want)


@pytest.mark.gpu
def test_device_nano_byte_exact_and_to_grid(ctx, oracle):
    from sharc.volrus_b200.io import NanoGrid
    from sharc.volrus_b200.tools import DeviceGrid
    for g in (random_grid(4), sphere_grid(oracle, 20.0, (3.0, -2.0, 1.0), 1.0), Grid(5.0, 1.0)):
        want = pf.nano_from_grid(g)
        got = NanoGrid.from_grid(DeviceGrid.upload(g, ctx)).as_bytes()
        assert got == want
        back = NanoGrid.from_bytes(want).to_grid(ctx)
        _same(back.download(), pf.nano_to_grid(want))
        # a grid read from a NanoGrid writes the same image back (inverse kept)
        again = NanoGrid.from_grid(back).as_bytes()
        assert again == pf.nano_from_grid(pf.nano_to_grid(want), affine_inv=pf.nano_header(want)["affine_inv"][:3])


@pytest.mark.gpu
def test_device_formats_reject_bad_data(ctx):
    from sharc.volrus_b200._lib import VolrusError
    from sharc.volrus_b200.io import NanoGrid, read_vol
    good = pf.write_vol(random_grid(5, n=4))
    cases = [b"NOPE" + good[4:], good[:4] + struct.pack("<I", 99) + good[8:], good[:8] + struct.pack("<I", 7) + good[12:],
             good[:-1], good[:20]]
    for bad in cases:
        with pytest.raises(VolrusError, match="VLR_ERR_FORMAT"):
            read_vol(bad, ctx)
    nb = pf.nano_from_grid(random_grid(6, n=4))
    swapped = bytearray(nb)
    a, b = pf.NANO_HEADER, pf.NANO_HEADER + pf.NANO_LEAF
    swapped[a:b], swapped[b:b + pf.NANO_LEAF] = nb[b:b + pf.NANO_LEAF], nb[a:b]
    for bad in (b"XYZW" + nb[4:], nb[:10], nb[:-1], bytes(swapped)):
        with pytest.raises(VolrusError, match="VLR_ERR_FORMAT"):
            NanoGrid.from_bytes(bad).to_grid(ctx)


@pytest.mark.gpu
def test_device_vol_round_trip_deformation_sphere(ctx, oracle, tmp_path):
    """The deformation test's sphere at 512^3 (2,392 leaves) through a file."""
    from sharc.volrus_b200.io import load_vol, save_vol
    from sharc.volrus_b200.tools import make_level_set_sphere
    d = make_level_set_sphere(0.15, (0.35, 0.35, 0.35), 1 / 512, 3.0, ctx=ctx, device=True)
    p = tmp_path / "sphere.vol"
    save_vol(d, str(p))
    assert p.stat().st_size == pf.VOL_HEADER + d.leaf_count() * pf.VOL_LEAF
    back = load_vol(str(p), ctx)
    _same(back.download(), d.download())


@pytest.mark.gpu
def test_device_nano_from_host_grid_with_rotated_affine(ctx):
    """A host grid built with ``Grid::with_affine`` over a rotated, scaled,
    translated map writes the inverse the crate's map holds (its 4x4
    cofactor inverse, src/grid.rs:205-234, 301-345) into the NanoGrid header,
    byte for byte as the oracle writer given that inverse."""
    from sharc.volrus_b200.grid import AffineMap, invert_4x4
    from sharc.volrus_b200.io import NanoGrid
    rot = [[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]]
    am = AffineMap.from_scale_rotate_translate((0.5, 0.5, 0.5), rot, (100.0, -50.0, 25.0))
    g = Grid.with_affine(0.0, am)
    for c in ((1, 2, 3), (-9, 0, 17), (40, -33, 5)):
        g.set(c, float(sum(c)))
    got = NanoGrid.from_grid(g).as_bytes()
    inv = invert_4x4(am.forward())[:3]
    assert np.array_equal(pf.nano_header(got)["affine_inv"][:3], inv)
    assert got == pf.nano_from_grid(g, affine_inv=inv)
    # a uniform map's inverse is 1 / voxel size exactly, as the crate stores it
    u = Grid.with_affine(0.0, AffineMap.from_uniform_scale(0.3))
    u.set((0, 0, 0), 1.0)
    assert pf.nano_header(NanoGrid.from_grid(u).as_bytes())["affine_inv"][0][0] == 1.0 / 0.3
