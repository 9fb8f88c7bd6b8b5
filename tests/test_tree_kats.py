"""The crate's own tree unit tests, restated over the oracle grid and the
library's host grid.

src/tree/leaf.rs:188-299, src/tree/internal.rs:364-538 and
src/tree/root.rs:173-296 pin the 5-4-3 tree's semantics at node level; the
oracle (oracle/ref_tree.hpp) restates them behind the grid facade the
advection path uses, so each assertion is checked here through that facade
(get, set, is_active, deactivate, leaf and voxel counts, leaf export,
remove_empty_leaves); the library's host ``Grid`` (sharc/volrus_b200/grid.py),
which assembles the leaf arrays the C ABI uploads, passes the same cases.
The internal-node count is read as the number of
distinct 128^3-aligned origins among the leaves.  Not restated, because the
path never creates them: tiles, and the `prune(tolerance)` that makes them
(internal.rs:470-538, root.rs:276-285); and `clear` (root.rs:262-274).  A
pruned tree still crosses the C ABI: its tiles travel as leaf records
(``Grid.add_tiles``), checked by the last test here.
"""
import numpy as np
import pytest


@pytest.fixture(params=["oracle", "library"])
def new(request):
    """Factory of empty grids (background, voxel size 1) of either implementation."""
    if request.param == "oracle":
        from oracle import pyoracle
        pyoracle.load()
        return lambda bg: pyoracle.OGrid.new(bg, 1.0)
    from sharc.volrus_b200.grid import Grid

    class HostGrid(Grid):
        def arrays(self):
            return self.to_arrays()

    return lambda bg: HostGrid(bg, 1.0)


def _active(g):
    """{(x, y, z): value} of every active voxel, from the leaf export."""
    o, m, v = g.arrays()
    out = {}
    bits = np.unpackbits(m.view(np.uint8).reshape(-1, 64), axis=1, bitorder="little").astype(bool)
    for i in range(len(o)):
        for off in np.nonzero(bits[i])[0]:
            c = (int(o[i][0]) + (off >> 6), int(o[i][1]) + ((off >> 3) & 7), int(o[i][2]) + (off & 7))
            out[c] = float(v[i][off])
    return out


def _internal_count(g):
    o, _, _ = g.arrays()
    return len({tuple(int(c) >> 7 for c in oo) for oo in o})


# ---- leaf.rs:188-299

def test_leaf_new_all_inactive(new):  # leaf.rs:192-197
    g = new(0.0)
    assert g.active_voxel_count() == 0 and g.leaf_count() == 0


def test_leaf_set_get_active(new):  # leaf.rs:199-207
    g = new(-1.0)
    g.set((3, 5, 7), 42.0)
    assert g.get((3, 5, 7)) == 42.0 and g.is_active((3, 5, 7))
    assert g.active_voxel_count() == 1


def test_leaf_set_inactive_resets(new):  # leaf.rs:209-218, deactivate alias :258-266
    g = new(-1.0)
    g.set((1, 1, 1), 5.0)
    assert g.is_active((1, 1, 1))
    g.deactivate((1, 1, 1))
    assert not g.is_active((1, 1, 1)) and g.get((1, 1, 1)) == -1.0


def test_leaf_origin_aligned(new):  # leaf.rs:220-224
    g = new(0.0)
    g.set((13, 7, 20), 1.0)
    o, _, _ = g.arrays()
    assert o.tolist() == [[8, 0, 16]]


def test_leaf_active_mask_512_bits(new):  # leaf.rs:226-238
    g = new(0.0)
    for x in range(8):
        for y in range(8):
            for z in range(8):
                g.set((x, y, z), 1.0)
    _, m, _ = g.arrays()
    assert g.active_voxel_count() == 512
    assert m.tolist() == [[0xFFFFFFFFFFFFFFFF] * 8]


def test_leaf_iter_active(new):  # leaf.rs:240-256
    g = new(0.0)
    assert _active(g) == {}
    g.set((1, 2, 3), 10.0)
    g.set((7, 7, 7), 20.0)
    assert _active(g) == {(1, 2, 3): 10.0, (7, 7, 7): 20.0}


def test_leaf_empty_after_deactivation(new):  # leaf.rs:268-287
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    assert g.active_voxel_count() == 1
    g.deactivate((0, 0, 0))
    assert g.active_voxel_count() == 0 and g.leaf_count() == 1
    g.remove_empty_leaves()
    assert g.leaf_count() == 0


def test_leaf_iter_active_with_offset_origin(new):  # leaf.rs:289-298
    g = new(0.0)
    g.set((8, 16, 24), 1.0)
    g.set((10, 18, 26), 2.0)
    assert _active(g) == {(8, 16, 24): 1.0, (10, 18, 26): 2.0}
    assert g.leaf_count() == 1


# ---- internal.rs:364-538

def test_internal_new_empty_and_unset(new):  # internal.rs:368-374, 392-397
    g = new(-1.0)
    assert g.leaf_count() == 0 and g.active_voxel_count() == 0
    assert g.get((5, 5, 5)) == -1.0 and not g.is_active((5, 5, 5))


def test_internal_origin_aligned(new):  # internal.rs:376-381
    g = new(0.0)
    g.set((13, 200, 50), 1.0)
    o, _, _ = g.arrays()
    assert [int(c) >> 7 << 7 for c in o[0]] == [0, 128, 0]


def test_internal_set_get(new):  # internal.rs:383-390
    g = new(-1.0)
    g.set((5, 5, 5), 42.0)
    assert g.get((5, 5, 5)) == 42.0 and g.is_active((5, 5, 5)) and g.leaf_count() == 1


def test_internal_different_and_same_leaves(new):  # internal.rs:399-416
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    g.set((8, 0, 0), 2.0)
    assert g.leaf_count() == 2 and g.get((0, 0, 0)) == 1.0 and g.get((8, 0, 0)) == 2.0
    h = new(0.0)
    h.set((0, 0, 0), 1.0)
    h.set((7, 7, 7), 2.0)
    assert h.leaf_count() == 1 and h.active_voxel_count() == 2


def test_internal_leaves_and_leaf_at(new):  # internal.rs:418-440
    g = new(0.0)
    for x in (0, 8, 16):
        g.set((x, 0, 0), 1.0 + x)
    assert g.leaf_count() == 3
    h = new(0.0)
    assert h.leaf_count() == 0
    h.set((5, 5, 5), 42.0)
    o, _, v = h.arrays()
    assert o.tolist() == [[0, 0, 0]] and v[0][(5 << 6) | (5 << 3) | 5] == 42.0


def test_internal_iter_active(new):  # internal.rs:442-451
    g = new(0.0)
    g.set((1, 2, 3), 10.0)
    g.set((9, 10, 11), 20.0)
    assert _active(g) == {(1, 2, 3): 10.0, (9, 10, 11): 20.0}


def test_internal_wide_coord_range(new):  # internal.rs:453-462
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    g.set((127, 127, 127), 2.0)
    assert g.leaf_count() == 2 and _internal_count(g) == 1
    assert g.get((0, 0, 0)) == 1.0 and g.get((127, 127, 127)) == 2.0


def test_internal_deactivate_voxel(new):  # internal.rs:470-478
    g = new(0.0)
    g.set((1, 1, 1), 5.0)
    g.deactivate((1, 1, 1))
    assert not g.is_active((1, 1, 1)) and g.get((1, 1, 1)) == 0.0


def test_internal_remove_empty_leaves(new):  # internal.rs:480-494
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    g.set((8, 0, 0), 2.0)
    g.deactivate((0, 0, 0))
    g.remove_empty_leaves()
    assert g.leaf_count() == 1 and g.get((0, 0, 0)) == 0.0


# ---- root.rs:173-296

def test_root_empty_returns_background(new):  # root.rs:177-182
    g = new(1.0)
    assert g.get((100, 200, 300)) == 1.0 and g.leaf_count() == 0


def test_root_set_allocates_leaf(new):  # root.rs:184-191
    g = new(0.0)
    g.set((5, 5, 5), 3.14)
    assert g.leaf_count() == 1 and g.get((5, 5, 5)) == np.float32(3.14) and g.is_active((5, 5, 5))


def test_root_tiles_and_internal_nodes(new):  # root.rs:193-230
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    g.set((8, 0, 0), 2.0)
    assert g.leaf_count() == 2 and _internal_count(g) == 1
    h = new(0.0)
    h.set((0, 0, 0), 1.0)
    h.set((7, 7, 7), 2.0)
    assert h.leaf_count() == 1 and h.active_voxel_count() == 2
    k = new(0.0)
    k.set((0, 0, 0), 1.0)
    k.set((128, 0, 0), 2.0)
    assert _internal_count(k) == 2 and k.leaf_count() == 2
    k.set((8, 0, 0), 3.0)
    assert k.leaf_count() == 3


def test_root_iter_active(new):  # root.rs:232-241
    g = new(0.0)
    g.set((1, 2, 3), 10.0)
    g.set((130, 130, 130), 20.0)
    assert _active(g) == {(1, 2, 3): 10.0, (130, 130, 130): 20.0}


def test_root_deactivate(new):  # root.rs:243-259
    g = new(0.0)
    g.set((5, 5, 5), 42.0)
    g.deactivate((5, 5, 5))
    assert not g.is_active((5, 5, 5)) and g.get((5, 5, 5)) == 0.0
    g.deactivate((999, 999, 999))  # a region that does not exist: no-op
    assert not g.is_active((999, 999, 999)) and g.leaf_count() == 1


def test_root_remove_empty_leaves(new):  # root.rs:287-295
    g = new(0.0)
    g.set((0, 0, 0), 1.0)
    g.set((8, 0, 0), 2.0)
    g.deactivate((0, 0, 0))
    g.remove_empty_leaves()
    assert g.leaf_count() == 1


# ---- tiles at the boundary: a pruned tree crosses the C ABI as leaf records

def test_pruned_tiles_cross_as_leaf_records():
    """internal.rs:497-509 prunes a leaf of constant 5.0 with an active voxel
    into an active tile; the tree then reads 5.0 at its voxels and iterates it
    as 512 active voxels (internal.rs:169-184, 319-349).  ``Grid.add_tiles``
    carries that tile, and an inactive one, as leaf records that read and
    iterate the same."""
    from sharc.volrus_b200.grid import Grid
    g = Grid(5.0, 1.0)
    g.set((20, 0, 0), 1.0)
    g.add_tiles([(0, 0, 0), (0, 8, 0)], [5.0, -2.5], [True, False])
    assert g.leaf_count() == 3
    assert g.active_voxel_count() == 1 + 512
    act = dict(g.iter_active())
    tile = {(x, y, z) for x in range(8) for y in range(8) for z in range(8)}
    assert tile <= set(act) and all(act[c] == 5.0 for c in tile)
    assert all(g.get((x, 8 + y, z)) == -2.5 and not g.is_active((x, 8 + y, z)) for x, y, z in tile)
    assert g.get((100, 100, 100)) == 5.0
    with pytest.raises(ValueError):
        g.add_tiles([(16, 0, 0)], [0.0], [True])  # holds a leaf
    with pytest.raises(ValueError):
        g.add_tiles([(4, 0, 64)], [0.0], [True])  # not leaf-aligned
