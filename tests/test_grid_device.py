"""vlr_grid_create_device: a grid from leaves already on the device is the grid
vlr_grid_create makes from the same leaves on the host, and unsorted or
misaligned device leaves are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sphere_arrays():
    from sharc.volrus_b200 import make_level_set_sphere
    g = make_level_set_sphere(20.0, (3.5, -2.25, 1.0), 1.0, 3.0)
    return g.to_arrays()


def test_device_creation_equals_host_creation(ctx):
    import torch
    from sharc.volrus_b200 import Grid
    from sharc.volrus_b200.tools import DeviceGrid
    o, m, v = _sphere_arrays()
    host = DeviceGrid.upload(Grid.from_arrays(o, m, v, 3.0), ctx)
    do = torch.from_numpy(o).cuda()
    dm = torch.from_numpy(m.view(np.int64)).cuda()
    dv = torch.from_numpy(v).cuda()
    torch.cuda.synchronize()
    dev = DeviceGrid.from_device(do.data_ptr(), dm.data_ptr(), dv.data_ptr(), len(o), 3.0, 1.0, ctx)
    a, b = host.download().to_arrays(), dev.download().to_arrays()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))
    assert dev.active_voxel_count() == host.active_voxel_count() == int(np.unpackbits(m.view(np.uint8)).sum())
    host.close()
    dev.close()


def test_device_creation_refuses_bad_leaves(ctx):
    import torch
    from sharc.volrus_b200 import VolrusError
    from sharc.volrus_b200.tools import DeviceGrid
    o, m, v = _sphere_arrays()
    swapped = o.copy()
    swapped[[0, 1]] = swapped[[1, 0]]
    shifted = o.copy()
    shifted[3, 1] += 4
    for bad in (swapped, shifted):
        do = torch.from_numpy(bad).cuda()
        dm = torch.from_numpy(m.view(np.int64)).cuda()
        dv = torch.from_numpy(v).cuda()
        torch.cuda.synchronize()
        with pytest.raises(VolrusError):
            DeviceGrid.from_device(do.data_ptr(), dm.data_ptr(), dv.data_ptr(), len(o), 3.0, 1.0, ctx)
