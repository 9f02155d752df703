"""The host mesh container (CPU): whatever integer and float types a caller
hands it, it holds the int32 / float32 x 4 arrays the C ABI reads, and refuses
what does not fit instead of letting the library reinterpret it."""
import numpy as np
import pytest

from slak_b200.mesh import POLY, QUAD, Mesh


def test_types_converted():
    ids = np.array([0, 1, 2, 3], np.int64)
    verts = np.arange(16, dtype=np.float64).reshape(4, 4)
    m = Mesh(QUAD, ids, verts, np.array([0, 4], np.int64), np.array([1, 2, 3, 4], np.uint8), 1, 4)
    assert m.ids.dtype == np.int32 and m.ptr.dtype == np.int32 and m.vals.dtype == np.int32
    assert m.verts.dtype == np.float32 and m.verts.flags.c_contiguous
    assert np.array_equal(m.ids, [0, 1, 2, 3]) and np.array_equal(m.verts, verts.astype(np.float32))


def test_strided_input_made_contiguous():
    ids = np.arange(8, dtype=np.int32)[::2]
    m = Mesh(QUAD, ids, np.zeros((4, 4), np.float32))
    assert m.ids.flags.c_contiguous and np.array_equal(m.ids, [0, 2, 4, 6])


def test_out_of_range_refused():
    with pytest.raises(ValueError):
        Mesh(POLY, np.array([0, 1, 2**31], np.int64), np.zeros((3, 4), np.float32), np.array([0, 3]))
    with pytest.raises(ValueError):
        Mesh(POLY, np.array([0, 1, 2]), np.zeros((3, 4), np.float32), np.array([0, -2**31 - 1], np.int64))


def test_verts_shape_checked():
    with pytest.raises(ValueError):
        Mesh(QUAD, np.array([0, 1, 2, 3]), np.zeros((4, 3), np.float32))
    with pytest.raises(ValueError):
        Mesh(QUAD, np.array([0, 1, 2, 3]), np.zeros(16, np.float32))


def test_device_mesh_refuses_what_the_abi_would_misread():
    """DeviceMesh.as_c hands raw pointers to the C ABI, so a tensor of another
    dtype, a strided view, a host tensor or too few elements is refused before
    any library call."""
    import torch
    from slak_b200 import api
    ok_ids = torch.zeros(4, dtype=torch.int32)
    for bad, err in ((dict(ids=torch.zeros(4, dtype=torch.int64)), TypeError),
                     (dict(ids=torch.zeros(8, dtype=torch.int32)[::2]), TypeError),
                     (dict(ids=ok_ids), TypeError),                                   # host memory
                     (dict(verts=torch.zeros(16, dtype=torch.float64)), TypeError)):
        dm = api.DeviceMesh(QUAD, 1, 4, 4, 4, True, **bad)
        with pytest.raises(err):
            dm.as_c()
    assert api.DeviceMesh().as_c().ids is None                                       # an empty output is fine


def test_batch_level_counts_must_match():
    from slak_b200 import api
    from slak_b200.mesh import SLAK
    for levels in ([1], [1, 2, 3]):
        with pytest.raises(ValueError):
            api.subdivide_batched([api.DeviceMesh(), api.DeviceMesh()], levels, SLAK)
        with pytest.raises(ValueError):
            api.Batch([api.DeviceMesh(), api.DeviceMesh()], levels, SLAK)
