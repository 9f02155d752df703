"""slak_subdivide_level_noalloc: one subdivision level with all scratch in a
fixed device array inside the library, for callers that cannot call cudaMalloc
(a pool allocator owns their device memory, or their loop must not block on
cudaMalloc/cudaFree).  Its output must equal slak_subdivide's (target_level 1)
bit for bit, the tolerance of the other parity tests, on two calls in a row
that share the array.  This file sorts last so that a run stopping at the
first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _reference_level(mesh, scheme):
    """The existing entry point: slak_subdivide with target_level 1."""
    cm = api.DeviceMesh.from_host(mesh)
    rm = api.DeviceMesh()
    (api.LAKCatmullClark if scheme == LAK else api.CatmullClark).subdivideIteratively(cm, rm, 1)
    return rm.to_host()


def _no_alloc_level(mesh, scheme, cm):
    """Calls the allocation-free entry point; the test (the caller) owns every buffer."""
    import torch
    N, V, F = mesh.nnz, mesh.nverts, mesh.nfaces
    cap = V + F + N
    ids = torch.full((4 * N,), -1, dtype=torch.int32, device="cuda")
    verts = torch.full((4 * cap,), float("nan"), dtype=torch.float32, device="cuda")
    ptr = torch.zeros(N + 1, dtype=torch.int32, device="cuda") if scheme == LAK else None
    vals = torch.zeros(4 * N, dtype=torch.int32, device="cuda") if scheme == LAK else None
    out = _abi.SlakMesh()
    out.nverts = cap
    out.ids, out.verts = ids.data_ptr(), verts.data_ptr()
    if scheme == LAK:
        out.ptr, out.vals = ptr.data_ptr(), vals.data_ptr()
    cin = cm.as_c()
    rc = _abi.lib().slak_subdivide_level_noalloc(ctypes.byref(cin), ctypes.byref(out), scheme,
                                                 int(torch.cuda.current_stream().cuda_stream) or None)
    _abi.check(rc, "slak_subdivide_level_noalloc")
    torch.cuda.synchronize()
    nv = int(out.nverts)
    return (out, ids.cpu().numpy(), verts[:4 * nv].cpu().numpy().reshape(-1, 4),
            None if ptr is None else ptr.cpu().numpy(), None if vals is None else vals.cpu().numpy())


CASES = [("icosphere-SLAK", lambda: meshgen.workload("icosphere").mesh, SLAK),
         ("mixed-LAK", lambda: meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=3), LAK),
         ("torus-SLAK", lambda: meshgen.torus(24, 20, seed=5), SLAK),
         ("cylinder-LAK", lambda: meshgen.capped_cylinder(64, 32, 0.001, seed=15), LAK)]


@pytest.mark.parametrize("name,make,scheme", CASES, ids=[c[0] for c in CASES])
def test_no_alloc_matches_slak_subdivide_twice(name, make, scheme):
    mesh = make()
    ref = _reference_level(mesh, scheme)
    cm = api.DeviceMesh.from_host(mesh)
    for _ in range(2):          # the second call reuses the array the first one left behind
        out, ids, verts, ptr, vals = _no_alloc_level(mesh, scheme, cm)
        assert (out.nfaces, out.nnz, out.nverts) == (ref.nfaces, ref.nnz, ref.nverts)
        assert out.type == 1 and bool(out.is_reduced) == ref.is_reduced
        assert np.array_equal(ids, ref.ids)
        assert np.array_equal(verts.view(np.uint32), ref.verts.view(np.uint32))
        if scheme == LAK:
            assert np.array_equal(ptr, ref.ptr) and np.array_equal(vals, ref.vals)


def test_no_alloc_rejects_meshes_beyond_the_fixed_scratch():
    big = meshgen.torus(512, 512, seed=1)          # 1M corners: more than 32 MiB of scratch
    cm = api.DeviceMesh.from_host(big)
    with pytest.raises(_abi.SlakError) as e:
        _no_alloc_level(big, SLAK, cm)
    assert e.value.code == 6 and "scratch" in str(e.value)
