"""slak_subdivide_level_noalloc: one subdivision level with all scratch in a
fixed device array inside the library, for callers that cannot call cudaMalloc
(a pool allocator owns their device memory, or their loop must not block on
cudaMalloc/cudaFree).  Its output must equal slak_subdivide's (target_level 1)
and the oracle's bit for bit, the tolerance of the other parity tests, on two
calls in a row that share the array.  This file sorts last so that a run
stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import oracle
from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20          # the fixed array's size (kNoAllocScratchBytes)


def _reference_level(mesh, scheme):
    """The existing entry point: slak_subdivide with target_level 1."""
    cm = api.DeviceMesh.from_host(mesh)
    rm = api.DeviceMesh()
    (api.LAKCatmullClark if scheme == LAK else api.CatmullClark).subdivideIteratively(cm, rm, 1)
    return rm.to_host()


def _buffers(mesh, scheme, cap):
    import torch
    N = mesh.nnz
    ids = torch.full((4 * N,), -1, dtype=torch.int32, device="cuda")
    verts = torch.full((4 * cap,), float("nan"), dtype=torch.float32, device="cuda")
    ptr = torch.zeros(N + 1, dtype=torch.int32, device="cuda") if scheme == LAK else None
    vals = torch.zeros(4 * N, dtype=torch.int32, device="cuda") if scheme == LAK else None
    return ids, verts, ptr, vals


def _call(cm, scheme, out):
    import torch
    cin = cm.as_c()
    return _abi.lib().slak_subdivide_level_noalloc(ctypes.byref(cin), ctypes.byref(out), scheme,
                                                   int(torch.cuda.current_stream().cuda_stream) or None)


def _no_alloc_level(mesh, scheme, cm, cap=None):
    """Calls the allocation-free entry point; the test (the caller) owns every buffer."""
    import torch
    cap = mesh.nverts + mesh.nfaces + mesh.nnz if cap is None else cap
    ids, verts, ptr, vals = _buffers(mesh, scheme, cap)
    out = _abi.SlakMesh()
    out.nverts = cap
    out.ids, out.verts = ids.data_ptr(), verts.data_ptr()
    if scheme == LAK:
        out.ptr, out.vals = ptr.data_ptr(), vals.data_ptr()
    _abi.check(_call(cm, scheme, out), "slak_subdivide_level_noalloc")
    torch.cuda.synchronize()
    nv = int(out.nverts)
    return (out, ids.cpu().numpy(), verts[:4 * nv].cpu().numpy().reshape(-1, 4),
            None if ptr is None else ptr.cpu().numpy(), None if vals is None else vals.cpu().numpy())


def _same(out, ids, verts, ptr, vals, ref, scheme):
    assert (out.nfaces, out.nnz, out.nverts) == (ref.nfaces, ref.nnz, ref.nverts)
    assert out.type == 1 and bool(out.is_reduced) == ref.is_reduced
    assert np.array_equal(ids, ref.ids)
    assert np.array_equal(verts.view(np.uint32), ref.verts.view(np.uint32))
    if scheme == LAK:
        assert np.array_equal(ptr, ref.ptr) and np.array_equal(vals, ref.vals)


CASES = [("icosphere-SLAK", lambda: meshgen.workload("icosphere").mesh, SLAK),
         ("mixed-LAK", lambda: meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=3), LAK),
         ("torus-SLAK", lambda: meshgen.torus(24, 20, seed=5), SLAK),
         ("cylinder-LAK", lambda: meshgen.capped_cylinder(64, 32, 0.001, seed=15), LAK),
         ("open-grid-SLAK", lambda: meshgen.open_grid(37, 23, seed=4), SLAK),
         ("open-grid-LAK", lambda: meshgen.open_grid(29, 31, seed=6), LAK)]


@pytest.mark.parametrize("name,make,scheme", CASES, ids=[c[0] for c in CASES])
def test_no_alloc_matches_slak_subdivide_twice(name, make, scheme):
    mesh = make()
    ref = _reference_level(mesh, scheme)
    orc = oracle.subdivide(mesh, 1, scheme)
    cm = api.DeviceMesh.from_host(mesh)
    for _ in range(2):          # the second call reuses the array the first one left behind
        got = _no_alloc_level(mesh, scheme, cm)
        _same(*got, ref, scheme)
        _same(*got, orc, scheme)


def test_no_alloc_refuses_a_short_position_buffer_and_writes_nothing():
    import torch
    mesh = meshgen.mixed_torus(24, 20, 0.05, 0.03, 0.005, seed=8)
    need = oracle.subdivide(mesh, 1, SLAK).nverts
    cm = api.DeviceMesh.from_host(mesh)
    ids, verts, _, _ = _buffers(mesh, SLAK, need - 1)
    out = _abi.SlakMesh()
    out.nverts = need - 1
    out.ids, out.verts = ids.data_ptr(), verts.data_ptr()
    assert _call(cm, SLAK, out) == 1                      # SLAK_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert out.nverts == need - 1 and out.nfaces == 0 and out.nnz == 0
    assert bool((ids == -1).all()) and bool(torch.isnan(verts).all())
    got = _no_alloc_level(mesh, SLAK, cm, cap=need)       # exactly enough is accepted
    _same(*got, oracle.subdivide(mesh, 1, SLAK), SLAK)


def _scratch_bytes(N, V, poly):
    """carve_scratch's layout: each array rounded up to 256 bytes."""
    up = lambda b: (max(b, 1) + 255) // 256 * 256
    ints = [V, V + 1] + [N] * 7 + [V, V + 1, (max(N, V) + 2047) // 2048 + 2] + ([N] if poly else [])
    return sum(up(4 * n) for n in ints) + up(8 * N) + up(4 * (4 + 32 + 17))


def test_no_alloc_limit_is_the_scratch_formula():
    # the largest W x W quad torus whose scratch fits, and the next size up
    w = 1
    while _scratch_bytes(4 * (w + 1) ** 2, (w + 1) ** 2, False) <= SCRATCH_BYTES:
        w += 1
    assert _scratch_bytes(4 * w * w, w * w, False) <= SCRATCH_BYTES < _scratch_bytes(4 * (w + 1) ** 2, (w + 1) ** 2, False)
    assert 4 * w * w > 800_000                       # about 830k corners, as documented
    under = meshgen.torus(w, w, seed=2)
    got = _no_alloc_level(under, SLAK, api.DeviceMesh.from_host(under))
    _same(*got, _reference_level(under, SLAK), SLAK)
    over = meshgen.torus(w + 1, w + 1, seed=2)
    with pytest.raises(_abi.SlakError) as e:
        _no_alloc_level(over, SLAK, api.DeviceMesh.from_host(over))
    assert e.value.code == 6 and "scratch" in str(e.value)


def test_no_alloc_rejects_meshes_beyond_the_fixed_scratch():
    big = meshgen.torus(512, 512, seed=1)          # 1M corners: more than 32 MiB of scratch
    cm = api.DeviceMesh.from_host(big)
    with pytest.raises(_abi.SlakError) as e:
        _no_alloc_level(big, SLAK, cm)
    assert e.value.code == 6 and "scratch" in str(e.value)
