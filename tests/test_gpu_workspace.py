"""slak_subdivide's cached per-device workspace: results stay bit-exact with
the oracle when the workspace is reused, grown, held by another thread,
released, or switched off (SLAK_WORKSPACE_CACHE=0)."""
import ctypes
import threading

import numpy as np
import pytest

import oracle
from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _same(mesh, levels, scheme):
    ref = oracle.subdivide(mesh, levels, scheme)
    rm = api.DeviceMesh()
    cls = api.CatmullClark if scheme == SLAK else api.LAKCatmullClark
    cls.subdivideIteratively(api.DeviceMesh.from_host(mesh), rm, levels)      # slak_subdivide
    got = rm.to_host()
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(np.asarray(got.verts, np.float32).view(np.uint32), ref.verts.view(np.uint32))


def test_reuse_grow_and_release():
    small = meshgen.torus(8, 6)
    big = meshgen.mixed_torus(96, 96, 0.05, 0.03, 0.005, seed=5)
    for mesh, levels in ((small, 2), (big, 3), (small, 3), (big, 2), (small, 1)):
        for scheme in (SLAK, LAK):
            m = mesh if scheme == SLAK or mesh.ptr is not None else mesh.with_quad_ptr()
            _same(m, levels, scheme)
    assert _abi.lib().slak_workspace_release() == _abi.SLAK_OK
    assert _abi.lib().slak_workspace_release() == _abi.SLAK_OK      # nothing cached: still fine
    _same(big, 2, SLAK)                                               # re-created on demand


def test_cache_off(monkeypatch):
    monkeypatch.setenv("SLAK_WORKSPACE_CACHE", "0")
    _same(meshgen.icosphere(4, 0.02, seed=3), 3, SLAK)
    _same(meshgen.icosphere(4, 0.02, seed=3), 3, LAK)


def test_concurrent_calls_from_threads():
    import torch
    meshes = [meshgen.mixed_torus(48 + 8 * k, 40, 0.05, 0.03, 0.005, seed=k) for k in range(4)]
    refs = [oracle.subdivide(m, 3, SLAK) for m in meshes]
    dms = [api.DeviceMesh.from_host(m) for m in meshes]
    out = [None] * len(meshes)
    errs = []

    def work(k):
        try:
            torch.cuda.set_device(0)
            s = torch.cuda.Stream()
            for _ in range(3):
                cout = _abi.SlakMesh()
                rc = _abi.lib().slak_subdivide(ctypes.byref(dms[k].as_c()), ctypes.byref(cout), 3, SLAK,
                                               int(s.cuda_stream))
                _abi.check(rc, "slak_subdivide")
                host = api._wrap_c(cout, None).to_host()
                _abi.lib().slak_mesh_free(ctypes.byref(cout))
                out[k] = host
        except Exception as e:       # reported on the main thread
            errs.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(meshes))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for h, r in zip(out, refs):
        assert np.array_equal(h.ids, r.ids)
        assert np.array_equal(np.asarray(h.verts, np.float32).view(np.uint32), r.verts.view(np.uint32))
