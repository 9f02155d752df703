"""Batched refinement: every mesh's output equals slak_subdivide on that mesh
alone, bit for bit, across mixed mesh kinds, level counts, waves and graph
replay."""
import os

import numpy as np
import pytest

from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, QUAD, SLAK

from meshes import cube_quad_type, open_grid, tetrahedron

pytestmark = pytest.mark.gpu


def _meshes():
    out = []
    for k, item in enumerate(meshgen.batch_specs(24, seed=77, fmin=20, fmax=3000)):
        out.append((meshgen.batch_mesh(item), item.levels))
    out += [(tetrahedron(), 3), (open_grid(4, 3), 2), (cube_quad_type(), 2), (cube_quad_type(), 0),
            (meshgen.torus(8, 6), 0)]
    return out


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("mode", ["eager", "graph", "waves"])
def test_batch_matches_single(scheme, mode, monkeypatch):
    import torch
    items = _meshes()
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    if mode == "waves":
        monkeypatch.setenv("SLAK_BATCH_WAVE_BYTES", str(8 << 20))
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    s = torch.cuda.Stream()
    flags = api._abi.PLAN_GRAPH if mode == "graph" else 0
    with torch.cuda.stream(s):
        b = api.Batch(dms, [l for _, l in items], scheme, flags, stream=s)
        if mode == "waves":
            assert b.waves > 1
        for _ in range(2 if mode == "graph" else 1):
            b.execute(s)
            b.check(s)
        outs = [b.output(i) for i in range(len(items))]
        hosts = [None if o is None else o.to_host() for o in outs]
    for (m, l), h in zip(items, hosts):
        if m.type == QUAD and l <= 0:
            assert h is None
            continue
        ref = api.subdivide(m, l, scheme)
        assert (h.nfaces, h.nverts, h.nnz) == (ref.nfaces, ref.nverts, ref.nnz)
        assert np.array_equal(h.ids, ref.ids)
        assert np.array_equal(_bits(h.verts), _bits(ref.verts))
        if scheme == LAK:
            assert np.array_equal(h.ptr, ref.ptr) and np.array_equal(h.vals, ref.vals)
    assert b.launches > 0
    b.close()


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("waves", [False, True])
def test_subdivide_batched_one_call(scheme, waves, monkeypatch):
    """slak_subdivide_batched: caller-owned outputs, each equal to
    slak_subdivide on that mesh alone; meshes with nothing to refine stay zeroed."""
    import torch
    items = _meshes()
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    if waves:
        monkeypatch.setenv("SLAK_BATCH_WAVE_BYTES", str(8 << 20))
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    outs = api.subdivide_batched(dms, [l for _, l in items], scheme)
    torch.cuda.synchronize()
    for (m, l), o in zip(items, outs):
        if m.type == QUAD and l <= 0:
            assert o.nfaces == 0 and o.ids is None
            continue
        h = o.to_host()
        ref = api.subdivide(m, l, scheme)
        assert (h.nfaces, h.nverts, h.nnz) == (ref.nfaces, ref.nverts, ref.nnz)
        assert np.array_equal(h.ids, ref.ids)
        assert np.array_equal(_bits(h.verts), _bits(ref.verts))
        if scheme == LAK:
            assert np.array_equal(h.ptr, ref.ptr) and np.array_equal(h.vals, ref.vals)
    del outs                                   # the caller's arrays go back through slak_mesh_free
    torch.cuda.synchronize()
