"""Batched refinement: every mesh's output equals slak_subdivide on that mesh
alone, bit for bit, across mixed mesh kinds, level counts, grouped launches,
chains, waves and graph replay."""
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


# mode: (graph, SLAK_BATCH_GROUP_QUADS, SLAK_BATCH_WAVE_BYTES); these meshes
# refine to at most 768k quads, so a bound of 4M groups all of them
MODES = {"grouped": (False, "4000000", None), "grouped-graph": (True, "4000000", None),
         "chains": (False, "0", None), "chains-graph": (True, "0", None),
         "mixed-graph": (True, "20000", None), "waves": (False, "0", "1")}


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("mode", list(MODES))
def test_batch_matches_single(scheme, mode, monkeypatch):
    import torch
    items = _meshes()
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    graph, gq, wb = MODES[mode]
    if gq is not None:
        monkeypatch.setenv("SLAK_BATCH_GROUP_QUADS", gq)
    if wb is not None:                         # a 1-byte budget: every chain reuses its slice
        monkeypatch.setenv("SLAK_BATCH_WAVE_BYTES", wb)
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    s = torch.cuda.Stream()
    flags = api._abi.PLAN_GRAPH if graph else 0
    with torch.cuda.stream(s):
        b = api.Batch(dms, [l for _, l in items], scheme, flags, stream=s)
        if mode.startswith("grouped"):
            assert b.groups >= 1 and b.waves == 0
        elif mode.startswith("chains") or mode == "waves":
            assert b.groups == 0 and b.waves >= 1
        else:
            assert b.groups >= 1 and b.waves >= 1
        for _ in range(2 if graph else 1):
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


def test_groups_cut_launches(monkeypatch):
    """Grouped launches: one launch per step of each group instead of one per
    step of each mesh."""
    import torch
    items = _meshes()
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    s = torch.cuda.Stream()
    counts = {}
    with torch.cuda.stream(s):
        for gq in ("0", "4000000"):
            monkeypatch.setenv("SLAK_BATCH_GROUP_QUADS", gq)
            b = api.Batch(dms, [l for _, l in items], SLAK, 0, stream=s)
            b.execute(s)
            b.check(s)
            counts[gq] = (b.launches, b.groups)
            b.close()
    (chained, _), (grouped, ngroups) = counts["0"], counts["4000000"]
    assert 1 <= ngroups < len(items)
    assert grouped * 2 < chained               # 29 meshes of many kinds: 174 against 510 on B200


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("waves", [False, True])
def test_subdivide_batched_one_call(scheme, waves, monkeypatch):
    """slak_subdivide_batched: caller-owned outputs, each equal to
    slak_subdivide on that mesh alone; meshes with nothing to refine stay zeroed."""
    import torch
    items = _meshes()
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    if waves:                                  # chains only, on a 1-byte budget
        monkeypatch.setenv("SLAK_BATCH_GROUP_QUADS", "0")
        monkeypatch.setenv("SLAK_BATCH_WAVE_BYTES", "1")
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
