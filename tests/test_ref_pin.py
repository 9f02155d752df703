"""Pins the oracle against the reference's own CUDA build (oracle/_ref).

The reference numbers edge points in atomicAdd order and sums some floats with
atomics, so it is compared after canonical edge relabelling: topology must be
identical, positions equal to a few float ulps of the coordinate scale."""
import numpy as np
import pytest

import oracle
from oracle import ref
from slak_b200 import canon, meshgen
from slak_b200.mesh import LAK, SLAK

from meshes import small_set

pytestmark = pytest.mark.gpu

TOL_ULPS = 64   # atomic float sums in another order + FMA contraction choices


def _ref_or_skip():
    if not ref.available():
        pytest.skip("reference library not built (no reference tree where build() ran)")


def _compare(mesh, levels, scheme):
    r = ref.run(mesh, levels, scheme)
    o = oracle.subdivide(mesh, levels, scheme)
    assert (r.nfaces, r.nnz, r.nverts) == (o.nfaces, o.nnz, o.nverts)
    assert r.is_reduced == o.is_reduced
    if scheme == LAK:
        assert np.array_equal(r.ptr, o.ptr) and np.array_equal(r.vals, o.vals)
        assert r.max_face_order == o.max_face_order == 4
    cr, vr = canon.canonicalize(mesh, levels, r.ids, r.verts)
    co, vo = canon.canonicalize(mesh, levels, o.ids, o.verts)
    assert np.array_equal(cr, co)
    scale = float(np.abs(vo[:, :3]).max())
    tol = TOL_ULPS * np.finfo(np.float32).eps * max(scale, 1.0)
    assert np.abs(vr - vo).max() <= tol, np.abs(vr - vo).max()
    return r, o


@pytest.mark.parametrize("scheme", [LAK, SLAK])
@pytest.mark.parametrize("case", small_set(), ids=lambda c: c[0])
def test_reference_matches_oracle_small(case, scheme):
    _ref_or_skip()
    name, mesh, levels = case
    if scheme == LAK and mesh.ptr is None:
        mesh = mesh.with_quad_ptr()
    _compare(mesh, levels, scheme)


@pytest.mark.parametrize("scheme", [LAK, SLAK])
@pytest.mark.parametrize("name,levels", [("torus32", 3), ("icosphere", 4), ("cylinder", 3)])
def test_reference_matches_oracle_workloads(name, levels, scheme):
    _ref_or_skip()
    _compare(meshgen.workload(name).mesh, levels, scheme)


@pytest.mark.parametrize("scheme", [LAK, SLAK])
def test_reference_matches_oracle_mixed_polygons(scheme):
    """The large mixed-polygon workload's structure (5% of face pairs merged,
    3% of quads split: n-gons of 3-8 sides, valence 3-10, closed) at 128 x 128,
    3 levels: the reference's own output against the oracle."""
    _ref_or_skip()
    mesh = meshgen.mixed_torus(128, 128, 0.05, 0.03, 0.005)
    order = np.diff(mesh.ptr)
    assert order.min() == 3 and order.max() >= 6
    _compare(mesh, 3, scheme)
