"""CPU tests of the oracle (the CPU restatement used as checker) and of the
canonical relabelling.  No GPU needed."""
import numpy as np
import pytest

import oracle
from slak_b200 import canon
from slak_b200.mesh import LAK, QUAD, SLAK, Mesh

from meshes import closed, cube, open_grid, small_set


def _next(ptr, N):
    orders = np.diff(ptr)
    start = np.repeat(ptr[:-1], orders)
    end = np.repeat(ptr[1:], orders)
    c = np.arange(N)
    return np.where(c + 1 < end, c + 1, start)


@pytest.mark.parametrize("scheme", [LAK, SLAK])
def test_cube_known_answer(scheme):
    """Published Catmull-Clark rules on the cube [-1,1]^3: corners go to +-5/9,
    face points to the face centres, edge points to 3/4 of the edge midpoint."""
    r = oracle.subdivide(cube(), 1, scheme, fp64=True)
    assert (r.nfaces, r.nnz, r.nverts) == (24, 96, 26)
    assert np.allclose(np.abs(r.verts[:8, :3]), 5.0 / 9.0, atol=1e-6)
    fp = r.verts[8:14, :3]
    assert np.allclose(np.sort(np.abs(fp), 1), [[0, 0, 1]] * 6)
    ep = r.verts[14:26, :3]
    assert np.allclose(np.sort(np.abs(ep), 1), [[0, 0.75, 0.75]] * 12)
    assert np.allclose(r.verts[:, 3], 1.0, atol=1e-6)


def _invariants(mesh, levels, scheme):
    r = oracle.subdivide(mesh, levels, scheme)
    sizes = canon.level_sizes(mesh, levels)
    F, V, N = sizes[-1]
    assert r.nfaces == N and r.nnz == 4 * N
    B = 0 if closed(mesh) else None
    if B == 0:
        assert r.nverts == V + F + N // 2
    # quad q = coarse corner q: {v, e_out, V + face, e_in}; face entry constant per coarse face
    q = r.ids.reshape(-1, 4)
    assert (q[:, 2] >= V).all() and (q[:, 2] < V + F).all()
    assert (q[:, 1] >= V + F).all() and (q[:, 3] >= V + F).all() and (q.max() < r.nverts)
    # e_in of corner c is e_out of the previous corner of the same face (quads: c-1 mod 4)
    if levels >= 2:
        c = np.arange(N)
        prv = (c & ~3) | ((c + 3) & 3)
        assert (q[:, 3] == q[prv, 1]).all()
    # every edge point is used by exactly 2 refined quads per side (interior) => closed mesh Euler
    if B == 0:
        ptr = np.arange(r.nfaces + 1) * 4
        nxt = _next(ptr, r.nnz)
        a, b = r.ids.astype(np.int64), r.ids[nxt].astype(np.int64)
        E = np.unique(np.minimum(a, b) * r.nverts + np.maximum(a, b)).size
        ptr0 = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
        n0 = _next(ptr0, mesh.nnz)
        a0, b0 = mesh.ids.astype(np.int64), mesh.ids[n0].astype(np.int64)
        E0 = np.unique(np.minimum(a0, b0) * mesh.nverts + np.maximum(a0, b0)).size
        assert r.nverts - E + r.nfaces == mesh.nverts - E0 + mesh.nfaces
    return r


@pytest.mark.parametrize("scheme", [LAK, SLAK])
@pytest.mark.parametrize("case", small_set(), ids=lambda c: c[0])
def test_invariants(case, scheme):
    name, mesh, levels = case
    if mesh.ptr is None and scheme == LAK:
        mesh = mesh.with_quad_ptr()
    _invariants(mesh, levels, scheme)


@pytest.mark.parametrize("case", small_set(), ids=lambda c: c[0])
def test_schemes_same_topology_up_to_edge_numbering(case):
    name, mesh, levels = case
    ms = mesh if mesh.ptr is not None else mesh.with_quad_ptr()
    a = oracle.subdivide(ms, levels, LAK)
    b = oracle.subdivide(mesh, levels, SLAK)
    ca, va = canon.canonicalize(ms, levels, a.ids, a.verts)
    cb, vb = canon.canonicalize(ms, levels, b.ids, b.verts)
    assert np.array_equal(ca, cb)
    # same subdivision matrices, different float operation order
    scale = max(1.0, float(np.abs(vb[:, :3]).max()))
    assert np.abs(va[:, :3] - vb[:, :3]).max() <= 1e-5 * scale


@pytest.mark.parametrize("scheme", [LAK, SLAK])
@pytest.mark.parametrize("case", small_set(), ids=lambda c: c[0])
def test_fp32_vs_fp64(case, scheme):
    name, mesh, levels = case
    if mesh.ptr is None and scheme == LAK:
        mesh = mesh.with_quad_ptr()
    r = oracle.subdivide(mesh, levels, scheme, fp64=True)
    diag = mesh.bbox_diag()
    err = np.abs(r.verts[:, :3].astype(np.float64) - r.verts64[:, :3]).max() / diag
    assert err <= 1e-6, err


def test_deterministic():
    name, mesh, levels = small_set()[8]
    a = oracle.subdivide(mesh, levels, SLAK)
    b = oracle.subdivide(mesh, levels, SLAK)
    assert np.array_equal(a.ids, b.ids) and np.array_equal(a.verts.view(np.uint32), b.verts.view(np.uint32))


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_single_thread_same_bits(scheme):
    """The single-thread timing of the CPU baseline runs the same arithmetic:
    one thread and the OpenMP default give identical results."""
    name, mesh, levels = small_set()[8]
    if scheme == LAK and mesh.ptr is None:
        mesh = mesh.with_quad_ptr()
    a = oracle.subdivide(mesh, levels, scheme)
    assert oracle.set_threads(1) == 1
    try:
        b = oracle.subdivide(mesh, levels, scheme)
    finally:
        oracle.set_threads(0)
    assert oracle.num_threads() >= 1
    assert np.array_equal(a.ids, b.ids) and np.array_equal(a.verts.view(np.uint32), b.verts.view(np.uint32))


def _slak_numbering_pure_python(mesh):
    """Independent pure-Python statement of the SLAK edge numbering rule
    (adjacency slots in corner order, owner = min->max half-edge or the only
    half-edge of a boundary edge, ids = owners ranked by (tail, corner))."""
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    nxt = _next(ptr, mesh.nnz)
    ids = mesh.ids.tolist()
    half = {(ids[c], ids[nxt[c]]): c for c in range(mesh.nnz)}
    owners = []
    for c in range(mesh.nnz):
        a, b = ids[c], ids[nxt[c]]
        if a < b or (b, a) not in half:
            owners.append((a, c))
    owners.sort()
    eid = {}
    for k, (a, c) in enumerate(owners):
        b = ids[nxt[c]]
        eid[(a, b)] = eid[(b, a)] = k
    V, F = mesh.nverts, mesh.nfaces
    return np.array([V + F + eid[(ids[c], ids[nxt[c]])] for c in range(mesh.nnz)])


def _lak_numbering_pure_python(mesh):
    """Independent statement of the LAK numbering: edges in ascending (max, min)."""
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    nxt = _next(ptr, mesh.nnz)
    ids = mesh.ids.tolist()
    edges = sorted({(max(ids[c], ids[nxt[c]]), min(ids[c], ids[nxt[c]])) for c in range(mesh.nnz)})
    rank = {e: k for k, e in enumerate(edges)}
    V, F = mesh.nverts, mesh.nfaces
    return np.array([V + F + rank[(max(ids[c], ids[nxt[c]]), min(ids[c], ids[nxt[c]]))] for c in range(mesh.nnz)])


@pytest.mark.parametrize("case", small_set(), ids=lambda c: c[0])
def test_edge_numbering_rule(case):
    name, mesh, _ = case
    ms = mesh if mesh.ptr is not None else mesh.with_quad_ptr()
    r = oracle.level(ms, SLAK, poly=mesh.type != QUAD)
    assert np.array_equal(r.ids[1::4], _slak_numbering_pure_python(ms))
    r = oracle.level(ms, LAK, poly=mesh.type != QUAD)
    assert np.array_equal(r.ids[1::4], _lak_numbering_pure_python(ms))


def test_canonicalize_is_invariant_to_edge_permutation():
    """Relabel every level's edge block at random; the canonical form must not change."""
    name, mesh, levels = small_set()[8]
    r = oracle.subdivide(mesh, levels, SLAK)
    c0, v0 = canon.canonicalize(mesh, levels, r.ids, r.verts)
    rng = np.random.default_rng(0)
    sizes = canon.level_sizes(mesh, levels)
    ids = r.ids.astype(np.int64).copy()
    verts = r.verts.copy()
    # permute the edge block of the last level only (earlier blocks feed later ids)
    F, V, N = sizes[-1]
    perm = np.arange(r.nverts)
    block = np.arange(V + F, r.nverts)
    perm[V + F:] = rng.permutation(block)
    ids = perm[ids]
    verts2 = np.empty_like(verts)
    verts2[perm] = verts
    c1, v1 = canon.canonicalize(mesh, levels, ids, verts2)
    assert np.array_equal(c0, c1) and np.array_equal(v0, v1)


def test_boundary_rules_open_grid():
    """Boundary vertex = 3/4 p + 1/8 (neighbours along the boundary); boundary edge point = midpoint."""
    m = open_grid(3, 2)
    for scheme in (LAK, SLAK):
        r = oracle.subdivide(m, 1, scheme, fp64=True)
        P = m.verts.astype(np.float64)
        # corner vertex 0 of the grid: boundary neighbours are vertices 1 (0,1) and 3 (1,0)
        exp = 0.75 * P[0] + 0.125 * P[1] + 0.125 * P[3]
        assert np.allclose(r.verts64[0], exp)
        assert np.allclose(r.verts[0], exp, atol=1e-6)


@pytest.mark.parametrize("scheme", [LAK, SLAK])
def test_unused_vertices_oracle(scheme):
    """Vertices no face uses (valence 0): at level 1 their refined positions
    are NaN (0/0 in the vertex rule) and every other output row equals the
    plain mesh's, with the old-vertex ids shifted past the inserted rows."""
    from slak_b200 import meshgen
    from slak_b200.mesh import from_arrays
    base = meshgen.mixed_torus(10, 8, 0.1, 0.05, 0.005, seed=7)
    V0 = base.nverts
    mid = V0 // 2
    P = np.asarray(base.verts, np.float32)[:, :3]
    ids = np.asarray(base.ids, np.int64)
    shift = lambda a: a + 1 + (a >= mid)                       # new id of an old vertex
    far = np.array([[3.0, 1.0, -2.0]], np.float32)
    m = from_arrays(np.asarray(base.ptr), shift(ids).astype(np.int32),
                    np.concatenate([far, P[:mid], far, P[mid:], far]))
    r0 = oracle.subdivide(base, 1, scheme)
    r1 = oracle.subdivide(m, 1, scheme)
    assert r1.nverts == r0.nverts + 3 and r1.nfaces == r0.nfaces
    old = np.arange(V0)
    v1 = np.asarray(r1.verts)
    v0 = np.asarray(r0.verts)
    nan_rows = np.flatnonzero(np.isnan(v1[:, :3]).any(1))
    assert np.array_equal(nan_rows, [0, mid + 1, V0 + 2])
    keep = v1[shift(old)]
    assert np.array_equal(keep.view(np.uint32), v0[:V0].view(np.uint32))
    assert np.array_equal(v1[V0 + 3:].view(np.uint32), v0[V0:].view(np.uint32))
    # refined quads: old-vertex ids shifted, face / edge point ids moved by 3
    q0 = np.asarray(r0.ids, np.int64)
    q1 = np.asarray(r1.ids, np.int64)
    expect = np.where(q0 < V0, shift(q0), q0 + 3)
    assert np.array_equal(q1, expect)


def _with_positions(mesh, xyz):
    v = np.ones((xyz.shape[0], 4), np.float32)
    v[:, :3] = xyz
    return Mesh(mesh.type, mesh.ids, v, mesh.ptr, mesh.vals, mesh.nfaces, mesh.max_face_order, mesh.is_reduced)


def _props_cases():
    from slak_b200 import meshgen
    return [(n, m, lv) for n, m, lv in small_set()] + [
        ("mixed", meshgen.mixed_torus(12, 10, 0.1, 0.05, 0.005, seed=4), 3),
        ("open_grid", open_grid(6, 5), 3)]


@pytest.mark.parametrize("scheme", [LAK, SLAK])
@pytest.mark.parametrize("case", _props_cases(), ids=lambda c: c[0])
def test_linear_and_affine(case, scheme):
    """Refinement is a fixed linear map of the positions whose rows sum to 1
    (every rule, boundary rules included, is an affine combination): in FP64,
    S(P + Q) = S(P) + S(Q) and S(P + t) = S(P) + t.  Integer coordinates keep
    the float32 inputs and their sums exact."""
    name, mesh, levels = case
    if scheme == LAK and mesh.ptr is None:
        mesh = mesh.with_quad_ptr()
    rng = np.random.default_rng(11)
    V = mesh.nverts
    P = rng.integers(-50, 50, (V, 3)).astype(np.float32)
    Q = rng.integers(-50, 50, (V, 3)).astype(np.float32)
    t = np.array([7.0, -3.0, 12.0], np.float32)
    S = lambda X: oracle.subdivide(_with_positions(mesh, X), levels, scheme, fp64=True).verts64[:, :3]
    sp, sq = S(P), S(Q)
    assert np.abs(S(P + Q) - (sp + sq)).max() <= 1e-9
    assert np.abs(S(P + t) - (sp + t)).max() <= 1e-9
