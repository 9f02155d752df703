"""Semi-sharp creases on the CPU: the restatement (oracle/creases.py) against
known answers.  The reference leaves creases unimplemented
(LibSource/device/CatmullClarkImpl.cu:94-96), so these answers come from the
published rules themselves: an all-sharp cube keeps its flat faces and
corners, sharpness 0 is the smooth surface, a sharp edge refines to its
midpoint and decays by one per level, and a crease ending on the boundary
pins the boundary vertex."""
import numpy as np
import pytest

import oracle
from oracle import creases as oc
from slak_b200.mesh import LAK, SLAK

from meshes import cube, open_grid, small_set


def _edges(mesh):
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    ids = np.asarray(mesh.ids, np.int64)
    nxt = oc._next_corner(ptr, ids.size, mesh.type == 1)
    e = np.unique(np.sort(np.stack([ids, ids[nxt]], 1), 1), axis=0)
    return e


def _lak(mesh, scheme):
    return mesh.with_quad_ptr() if scheme == LAK and mesh.ptr is None else mesh


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_all_sharp_cube_stays_a_cube(scheme):
    m = _lak(cube(), scheme)
    e = _edges(m)
    assert e.shape[0] == 12
    r = oc.subdivide_creased(m, 4, scheme, e, np.full(12, 10.0, np.float32))
    xyz = r.verts[:, :3]
    assert (np.abs(xyz).max(1) == 1.0).all()                       # every vertex on a face plane
    assert np.array_equal(r.verts[:8], np.asarray(m.verts, np.float32)[:8])   # corners fixed
    # points on the cube's edges keep two coordinates at +-1
    on_edge = (np.abs(xyz) == 1.0).sum(1) >= 2
    assert on_edge.sum() == 8 + 12 * (2 ** 4 - 1)
    smooth = oracle.subdivide(m, 4, scheme)
    assert np.abs(smooth.verts[:, :3]).max() < 1.0                  # without creases it shrinks


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_zero_sharpness_is_smooth(scheme):
    name, m, levels = small_set()[8]
    m = _lak(m, scheme)
    e = _edges(m)
    r = oc.subdivide_creased(m, levels, scheme, e, np.zeros(e.shape[0], np.float32))
    ref = oracle.subdivide(m, levels, scheme)
    assert np.array_equal(r.ids, ref.ids) and np.array_equal(r.verts.view(np.uint32), ref.verts.view(np.uint32))


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_sharp_edge_is_midpoint_then_decays(scheme):
    m = _lak(cube(), scheme)
    a, b = 4, 6                                       # an edge of the x = +1 face
    r1 = oc.subdivide_creased(m, 1, scheme, [[a, b]], [1.0])
    ref1 = oracle.subdivide(m, 1, scheme)
    ids = np.asarray(m.ids)
    c = [k for k in range(ids.size) if ids[k] == min(a, b) and ids[(k & ~3) | ((k + 1) & 3)] == max(a, b)][0]
    ep = r1.ids[4 * c + 1]
    V = np.asarray(m.verts, np.float32)
    assert np.array_equal(r1.verts[ep], (V[a] + V[b]) * np.float32(0.5))
    # the two ends are darts (one crease edge each): smooth
    assert np.array_equal(r1.verts[a], ref1.verts[a]) and np.array_equal(r1.verts[b], ref1.verts[b])
    changed = np.flatnonzero((r1.verts != ref1.verts).any(1))
    assert changed.tolist() == [ep]
    # sharpness 1 is spent after one level: level 2 is the smooth rule on level 1's result
    r2 = oc.subdivide_creased(m, 2, scheme, [[a, b]], [1.0])
    from oracle import _LevelMesh
    lm = _LevelMesh(r1)
    ref2 = oracle.level(lm, scheme, poly=False)
    assert np.array_equal(r2.verts.view(np.uint32), ref2.verts.view(np.uint32))


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_fractional_sharpness_blends_linearly(scheme):
    m = _lak(cube(), scheme)
    smooth = oracle.subdivide(m, 1, scheme).verts.astype(np.float64)
    sharp = oc.subdivide_creased(m, 1, scheme, [[4, 6]], [1.0]).verts.astype(np.float64)
    half = oc.subdivide_creased(m, 1, scheme, [[4, 6]], [0.5]).verts.astype(np.float64)
    assert np.allclose(half, 0.5 * smooth + 0.5 * sharp, atol=1e-6)


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_crease_ending_on_boundary_pins_the_boundary_vertex(scheme):
    m = _lak(open_grid(4, 3), scheme)
    H = 3
    vid = lambda i, j: i * (H + 1) + j
    # a crease from the bottom boundary vertex (2, 0) up to the interior vertex (2, 1)
    pairs = [[vid(2, 0), vid(2, 1)]]
    r = oc.subdivide_creased(m, 1, scheme, pairs, [3.0])
    V = np.asarray(m.verts, np.float32)
    assert np.array_equal(r.verts[vid(2, 0)], V[vid(2, 0)])            # boundary vertex: corner
    # a boundary edge named as a crease does nothing
    rb = oc.subdivide_creased(m, 2, scheme, [[vid(0, 0), vid(1, 0)]], [5.0])
    ref = oracle.subdivide(m, 2, scheme)
    assert np.array_equal(rb.verts.view(np.uint32), ref.verts.view(np.uint32))


def test_invalid_pairs_rejected():
    m = cube()
    with pytest.raises(ValueError):
        oc.subdivide_creased(m, 1, SLAK, [[0, 7]], [1.0])        # not an edge
    with pytest.raises(ValueError):
        oc.subdivide_creased(m, 1, SLAK, [[4, 6], [6, 4]], [1.0, 2.0])   # named twice
    with pytest.raises(ValueError):
        oc.subdivide_creased(m, 1, SLAK, [[0, 8]], [1.0])        # out of range


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_corner_tags_pin_vertices(scheme):
    """Vertex sharpness ("t corner" tags): a corner of sharpness >= the level
    count never moves; sharpness 0.5 blends the first level's smooth point
    half-way to the original; a corner on a crease vertex wins the rule."""
    m = _lak(cube(), scheme)
    V = np.asarray(m.verts, np.float32)
    none = np.zeros((0, 2), np.int32), np.zeros(0, np.float32)
    r = oc.subdivide_creased(m, 3, scheme, *none, corners=(np.arange(8), np.full(8, 5.0, np.float32)))
    assert np.array_equal(r.verts[:8], V[:8])
    smooth = oracle.subdivide(m, 3, scheme)
    assert not np.array_equal(smooth.verts[:8], V[:8])
    half = oc.subdivide_creased(m, 1, scheme, *none, corners=([2], [0.5]))
    s1 = oracle.subdivide(m, 1, scheme).verts
    assert np.allclose(half.verts[2], 0.5 * s1[2] + 0.5 * V[2], atol=1e-6)
    changed = np.flatnonzero((half.verts != s1).any(1))
    assert changed.tolist() == [2]
    # sharpness 1 is spent after one level: level 2 moves the vertex again
    r2 = oc.subdivide_creased(m, 2, scheme, *none, corners=([2], [1.0]))
    assert not np.array_equal(r2.verts[2], V[2])
    # a crease through vertex 4 (crease rule) plus a corner tag on it: corner wins
    both = oc.subdivide_creased(m, 1, scheme, [[4, 6], [4, 5]], [3.0, 3.0], corners=([4], [2.0]))
    assert np.array_equal(both.verts[4], V[4])


def test_invalid_corners_rejected():
    m = cube()
    none = np.zeros((0, 2), np.int32), np.zeros(0, np.float32)
    with pytest.raises(ValueError):
        oc.subdivide_creased(m, 1, SLAK, *none, corners=([8], [1.0]))           # out of range
    with pytest.raises(ValueError):
        oc.subdivide_creased(m, 1, SLAK, *none, corners=([3, 3], [1.0, 2.0]))   # named twice
