"""Semi-sharp creases on the GPU (slak_plan_create_creased): bit for bit
against the CPU restatement (oracle/creases.py) on closed and open meshes,
quad and polygon inputs, both schemes, integer and fractional sharpness, on
the fast path, the general path and a graph replay; and the errors."""
import ctypes

import numpy as np
import pytest

import oracle
from oracle import creases as oc
from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

from meshes import cube, open_grid, open_mixed

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def _edges(mesh):
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    ids = np.asarray(mesh.ids, np.int64)
    nxt = oc._next_corner(ptr, ids.size, mesh.type == 1)
    return np.unique(np.sort(np.stack([ids, ids[nxt]], 1), 1), axis=0)


def _random_creases(mesh, frac, seed, values=(0.5, 1.0, 1.5, 2.0, 3.0, 10.0)):
    rng = np.random.default_rng(seed)
    e = _edges(mesh)
    pick = e[rng.random(e.shape[0]) < frac]
    flip = rng.random(pick.shape[0]) < 0.5                       # either order names the edge
    pick[flip] = pick[flip][:, ::-1]
    return pick.astype(np.int32), rng.choice(np.array(values, np.float32), pick.shape[0])


def _lak(mesh, scheme):
    return mesh.with_quad_ptr() if scheme == LAK and mesh.ptr is None else mesh


def _same(mesh, levels, scheme, pairs, sharp, flags=0):
    ref = oc.subdivide_creased(mesh, levels, scheme, pairs, sharp)
    got = api.subdivide(mesh, levels, scheme, flags, creases=(pairs, sharp))
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(_bits(got.verts), _bits(ref.verts))
    return got


CASES = [
    ("cube_all_sharp", lambda: cube(), 4, lambda m: (_edges(m).astype(np.int32), np.full(12, 10.0, np.float32))),
    ("cube_fractional", lambda: cube(), 3, lambda m: (_edges(m).astype(np.int32),
                                                      np.linspace(0.25, 2.75, 12).astype(np.float32))),
    ("mixed_torus", lambda: meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=4), 4,
     lambda m: _random_creases(m, 0.15, 1)),
    ("icosphere", lambda: meshgen.icosphere(3, 0.02, seed=3), 3, lambda m: _random_creases(m, 0.3, 2)),
    ("open_grid", lambda: open_grid(24, 20), 3, lambda m: _random_creases(m, 0.2, 3)),
    ("open_mixed", lambda: open_mixed(), 3, lambda m: _random_creases(m, 0.1, 4)),
]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make,levels,creases", CASES, ids=[c[0] for c in CASES])
def test_creases_bit_exact(name, make, levels, creases, scheme):
    m = _lak(make(), scheme)
    pairs, sharp = creases(m)
    assert pairs.shape[0] > 0
    _same(m, levels, scheme, pairs, sharp)


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_creases_general_path_and_graph(scheme):
    m = _lak(meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=4), scheme)
    pairs, sharp = _random_creases(m, 0.15, 1)
    a = _same(m, 4, scheme, pairs, sharp, _abi.PLAN_GENERAL)
    import torch
    dm = api.DeviceMesh.from_host(m)
    s = torch.cuda.Stream()
    plan = api.Plan(dm, 4, scheme, _abi.PLAN_GRAPH, stream=s, creases=(pairs, sharp))
    for _ in range(3):                                   # replays re-run the crease passes from the snapshot
        plan.execute(s)
    plan.check(s)
    out = plan.output().to_host()
    torch.cuda.synchronize()
    plan.close()
    assert np.array_equal(out.ids, a.ids) and np.array_equal(_bits(out.verts), _bits(a.verts))


def test_all_sharp_cube_known_answer():
    m = cube()
    got = api.subdivide(m, 5, SLAK, creases=(_edges(m).astype(np.int32), np.full(12, 8.0, np.float32)))
    assert (np.abs(got.verts[:, :3]).max(1) == 1.0).all()
    assert np.array_equal(got.verts[:8], np.asarray(m.verts, np.float32)[:8])


def test_zero_sharpness_equals_plain_plan():
    m = meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=4)
    e = _edges(m).astype(np.int32)
    got = api.subdivide(m, 3, SLAK, creases=(e, np.zeros(e.shape[0], np.float32)))
    plain = api.subdivide(m, 3, SLAK)
    assert np.array_equal(got.ids, plain.ids) and np.array_equal(_bits(got.verts), _bits(plain.verts))


def test_subdivide_creased_one_shot():
    import torch
    m = cube()
    pairs, sharp = _edges(m).astype(np.int32), np.full(12, 2.5, np.float32)
    ref = oc.subdivide_creased(m, 3, SLAK, pairs, sharp)
    dm = api.DeviceMesh.from_host(m)
    tp, ts = api._crease_tensors((pairs, sharp))
    out = _abi.SlakMesh()
    rc = _abi.lib().slak_subdivide_creased(ctypes.byref(dm.as_c()), ctypes.byref(out), 3, SLAK, tp.data_ptr(),
                                           ts.data_ptr(), 12, None)
    _abi.check(rc, "slak_subdivide_creased")
    host = api._wrap_c(out, None).to_host()
    torch.cuda.synchronize()
    _abi.lib().slak_mesh_free(ctypes.byref(out))
    assert np.array_equal(host.ids, ref.ids) and np.array_equal(_bits(host.verts), _bits(ref.verts))


@pytest.mark.parametrize("pairs,sharp,code", [
    ([[0, 7]], [1.0], _abi.SLAK_ERR_BAD_MESH),              # not an edge
    ([[4, 6], [6, 4]], [1.0, 2.0], _abi.SLAK_ERR_BAD_MESH),  # named twice
    ([[0, 8]], [1.0], _abi.SLAK_ERR_BAD_MESH),              # out of range
    ([[4, 6]], [float("nan")], _abi.SLAK_ERR_INVALID_ARG),  # not finite
])
def test_invalid_creases_rejected(pairs, sharp, code):
    m = cube()
    with pytest.raises(_abi.SlakError) as ei:
        api.subdivide(m, 2, SLAK, creases=(np.array(pairs, np.int32), np.array(sharp, np.float32)))
    assert ei.value.code == code


def _same_sharp(mesh, levels, scheme, pairs, sharp, corners, flags=0):
    ref = oc.subdivide_creased(mesh, levels, scheme, pairs, sharp, corners=corners)
    got = api.subdivide(mesh, levels, scheme, flags, creases=(pairs, sharp), corners=corners)
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(_bits(got.verts), _bits(ref.verts))
    return got


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_corners_bit_exact(scheme):
    """Corner tags alone, with creases, fractional, on crease vertices and on
    boundary vertices: bit for bit against the restatement, on the fast path,
    the general path and a graph replay."""
    rng = np.random.default_rng(7)
    none = (np.zeros((0, 2), np.int32), np.zeros(0, np.float32))
    cube_m = _lak(cube(), scheme)
    _same_sharp(cube_m, 4, scheme, *none, (np.arange(8, dtype=np.int32), np.full(8, 10.0, np.float32)))
    _same_sharp(cube_m, 3, scheme, *none, (np.array([1, 6], np.int32), np.array([0.5, 1.5], np.float32)))
    for make, levels in ((lambda: meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=4), 4),
                         (lambda: open_mixed(), 3)):
        m = _lak(make(), scheme)
        pairs, sharp = _random_creases(m, 0.15, 1)
        kv = np.unique(np.concatenate([pairs[:40, 0], rng.integers(0, m.nverts, 60)])).astype(np.int32)
        ks = rng.choice(np.array([0.25, 0.5, 1.0, 2.5, 6.0], np.float32), kv.size)
        a = _same_sharp(m, levels, scheme, pairs, sharp, (kv, ks))
        g = api.subdivide(m, levels, scheme, _abi.PLAN_GENERAL, creases=(pairs, sharp), corners=(kv, ks))
        assert np.array_equal(_bits(g.verts), _bits(a.verts))
        _same_sharp(m, levels, scheme, *none, (kv, ks))            # corners without creases


@pytest.mark.parametrize("kv,ks,code", [
    ([8], [1.0], _abi.SLAK_ERR_BAD_MESH),                  # out of range
    ([3, 3], [1.0, 2.0], _abi.SLAK_ERR_BAD_MESH),          # named twice
    ([3], [float("inf")], _abi.SLAK_ERR_INVALID_ARG),      # not finite
])
def test_invalid_corners_rejected(kv, ks, code):
    with pytest.raises(_abi.SlakError) as ei:
        api.subdivide(cube(), 2, SLAK, corners=(np.array(kv, np.int32), np.array(ks, np.float32)))
    assert ei.value.code == code
