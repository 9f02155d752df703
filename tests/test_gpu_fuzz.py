"""Seeded random inputs through the CUDA path, bit for bit against the oracle
(topology and positions) and against the general path: mixed-polygon tori of
random size and merge / split rates, the same cut open by random angular
windows (one or two boundary loops), fans and capped cylinders of random
valence (the single-thread, warp and long-column paths), open grids and
icospheres, at 1-3 levels, both schemes."""
import numpy as np
import pytest

import oracle
from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, SLAK

from meshes import cut_mesh, fan_disk, open_grid

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def _face_centres(m):
    ptr = np.asarray(m.ptr if m.ptr is not None else np.arange(m.nfaces + 1) * 4)
    P = np.asarray(m.verts, np.float64)[np.asarray(m.ids), :3]
    return np.add.reduceat(P, ptr[:-1]) / np.diff(ptr)[:, None]


def _bowtie_free(m):
    """No vertex with two outgoing boundary half-edges (where SLAK's boundary
    correction in the reference races; see the bowtie tests)."""
    ptr = np.asarray(m.ptr if m.ptr is not None else np.arange(m.nfaces + 1) * 4, np.int64)
    ids = np.asarray(m.ids, np.int64)
    face = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    c = np.arange(ids.size)
    nxt = np.where(c + 1 == ptr[face + 1], ptr[face], c + 1)
    a, b = ids, ids[nxt]
    half = set(zip(a.tolist(), b.tolist()))
    out = [u for u, w in zip(a.tolist(), b.tolist()) if (w, u) not in half]
    return len(out) == len(set(out))


def _random_case(seed):
    rng = np.random.default_rng(seed)
    kind = seed % 5
    levels = int(rng.integers(1, 4))
    if kind == 0:
        m = meshgen.mixed_torus(int(rng.integers(6, 40)), int(rng.integers(4, 30)), float(rng.uniform(0, 0.15)),
                                float(rng.uniform(0, 0.1)), 0.005, seed=seed)
    elif kind == 1:
        m = meshgen.mixed_torus(int(rng.integers(12, 48)), int(rng.integers(8, 32)), float(rng.uniform(0, 0.1)),
                                float(rng.uniform(0, 0.08)), 0.005, seed=seed)
        ctr = _face_centres(m)
        ang = np.arctan2(ctr[:, 1], ctr[:, 0])
        lo = float(rng.uniform(-np.pi, 2.0))
        keep = ~((ang > lo) & (ang < lo + float(rng.uniform(0.4, 1.0))))
        if rng.random() < 0.5:                      # a second window: two patches, four boundary loops
            lo2 = lo + 2.5
            keep &= ~((ang > lo2 - 2 * np.pi) & (ang < lo2 - 2 * np.pi + 0.5)) & ~((ang > lo2) & (ang < lo2 + 0.5))
        m = cut_mesh(m, keep)
    elif kind == 2:
        m = fan_disk(int(rng.integers(3, 72)))
    elif kind == 3:
        m = meshgen.capped_cylinder(int(rng.integers(3, 80)), int(rng.integers(2, 7)), 0.001, seed=seed)
    else:
        m = (open_grid(int(rng.integers(1, 30)), int(rng.integers(1, 30))) if rng.random() < 0.5
             else meshgen.icosphere(int(rng.integers(1, 4)), 0.02, seed=seed))
    return m, levels


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("seed", list(range(30)))
def test_random_meshes_bit_exact(seed, scheme):
    mesh, levels = _random_case(seed)
    if scheme == LAK and mesh.ptr is None:
        mesh = mesh.with_quad_ptr()
    if scheme == SLAK and not _bowtie_free(mesh):
        pytest.skip("a bowtie boundary vertex (SLAK differs there by design)")
    ref = oracle.subdivide(mesh, levels, scheme)
    got = api.subdivide(mesh, levels, scheme)
    assert (got.nfaces, got.nverts) == (ref.nfaces, ref.nverts)
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(_bits(got.verts), _bits(ref.verts))
    gen = api.subdivide(mesh, levels, scheme, api._abi.PLAN_GENERAL)
    assert np.array_equal(gen.ids, got.ids) and np.array_equal(_bits(gen.verts), _bits(got.verts))


def _random_sharp(mesh, seed):
    """A random share of the edges tagged with random sharpness (whole and
    fractional, some above the level count) and a few random corners."""
    from oracle import creases as oc
    rng = np.random.default_rng(1000 + seed)
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    ids = np.asarray(mesh.ids, np.int64)
    nxt = oc._next_corner(ptr, ids.size, mesh.type == 1)
    e = np.unique(np.sort(np.stack([ids, ids[nxt]], 1), 1), axis=0)
    pick = e[rng.random(e.shape[0]) < rng.uniform(0.02, 0.4)]
    sharp = np.where(rng.random(pick.shape[0]) < 0.5, rng.integers(1, 6, pick.shape[0]),
                     rng.uniform(0.05, 4.0, pick.shape[0])).astype(np.float32)
    V = int(np.asarray(mesh.verts).shape[0])
    kv = rng.choice(V, int(rng.integers(0, min(V, 8) + 1)), replace=False).astype(np.int32)
    ks = rng.uniform(0.1, 5.0, kv.size).astype(np.float32)
    return pick.astype(np.int32), sharp, (kv, ks)


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("seed", list(range(20)))
def test_random_creases_bit_exact(seed, scheme):
    from oracle import creases as oc
    mesh, levels = _random_case(seed)
    if scheme == LAK and mesh.ptr is None:
        mesh = mesh.with_quad_ptr()
    if scheme == SLAK and not _bowtie_free(mesh):
        pytest.skip("a bowtie boundary vertex (SLAK differs there by design)")
    pairs, sharp, corners = _random_sharp(mesh, seed)
    ref = oc.subdivide_creased(mesh, levels, scheme, pairs, sharp, corners=corners)
    got = api.subdivide(mesh, levels, scheme, creases=(pairs, sharp), corners=corners)
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(_bits(got.verts), _bits(ref.verts))
    gen = api.subdivide(mesh, levels, scheme, api._abi.PLAN_GENERAL, creases=(pairs, sharp), corners=corners)
    assert np.array_equal(gen.ids, got.ids) and np.array_equal(_bits(gen.verts), _bits(got.verts))
