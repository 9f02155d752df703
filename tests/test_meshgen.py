"""Synthetic workload generators: sizes and mesh validity (CPU)."""
import numpy as np
import pytest

from slak_b200 import meshgen
from slak_b200.mesh import POLY, QUAD, TRI

from meshes import closed


def _valences(m):
    return np.bincount(m.ids, minlength=m.nverts)


def test_torus32():
    w = meshgen.workload("torus32")
    m = w.mesh
    assert m.type == QUAD and m.nfaces == 1024 and m.nverts == 1024 and w.levels == 3
    assert closed(m) and (_valences(m) == 4).all()
    assert np.allclose(m.verts[:, 3], 1.0)


def test_icosphere():
    w = meshgen.workload("icosphere")
    m = w.mesh
    assert m.type == TRI and m.nfaces == 1280 and m.nverts == 642 and w.levels == 4
    v = _valences(m)
    assert closed(m) and set(np.unique(v)) == {5, 6} and (v == 5).sum() == 12


def test_cylinder():
    w = meshgen.workload("cylinder")
    m = w.mesh
    assert m.type == POLY and m.nfaces == 2112 and m.nverts == 2050 and m.nnz == 8320 and w.levels == 7
    v = _valences(m)
    assert closed(m) and v.max() == 64 and (v == 64).sum() == 2


def test_mixed_torus_small_and_spec():
    m = meshgen.mixed_torus(64, 64, 0.05, 0.03, 0.005, seed=13)
    orders = np.diff(m.ptr)
    assert m.type == POLY and closed(m)
    assert orders.min() == 3 and orders.max() <= 8
    v = _valences(m)
    assert v.min() >= 3
    # Euler characteristic of a torus
    ptr = m.ptr
    st = np.repeat(ptr[:-1], orders)
    en = np.repeat(ptr[1:], orders)
    c = np.arange(m.nnz)
    nx = np.where(c + 1 < en, c + 1, st)
    a, b = m.ids.astype(np.int64), m.ids[nx].astype(np.int64)
    E = np.unique(np.minimum(a, b) * m.nverts + np.maximum(a, b)).size
    assert m.nverts - E + m.nfaces == 0


def test_seeded():
    a = meshgen.mixed_torus(32, 32, seed=9)
    b = meshgen.mixed_torus(32, 32, seed=9)
    assert np.array_equal(a.ids, b.ids) and np.array_equal(a.verts, b.verts)


def test_batch_specs():
    specs = meshgen.batch_specs(2000)
    assert len(specs) == 2000
    faces = np.array([s.faces for s in specs])
    assert faces.min() >= 100 and faces.max() <= 200000
    kinds = [s.kind for s in specs]
    assert 0.35 < kinds.count("torus") / 2000 < 0.45
    assert set(s.levels for s in specs) == {1, 2, 3, 4}
    assert meshgen.batch_specs(10) == meshgen.batch_specs(10)


def test_degenerate_parameters_refused():
    """Sizes a generator cannot build (a torus of fewer than 3 x 3 quads, an
    icosphere of frequency < 1, a cylinder of < 3 segments or < 2 rings, an
    empty grid) raise instead of returning a broken mesh."""
    import pytest
    for call in (lambda: meshgen.torus(0, 4), lambda: meshgen.torus(2, 2), lambda: meshgen.icosphere(0),
                 lambda: meshgen.mixed_torus(0, 4), lambda: meshgen.capped_cylinder(2, 4),
                 lambda: meshgen.capped_cylinder(8, 1), lambda: meshgen.open_grid(0, 3), lambda: meshgen.open_grid(4, 0)):
        with pytest.raises(ValueError):
            call()
