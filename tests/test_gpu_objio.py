"""OBJ in, GPU refinement, OBJ out: the file written after slak_subdivide
reads back as the oracle's refined mesh (exact positions)."""
import numpy as np
import pytest

import oracle
from slak_b200 import meshgen, meshio, objsubdiv
from slak_b200.mesh import LAK, QUAD, SLAK

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", ["slak", "lak"])
def test_obj_subdivide_round_trip(tmp_path, scheme):
    src = meshgen.mixed_torus(24, 20, 0.05, 0.03, 0.005, seed=9)
    inp, out = tmp_path / "in.obj", tmp_path / "out.obj"
    meshio.write_obj(str(inp), src)
    assert objsubdiv.main([str(inp), str(out), "--levels", "2", "--scheme", scheme]) == 0
    got = meshio.read_obj(str(out))
    mesh = meshio.read_obj(str(inp))
    ref = oracle.subdivide(mesh, 2, SLAK if scheme == "slak" else LAK)
    assert got.type == QUAD and got.nfaces == ref.nfaces and got.nverts == ref.nverts
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(got.verts[:, :3].view(np.uint32), ref.verts[:, :3].view(np.uint32))


@pytest.mark.parametrize("scheme", ["slak", "lak"])
def test_obj_crease_tags_subdivide(tmp_path, scheme):
    """A file with "t crease" and "t corner" tags is refined with them: the
    result reads back as the restatement's refined mesh."""
    from oracle import creases as oc
    src = meshgen.mixed_torus(24, 20, 0.05, 0.03, 0.005, seed=9)
    ids = np.asarray(src.ids)
    ptr = np.asarray(src.ptr)
    first = ptr[:-1]
    rng = np.random.default_rng(3)
    pick = first[rng.random(first.size) < 0.2]
    pairs = np.stack([ids[pick], ids[pick + 1]], 1).astype(np.int32)       # each face's first edge
    pairs = np.unique(np.sort(pairs, 1), axis=0)
    sharp = rng.choice(np.array([0.5, 1.0, 2.5, 4.0], np.float32), pairs.shape[0])
    kv = np.unique(rng.integers(0, src.nverts, 30)).astype(np.int32)
    ks = rng.choice(np.array([0.5, 1.0, 3.0], np.float32), kv.size)
    inp, out = tmp_path / "in.obj", tmp_path / "out.obj"
    meshio.write_obj(str(inp), src, creases=(pairs, sharp), corners=(kv, ks))
    assert objsubdiv.main([str(inp), str(out), "--levels", "3", "--scheme", scheme]) == 0
    got = meshio.read_obj(str(out))
    mesh, cr, ko = meshio.read_obj_sharp(str(inp))
    ref = oc.subdivide_creased(mesh, 3, SLAK if scheme == "slak" else LAK, *cr, corners=ko)
    assert np.array_equal(got.ids, ref.ids)
    assert np.array_equal(got.verts[:, :3].view(np.uint32), ref.verts[:, :3].view(np.uint32))
