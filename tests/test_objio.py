"""OBJ reading and writing (CPU): the multi-threaded C++ parser against a
plain-Python restatement of the reference's OBJ::read + CSCMesh layout, the
index forms and negative indices, errors, and exact round trips."""
import numpy as np
import pytest

from slak_b200 import _abi, meshgen, meshio
from slak_b200.mesh import POLY, QUAD, TRI


def py_read(text):
    """Restatement of OBJ::read (include/obj.h:107-257) followed by the CSCMesh
    arrays (include/Mesh.h:153-176), for small files."""
    v, ptr, ids, vals = [], [0], [], []
    for line in text.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            v.append([float(x) for x in t[1:4]] + [1.0])
        elif t[0] == "f":
            for k, c in enumerate(t[1:]):
                i = int(c.split("/")[0])
                ids.append(len(v) + i if i < 0 else i - 1)
                vals.append(k + 1)
            ptr.append(len(ids))
    orders = np.diff(ptr)
    typ = TRI if (orders == 3).all() else QUAD if (orders == 4).all() else POLY
    return typ, np.array(ptr), np.array(ids), np.array(vals), np.array(v, np.float32), int(orders.max())


SAMPLE = """# a pyramid with mixed index forms
o pyramid
v 0 0 0
v 1 0 0
v 1 1 0
vt 0 0
vn 0 0 1
v 0 1 0
v 0.5 0.5 1.25
f 1/1/1 4//1 3 2/1
f 1 2 5
f -4/1 -3//1 -1
  f 3 4 5
f 4 1 5
s off
"""


def test_sample_matches_python_restatement(tmp_path):
    path = tmp_path / "pyr.obj"
    path.write_text(SAMPLE)
    m = meshio.read_obj(str(path))
    typ, ptr, ids, vals, verts, mfo = py_read(SAMPLE)
    assert m.type == typ == POLY and m.max_face_order == mfo == 4
    assert np.array_equal(m.ptr, ptr) and np.array_equal(m.ids, ids) and np.array_equal(m.vals, vals)
    assert np.array_equal(m.verts, verts)


@pytest.mark.parametrize("make,typ", [(lambda: meshgen.torus(30, 20, seed=2), QUAD),
                                      (lambda: meshgen.icosphere(6, 0.02, seed=3), TRI),
                                      (lambda: meshgen.mixed_torus(40, 30, 0.05, 0.03, 0.005, seed=4), POLY)])
def test_round_trip_is_exact(tmp_path, make, typ):
    m = make()
    path = tmp_path / "m.obj"
    meshio.write_obj(str(path), m)
    r = meshio.read_obj(str(path))
    assert r.type == typ and r.nfaces == m.nfaces and r.nverts == m.nverts
    assert np.array_equal(r.ids, m.ids)
    assert np.array_equal(r.verts[:, :3].view(np.uint32), np.asarray(m.verts, np.float32)[:, :3].view(np.uint32))
    assert (r.verts[:, 3] == 1.0).all()
    expect_ptr = m.ptr if m.ptr is not None else np.arange(m.nfaces + 1, dtype=np.int32) * 4
    assert np.array_equal(r.ptr, expect_ptr)


def test_large_file_parsed_in_parallel_chunks(tmp_path):
    # several MB, so the parse is split over threads; negative indices across chunk borders
    rng = np.random.default_rng(5)
    n = 120000
    lines = []
    for k in range(n):
        lines.append(f"v {rng.normal():.6f} {rng.normal():.6f} {rng.normal():.6f}")
        if k >= 3 and k % 2:
            lines.append("f -1 -2 -3 -4" if k % 4 == 1 else f"f {k + 1} {k} {k - 1}")
    text = "\n".join(lines) + "\n"
    path = tmp_path / "big.obj"
    path.write_text(text)
    m = meshio.read_obj(str(path))
    typ, ptr, ids, vals, verts, mfo = py_read(text)
    assert m.type == typ and np.array_equal(m.ptr, ptr) and np.array_equal(m.ids, ids)
    assert np.array_equal(m.vals, vals) and np.array_equal(m.verts, verts)


@pytest.mark.parametrize("bad", ["v 0 0 0\nv 1 0 0\nf 1 2\n", "v 0 0 0\nf 1 2 7\n", "v 0 0 0\nf 1 0 1\n",
                                 "v 0 0 0\nf 1 x 1\n"])
def test_malformed_faces_rejected(tmp_path, bad):
    path = tmp_path / "bad.obj"
    path.write_text(bad)
    with pytest.raises(_abi.SlakError):
        meshio.read_obj(str(path))


def test_missing_file_rejected(tmp_path):
    with pytest.raises(_abi.SlakError):
        meshio.read_obj(str(tmp_path / "none.obj"))


CREASED = """v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0.5 0.5 1
f 1 2 3 4
t crease 2/1/0 0 1 4.5
t crease 3/1/0 1 2 3 2
t corner 1/1/0 4 10
t crease 3/2/0 3 0 4 0.5 1.5
t interpolateboundary 1/0/0 1
"""


def test_crease_tags(tmp_path):
    path = tmp_path / "c.obj"
    path.write_text(CREASED)
    m, (pairs, sharp) = meshio.read_obj_creased(str(path))
    assert m.nfaces == 1 and m.nverts == 5
    assert pairs.tolist() == [[0, 1], [1, 2], [2, 3], [3, 0], [0, 4]]
    assert sharp.tolist() == [4.5, 2.0, 2.0, 0.5, 1.5]
    # the plain reader skips tags; a file without tags has no creases
    assert np.array_equal(meshio.read_obj(str(path)).ids, m.ids)
    plain = tmp_path / "p.obj"
    plain.write_text(SAMPLE)
    assert meshio.read_obj_creased(str(plain))[1][1].size == 0


def test_crease_tags_round_trip(tmp_path):
    m = meshgen.torus(12, 8, seed=2)
    rng = np.random.default_rng(1)
    ids = np.asarray(m.ids).reshape(-1, 4)
    pairs = np.stack([ids[:, 0], ids[:, 1]], 1)[rng.random(ids.shape[0]) < 0.3].astype(np.int32)
    sharp = rng.random(pairs.shape[0]).astype(np.float32) * 5
    path = tmp_path / "t.obj"
    meshio.write_obj(str(path), m, creases=(pairs, sharp))
    r, (p2, s2) = meshio.read_obj_creased(str(path))
    assert np.array_equal(r.ids, m.ids)
    assert np.array_equal(p2, pairs) and np.array_equal(s2.view(np.uint32), sharp.view(np.uint32))


def test_crease_tags_across_parallel_chunks(tmp_path):
    rng = np.random.default_rng(9)
    n = 150000
    lines = [f"v {rng.normal():.6f} {rng.normal():.6f} {rng.normal():.6f}" for _ in range(n)]
    expect = []
    for k in range(0, n - 1, 37):
        lines.insert(k + len(expect), f"t crease 2/1/0 {k} {k + 1} {k % 7 + 0.5}")
        expect.append((k, k + 1, k % 7 + 0.5))
    lines += ["f 1 2 3"]
    path = tmp_path / "big.obj"
    path.write_text("\n".join(lines) + "\n")
    m, (pairs, sharp) = meshio.read_obj_creased(str(path))
    assert m.nverts == n
    assert pairs.tolist() == [[a, b] for a, b, _ in expect]
    assert np.allclose(sharp, [s for _, _, s in expect])


@pytest.mark.parametrize("bad", ["v 0 0 0\nv 1 0 0\nt crease 2/1/0 0 5 1\n",     # id out of range
                                 "v 0 0 0\nv 1 0 0\nt crease 1/1/0 0 1\n",       # one id
                                 "v 0 0 0\nv 1 0 0\nt crease 2/2/0 0 1 1 2\n",   # float count
                                 "v 0 0 0\nv 1 0 0\nt crease 2/1/0 0 x 1\n",     # not a number
                                 "v 0 0 0\nv 1 0 0\nt crease 2 1 0 0 1 1\n"])    # counts not n/n/n
def test_malformed_crease_tags_rejected(tmp_path, bad):
    path = tmp_path / "bad.obj"
    path.write_text(bad)
    with pytest.raises(_abi.SlakError):
        meshio.read_obj_creased(str(path))
    meshio.read_obj(str(path))           # the plain reader skips tags


def test_corner_tags(tmp_path):
    path = tmp_path / "k.obj"
    path.write_text(CREASED + "t corner 2/1/0 3 4 7.5\nt corner 1/1/0 0 0.25\nt corner 2/2/0 1 2 1 2\n")
    m, (pairs, sharp), (kv, ks) = meshio.read_obj_sharp(str(path))
    assert pairs.shape == (5, 2)
    # CREASED's own "t corner 1/1/0 4 10" first (the plan, not the reader, rejects a vertex named twice)
    assert kv.tolist() == [4, 3, 4, 0, 1, 2] and ks.tolist() == [10.0, 7.5, 7.5, 0.25, 1.0, 2.0]
    # the crease-only reader skips corner tags, even malformed ones
    bad = tmp_path / "kb.obj"
    bad.write_text(CREASED + "t corner 2/5/0 3 4 1\n")
    assert meshio.read_obj_creased(str(bad))[1][1].size == 5
    with pytest.raises(_abi.SlakError):
        meshio.read_obj_sharp(str(bad))
    oor = tmp_path / "ko.obj"
    oor.write_text(CREASED + "t corner 1/1/0 9 1\n")          # vertex out of range
    with pytest.raises(_abi.SlakError):
        meshio.read_obj_sharp(str(oor))


def test_corner_tags_round_trip(tmp_path):
    m = meshgen.torus(8, 6, seed=2)
    kv = np.array([0, 5, 17], np.int32)
    ks = np.array([0.5, 3.0, 10.0], np.float32)
    pairs = np.array([[0, 1]], np.int32)
    path = tmp_path / "r.obj"
    meshio.write_obj(str(path), m, creases=(pairs, np.array([2.0], np.float32)), corners=(kv, ks))
    r, (p2, s2), (k2, w2) = meshio.read_obj_sharp(str(path))
    assert np.array_equal(r.ids, m.ids) and np.array_equal(p2, pairs)
    assert np.array_equal(k2, kv) and np.array_equal(w2.view(np.uint32), ks.view(np.uint32))


def test_writer_refuses_offsets_that_leave_ids(tmp_path):
    """The writer reads faces through ptr / nnz: offsets that do not start at
    0, do not end at nnz or go down, and a QUAD / TRI corner count that is not
    4 or 3 per face, are refused (SLAK_ERR_BAD_MESH) before any byte is written."""
    from slak_b200.mesh import Mesh
    V = np.zeros((4, 4), np.float32)
    ids = np.array([0, 1, 2, 0, 2, 3], np.int32)
    for ptr in ([0, 3, 7], [1, 3, 6], [0, 4, 3, 6]):
        m = Mesh(POLY, ids, V, np.array(ptr, np.int32), None, len(ptr) - 1, 3)
        path = tmp_path / "w.obj"
        with pytest.raises(_abi.SlakError) as e:
            meshio.write_obj(str(path), m)
        assert e.value.code == _abi.SLAK_ERR_BAD_MESH and not path.exists()
    m = Mesh(QUAD, ids, V, None, None, 2, 4)                      # 6 corners for 2 quads
    with pytest.raises(_abi.SlakError):
        meshio.write_obj(str(tmp_path / "q.obj"), m)
