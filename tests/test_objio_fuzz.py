"""The C++ OBJ reader on damaged and hostile input (CPU): seeded mutations of
valid files (bytes flipped, lines dropped or repeated, tokens swapped for
extreme numbers, truncation) and hand-written edge cases.  Every file either
reads into a consistent mesh (offsets from 0 rising by at least 3, ids in
range, vals counting 1..order, crease / corner ids in range) or is refused with
a status code; none may crash the process."""
import numpy as np
import pytest

from slak_b200 import _abi, meshio

BASE = """v 0 0 0
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
t crease 2/1/0 0 1 4.5
t crease 3/1/0 1 2 3 2
t corner 1/1/0 4 10
"""

TOKENS = ["0", "-1", "-0", "1e38", "1e39", "-1e39", "nan", "inf", "2147483647", "2147483648", "-2147483649",
          "99999999999999999999", "1/", "//", "/1/", "1//", "f", "v", "t", "crease", "corner", "", "\t", "#",
          "0x10", "1.5", "-7", "3/3/3/3", "\x00", "\xff", "é"]


def _mutate(text, rng):
    lines = text.split("\n")
    for _ in range(int(rng.integers(1, 5))):
        op = int(rng.integers(0, 6))
        k = int(rng.integers(0, len(lines)))
        if op == 0 and len(lines) > 1:
            del lines[k]
        elif op == 1:
            lines.insert(k, lines[int(rng.integers(0, len(lines)))])
        elif op == 2:
            t = lines[k].split(" ")
            t[int(rng.integers(0, len(t)))] = TOKENS[int(rng.integers(0, len(TOKENS)))]
            lines[k] = " ".join(t)
        elif op == 3:
            s = lines[k]
            if s:
                i = int(rng.integers(0, len(s)))
                lines[k] = s[:i] + chr(int(rng.integers(1, 256))) + s[i + 1:]
        elif op == 4:
            lines[k] = lines[k] + " " + TOKENS[int(rng.integers(0, len(TOKENS)))]
        else:
            lines = lines[:k + 1]
            lines[-1] = lines[-1][:int(rng.integers(0, len(lines[-1]) + 1))]
    return "\n".join(lines)


def _consistent(mesh, creases, corners):
    ptr, ids, vals = np.asarray(mesh.ptr, np.int64), np.asarray(mesh.ids, np.int64), np.asarray(mesh.vals)
    V = mesh.nverts
    assert ptr[0] == 0 and ptr[-1] == ids.size and ptr.size == mesh.nfaces + 1
    d = np.diff(ptr)
    assert (d >= 3).all()
    assert ((ids >= 0) & (ids < V)).all()
    face = np.repeat(np.arange(d.size), d)
    assert np.array_equal(vals, np.arange(ids.size) - ptr[face] + 1)
    pairs, sharp = creases
    assert pairs.shape[0] == sharp.shape[0] and ((pairs >= 0) & (pairs < V)).all()
    kv, ks = corners
    assert kv.shape[0] == ks.shape[0] and ((kv >= 0) & (kv < V)).all()


def _read(path):
    try:
        return meshio.read_obj_sharp(str(path))
    except _abi.SlakError:
        return None


@pytest.mark.parametrize("seed", range(400))
def test_mutated_files(tmp_path, seed):
    rng = np.random.default_rng(seed)
    path = tmp_path / "m.obj"
    path.write_bytes(_mutate(BASE, rng).encode("utf-8", "surrogateescape"))
    r = _read(path)
    if r is not None:
        _consistent(*r)


EDGE = {
    "empty": b"",
    "comments_only": b"# nothing\n# here\n",
    "no_trailing_newline": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3",
    "crlf": b"v 0 0 0\r\nv 1 0 0\r\nv 0 1 0\r\nf 1 2 3\r\n",
    "tabs": b"v\t0\t0\t0\nv\t1\t0\t0\nv\t0\t1\t0\nf\t1\t2\t3\n",
    "nul_bytes": b"v 0 0 0\nv 1 0\x00 0\nv 0 1 0\nf 1 2 3\n",
    "long_line": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3 " + b"1 " * 200000 + b"\n",
    "huge_index": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 99999999999999999999\n",
    "negative_past_start": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf -1 -2 -4\n",
    "vertex_missing_coords": b"v 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "faces_before_vertices": b"f 1 2 3\nv 0 0 0\nv 1 0 0\nv 0 1 0\n",
    "crease_count_too_large": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nt crease 1000000/1/0 0 1 2\n",
    "crease_negative_count": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nt crease -2/1/0 0 1 2\n",
    "crease_count_huge": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nt crease 99999999999999/1/0 0 1 2\n",
    "corner_count_huge": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nt corner 99999999999999/99999999999999/0 0 1\n",
    "index_past_int32": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4294967298\n",
    "corner_nan": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nt corner 1/1/0 0 nan\n",
    "inf_position": b"v 1e39 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
}


# must be refused: an index out of range or past 32 bits, a malformed tag
REFUSED = {"huge_index", "index_past_int32", "negative_past_start",
           "crease_count_too_large", "crease_negative_count", "crease_count_huge", "corner_count_huge"}
# must read as the one triangle they hold (positive indices are absolute, as in the reference's
# OBJ::read, so a face may come before its vertices)
ONE_TRIANGLE = {"no_trailing_newline", "crlf", "tabs", "vertex_missing_coords", "inf_position",
                "faces_before_vertices"}


@pytest.mark.parametrize("name", sorted(EDGE))
def test_edge_cases(tmp_path, name):
    path = tmp_path / "e.obj"
    path.write_bytes(EDGE[name])
    r = _read(path)
    if name in REFUSED:
        assert r is None
    if name in ONE_TRIANGLE:
        assert r is not None and r[0].nfaces == 1 and r[0].nverts == 3
    if r is not None:
        _consistent(*r)
