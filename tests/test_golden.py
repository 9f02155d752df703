"""The oracle against golden fixtures of the reference's own output
(tests/golden/*.npz, written by tests/golden/make_golden.py from
GPUPeople/SLAK's CUDA path run on a B200).  Runs on the CPU: topology must be
identical after canonical edge relabelling, positions equal to 64 float ulps
of the coordinate scale (the reference sums some floats with atomics in a
varying order and lets its compiler contract a few products into FMAs)."""
import glob
import os

import numpy as np
import pytest

import oracle
from slak_b200 import canon
from slak_b200.mesh import LAK, Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
TOL_ULPS = 64


def test_fixtures_present():
    assert len(FIXTURES) >= 20


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference_fixture(path):
    g = np.load(path)
    mesh = Mesh(int(g["type"]), g["ids"], g["verts"], g["ptr"] if "ptr" in g else None,
                g["vals"] if "vals" in g else None, int(g["nfaces"]), int(g["max_face_order"]),
                bool(g["is_reduced"]))
    levels, scheme = int(g["levels"]), int(g["scheme"])
    o = oracle.subdivide(mesh, levels, scheme)
    assert [o.nfaces, o.nnz, o.nverts] == list(g["out_counts"])
    assert int(o.is_reduced) == int(g["out_is_reduced"])
    if scheme == LAK:
        assert np.array_equal(o.ptr, g["out_ptr"]) and np.array_equal(o.vals, g["out_vals"])
    cids, cverts = canon.canonicalize(mesh, levels, o.ids, o.verts)
    assert np.array_equal(cids, g["canon_ids"])
    scale = max(float(np.abs(cverts[:, :3]).max()), 1.0)
    assert np.abs(cverts - g["canon_verts"]).max() <= TOL_ULPS * np.finfo(np.float32).eps * scale
