"""The drop-in headers (include/CatmullClark.h, include/LAKCatmullClark.h) used
from a compiled C++ program, like the reference's own driver, give the
oracle's result bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from slak_b200 import _paths, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path, "rb") as f:
        nf, nv, nnz, has_ptr = np.frombuffer(f.read(32), dtype=np.int64)
        ids = np.frombuffer(f.read(4 * nnz), dtype=np.int32)
        verts = np.frombuffer(f.read(16 * nv), dtype=np.float32).reshape(-1, 4)
        ptr = vals = None
        if has_ptr:
            ptr = np.frombuffer(f.read(4 * (nf + 1)), dtype=np.int32)
            vals = np.frombuffer(f.read(4 * nnz), dtype=np.int32)
    return int(nf), int(nv), ids, verts, ptr, vals


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,levels", [("torus", 3), ("icosphere", 3)])
def test_demo_program(tmp_path, name, levels, scheme):
    if not os.path.exists(_paths.DEMO_BIN):
        pytest.fail("slak_demo was not built")
    out = tmp_path / "r.bin"
    r = subprocess.run([_paths.DEMO_BIN, name, str(scheme), str(levels), str(out)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    nf, nv, ids, verts, ptr, vals = _read(out)
    m = meshgen.workload("torus32" if name == "torus" else name).mesh
    ref = oracle.subdivide(m, levels, scheme)
    assert (nf, nv) == (ref.nfaces, ref.nverts)
    assert np.array_equal(ids, ref.ids)
    assert np.array_equal(verts.view(np.uint32), ref.verts.view(np.uint32))
    if scheme == LAK:
        assert np.array_equal(ptr, ref.ptr) and np.array_equal(vals, ref.vals)
    else:
        assert ptr is None
