"""The reference's own driver program (source/main.cpp of GPUPeople/SLAK),
compiled unchanged against include/CatmullClark.h and
include/LAKCatmullClark.h and linked with libslak_b200.so
(oracle/_ref/slak_main_dropin, built where the reference sources were
present).  Run as its users run it -- OBJ in, "<scheme> <level> 1" on the
command line, OBJ out through its own writer -- it gives the oracle's refined
mesh: identical faces, positions to the writer's 6 significant digits."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from slak_b200 import _paths, meshgen, meshio
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("make,levels", [(lambda: meshgen.mixed_torus(24, 20, 0.05, 0.03, 0.005, seed=9), 3),
                                         (lambda: meshgen.icosphere(2, 0.02, seed=3), 3)])
def test_reference_driver_on_the_drop_in_library(tmp_path, make, levels, scheme):
    if not os.path.exists(_paths.DROPIN_MAIN):
        pytest.skip("oracle/_ref/slak_main_dropin was not built (the reference sources were absent)")
    src = make()
    inp = tmp_path / "in.obj"
    meshio.write_obj(str(inp), src)
    r = subprocess.run([_paths.DROPIN_MAIN, str(inp), str(scheme), str(levels), "1"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = tmp_path / f"in_{levels}_{'SLAK' if scheme == SLAK else 'LAK'}.obj"
    assert out.exists(), r.stdout + r.stderr
    got = meshio.read_obj(str(out))
    mesh = meshio.read_obj(str(inp))
    ref = oracle.subdivide(mesh, levels, scheme)
    assert got.nfaces == ref.nfaces and got.nverts == ref.nverts
    assert np.array_equal(got.ids, ref.ids)
    xyz = ref.verts[:, :3].astype(np.float64)
    assert np.allclose(got.verts[:, :3], xyz, rtol=1e-5, atol=1e-6)
