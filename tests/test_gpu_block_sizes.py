"""Every launch shape of the fast kernels gives the same bits.

k_g1 writes its refined quads by one TMA tensor store per block for blocks of
128 and 256 threads and through a shared-memory staging buffer for blocks of
512 (beyond the tensor map's 256-row box); k_g2 and k_g3 run in all three
sizes too.  The autotuner may pick any of them, so each size is forced on
every fast level (through a SLAK_TUNE_FILE read by a fresh process, since the
file is read once per process) and the output compared with the oracle, on a
closed mixed mesh (polygon parent at level 1, the SG last level) and an open
one (the boundary path), in both schemes."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

MESHES = {"mixed": lambda: meshgen.mixed_torus(37, 29, 0.05, 0.03, 0.005, seed=31),
          "open": lambda: meshgen.open_grid(33, 27, seed=32)}
LEVELS = 4

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, SLAK
meshes = {"mixed": lambda: meshgen.mixed_torus(37, 29, 0.05, 0.03, 0.005, seed=31),
          "open": lambda: meshgen.open_grid(33, 27, seed=32)}
bs = int(sys.argv[2])
res = []
for name, make in meshes.items():
    for scheme in (SLAK, LAK):
        m = make()
        if scheme == LAK and m.ptr is None:
            m = m.with_quad_ptr()
        plan = api.Plan(api.DeviceMesh.from_host(m), 4, scheme, 0)
        plan.execute()
        plan.check()
        out = plan.output().to_host()
        blocks = [t["block"] for t in plan.tuning() if t["state"] >= 0]
        plan.close()
        ref = oracle.subdivide(m, 4, scheme)
        same = (np.array_equal(out.ids, ref.ids)
                and np.array_equal(np.asarray(out.verts, np.float32).view(np.uint32), ref.verts.view(np.uint32)))
        if scheme == LAK:
            same = same and np.array_equal(out.ptr, ref.ptr) and np.array_equal(out.vals, ref.vals)
        res.append({"mesh": name, "scheme": scheme, "same": bool(same), "blocks": blocks})
print(json.dumps(res))
"""


def _keys():
    """The tuning keys of every fast level of the meshes in both schemes."""
    keys = set()
    for make in MESHES.values():
        for scheme in (SLAK, LAK):
            m = make()
            if scheme == LAK and m.ptr is None:
                m = m.with_quad_ptr()
            plan = api.Plan(api.DeviceMesh.from_host(m), LEVELS, scheme, 0)
            keys |= {t["key"] for t in plan.tuning() if t["state"] >= 0}
            plan.close()
    return sorted(keys)


@pytest.mark.parametrize("bs", [128, 256, 512])
def test_every_block_size_bit_exact(bs, tmp_path):
    keys = _keys()
    assert keys
    path = tmp_path / "tune.txt"
    path.write_text("".join(f"{k} {bs} {bs} {bs}\n" for k in keys))
    env = dict(os.environ, SLAK_TUNE_FILE=str(path))
    r = subprocess.run([sys.executable, "-c", CHILD, REPO, str(bs)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(res) == 4
    for row in res:
        assert row["same"], row
        assert row["blocks"] and all(b == [bs, bs, bs] for b in row["blocks"]), row
