"""Run-to-run stability of the reference's raw output on this GPU.

TEST / BASELINE INFRASTRUCTURE ONLY.  Runs the reference's own CUDA path
(oracle/_ref) five times per case and hashes the raw refined ids and positions
(SHA-256).  Where all five runs agree, the raw bytes are also compared with
the oracle's (the serialized-atomic order this repository emits); where they
do not, only the canonical comparison of tests/test_ref_pin.py applies.

    python -m oracle.ref_stability
"""
from __future__ import annotations

import hashlib
import sys

import numpy as np

from . import ref, subdivide

RUNS = 5


def _cases():
    from slak_b200 import meshgen
    yield "torus32", meshgen.torus(32, 32, seed=1), 3
    yield "icosphere", meshgen.icosphere(3, 0.02, seed=3), 4
    yield "mixed128", meshgen.mixed_torus(128, 128, 0.05, 0.03, 0.005, seed=4), 3
    yield "cylinder", meshgen.capped_cylinder(64, 32, 0.001, seed=6), 3


def main() -> int:
    if not ref.available():
        print("reference library not built")
        return 1
    for name, mesh, levels in _cases():
        for scheme, sname in ((1, "SLAK"), (0, "LAK")):
            m = mesh if scheme == 1 or mesh.ptr is not None else mesh.with_quad_ptr()
            ids_h, verts_h = set(), set()
            last = None
            for _ in range(RUNS):
                r = ref.run(m, levels, scheme)
                ids_h.add(hashlib.sha256(np.ascontiguousarray(r.ids).tobytes()).hexdigest()[:16])
                verts_h.add(hashlib.sha256(np.ascontiguousarray(r.verts).tobytes()).hexdigest()[:16])
                last = r
            stable = len(ids_h) == 1 and len(verts_h) == 1
            line = (f"{name:10s} {sname:4s} {levels} levels: {len(ids_h)} distinct id hashes, "
                    f"{len(verts_h)} distinct position hashes in {RUNS} runs")
            if stable:
                o = subdivide(m, levels, scheme)
                same_ids = np.array_equal(last.ids, o.ids)
                same_verts = same_ids and np.array_equal(last.verts.view(np.uint32), o.verts.view(np.uint32))
                line += f"; raw bytes equal to the oracle: ids {same_ids}, positions {same_verts}"
            print(line, flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
