"""Writes the golden fixtures of tests/test_golden.py: GPUPeople/SLAK's own
output on small meshes.

The reference's only implementation is CUDA, so this runs on a machine with a
GPU and the reference built from its sources (oracle/_ref, oracle/build_ref.py):

    python tests/golden/make_golden.py [out_dir]     # default: tests/golden

For every small test mesh and both schemes it stores the input mesh, the
reference's refined counts, LAK's ptr / vals, and the refined ids and
positions after canonical edge relabelling (slak_b200/canon.py: the reference
numbers edge points in atomicAdd order, which varies from run to run).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import ref                      # noqa: E402
from slak_b200 import canon                 # noqa: E402
from slak_b200.mesh import LAK, SLAK        # noqa: E402
from meshes import small_set                # noqa: E402


def main(out_dir=HERE):
    if not ref.available():
        raise SystemExit("oracle/_ref/libslak_ref.so is not built")
    os.makedirs(out_dir, exist_ok=True)
    for name, mesh, levels in small_set():
        for scheme in (SLAK, LAK):
            m = mesh if scheme == SLAK or mesh.ptr is not None else mesh.with_quad_ptr()
            r = ref.run(m, levels, scheme)
            cids, cverts = canon.canonicalize(m, levels, r.ids, r.verts)
            arrays = dict(type=m.type, nfaces=m.nfaces, nverts=m.nverts, max_face_order=m.max_face_order,
                          is_reduced=int(m.is_reduced), ids=m.ids.astype(np.int32),
                          verts=np.asarray(m.verts, np.float32), levels=levels, scheme=scheme,
                          out_counts=np.array([r.nfaces, r.nnz, r.nverts], np.int64),
                          out_is_reduced=int(r.is_reduced), canon_ids=cids.astype(np.int32),
                          canon_verts=np.asarray(cverts, np.float32))
            if m.ptr is not None:
                arrays["ptr"] = m.ptr.astype(np.int32)
            if m.vals is not None:
                arrays["vals"] = m.vals.astype(np.int32)
            if scheme == LAK:
                arrays["out_ptr"] = r.ptr.astype(np.int32)
                arrays["out_vals"] = r.vals.astype(np.int32)
            path = os.path.join(out_dir, f"{name}_{'slak' if scheme == SLAK else 'lak'}.npz")
            np.savez_compressed(path, **arrays)
            print(path, r.nfaces, "quads")


if __name__ == "__main__":
    main(*sys.argv[1:])
