"""Precision study on the capped cylinder (64 x 32, two valence-64 poles,
jitter +-0.001), 7 levels, and on the 512 x 512 mixed-polygon torus, 4 levels:
per level, the max-abs error of the xyz positions
relative to the input's bounding-box diagonal, for plain FP32 (the reference's
operation order) and compensated FP32 (SLAK_PLAN_COMPENSATED: TwoSum sums and
exact-remainder quotients in the vertex points of valence > 4), both against an
FP64 evaluation of the same subdivision matrices (the oracle carried in
double).  Bound: 1e-6 at every level.  The per-level table, with the device
time of each variant, is written as JSON to $SLAK_REPORT_DIR (if set)."""
import json
import os

import numpy as np
import pytest

import oracle
from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _timed(mesh, levels, scheme, flags, reps=5):
    import torch
    dm = api.DeviceMesh.from_host(mesh)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan = api.Plan(dm, levels, scheme, flags | api._abi.PLAN_GRAPH, stream=s)
        for _ in range(2):
            plan.execute(s)
        plan.check(s)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in ev:
            a.record(s)
            plan.execute(s)
            b.record(s)
        torch.cuda.synchronize()
        plan.check(s)
        ms = float(np.median([a.elapsed_time(b) for a, b in ev]))
        out = plan.output().to_host()
        faces = plan.level_stats()[-1]["out_faces"]
    plan.close()
    return out, ms, faces


CASES = {"cylinder": ("capped cylinder 64x32, valence-64 poles, jitter 0.001", {SLAK: 7, LAK: 7}),
         "mixed512": ("512x512 mixed-polygon torus (n-gons 3-8, valence 3-10), jitter 0.005", {SLAK: 4, LAK: 4})}


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name", list(CASES))
def test_per_level_error(name, scheme):
    mesh = meshgen.workload(name).mesh
    what, lv = CASES[name]
    levels = lv[scheme]
    ref = oracle.subdivide_levels(mesh, levels, scheme)
    diag = mesh.bbox_diag()
    rows = []
    for L in range(1, levels + 1):
        r64 = ref[L - 1].verts64[:, :3]
        plain, ms_p, faces = _timed(mesh, L, scheme, 0)
        comp, ms_c, _ = _timed(mesh, L, scheme, api._abi.PLAN_COMPENSATED)
        assert np.array_equal(plain.ids, ref[L - 1].ids) and np.array_equal(comp.ids, ref[L - 1].ids)
        # the plain path is the oracle's FP32 bit for bit
        assert np.array_equal(plain.verts.view(np.uint32), ref[L - 1].verts.view(np.uint32))
        e_p = float(np.abs(plain.verts[:, :3].astype(np.float64) - r64).max() / diag)
        e_c = float(np.abs(comp.verts[:, :3].astype(np.float64) - r64).max() / diag)
        rows.append({"level": L, "faces": faces, "err_fp32": e_p, "err_compensated": e_c,
                     "ms_fp32": ms_p, "ms_compensated": ms_c})
        assert e_p <= 1e-6 and e_c <= 1e-6, rows[-1]
    if name == "cylinder":     # the poles: compensation must help where it applies
        assert rows[-1]["err_compensated"] <= rows[-1]["err_fp32"]
    d = os.environ.get("SLAK_REPORT_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        fn = f"precision_{name}_{'slak' if scheme == SLAK else 'lak'}.json"
        with open(os.path.join(d, fn), "w") as f:
            json.dump({"workload": what, "scheme": "SLAK" if scheme == SLAK else "LAK", "bbox_diag": diag,
                       "levels": rows}, f, indent=1)
