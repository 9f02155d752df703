"""One eager plan execution per repetition, for profilers (ncu).

    python -m slak_b200.profile_case --workload mixed:384 --levels 4 --scheme slak --reps 2

``--workload`` is a named workload (torus32, icosphere, mixed512, cylinder) or
``mixed:W`` for a WxW mixed-polygon torus (5% merged, 3% split), so that a
profile can run on a smaller case of the same structure.  Each repetition runs
every level's kernels once, in launch order, and the result is checked against
the device status.
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixed:384")
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--scheme", default="slak", choices=["slak", "lak"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--flags", type=int, default=0)
    a = ap.parse_args(argv)
    import torch
    from . import api, meshgen
    from .mesh import LAK, SLAK
    if a.workload.startswith("mixed:"):
        w = int(a.workload.split(":")[1])
        mesh = meshgen.mixed_torus(w, w, 0.05, 0.03, 0.005, seed=13)
    else:
        mesh = meshgen.workload(a.workload).mesh
    scheme = SLAK if a.scheme == "slak" else LAK
    dm = api.DeviceMesh.from_host(mesh)
    plan = api.Plan(dm, a.levels, scheme, a.flags)
    for _ in range(a.reps):
        t0 = time.perf_counter()
        plan.execute()
        plan.check()
        print(f"execution: {1e3 * (time.perf_counter() - t0):.3f} ms wall, {plan.launches} launches", flush=True)
    st = plan.level_stats()[-1]
    print(f"{mesh.nfaces} faces -> {st['out_faces']} quads, {st['out_verts']} verts")
    plan.close()
    torch.cuda.synchronize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
