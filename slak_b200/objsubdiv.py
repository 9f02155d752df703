"""Subdivide an OBJ file on the GPU and write the refined mesh as OBJ.

    python -m slak_b200.objsubdiv in.obj out.obj --levels 3 --scheme slak

The mesh is read on the host (multi-threaded parse), refined by slak_subdivide
(the drop-in call, host buffers copied in and out) and written with exact
float32 positions, for visual checks of the refinement.
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("input")
    ap.add_argument("output")
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--scheme", default="slak", choices=["slak", "lak"])
    a = ap.parse_args(argv)
    from . import api, meshio
    from .mesh import LAK, SLAK
    t0 = time.perf_counter()
    mesh = meshio.read_obj(a.input)
    scheme = SLAK if a.scheme == "slak" else LAK
    cls = api.CatmullClark if scheme == SLAK else api.LAKCatmullClark
    rm = api.DeviceMesh()
    cls.subdivideIteratively(api.DeviceMesh.from_host(mesh), rm, a.levels)
    out = rm.to_host()
    meshio.write_obj(a.output, out)
    print(f"{a.input}: {mesh.nfaces} faces, {mesh.nverts} verts -> {out.nfaces} quads, {out.nverts} verts "
          f"({a.scheme.upper()}, {a.levels} levels) in {time.perf_counter() - t0:.2f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
