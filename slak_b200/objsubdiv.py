"""Subdivide an OBJ file on the GPU and write the refined mesh as OBJ.

    python -m slak_b200.objsubdiv in.obj out.obj --levels 3 --scheme slak

The mesh is read on the host (multi-threaded parse), refined by slak_subdivide
(the drop-in call, host buffers copied in and out) and written with exact
float32 positions, for visual checks of the refinement.  A file with
"t crease" / "t corner" tags is refined with that sharpness
(slak_plan_create_sharp), unless --no-creases is given.
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
    ap.add_argument("--no-creases", action="store_true", help="ignore the file's crease and corner tags")
    a = ap.parse_args(argv)
    from . import api, meshio
    from .mesh import LAK, SLAK
    t0 = time.perf_counter()
    mesh, creases, corners = meshio.read_obj_sharp(a.input)
    scheme = SLAK if a.scheme == "slak" else LAK
    ncr = 0 if a.no_creases else int(creases[1].size)
    nco = 0 if a.no_creases else int(corners[1].size)
    if ncr or nco:
        out = api.subdivide(mesh, a.levels, scheme, creases=creases, corners=corners)
    else:
        cls = api.CatmullClark if scheme == SLAK else api.LAKCatmullClark
        rm = api.DeviceMesh()
        cls.subdivideIteratively(api.DeviceMesh.from_host(mesh), rm, a.levels)
        out = rm.to_host()
    meshio.write_obj(a.output, out)
    print(f"{a.input}: {mesh.nfaces} faces, {mesh.nverts} verts, {ncr} crease edges, {nco} corners -> {out.nfaces} quads, "
          f"{out.nverts} verts ({a.scheme.upper()}, {a.levels} levels) in {time.perf_counter() - t0:.2f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
