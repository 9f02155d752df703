"""Recipe: compile GPUPeople/SLAK's own CUDA sources for sm_100a, and its
driver program against this repository's drop-in headers.

TEST / BASELINE INFRASTRUCTURE ONLY.  The reference's files are compiled
where they lie (never copied); outputs go to oracle/_ref/ only.  The
reference's own CMake build (arch 61;75) is not used: its two scheme sources
are compiled directly, with ref_shim.h force-included to stand in for the
legacy texture reference CUDA 12 removed (used only by the disabled
EXPLICIT_MAP_LOOKUP multiply of LibInclude/device/math/spgemm.cuh).

    python oracle/build_ref.py REFERENCE_DIR       (or $SLAK_REFERENCE_ROOT)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(ref_root: str, out_dir: str, nvcc: str = "nvcc", verbose: bool = False, force: bool = False):
    srcs = [os.path.join(ref_root, "LibSource", "device", "CatmullClarkImpl.cu"),
            os.path.join(ref_root, "LibSource", "device", "LAKCatmullClarkImpl.cu"),
            os.path.join(HERE, "ref_harness.cu")]
    for s in srcs:
        if not os.path.exists(s):
            raise FileNotFoundError(s)
    os.makedirs(out_dir, exist_ok=True)
    target = os.path.join(out_dir, "libslak_ref.so")
    deps = srcs + [os.path.join(HERE, "ref_shim.h")]
    if not force and os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target) for d in deps):
        return target
    inc = ["-I", os.path.join(ref_root, "LibInclude", "device"), "-I", os.path.join(ref_root, "LibInclude")]
    flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
             "-include", os.path.join(HERE, "ref_shim.h"), "-w"]
    objs = []
    for s in srcs:
        o = os.path.join(out_dir, os.path.basename(s) + ".o")
        cmd = [nvcc] + flags + inc + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"compiling {s} failed")
        objs.append(o)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", target] + objs + ["-lcusparse"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("linking the reference failed")
    for o in objs:
        os.remove(o)
    return target


def build_dropin_main(ref_root: str, out_dir: str, include_dir: str, lib_dir: str, cuda_home: str = "/usr/local/cuda",
                      cxx: str = "g++", verbose: bool = False, force: bool = False):
    """The reference's own driver (source/main.cpp), compiled unchanged against
    this repository's drop-in headers (include/CatmullClark.h,
    include/LAKCatmullClark.h, found first on the include path) and linked
    with libslak_b200.so instead of the reference's library.  Its mesh I/O
    headers (include/Mesh.h, include/obj.h, LibInclude/cuda_host_helpers.h,
    LibInclude/math/) are the reference's, read where they lie."""
    src = os.path.join(ref_root, "source", "main.cpp")
    lib = os.path.join(lib_dir, "libslak_b200.so")
    for f in (src, lib):
        if not os.path.exists(f):
            raise FileNotFoundError(f)
    os.makedirs(out_dir, exist_ok=True)
    target = os.path.join(out_dir, "slak_main_dropin")
    deps = [src, lib, os.path.join(include_dir, "CatmullClark.h"), os.path.join(include_dir, "LAKCatmullClark.h")]
    if not force and os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target) for d in deps):
        return target
    rel = os.path.relpath(lib_dir, out_dir)
    cmd = [cxx, "-std=c++17", "-O2", "-w", "-I", include_dir, "-I", os.path.join(ref_root, "include"),
           "-I", os.path.join(ref_root, "LibInclude"), "-I", os.path.join(cuda_home, "include"), src,
           "-L", lib_dir, "-lslak_b200", "-L", os.path.join(cuda_home, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN/" + rel, "-Wl,-rpath," + os.path.join(cuda_home, "lib64"), "-o", target]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("compiling the reference's main.cpp against the drop-in headers failed")
    return target


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLAK_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: python oracle/build_ref.py REFERENCE_DIR (or set SLAK_REFERENCE_ROOT)")
    print(build(root, os.path.join(HERE, "_ref"), verbose=True, force=True))
    repo = os.path.dirname(HERE)
    print(build_dropin_main(root, os.path.join(HERE, "_ref"), os.path.join(repo, "include"),
                            os.path.join(repo, "slak_b200", "lib"), verbose=True, force=True))
