"""Builds the in-tree shared libraries.

* ``slak_b200/lib/libslak_b200.so``    CUDA product library (C ABI of include/slak_b200.h),
                                        sm_100a only, IEEE float (no FMA contraction)
* ``slak_b200/lib/libslak_meshgen.so`` host mesh generators
* ``slak_b200/lib/slak_demo``           drop-in demo: include/CatmullClark.h callers
* ``oracle/_build/libslak_oracle.so``  CPU restatement (test infrastructure)
* ``oracle/_ref/libslak_ref.so``       the reference's own CUDA sources compiled for
                                        sm_100a (only where the reference tree exists)

Run ``python -m slak_b200.build`` or ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

from . import _paths

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _csrc(*names):
    return [os.path.join(_paths.CSRC_DIR, n) for n in names]


def build_cuda(verbose=False, force=False, extra=None):
    os.makedirs(_paths.LIB_DIR, exist_ok=True)
    srcs = _csrc("slak_abi.cu") + _csrc("objio.cpp")
    deps = srcs + [os.path.join(_paths.CSRC_DIR, f) for f in os.listdir(_paths.CSRC_DIR)
                   if f.endswith((".cuh", ".h"))] + [os.path.join(_paths.INCLUDE_DIR, "slak_b200.h")]
    if not force and not _stale(_paths.LIB_SLAK, deps):
        return _paths.LIB_SLAK
    cmd = [NVCC] + CUDA_FLAGS + (extra or []) + ["-shared", "-I", _paths.INCLUDE_DIR, "-I", _paths.CSRC_DIR,
                                                 "-o", _paths.LIB_SLAK] + srcs
    _run(cmd, verbose)
    return _paths.LIB_SLAK


def build_meshgen(verbose=False, force=False):
    os.makedirs(_paths.LIB_DIR, exist_ok=True)
    src = _csrc("meshgen.cpp")
    if force or _stale(_paths.LIB_MESHGEN, src):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", _paths.LIB_MESHGEN] + src, verbose)
    return _paths.LIB_MESHGEN


def build_demo(verbose=False, force=False):
    """Links a small C++ program written against include/CatmullClark.h and
    include/LAKCatmullClark.h (the reference's headers' API) to the C ABI."""
    src = _csrc("demo_main.cpp")
    if not os.path.exists(src[0]):
        return None
    hdrs = [os.path.join(_paths.INCLUDE_DIR, h) for h in ("CatmullClark.h", "LAKCatmullClark.h", "slak_b200.h")]
    if force or _stale(_paths.DEMO_BIN, src + hdrs + [_paths.LIB_SLAK, _paths.LIB_MESHGEN]):
        cmd = [NVCC, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-I", _paths.INCLUDE_DIR, "-o", _paths.DEMO_BIN] + src + [
            "-L", _paths.LIB_DIR, "-lslak_b200", "-lslak_meshgen", "-Xlinker", "-rpath=$ORIGIN"]
        _run(cmd, verbose)
    return _paths.DEMO_BIN


def build_oracle(verbose=False, force=False):
    odir = os.path.join(_paths.REPO_DIR, "oracle")
    src = [os.path.join(odir, "slak_oracle.c")]
    hdr = [os.path.join(odir, "slak_oracle.h")]
    os.makedirs(os.path.dirname(_paths.LIB_ORACLE), exist_ok=True)
    if force or _stale(_paths.LIB_ORACLE, src + hdr):
        _run(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              "-fno-fast-math", "-o", _paths.LIB_ORACLE] + src, verbose)
    return _paths.LIB_ORACLE


def build_reference(verbose=False, force=False, ref_root=None):
    """Compiles the reference's CUDA sources (never copied) with oracle/build_ref.py,
    and the reference's driver against the drop-in headers (oracle/_ref/slak_main_dropin).
    The reference tree is `ref_root`, else $SLAK_REFERENCE_ROOT; with neither
    (or no such directory) nothing is built and None is returned."""
    ref_root = ref_root or os.environ.get("SLAK_REFERENCE_ROOT")
    if not ref_root or not os.path.isdir(ref_root):
        return None
    sys.path.insert(0, _paths.REPO_DIR)
    try:
        from oracle import build_ref
    finally:
        sys.path.pop(0)
    out = build_ref.build(ref_root, os.path.dirname(_paths.LIB_REF), nvcc=NVCC, verbose=verbose, force=force)
    build_ref.build_dropin_main(ref_root, os.path.dirname(_paths.LIB_REF), _paths.INCLUDE_DIR, _paths.LIB_DIR,
                                verbose=verbose, force=force)
    return out


def build_all(verbose=False, force=False, ref_root=None):
    build_meshgen(verbose, force)
    build_cuda(verbose, force)
    build_demo(verbose, force)
    build_oracle(verbose, force)
    build_reference(verbose, force, ref_root)


if __name__ == "__main__":
    # python -m slak_b200.build [-v] [-f] [--reference DIR]
    ref = sys.argv[sys.argv.index("--reference") + 1] if "--reference" in sys.argv else None
    build_all(verbose="-v" in sys.argv, force="-f" in sys.argv, ref_root=ref)
    print("built:", _paths.LIB_SLAK)
