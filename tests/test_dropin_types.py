"""The drop-in headers carry the reference's public nested types, so host code
that names them compiles: Context<MESH_INFO>, ProfilinInfo<PROFILER,
MEM_MANAGER> and MeshInfo::freeAndReset(MEM_MANAGER&) of both schemes
(LibInclude/CatmullClark.h:38-67,108-129, LibInclude/LAKCatmullClark.h:38-83).
tests/dropin_types.cpp is compiled with g++ against include/ and run on the
CPU; its memory manager is a fake, so no GPU is touched."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(os.path.join(CUDA, "include")),
                    reason="g++ and the CUDA headers are needed")
def test_reference_nested_types_compile_and_free_through_the_manager(tmp_path):
    exe = tmp_path / "dropin_types"
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(HERE, "dropin_types.cpp"),
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64"),
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")      # the fallback cudaFree must find no device
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "CatmullClark: ok (fallback threw)" in r.stdout
    assert "LAKCatmullClark: ok (fallback threw)" in r.stdout
