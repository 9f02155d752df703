"""The C ABI library loads without a GPU and exports what include/slak_b200.h declares."""
import ctypes
import os
import re

import pytest

from slak_b200 import _abi, _paths


def _declared():
    src = open(os.path.join(_paths.INCLUDE_DIR, "slak_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(slak_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from slak_b200 import build
    build.build_cuda()
    return _abi.lib()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 12
    assert sorted(names) == sorted(_abi.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_status_strings(lib):
    hdr = open(os.path.join(_paths.INCLUDE_DIR, "slak_b200.h")).read()
    declared = int(re.search(r"#define SLAK_B200_ABI_VERSION (\d+)", hdr).group(1))
    assert lib.slak_abi_version() == declared == _abi.ABI_VERSION
    for code in range(0, 8):
        s = _abi.status_string(code)
        assert s and s != "unknown status"
    assert _abi.status_string(99) == "unknown status"


def test_invalid_arguments_rejected_before_cuda(lib):
    h = ctypes.c_void_p()
    assert lib.slak_plan_create(None, 1, 1, 0, None, ctypes.byref(h)) == _abi.SLAK_OK + 1
    m = _abi.SlakMesh()
    m.type, m.nfaces, m.nnz, m.nverts = 1, 1, 4, 4
    assert lib.slak_plan_create(ctypes.byref(m), 1, 7, 0, None, ctypes.byref(h)) == 1      # bad scheme
    m.ids = None
    assert lib.slak_plan_create(ctypes.byref(m), 1, 1, 0, None, ctypes.byref(h)) == 1      # no ids
    m.type = 2
    assert lib.slak_plan_create(ctypes.byref(m), 1, 1, 0, None, ctypes.byref(h)) == 1      # poly without ptr
    assert lib.slak_subdivide(None, None, 1, 1, None) == 1
    assert lib.slak_mesh_free(None) == 1
    assert lib.slak_plan_destroy(None) == 0
    assert lib.slak_plan_num_levels(None) == 0


def test_meshgen_and_oracle_libraries_load():
    import oracle
    from slak_b200 import meshgen
    assert oracle.num_threads() >= 1
    assert meshgen.torus(4, 4).nfaces == 16


def test_every_entry_point_checks_its_arguments_first(lib):
    """Null handles, negative counts and unknown schemes give
    SLAK_ERR_INVALID_ARG before any CUDA call (this runs with no GPU); the
    destroy calls accept null, as free() does."""
    m = _abi.SlakMesh()
    m.type, m.nfaces, m.nnz, m.nverts = 1, 1, 4, 4
    out = _abi.SlakMesh()
    lv = (ctypes.c_int * 1)(1)
    h = ctypes.c_void_p()
    M, O = ctypes.byref(m), ctypes.byref(out)
    calls = [
        lambda: lib.slak_subdivide_batched(None, lv, 1, 1, O, None),
        lambda: lib.slak_subdivide_batched(M, lv, -1, 1, O, None),
        lambda: lib.slak_subdivide_batched(M, lv, 1, 9, O, None),
        lambda: lib.slak_batch_create(None, lv, 1, 1, 0, None, ctypes.byref(h)),
        lambda: lib.slak_batch_create(M, lv, 1, 1, 0, None, None),
        lambda: lib.slak_subdivide_level_noalloc(None, None, 1, None),
        lambda: lib.slak_subdivide_level_noalloc(M, O, 5, None),
        lambda: lib.slak_plan_create_sharp(M, 1, 1, 0, None, None, -1, None, None, 0, None, ctypes.byref(h)),
        lambda: lib.slak_plan_create_sharp(M, 1, 1, 0, None, None, 3, None, None, 0, None, ctypes.byref(h)),
        lambda: lib.slak_obj_read(None, O),
        lambda: lib.slak_obj_write(None, O),
        lambda: lib.slak_plan_execute(None, None),
        lambda: lib.slak_plan_status(None, None),
        lambda: lib.slak_plan_output(None, O),
        lambda: lib.slak_batch_execute(None, None),
        lambda: lib.slak_batch_status(None, None),
        lambda: lib.slak_batch_output(None, 0, O),
    ]
    for k, call in enumerate(calls):
        assert call() == _abi.SLAK_ERR_INVALID_ARG, k
    assert lib.slak_batch_destroy(None) == 0
