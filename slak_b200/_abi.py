"""ctypes declarations of the C ABI in include/slak_b200.h.

Loading fails loudly when the CUDA library has not been built: there is no
CPU fallback in this package.
"""
from __future__ import annotations

import ctypes
import os

from . import _paths

SLAK_OK = 0
SLAK_ERR_INVALID_ARG, SLAK_ERR_CUDA, SLAK_ERR_OOM, SLAK_ERR_BAD_MESH = 1, 2, 3, 4
SLAK_ERR_TIMEOUT, SLAK_ERR_UNSUPPORTED, SLAK_ERR_NOT_READY = 5, 6, 7
STATUS_NAMES = {0: "SLAK_OK", 1: "SLAK_ERR_INVALID_ARG", 2: "SLAK_ERR_CUDA", 3: "SLAK_ERR_OOM",
                4: "SLAK_ERR_BAD_MESH", 5: "SLAK_ERR_TIMEOUT", 6: "SLAK_ERR_UNSUPPORTED", 7: "SLAK_ERR_NOT_READY"}

PLAN_GRAPH, PLAN_GENERAL, PLAN_COMPENSATED, PLAN_TIMING, PLAN_AUTOTUNE, PLAN_GQ, PLAN_BULK_RECORDS = (
    1, 2, 4, 8, 16, 32, 64)

# SLAK_B200_ABI_VERSION of include/slak_b200.h, which the structs and signatures here follow
ABI_VERSION = 1

# every symbol include/slak_b200.h declares
EXPORTS = ["slak_status_string", "slak_abi_version", "slak_last_error_detail", "slak_subdivide", "slak_mesh_free",
           "slak_workspace_release", "slak_subdivide_level_noalloc", "slak_obj_read", "slak_obj_write",
           "slak_obj_free", "slak_obj_read_creased", "slak_obj_write_creased", "slak_obj_free_creases",
           "slak_obj_read_sharp", "slak_obj_write_sharp", "slak_obj_free_corners",
           "slak_plan_create", "slak_plan_create_creased", "slak_subdivide_creased", "slak_plan_create_sharp",
           "slak_subdivide_sharp",
           "slak_plan_execute", "slak_plan_status", "slak_plan_output", "slak_plan_release_output",
           "slak_plan_num_levels", "slak_plan_level_stats", "slak_plan_launches", "slak_plan_kernel_timings",
           "slak_plan_tuning", "slak_autotune_reset",
           "slak_plan_destroy", "slak_subdivide_batched", "slak_batch_create", "slak_batch_execute", "slak_batch_status", "slak_batch_output",
           "slak_batch_num_waves", "slak_batch_num_groups", "slak_batch_launches", "slak_batch_destroy"]


class SlakCorners(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int64), ("verts", ctypes.POINTER(ctypes.c_int32)),
                ("sharpness", ctypes.POINTER(ctypes.c_float))]


class SlakCreases(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int64), ("verts", ctypes.POINTER(ctypes.c_int32)),
                ("sharpness", ctypes.POINTER(ctypes.c_float))]


class SlakMesh(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("is_reduced", ctypes.c_int32),
                ("nfaces", ctypes.c_int64), ("nverts", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("max_face_order", ctypes.c_int64),
                ("ptr", ctypes.c_void_p), ("ids", ctypes.c_void_p),
                ("vals", ctypes.c_void_p), ("verts", ctypes.c_void_p)]


class LevelStats(ctypes.Structure):
    _fields_ = [("nfaces", ctypes.c_int64), ("nverts", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("nedges", ctypes.c_int64), ("nboundary", ctypes.c_int64),
                ("out_faces", ctypes.c_int64), ("out_verts", ctypes.c_int64),
                ("algorithmic_bytes", ctypes.c_int64)]


class KernelTiming(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("level", ctypes.c_int32), ("ms", ctypes.c_float),
                ("algorithmic_bytes", ctypes.c_int64)]


class Tuning(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("block", ctypes.c_int32 * 3), ("ms", (ctypes.c_float * 3) * 3),
                ("key", ctypes.c_char * 64)]


class SlakError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        try:
            detail = lib().slak_last_error_detail().decode()
        except Exception:
            detail = ""
        super().__init__(f"{what}: {STATUS_NAMES.get(code, code)} ({status_string(code)}) {detail}")


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_paths.LIB_SLAK):
            raise RuntimeError(f"CUDA library {_paths.LIB_SLAK} is missing: run __graft_entry__.build(); "
                               "slak_b200 has no CPU fallback")
        L = ctypes.CDLL(_paths.LIB_SLAK)
        P, V, I, I64 = ctypes.POINTER(SlakMesh), ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        L.slak_status_string.argtypes = [I]
        L.slak_status_string.restype = ctypes.c_char_p
        L.slak_abi_version.restype = I
        L.slak_last_error_detail.restype = ctypes.c_char_p
        L.slak_subdivide.argtypes = [P, P, I, I, V]
        L.slak_mesh_free.argtypes = [P]
        L.slak_obj_read.argtypes = [ctypes.c_char_p, P]
        L.slak_obj_write.argtypes = [ctypes.c_char_p, P]
        L.slak_obj_free.argtypes = [P]
        PC = ctypes.POINTER(SlakCreases)
        L.slak_obj_read_creased.argtypes = [ctypes.c_char_p, P, PC]
        L.slak_obj_write_creased.argtypes = [ctypes.c_char_p, P, PC]
        L.slak_obj_free_creases.argtypes = [PC]
        PK = ctypes.POINTER(SlakCorners)
        L.slak_obj_read_sharp.argtypes = [ctypes.c_char_p, P, PC, PK]
        L.slak_obj_write_sharp.argtypes = [ctypes.c_char_p, P, PC, PK]
        L.slak_obj_free_corners.argtypes = [PK]
        for n in ("slak_obj_read", "slak_obj_write", "slak_obj_free", "slak_obj_read_creased", "slak_obj_write_creased",
                  "slak_obj_free_creases", "slak_obj_read_sharp", "slak_obj_write_sharp", "slak_obj_free_corners"):
            getattr(L, n).restype = I
        L.slak_workspace_release.argtypes = []
        L.slak_workspace_release.restype = I
        L.slak_subdivide_level_noalloc.argtypes = [P, P, I, V]
        L.slak_plan_create.argtypes = [P, I, I, I, V, ctypes.POINTER(V)]
        L.slak_plan_create_creased.argtypes = [P, I, I, I, V, V, I64, V, ctypes.POINTER(V)]
        L.slak_subdivide_creased.argtypes = [P, P, I, I, V, V, I64, V]
        L.slak_plan_create_sharp.argtypes = [P, I, I, I, V, V, I64, V, V, I64, V, ctypes.POINTER(V)]
        L.slak_subdivide_sharp.argtypes = [P, P, I, I, V, V, I64, V, V, I64, V]
        L.slak_plan_execute.argtypes = [V, V]
        L.slak_plan_status.argtypes = [V, V]
        L.slak_plan_output.argtypes = [V, P]
        L.slak_plan_release_output.argtypes = [V, P]
        L.slak_plan_num_levels.argtypes = [V]
        L.slak_plan_level_stats.argtypes = [V, I, ctypes.POINTER(LevelStats)]
        L.slak_plan_launches.argtypes = [V]
        L.slak_plan_launches.restype = I64
        L.slak_plan_destroy.argtypes = [V]
        L.slak_plan_kernel_timings.argtypes = [V, ctypes.POINTER(KernelTiming), I]
        L.slak_plan_kernel_timings.restype = I
        L.slak_plan_tuning.argtypes = [V, I, ctypes.POINTER(Tuning)]
        L.slak_plan_tuning.restype = I
        L.slak_autotune_reset.argtypes = []
        L.slak_autotune_reset.restype = I
        L.slak_batch_create.argtypes = [P, ctypes.POINTER(ctypes.c_int), I64, I, I, V, ctypes.POINTER(V)]
        L.slak_subdivide_batched.argtypes = [P, ctypes.POINTER(ctypes.c_int), I64, I, P, V]
        L.slak_subdivide_batched.restype = I
        L.slak_batch_execute.argtypes = [V, V]
        L.slak_batch_status.argtypes = [V, V]
        L.slak_batch_output.argtypes = [V, I64, P]
        L.slak_batch_num_waves.argtypes = [V]
        L.slak_batch_num_groups.argtypes = [V]
        L.slak_batch_launches.argtypes = [V]
        L.slak_batch_launches.restype = I64
        L.slak_batch_destroy.argtypes = [V]
        for n in ("slak_batch_create", "slak_batch_execute", "slak_batch_status", "slak_batch_output",
                  "slak_batch_num_waves", "slak_batch_num_groups", "slak_batch_destroy"):
            getattr(L, n).restype = I
        for n in ("slak_subdivide", "slak_mesh_free", "slak_subdivide_level_noalloc", "slak_plan_create",
                  "slak_plan_create_creased", "slak_subdivide_creased", "slak_plan_create_sharp",
                  "slak_subdivide_sharp", "slak_plan_execute", "slak_plan_status",
                  "slak_plan_output", "slak_plan_release_output", "slak_plan_num_levels",
                  "slak_plan_level_stats", "slak_plan_destroy"):
            getattr(L, n).restype = I
        if L.slak_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{_paths.LIB_SLAK} has ABI version {L.slak_abi_version()}, these bindings "
                               f"expect {ABI_VERSION}: rebuild it with __graft_entry__.build()")
        _lib = L
    return _lib


def status_string(code: int) -> str:
    try:
        return lib().slak_status_string(code).decode()
    except RuntimeError:
        return "library not loaded"


def check(code: int, what: str):
    if code != SLAK_OK:
        raise SlakError(code, what)
