"""ctypes bindings of oracle/_ref/libslak_ref.so: the reference's own CUDA path.

TEST / BASELINE INFRASTRUCTURE ONLY: pins the oracle against the real
reference on a GPU and times the reference arm of bench.py.  The library is
built by oracle/build_ref.py from the reference's sources.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libslak_ref.so")


class RefMesh(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("is_reduced", ctypes.c_int32),
                ("nfaces", ctypes.c_int64), ("nverts", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("max_face_order", ctypes.c_int64),
                ("ptr", ctypes.POINTER(ctypes.c_int32)), ("ids", ctypes.POINTER(ctypes.c_int32)),
                ("vals", ctypes.POINTER(ctypes.c_int32)), ("verts", ctypes.POINTER(ctypes.c_float))]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} missing: the reference was not built (oracle/build_ref.py)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(RefMesh)
        L.ref_run.argtypes = [ctypes.c_int, P, ctypes.c_int, P, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        L.ref_time.argtypes = [ctypes.c_int, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        L.ref_time_e2e.argtypes = [ctypes.c_int, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64),
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.ref_time_e2e.restype = ctypes.c_int
        L.ref_free.argtypes = [P]
        L.ref_run.restype = L.ref_time.restype = ctypes.c_int
        _lib = L
    return _lib


def _in(mesh, keep):
    def p(a, ct):
        if a is None:
            return None
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ct))
    m = RefMesh()
    m.type, m.is_reduced = mesh.type, int(mesh.is_reduced)
    m.nfaces, m.nverts, m.nnz, m.max_face_order = mesh.nfaces, mesh.nverts, mesh.nnz, mesh.max_face_order
    ptr = mesh.ptr if mesh.ptr is not None else (np.arange(mesh.nfaces + 1) * 4).astype(np.int32)
    m.ptr = p(ptr.astype(np.int32), ctypes.c_int32)
    m.ids = p(mesh.ids.astype(np.int32), ctypes.c_int32)
    m.vals = p(None if mesh.vals is None else mesh.vals.astype(np.int32), ctypes.c_int32)
    m.verts = p(mesh.verts.astype(np.float32).reshape(-1), ctypes.c_float)
    return m


class RefResult:
    def __init__(self, m: RefMesh, self_ms: float):
        F, N, V = m.nfaces, m.nnz, m.nverts
        self.type, self.nfaces, self.nnz, self.nverts = int(m.type), int(F), int(N), int(V)
        self.max_face_order, self.is_reduced = int(m.max_face_order), bool(m.is_reduced)
        self.ids = np.ctypeslib.as_array(m.ids, shape=(N,)).copy() if m.ids else None
        self.verts = np.ctypeslib.as_array(m.verts, shape=(4 * V,)).copy().reshape(V, 4) if m.verts else None
        self.ptr = np.ctypeslib.as_array(m.ptr, shape=(F + 1,)).copy() if m.ptr else None
        self.vals = np.ctypeslib.as_array(m.vals, shape=(N,)).copy() if m.vals else None
        self.self_ms = self_ms


def run(mesh, levels: int, scheme: int, quiet: bool = True) -> RefResult:
    keep = []
    cin = _in(mesh, keep)
    out = RefMesh()
    ms = ctypes.c_float(-1)
    rc = lib().ref_run(scheme, ctypes.byref(cin), levels, ctypes.byref(out), ctypes.byref(ms), int(quiet))
    if rc != 0:
        lib().ref_free(ctypes.byref(out))
        raise RuntimeError(f"reference run failed with code {rc}")
    res = RefResult(out, ms.value)
    lib().ref_free(ctypes.byref(out))
    return res


def time(mesh, levels: int, scheme: int, warmup: int, reps: int, quiet: bool = True):
    """Per-call device time (ms, CUDA events around subdivideIteratively) and the
    reference's own printed time, on device-resident input."""
    keep = []
    cin = _in(mesh, keep)
    ms = (ctypes.c_double * reps)()
    self_ms = (ctypes.c_float * reps)()
    rc = lib().ref_time(scheme, ctypes.byref(cin), levels, warmup, reps, ms, self_ms, int(quiet))
    if rc != 0:
        raise RuntimeError(f"reference timing failed with code {rc}")
    return list(ms), list(self_ms)


def time_e2e(mesh, levels: int, scheme: int, warmup: int, reps: int, quiet: bool = True):
    """Per-call wall time (ms) with host buffers: pinned H2D of the input,
    subdivideIteratively, D2H of the refined ids and positions.  Returns
    (ms list, h2d bytes, d2h bytes)."""
    keep = []
    cin = _in(mesh, keep)
    ms = (ctypes.c_double * reps)()
    hb, db = ctypes.c_int64(0), ctypes.c_int64(0)
    rc = lib().ref_time_e2e(scheme, ctypes.byref(cin), levels, warmup, reps, ms, ctypes.byref(hb),
                            ctypes.byref(db), int(quiet))
    if rc != 0:
        raise RuntimeError(f"reference end-to-end timing failed with code {rc}")
    return list(ms), int(hb.value), int(db.value)
