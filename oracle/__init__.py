"""CPU oracle of the SLAK / LAK Catmull-Clark schemes (ctypes bindings).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the CPU
baseline, never as the implementation under measurement.  The product package
``slak_b200`` does not import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libslak_oracle.so")


class OrMesh(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("is_reduced", ctypes.c_int32),
                ("nfaces", ctypes.c_int64), ("nverts", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("max_face_order", ctypes.c_int64),
                ("ptr", ctypes.POINTER(ctypes.c_int32)), ("ids", ctypes.POINTER(ctypes.c_int32)),
                ("vals", ctypes.POINTER(ctypes.c_int32)), ("verts", ctypes.POINTER(ctypes.c_float)),
                ("verts64", ctypes.POINTER(ctypes.c_double))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run __graft_entry__.build() first")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(OrMesh)
        L.or_level.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_subdivide.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_mesh_free.argtypes = [P]
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_level.restype = L.or_subdivide.restype = L.or_num_threads.restype = ctypes.c_int
        L.or_set_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def num_threads() -> int:
    return lib().or_num_threads()


def set_threads(n: int) -> int:
    """Thread count of later calls (n <= 0: the OpenMP default); returns it."""
    return lib().or_set_threads(int(n))


class Result:
    """Oracle output: refined mesh arrays plus optional FP64 positions."""

    def __init__(self, m: OrMesh):
        F, N, V = m.nfaces, m.nnz, m.nverts
        self.type = int(m.type)
        self.nfaces, self.nnz, self.nverts = int(F), int(N), int(V)
        self.max_face_order = int(m.max_face_order)
        self.is_reduced = bool(m.is_reduced)
        self.ids = np.ctypeslib.as_array(m.ids, shape=(N,)).copy() if N else np.zeros(0, np.int32)
        self.ptr = np.ctypeslib.as_array(m.ptr, shape=(F + 1,)).copy() if m.ptr else None
        self.vals = np.ctypeslib.as_array(m.vals, shape=(N,)).copy() if m.vals else None
        self.verts = (np.ctypeslib.as_array(m.verts, shape=(V * 4,)).copy().reshape(V, 4)
                      if V else np.zeros((0, 4), np.float32))
        self.verts64 = (np.ctypeslib.as_array(m.verts64, shape=(V * 4,)).copy().reshape(V, 4)
                        if m.verts64 else None)


def _as_or(mesh, keep):
    def p(a, ct):
        if a is None:
            return None
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ct))
    m = OrMesh()
    m.type = mesh.type
    m.is_reduced = int(mesh.is_reduced)
    m.nfaces, m.nverts, m.nnz = mesh.nfaces, mesh.nverts, mesh.nnz
    m.max_face_order = mesh.max_face_order
    m.ptr = p(None if mesh.ptr is None else mesh.ptr.astype(np.int32), ctypes.c_int32)
    m.ids = p(mesh.ids.astype(np.int32), ctypes.c_int32)
    m.vals = p(None if mesh.vals is None else mesh.vals.astype(np.int32), ctypes.c_int32)
    m.verts = p(mesh.verts.astype(np.float32).reshape(-1), ctypes.c_float)
    v64 = getattr(mesh, "verts64", None)
    m.verts64 = p(None if v64 is None else np.asarray(v64, np.float64).reshape(-1), ctypes.c_double)
    return m


def subdivide(mesh, levels: int, scheme: int, fp64: bool = False) -> Result:
    """Oracle of ``subdivideIteratively`` (scheme 0 = LAK, 1 = SLAK)."""
    keep = []
    cin = _as_or(mesh, keep)
    out = OrMesh()
    rc = lib().or_subdivide(ctypes.byref(cin), ctypes.byref(out), levels, scheme, int(fp64))
    if rc != 0:
        raise ValueError(f"oracle rejected the mesh (code {rc})")
    res = Result(out)
    lib().or_mesh_free(ctypes.byref(out))
    return res


def level(mesh, scheme: int, poly: bool, fp64: bool = False) -> Result:
    """One oracle level (poly=True runs the reference's first-level functions)."""
    keep = []
    cin = _as_or(mesh, keep)
    out = OrMesh()
    rc = lib().or_level(ctypes.byref(cin), ctypes.byref(out), scheme, int(poly), int(fp64))
    if rc != 0:
        raise ValueError(f"oracle rejected the mesh (code {rc})")
    res = Result(out)
    lib().or_mesh_free(ctypes.byref(out))
    return res


class _LevelMesh:
    """Adapter: an oracle Result as the input of the next oracle level."""

    def __init__(self, r: Result):
        self.type, self.is_reduced = r.type, r.is_reduced
        self.nfaces, self.nverts, self.nnz = r.nfaces, r.nverts, r.nnz
        self.max_face_order = r.max_face_order or 4
        self.ptr, self.ids, self.vals = r.ptr, r.ids, r.vals
        self.verts, self.verts64 = r.verts, r.verts64


def subdivide_levels(mesh, levels: int, scheme: int):
    """Every level's oracle result (FP32 and FP64 positions), level 1 first.
    The FP64 shadow of level l feeds level l+1, so level l's verts64 is the
    FP64 evaluation of l levels of the same subdivision matrices."""
    out = []
    cur = mesh
    if getattr(cur, "verts64", None) is None:
        cur = _LevelMesh.__new__(_LevelMesh)
        for f in ("type", "is_reduced", "nfaces", "nverts", "nnz", "max_face_order", "ptr", "ids", "vals", "verts"):
            setattr(cur, f, getattr(mesh, f))
        cur.verts64 = mesh.verts.astype(np.float64)
    for l in range(levels):
        r = level(cur, scheme, poly=(l == 0 and mesh.type != 1), fp64=True)
        out.append(r)
        cur = _LevelMesh(r)
    return out
