"""Host-side mesh container mirroring ``MeshInfo<int,int,int,float>``.

The reference describes a control mesh by a face-vertex incidence matrix in
CSC form (one column per face): ``ptr`` (F+1 face offsets), ``ids`` (N corner
vertex ids), ``vals`` (N 1-based corner positions) and ``verts`` (float4
positions, w = 1); see ``LibInclude/CatmullClark.h:69-130`` and
``include/Mesh.h:153-176`` of GPUPeople/SLAK.  This class holds the same
arrays as numpy arrays on the host.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

TRI, QUAD, POLY = 0, 1, 2          # MeshInfo::MeshType order (CatmullClark.h:72)
LAK, SLAK = 0, 1                   # scheme ids of source/main.cpp:89-104


@dataclasses.dataclass
class Mesh:
    type: int
    ids: np.ndarray                        # int32 [N]
    verts: np.ndarray                      # float32 [V, 4]
    ptr: Optional[np.ndarray] = None       # int32 [F+1]
    vals: Optional[np.ndarray] = None      # int32 [N]
    nfaces: int = 0
    max_face_order: int = 0
    is_reduced: bool = True

    def __post_init__(self):
        # the C ABI reads int32 indices and float32 x 4 positions: arrays of
        # other types are converted here, never reinterpreted
        def i32(a, name):
            if a is None:
                return None
            a = np.asarray(a)
            if a.dtype != np.int32:
                if a.size and (a.min() < np.iinfo(np.int32).min or a.max() > np.iinfo(np.int32).max):
                    raise ValueError(f"{name}: values do not fit 32-bit indices")
                a = a.astype(np.int32)
            return np.ascontiguousarray(a)
        self.ids = i32(self.ids, "ids")
        self.ptr = i32(self.ptr, "ptr")
        self.vals = i32(self.vals, "vals")
        v = np.asarray(self.verts)
        if v.ndim != 2 or v.shape[1] != 4:
            raise ValueError(f"verts: expected shape (V, 4), got {v.shape}")
        self.verts = np.ascontiguousarray(v, dtype=np.float32)

    @property
    def nnz(self) -> int:
        return int(self.ids.shape[0])

    @property
    def nverts(self) -> int:
        return int(self.verts.shape[0])

    def face_orders(self) -> np.ndarray:
        if self.ptr is None:
            return np.full(self.nfaces, 4, dtype=np.int32)
        return np.diff(self.ptr).astype(np.int32)

    def bbox_diag(self) -> float:
        xyz = self.verts[:, :3].astype(np.float64)
        if xyz.shape[0] == 0:
            return 0.0
        return float(np.linalg.norm(xyz.max(0) - xyz.min(0)))

    def copy(self) -> "Mesh":
        return Mesh(self.type, self.ids.copy(), self.verts.copy(),
                    None if self.ptr is None else self.ptr.copy(),
                    None if self.vals is None else self.vals.copy(),
                    self.nfaces, self.max_face_order, self.is_reduced)

    def with_quad_ptr(self) -> "Mesh":
        """Adds explicit quad ``ptr``/``vals`` (what LAK expects on quad levels)."""
        m = self.copy()
        if m.ptr is None:
            m.ptr = (np.arange(m.nfaces + 1, dtype=np.int64) * 4).astype(np.int32)
        if m.vals is None:
            orders = np.diff(m.ptr)
            starts = np.repeat(m.ptr[:-1], orders)
            m.vals = (np.arange(m.nnz, dtype=np.int64) - starts + 1).astype(np.int32)
        if m.max_face_order == 0:
            m.max_face_order = int(np.diff(m.ptr).max()) if m.nfaces else 0
        return m


def from_arrays(ptr: np.ndarray, ids: np.ndarray, verts_xyz: np.ndarray) -> Mesh:
    """Builds a Mesh from face offsets, corner ids and xyz (w is set to 1)."""
    ptr = np.ascontiguousarray(ptr, dtype=np.int32)
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    v = np.ones((verts_xyz.shape[0], 4), dtype=np.float32)
    v[:, :3] = verts_xyz
    orders = np.diff(ptr)
    if orders.size and orders.min() == orders.max() == 4:
        t = QUAD
    elif orders.size and orders.min() == orders.max() == 3:
        t = TRI
    else:
        t = POLY
    starts = np.repeat(ptr[:-1], orders)
    vals = (np.arange(ids.shape[0], dtype=np.int64) - starts + 1).astype(np.int32)
    return Mesh(t, ids, v, ptr, vals, int(ptr.shape[0] - 1), int(orders.max()) if orders.size else 0)
