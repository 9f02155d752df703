"""Seeded synthetic control meshes (ctypes front end of ``csrc/meshgen.cpp``).

The named workloads are the five evaluation configurations of this project:

* ``torus32``      32x32 quad torus, R=1, r=0.3, jitter +-0.01; SLAK, 3 levels
* ``icosphere``    frequency-8 geodesic sphere (1280 tris, 642 verts), radial
                   noise N(0, 0.02); LAK and SLAK, 4 levels
* ``mixed512``     512x512 torus, 5% of adjacent pairs merged, 3% of quads split,
                   jitter +-0.005; 4 levels (~67 M output quads)
* ``batch2000``    2000 meshes, faces log-uniform in [100, 200000], 40% tori,
                   30% icospheres, 30% merged/split tori, levels U{1..4}
* ``cylinder``     capped cylinder 64 segments x 32 rings, valence-64 poles,
                   jitter +-0.001; 7 levels
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os
from typing import List

import numpy as np

from . import _paths
from .mesh import Mesh


class _MgMesh(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("is_reduced", ctypes.c_int32),
                ("nfaces", ctypes.c_int64), ("nverts", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("max_face_order", ctypes.c_int64),
                ("ptr", ctypes.POINTER(ctypes.c_int32)), ("ids", ctypes.POINTER(ctypes.c_int32)),
                ("vals", ctypes.POINTER(ctypes.c_int32)), ("verts", ctypes.POINTER(ctypes.c_float))]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_paths.LIB_MESHGEN):
            raise RuntimeError(f"{_paths.LIB_MESHGEN} is missing: run __graft_entry__.build() first")
        lib = ctypes.CDLL(_paths.LIB_MESHGEN)
        d, i, u64, p = ctypes.c_double, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_MgMesh)
        lib.mg_torus.argtypes = [i, i, d, d, d, u64, p]
        lib.mg_icosphere.argtypes = [i, d, u64, p]
        lib.mg_mixed_torus.argtypes = [i, i, d, d, d, d, d, i, u64, p]
        lib.mg_capped_cylinder.argtypes = [i, i, d, u64, p]
        lib.mg_free.argtypes = [p]
        for f in (lib.mg_torus, lib.mg_icosphere, lib.mg_mixed_torus, lib.mg_capped_cylinder):
            f.restype = ctypes.c_int
        _lib = lib
    return _lib


def _take(m: _MgMesh) -> Mesh:
    F, N, V = m.nfaces, m.nnz, m.nverts
    ptr = np.ctypeslib.as_array(m.ptr, shape=(F + 1,)).copy()
    ids = np.ctypeslib.as_array(m.ids, shape=(N,)).copy()
    vals = np.ctypeslib.as_array(m.vals, shape=(N,)).copy()
    verts = np.ctypeslib.as_array(m.verts, shape=(V * 4,)).copy().reshape(V, 4)
    out = Mesh(int(m.type), ids, verts, ptr, vals, int(F), int(m.max_face_order), True)
    _load().mg_free(ctypes.byref(m))
    return out


def _call(fn, *args) -> Mesh:
    m = _MgMesh()
    rc = fn(*args, ctypes.byref(m))
    if rc != 0:
        raise ValueError(f"mesh generator failed with code {rc}")
    return _take(m)


def torus(W: int, H: int, R: float = 1.0, r: float = 0.3, jitter: float = 0.01, seed: int = 1) -> Mesh:
    return _call(_load().mg_torus, W, H, R, r, jitter, seed)


def icosphere(freq: int, sigma: float = 0.02, seed: int = 2) -> Mesh:
    return _call(_load().mg_icosphere, freq, sigma, seed)


def mixed_torus(W: int, H: int, merge: float = 0.05, split: float = 0.03, jitter: float = 0.005,
                seed: int = 3, R: float = 1.0, r: float = 0.3, max_group: int = 3) -> Mesh:
    return _call(_load().mg_mixed_torus, W, H, R, r, merge, split, jitter, max_group, seed)


def capped_cylinder(segs: int = 64, rings: int = 32, jitter: float = 0.001, seed: int = 5) -> Mesh:
    return _call(_load().mg_capped_cylinder, segs, rings, jitter, seed)


def open_grid(W: int, H: int, jitter: float = 0.005, seed: int = 16) -> Mesh:
    """A flat W x H quad patch with height noise: an open mesh, its boundary a
    single loop of 2(W+H) edges (the boundary rules of both schemes)."""
    from .mesh import from_arrays
    if W < 1 or H < 1:
        raise ValueError(f"open_grid: W and H must be at least 1, got {W} x {H}")
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(W + 1), np.arange(H + 1), indexing="ij")
    xyz = np.stack([i.ravel() / W, j.ravel() / H, jitter * rng.standard_normal(i.size)], 1)
    vid = lambda a, b: a * (H + 1) + b
    a, b = np.meshgrid(np.arange(W), np.arange(H), indexing="ij")
    a, b = a.ravel(), b.ravel()
    faces = np.stack([vid(a, b), vid(a + 1, b), vid(a + 1, b + 1), vid(a, b + 1)], 1)
    return from_arrays(np.arange(W * H + 1) * 4, faces.reshape(-1), xyz.astype(np.float32))


@dataclasses.dataclass
class Workload:
    name: str
    mesh: Mesh
    levels: int
    schemes: tuple


def workload(name: str) -> Workload:
    if name == "torus32":
        return Workload(name, torus(32, 32, 1.0, 0.3, 0.01, seed=11), 3, (1,))
    if name == "icosphere":
        return Workload(name, icosphere(8, 0.02, seed=12), 4, (0, 1))
    if name == "mixed512":
        return Workload(name, mixed_torus(512, 512, 0.05, 0.03, 0.005, seed=13), 4, (1, 0))
    if name == "cylinder":
        return Workload(name, capped_cylinder(64, 32, 0.001, seed=15), 7, (1, 0))
    if name == "grid512":           # an open mesh (boundary rules), beside the closed configurations
        return Workload(name, open_grid(512, 512), 4, (1, 0))
    raise KeyError(name)


@dataclasses.dataclass
class BatchItem:
    kind: str        # "torus" | "icosphere" | "mixed"
    faces: int       # requested face count
    levels: int
    seed: int
    params: tuple


def batch_specs(count: int = 2000, seed: int = 14, fmin: int = 100, fmax: int = 200000) -> List[BatchItem]:
    """The seeded mesh list of the batched workload (no geometry generated yet)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        faces = int(round(math.exp(rng.uniform(math.log(fmin), math.log(fmax)))))
        u = rng.uniform()
        kind = "torus" if u < 0.4 else ("icosphere" if u < 0.7 else "mixed")
        levels = int(rng.integers(1, 5))
        s = int(rng.integers(1, 2**62))
        if kind == "icosphere":
            params = (max(1, int(round(math.sqrt(faces / 20.0)))),)
        else:
            a = rng.uniform(1.0, 4.0)
            H = max(4, int(round(math.sqrt(faces / a))))
            W = max(4, int(round(faces / H)))
            params = (W, H)
        out.append(BatchItem(kind, faces, levels, s, params))
    return out


def batch_mesh(item: BatchItem) -> Mesh:
    if item.kind == "torus":
        return torus(item.params[0], item.params[1], 1.0, 0.3, 0.005, seed=item.seed)
    if item.kind == "icosphere":
        return icosphere(item.params[0], 0.02, seed=item.seed)
    return mixed_torus(item.params[0], item.params[1], 0.05, 0.03, 0.005, seed=item.seed)
