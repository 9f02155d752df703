"""Canonical relabelling of a refined mesh's edge points.

The reference numbers edge points in atomicAdd order (SLAK: adjacency slots,
``CatmullClarkKernels.cuh:137-145`` + scan ``CatmullClarkImpl.cu:209-211``;
LAK: a global counter, ``spgemm.cuh:86-87``), so two runs on the same input
may permute every level's edge-point block, and through it the vertex ids of
all later levels.  Face order, face-point ids and original vertex ids are
deterministic.  This module rewrites a refined mesh so that, at every level,
edge point e is the rank of its endpoint pair (min, max) in lexicographic
order.  Two results that differ only by edge numbering then compare equal.

The level history is recovered from the final quads alone: quad q of level
l+1 is corner q of level l and starts with that corner's vertex, so the
level-l corner ids are the level-(l+1) ids taken every 4th entry.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .mesh import QUAD


def level_sizes(mesh, levels: int) -> List[Tuple[int, int, int]]:
    """(F, V, N) of the input of each level, assuming a closed or open 2-manifold.

    ``levels`` is the number of refinement levels actually run."""
    F, V, N = mesh.nfaces, mesh.nverts, mesh.nnz
    # boundary half-edges of level 0: a directed edge without its reverse
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(F + 1, dtype=np.int64) * 4
    nxt = _next_corner(ptr, N)
    a = mesh.ids.astype(np.int64)
    b = a[nxt]
    key = a * V + b
    rkey = b * V + a
    B = int(np.count_nonzero(~np.isin(key, rkey)))
    out = []
    for _ in range(levels):
        out.append((F, V, N))
        E = (N - B) // 2 + B
        F, V, N, B = N, V + F + E, 4 * N, 2 * B
    return out


def _next_corner(ptr: np.ndarray, N: int) -> np.ndarray:
    ptr = ptr.astype(np.int64)
    orders = np.diff(ptr)
    start = np.repeat(ptr[:-1], orders)
    end = np.repeat(ptr[1:], orders)
    c = np.arange(N, dtype=np.int64)
    return np.where(c + 1 < end, c + 1, start)


def canonicalize(mesh, levels: int, ids: np.ndarray, verts: np.ndarray):
    """Returns (ids, verts) of a ``levels``-level result with canonical edge numbering.

    ``mesh`` is the level-0 input (a slak_b200.Mesh), ``ids`` the final flat
    quad ids, ``verts`` the final positions ([V, 4])."""
    sizes = level_sizes(mesh, levels)
    ids = np.asarray(ids, dtype=np.int64)
    # level-l corner ids, raw numbering, for l = 0..levels
    hist = [None] * (levels + 1)
    hist[levels] = ids
    for l in range(levels - 1, 0, -1):
        hist[l] = hist[l + 1][0::4]
    hist[0] = mesh.ids.astype(np.int64)
    perm = np.arange(mesh.nverts, dtype=np.int64)        # raw -> canonical at level 0
    for l in range(levels):
        F, V, N = sizes[l]
        if l == 0:
            ptr = mesh.ptr if mesh.ptr is not None else np.arange(F + 1, dtype=np.int64) * 4
            if mesh.type == QUAD and mesh.ptr is None:
                ptr = np.arange(F + 1, dtype=np.int64) * 4
            nxt = _next_corner(ptr, N)
        else:
            c = np.arange(N, dtype=np.int64)
            nxt = (c & ~3) | ((c + 1) & 3)
        coarse = hist[l]
        a = perm[coarse]
        b = perm[coarse[nxt]]
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        key = lo * (V + 1) + hi
        raw_e = hist[l + 1][1::4]                       # e_out of every quad, raw id
        uk, inv = np.unique(key, return_inverse=True)
        E = uk.shape[0]
        Vn = V + F + E
        newperm = np.full(Vn, -1, dtype=np.int64)
        newperm[:V] = perm
        newperm[V:V + F] = np.arange(V, V + F)
        if raw_e.min() < V + F or raw_e.max() >= Vn:
            raise ValueError(f"level {l}: edge-point id out of range")
        newperm[raw_e] = V + F + inv
        if (newperm < 0).any():
            raise ValueError(f"level {l}: some edge point is never referenced")
        perm = newperm
    cids = perm[ids].astype(np.int32)
    cverts = np.empty_like(verts)
    cverts[perm] = verts
    return cids, cverts
