"""CPU restatement of the semi-sharp crease pass (numpy, float32).

TEST INFRASTRUCTURE ONLY, like the rest of ``oracle``: the tests compare the
CUDA crease pass with it bit for bit.

The reference declares this step but leaves it unimplemented
(LibSource/device/CatmullClarkImpl.cu:94-96 and :296-298,
LibSource/device/LAKCatmullClarkImpl.cu:240-242 call a handleCreases that is
commented out), so there is no reference output to pin it to.  It restates the
published rules of DeRose, Kass and Truong, "Subdivision Surfaces in Character
Animation" (SIGGRAPH 1998), with sharpness decaying by one per level, and the
tests pin it with known answers (a cube whose edges are all sharp stays a cube;
sharpness 0 is the smooth surface; the blend is linear in the sharpness).

The smooth level comes from the oracle (``oracle.level``); then, per level with
a live crease:
  * crease edge {a, b}, sharpness s: edge point = (p_a + p_b) * 0.5 for s >= 1,
    else smooth * (1 - s) + sharp * s;
  * vertex v with k crease edges, w = min(1, (sum of s in ascending other-end
    id) / k): a base-mesh boundary vertex or k >= 3 is a corner (sharp = p_v);
    k == 2 takes (p_v * 0.75 + p_o1 * 0.125) + p_o2 * 0.125 (o1 < o2); k == 1
    stays smooth; the result is sharp for w >= 1, else smooth * (1 - w) + sharp * w;
  * a crease half-edge c of sharpness s > 1 leaves the refined half-edges 4c
    and 4 next(c) + 3 with sharpness s - 1.
A crease pair is matched to the half-edge min -> max of the base mesh; a pair
on a boundary edge or with s <= 0 does nothing; a pair that is no edge, or an
interior edge named twice, is an error.

Corners (vertex sharpness, the "t corner" tags): a base vertex of sharpness
s_v takes the corner rule (p_v) while s_v - level > 0, blended by
max(min(1, s_v - level), min(1, mean crease sharpness)); an id out of range or
a vertex named twice is an error.
"""
from __future__ import annotations

import math

import numpy as np

from . import _LevelMesh, level

F32 = np.float32


def _next_corner(ptr, N, quad):
    c = np.arange(N, dtype=np.int64)
    if quad:
        return (c & ~3) | ((c + 1) & 3)
    ptr = np.asarray(ptr, np.int64)
    face = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    nxt = c + 1
    last = nxt == ptr[face + 1]
    nxt[last] = ptr[face[last]]
    return nxt


def resolve(mesh, pairs, sharp):
    """Base-mesh crease list (corner, sharpness) and the boundary flag of every
    base vertex.  Raises ValueError where the CUDA path reports SLAK_ERR_BAD_MESH."""
    quad = mesh.type == 1
    ids = np.asarray(mesh.ids, np.int64)
    nxt = _next_corner(mesh.ptr, ids.size, quad)
    half = {(int(a), int(b)): c for c, (a, b) in enumerate(zip(ids.tolist(), ids[nxt].tolist()))}
    V = int(mesh.nverts if hasattr(mesh, "nverts") else np.asarray(mesh.verts).shape[0])
    bnd = np.zeros(V, bool)
    for (a, b) in half:
        if (b, a) not in half:
            bnd[a] = bnd[b] = True
    cc, cs, seen = [], [], set()
    for (a, b), s in zip(np.asarray(pairs, np.int64).reshape(-1, 2).tolist(), np.asarray(sharp, F32).tolist()):
        if a == b or min(a, b) < 0 or max(a, b) >= V:
            raise ValueError("crease pair out of range")
        lo, hi = min(a, b), max(a, b)
        up, dn = half.get((lo, hi)), half.get((hi, lo))
        if up is None and dn is None:
            raise ValueError("crease pair is not an edge")
        if up is None or dn is None or not s > 0:
            continue
        if up in seen:
            raise ValueError("crease edge named twice")
        seen.add(up)
        cc.append(up)
        cs.append(s)
    return np.array(cc, np.int64), np.array(cs, F32), bnd


def resolve_corners(V, verts, sharp):
    """Dense corner sharpness of the base vertices (0: none).  Raises ValueError
    where the CUDA path rejects the tags (an id out of range, a vertex named
    twice)."""
    vcs = np.zeros(V, F32)
    seen = set()
    for v, s in zip(np.asarray(verts, np.int64).reshape(-1).tolist(), np.asarray(sharp, F32).tolist()):
        if v < 0 or v >= V:
            raise ValueError("corner vertex out of range")
        if v in seen:
            raise ValueError("corner vertex named twice")
        if not np.isfinite(s):
            raise ValueError("corner sharpness is not finite")
        seen.add(v)
        vcs[v] = max(F32(s), F32(0))
    return vcs


def crease_pass(cur, r, cc, cs, bnd0, last, vcs=None, lvl=0):
    """Applies one level's crease rules to the oracle level result ``r`` of the
    input ``cur`` (in place on r.verts); returns the next level's list.  With
    ``vcs`` (corner sharpness of the base vertices), a base vertex whose corner
    sharpness minus the level is positive takes the corner rule, blended by
    max(min(1, that), min(1, mean crease sharpness))."""
    quad = cur.type == 1
    ids = np.asarray(cur.ids, np.int64)
    nxt = _next_corner(cur.ptr, ids.size, quad)
    P = np.asarray(cur.verts, F32).reshape(-1, 4)
    R = r.verts
    rids = np.asarray(r.ids, np.int64)
    nc = nxt[cc]
    a, b = ids[cc], ids[nc]
    ep = rids[4 * cc + 1]
    sharp_e = (P[a] + P[b]) * F32(0.5)
    s = cs[:, None]
    blend = R[ep] * (F32(1) - s) + sharp_e * s
    R[ep] = np.where(s >= F32(1), sharp_e, blend)

    # vertices: incidence records sorted by (vertex, other end)
    v = np.concatenate([a, b])
    o = np.concatenate([b, a])
    sv = np.concatenate([cs, cs])
    order = np.lexsort((o, v))
    v, o, sv = v[order], o[order], sv[order]
    starts = np.flatnonzero(np.r_[True, v[1:] != v[:-1]]) if v.size else np.zeros(0, np.int64)
    ends = np.r_[starts[1:], v.size]
    V0 = bnd0.size
    groups = {int(v[st]): (st, en) for st, en in zip(starts.tolist(), ends.tolist())}
    corner = {}
    if vcs is not None:
        cv = vcs - F32(lvl)
        corner = {int(x): cv[x] for x in np.flatnonzero(cv > F32(0)).tolist()}
    for vx in sorted(set(groups) | set(corner)):
        st, en = groups.get(vx, (0, 0))
        k = en - st
        ssum = F32(0)
        for t in range(st, en):
            ssum = F32(ssum + sv[t])
        if vx in corner:
            wk = F32(0)
            if k > 0:
                wk = F32(ssum / F32(k))
                if wk > F32(1):
                    wk = F32(1)
            wc = corner[vx] if corner[vx] < F32(1) else F32(1)
            w = wc if wc > wk else wk
            if w >= F32(1):
                R[vx] = P[vx]
            else:
                R[vx] = R[vx] * (F32(1) - w) + P[vx] * w
            continue
        w = F32(ssum / F32(k))
        if w > F32(1):
            w = F32(1)
        boundary = vx < V0 and bool(bnd0[vx])
        if boundary or k >= 3:
            sharp_v = P[vx].copy()
        elif k == 1:
            continue
        else:
            sharp_v = (P[vx] * F32(0.75) + P[int(o[st])] * F32(0.125)) + P[int(o[st + 1])] * F32(0.125)
        if w >= F32(1):
            R[vx] = sharp_v
        else:
            R[vx] = R[vx] * (F32(1) - w) + sharp_v * w
    if last:
        return None, None
    live = cs > F32(1)
    ncc = np.concatenate([4 * cc[live], 4 * nc[live] + 3])
    ncs = np.concatenate([cs[live] - F32(1), cs[live] - F32(1)]).astype(F32)
    return ncc, ncs


def subdivide_creased(mesh, levels: int, scheme: int, pairs, sharp, corners=None):
    """Oracle levels with the crease pass after each level that has a live
    crease or corner; returns the last level's Result (positions float32).
    ``corners``: None or (vertex ids, sharpness)."""
    nlev = levels if mesh.type == 1 else max(levels, 1)
    cc, cs, bnd0 = resolve(mesh, np.asarray(pairs, np.int64).reshape(-1, 2), sharp)
    smax = float(np.max(np.asarray(sharp, F32))) if np.asarray(sharp).size else 0.0
    vcs = None
    if corners is not None and np.asarray(corners[1]).size:
        vcs = resolve_corners(bnd0.size, corners[0], corners[1])
        smax = max(smax, float(vcs.max()))
    crease_levels = min(nlev, math.ceil(smax)) if smax > 0 else 0
    cur = mesh
    r = None
    for l in range(nlev):
        r = level(cur, scheme, poly=(l == 0 and mesh.type != 1))
        r.verts = np.ascontiguousarray(r.verts, F32)
        if l < crease_levels:
            cc, cs = crease_pass(cur, r, cc, cs, bnd0, last=l + 1 >= crease_levels, vcs=vcs, lvl=l)
        nxt = _LevelMesh(r)
        nxt.verts64 = None
        cur = nxt
    return r
