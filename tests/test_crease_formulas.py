"""CPU check of how the CUDA crease pass finds each crease vertex's crease
edges without sorting.  Incidence is inherited from level to level:
  * a base vertex's level-0 entry j0 (side 0: the vertex is the origin of the
    entry's half-edge, side 1: its head) continues at level l as entry
    (j0 << l) + side (2^l - 1);
  * the edge point made by entry j of level t (sharpness > 1) touches, at
    level l > t, entries (2j << d) + 2^d - 1 (as their head) and (2j + 1) << d
    (as their origin), d = l - t - 1.
The emulation below follows those formulas and must give, at every level, the
same (vertex -> sorted other ends, sharpness) groups as grouping the level's
live crease edges by vertex, which is what the restatement does."""
import math

import numpy as np
import pytest

import oracle
from oracle import _LevelMesh
from oracle import creases as oc
from slak_b200 import meshgen
from slak_b200.mesh import LAK, SLAK

from meshes import cube, open_mixed


def _edges(mesh):
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    ids = np.asarray(mesh.ids, np.int64)
    nxt = oc._next_corner(ptr, ids.size, mesh.type == 1)
    return np.unique(np.sort(np.stack([ids, ids[nxt]], 1), 1), axis=0)


def _dense_lists(mesh, levels, scheme, pairs, sharp):
    """Per level: the input mesh and the dense crease list (dead = -1) in the
    CUDA layout (entry j of level l has children 2j, 2j + 1 at level l + 1),
    plus the edge-point id each entry makes."""
    cc, cs, _ = oc.resolve(mesh, pairs, sharp)
    # dense level-0 list in pair order, as k_crease_resolve writes it
    m = len(pairs)
    ids = np.asarray(mesh.ids, np.int64)
    nxt = oc._next_corner(mesh.ptr, ids.size, mesh.type == 1)
    half = {(int(a), int(b)): c for c, (a, b) in enumerate(zip(ids.tolist(), ids[nxt].tolist()))}
    c0 = np.full(m, -1, np.int64)
    s0 = np.zeros(m, np.float32)
    for i, ((a, b), s) in enumerate(zip(np.asarray(pairs).tolist(), np.asarray(sharp, np.float32).tolist())):
        lo, hi = min(a, b), max(a, b)
        if (lo, hi) in half and (hi, lo) in half and s > 0:
            c0[i], s0[i] = half[(lo, hi)], s
    smax = float(np.max(sharp))
    nlev = min(levels, math.ceil(smax))
    out = []
    cur, ccl, csl = mesh, c0, s0
    for l in range(nlev):
        r = oracle.level(cur, scheme, poly=(l == 0 and mesh.type != 1))
        quad = cur.type == 1
        idl = np.asarray(cur.ids, np.int64)
        nx = oc._next_corner(cur.ptr, idl.size, quad)
        live = ccl >= 0
        ep = np.full(ccl.size, -1, np.int64)
        ep[live] = np.asarray(r.ids, np.int64)[4 * ccl[live] + 1]
        nlive = live & (csl > 1)
        ncc = np.full(2 * ccl.size, -1, np.int64)
        ncs = np.zeros(2 * ccl.size, np.float32)
        ncc[0::2][nlive] = 4 * ccl[nlive]
        ncc[1::2][nlive] = 4 * nx[ccl[nlive]] + 3
        ncs[0::2][nlive] = csl[nlive] - np.float32(1)
        ncs[1::2][nlive] = csl[nlive] - np.float32(1)
        out.append(dict(mesh=cur, cc=ccl, cs=csl, next=nx, ep=np.where(nlive, ep, -1)))
        cur, ccl, csl = _LevelMesh(r), ncc, ncs
    return out, c0


def _groups_by_sorting(L):
    ids, cc, cs, nx = np.asarray(L["mesh"].ids, np.int64), L["cc"], L["cs"], L["next"]
    live = cc >= 0
    a, b, s = ids[cc[live]], ids[nx[cc[live]]], cs[live]
    g = {}
    for x, y, w in zip(np.r_[a, b].tolist(), np.r_[b, a].tolist(), np.r_[s, s].tolist()):
        g.setdefault(x, []).append((y, w))
    return {v: sorted(e) for v, e in g.items()}


def _groups_inherited(levels, l, c0, base_mesh):
    ids0 = np.asarray(base_mesh.ids, np.int64)
    nx0 = oc._next_corner(base_mesh.ptr, ids0.size, base_mesh.type == 1)
    # base CSR: level-0 live entries at each vertex, with side
    inc = {}
    for j, c in enumerate(c0.tolist()):
        if c >= 0:
            inc.setdefault(int(ids0[c]), []).append((j, 0))
            inc.setdefault(int(ids0[nx0[c]]), []).append((j, 1))
    L = levels[l]
    ids, cc, cs, nx = np.asarray(L["mesh"].ids, np.int64), L["cc"], L["cs"], L["next"]
    g = {}
    for v, lst in inc.items():
        e = []
        for j0, side in lst:
            jl = (j0 << l) + (((1 << l) - 1) if side else 0)
            c = cc[jl]
            if c < 0:
                continue
            e.append((int(ids[c]) if side else int(ids[nx[c]]), float(cs[jl])))
        if e:
            g[v] = sorted(e)
    for t in range(l):
        ep = levels[t]["ep"]
        d = l - t - 1
        for q in np.flatnonzero(ep >= 0).tolist():
            jb, ja = ((2 * q) << d) + ((1 << d) - 1), (2 * q + 1) << d
            cb, ca = cc[jb], cc[ja]
            assert (cb < 0) == (ca < 0)                  # the two descendants decay together
            if cb < 0:
                continue
            assert cs[jb] == cs[ja]
            g[int(ep[q])] = sorted([(int(ids[cb]), float(cs[jb])), (int(ids[nx[ca]]), float(cs[ja]))])
    return g


CASES = [("cube", lambda: cube(), 5, lambda m: (_edges(m), np.linspace(0.5, 6.0, 12).astype(np.float32))),
         ("mixed_torus", lambda: meshgen.mixed_torus(20, 16, 0.05, 0.03, 0.005, seed=4), 4, None),
         ("open_mixed", lambda: open_mixed(24, 20), 4, None)]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make,levels,creases", CASES, ids=[c[0] for c in CASES])
def test_inherited_incidence_equals_grouping(name, make, levels, creases, scheme):
    m = make()
    if scheme == LAK and m.ptr is None:
        m = m.with_quad_ptr()
    if creases is None:
        rng = np.random.default_rng(5)
        e = _edges(m)
        pairs = e[rng.random(e.shape[0]) < 0.25]
        sharp = rng.choice(np.array([0.5, 1.0, 1.5, 2.0, 3.0, 4.0], np.float32), pairs.shape[0])
    else:
        pairs, sharp = creases(m)
    lv, c0 = _dense_lists(m, levels, scheme, pairs, sharp)
    assert len(lv) >= 2
    for l in range(len(lv)):
        want = _groups_by_sorting(lv[l])
        got = _groups_inherited(lv, l, c0, m)
        assert got == want, l
