"""CPU check of the closed-form refinement for parents WITH a boundary (the
fast path's open-mesh case): restated in numpy, the formulas must reproduce
the oracle's refined quads of C = refine(P) refined once more, and C's
adjacency state (offsets, slots, twins, t, boundary-edge ranks) computed by
brute force.  A half-edge without a twin has twin -1; brank(e) counts the
boundary edges with a smaller id."""
import numpy as np
import pytest

import oracle
from slak_b200.mesh import LAK, QUAD, SLAK, Mesh

from meshes import bowtie, fan_disk, open_grid


def qn(x):
    return (x & ~3) | ((x + 1) & 3)


def qp(x):
    return (x & ~3) | ((x + 3) & 3)


def brute_state(ids, V, scheme):
    """State of a quad mesh that may have a boundary."""
    ids = ids.astype(np.int64)
    N = ids.size
    c = np.arange(N)
    sc = np.argsort(ids, kind="stable")
    sptr = np.concatenate([[0], np.cumsum(np.bincount(ids, minlength=V))])
    slot = np.empty(N, np.int64)
    slot[sc] = c
    a, b = ids, ids[qn(c)]
    key = a * V + b
    order = np.argsort(key)
    rk = b * V + a
    pos = np.clip(np.searchsorted(key[order], rk), 0, N - 1)
    tw = np.where(key[order[pos]] == rk, order[pos], -1)
    twp = tw[qp(c)]
    t = np.where(twp >= 0, slot[np.maximum(twp, 0)], -1)
    if scheme == SLAK:
        own = sc[(a[sc] < b[sc]) | (tw[sc] < 0)]             # owners in slot order
        H = np.stack([own, tw[own]], 1)
    else:
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        und = np.unique(np.stack([hi, lo], 1), axis=0)        # ascending (max, min)
        H = np.full((und.shape[0], 2), -1, np.int64)
        kk = {(int(h), int(l)): i for i, (h, l) in enumerate(und)}
        for x in range(N):
            i = kk[(int(hi[x]), int(lo[x]))]
            H[i, 0 if a[x] < b[x] else 1] = x
    eid = np.empty(N, np.int64)
    for i, (h0, h1) in enumerate(H):
        if h0 >= 0:
            eid[h0] = i
        if h1 >= 0:
            eid[h1] = i
    isb = (H < 0).any(1)
    brank = np.concatenate([[0], np.cumsum(isb)])[:-1]
    return dict(sptr=sptr, sc=sc, slot=slot, tw=tw, t=t, H=H, eid=eid, isb=isb, brank=brank)


def rank_in(x, group):
    """rank of corner x among the present corners of `group` (-1 = absent)."""
    r = np.zeros_like(x)
    for g in group:
        r += ((g >= 0) & (g < x)).astype(np.int64)
    return r


def emulate(P_ids, P_V, C_ids, C_V, st, scheme):
    N1 = P_ids.size
    V1, F1 = P_V, N1 // 4
    VF1 = V1 + F1
    B1 = int(st["isb"].sum())
    N = 4 * N1
    y = np.arange(N)
    x, k = y >> 2, y & 3
    vid = C_ids.astype(np.int64)
    tw, t, slot, brank = st["tw"], st["t"], st["slot"], st["brank"]
    eidp_x = vid[4 * x + 1] - VF1
    eidp_px = vid[4 * x + 3] - VF1
    tw1x, tw1px = tw[x], tw[qp(x)]
    if scheme == SLAK:
        e3 = np.where(t[x] >= 0, t[x], 2 * N1 + brank[eidp_px])
        eid = np.select([k == 0, k == 1, k == 2], [slot[x], N1 + qn(x), N1 + x], e3)
    else:
        base = lambda e: 4 * e - brank[e]
        vx, vnx, vpx = vid[4 * x], vid[4 * qn(x)], vid[4 * qp(x)]
        fx = x >> 2
        eid = np.select([k == 0, k == 1, k == 2],
                        [base(eidp_x) + (vx > vnx), base(eidp_x) + 2 + ((tw1x >= 0) & (fx > (tw1x >> 2))),
                         base(eidp_px) + 2 + ((tw1px >= 0) & (fx > (tw1px >> 2)))], base(eidp_px) + (vx > vpx))
    VFc = C_V + N1
    ein = eid[4 * x + ((k + 3) & 3)]
    refined = np.stack([vid, VFc + eid, C_V + x, VFc + ein], 1).reshape(-1)

    # C's state
    px, nxx = qp(x), qn(x)
    ntw = np.where(tw1x >= 0, qn(np.maximum(tw1x, 0)), -1)
    ntwp = np.where(tw1px >= 0, qn(np.maximum(tw1px, 0)), -1)
    A, B, Cc, D = 4 * x + 1, np.where(tw1x >= 0, 4 * tw1x + 1, -1), 4 * nxx + 3, np.where(tw1x >= 0, 4 * ntw + 3, -1)
    A2, B2, C2, D2 = 4 * px + 1, np.where(tw1px >= 0, 4 * tw1px + 1, -1), 4 * x + 3, np.where(tw1px >= 0, 4 * ntwp + 3, -1)
    colbase = lambda e: 2 * N1 + 4 * e - 2 * brank[e]
    bx, bpx = colbase(eidp_x), colbase(eidp_px)
    slot_c = np.select([k == 0, k == 1, k == 2], [slot[x], bx + rank_in(A, (B, Cc, D)), N1 + x],
                       bpx + rank_in(C2, (A2, B2, D2)))
    tw_c = np.select([k == 0, k == 1, k == 2], [np.where(tw1x >= 0, 4 * ntw + 3, -1), 4 * nxx + 2, 4 * px + 1],
                     np.where(tw1px >= 0, 4 * tw1px, -1))
    t_c = np.select([k == 0, k == 1, k == 2],
                    [t[x], np.where(tw1x >= 0, bx + rank_in(D, (A, B, Cc)), -1), N1 + nxx],
                    bpx + rank_in(A2, (B2, C2, D2)))
    E1 = st["H"].shape[0]
    sptr_c = np.empty(C_V + 1, np.int64)
    sptr_c[:V1] = st["sptr"][:V1]
    sptr_c[V1:V1 + F1] = N1 + 4 * np.arange(F1)
    sptr_c[VF1:VF1 + E1] = colbase(np.arange(E1))
    sptr_c[C_V] = N
    # boundary ranks of C's edges
    if scheme == SLAK:
        bout = (tw[st["sc"]] < 0).astype(np.int64)               # C edges 0..N1-1, slot order
        isb_c = np.concatenate([bout, np.zeros(N1, np.int64), np.ones(B1, np.int64)])
    else:
        isb_p = st["isb"]
        per = np.where(isb_p[:, None], np.array([[1, 1, 0, 0]]), 0)
        cnt = np.where(isb_p, 3, 4)
        isb_c = np.concatenate([per[e, :cnt[e]] for e in range(E1)])
    brank_c = np.concatenate([[0], np.cumsum(isb_c)])[:-1]
    return refined, dict(sptr=sptr_c, slot=slot_c, tw=tw_c, t=t_c, brank=brank_c)


def _quad_level(mesh, scheme):
    r = oracle.level(mesh, scheme, poly=mesh.type != QUAD)
    return Mesh(QUAD, r.ids, r.verts, None if scheme == SLAK else r.ptr, None if scheme == SLAK else r.vals,
                r.nfaces, 4, True)


CASES = [("grid", lambda: open_grid(5, 4)), ("fan", lambda: fan_disk(7)), ("grid_wide", lambda: open_grid(9, 2)),
         ("bowtie", lambda: bowtie())]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_closed_form_refinement_with_boundary(name, make, scheme):
    base = make()
    P = _quad_level(base, scheme)                        # P: quad mesh with a boundary
    Pm = P if scheme == SLAK else P.with_quad_ptr()
    C = oracle.level(Pm, scheme, poly=False)
    Cm = Mesh(QUAD, C.ids, C.verts, C.ptr if scheme == LAK else None, C.vals if scheme == LAK else None,
              C.nfaces, 4, True)
    R = oracle.level(Cm, scheme, poly=False)
    stP = brute_state(P.ids, P.nverts, scheme)
    assert stP["isb"].any()
    assert np.array_equal(stP["eid"] + P.nverts + P.nfaces, C.ids[1::4])   # state numbering = oracle's
    refined, stC = emulate(P.ids, P.nverts, C.ids, C.nverts, stP, scheme)
    assert np.array_equal(refined, R.ids)
    bC = brute_state(C.ids, C.nverts, scheme)
    for f in ("sptr", "slot", "tw", "brank"):
        assert np.array_equal(stC[f], bC[f]), f
    if scheme == SLAK:
        assert np.array_equal(stC["t"], bC["t"])
