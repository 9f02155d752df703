"""CPU check of the closed-form refinement used by the fast CUDA path
(slak_b200/csrc/fast.cuh): the kernels' index formulas, restated in numpy,
must reproduce (1) the oracle's refined quads of C = refine(P) refined once
more, and (2) C's adjacency state computed by brute force."""
import numpy as np
import pytest

import oracle
from slak_b200 import meshgen
from slak_b200.mesh import LAK, QUAD, SLAK, Mesh


def qn(x):
    return (x & ~3) | ((x + 1) & 3)


def qp(x):
    return (x & ~3) | ((x + 3) & 3)


class Faces:
    """Corner navigation of P: next / previous corner in its face, and its face.
    Quad faces are 4 consecutive corners; polygon faces come from `ptr`."""

    def __init__(self, N, ptr=None):
        c = np.arange(N)
        if ptr is None:
            self.next, self.prev, self.face = qn(c), qp(c), c >> 2
            self.start = 4 * np.arange(N // 4)
        else:
            ptr = np.asarray(ptr, np.int64)
            self.face = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
            b, e = ptr[self.face], ptr[self.face + 1]
            self.next = np.where(c + 1 == e, b, c + 1)
            self.prev = np.where(c == b, e - 1, c - 1)
            self.start = ptr[:-1]


def brute_state(ids, V, scheme, fc=None):
    """Adjacency state of a closed mesh: sptr, sc, slot, tw, t, H (scheme order), eid."""
    ids = ids.astype(np.int64)
    N = ids.size
    fc = fc or Faces(N)
    c = np.arange(N)
    sc = np.argsort(ids, kind="stable")
    sptr = np.concatenate([[0], np.cumsum(np.bincount(ids, minlength=V))])
    slot = np.empty(N, np.int64)
    slot[sc] = c
    a, b = ids, ids[fc.next]
    key = a * V + b
    order = np.argsort(key)
    rk = b * V + a
    pos = np.searchsorted(key[order], rk)
    tw = order[pos]
    assert (key[tw] == rk).all()
    t = slot[tw[fc.prev]]
    if scheme == SLAK:
        owners = sc[a[sc] < b[sc]]                      # owners in slot order
        H = np.stack([owners, tw[owners]], 1)
    else:
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        mm = c[a < b]                                   # min->max half-edges
        o = np.lexsort((lo[mm], hi[mm]))
        H = np.stack([mm[o], tw[mm[o]]], 1)
    eid = np.empty(N, np.int64)
    eid[H[:, 0]] = np.arange(H.shape[0])
    eid[H[:, 1]] = np.arange(H.shape[0])
    return dict(sptr=sptr, sc=sc, slot=slot, tw=tw, t=t, H=H, eid=eid)


def rank4(a, b, c, d):
    return (b < a).astype(np.int64) + (c < a) + (d < a)


def emulate(P_ids, P_V, C_ids, C_V, st, scheme, fc=None):
    """The index math of k_g1 / k_gf / k_g2 / k_g3: refined quads of C and C's
    state (fc: P's corner navigation, quad faces by default)."""
    N1 = P_ids.size
    fc = fc or Faces(N1)
    nx_, pv_, fa_ = fc.next, fc.prev, fc.face
    V1, F1, E1 = P_V, fc.start.size, N1 // 2
    VF1 = V1 + F1
    N = 4 * N1
    y = np.arange(N)
    x, k = y >> 2, y & 3
    vid = C_ids.astype(np.int64)
    eidp_x = vid[4 * x + 1] - VF1
    eidp_px = vid[4 * x + 3] - VF1
    tw1x, tw1px = st["tw"][x], st["tw"][pv_[x]]
    if scheme == SLAK:
        eid = np.select([k == 0, k == 1, k == 2], [st["slot"][x], N1 + nx_[x], N1 + x], st["t"][x])
    else:
        vx, vnx, vpx = vid[4 * x], vid[4 * nx_[x]], vid[4 * pv_[x]]
        fx = fa_[x]
        eid = np.select([k == 0, k == 1, k == 2],
                        [4 * eidp_x + (vx > vnx), 4 * eidp_x + 2 + (fx > fa_[tw1x]),
                         4 * eidp_px + 2 + (fx > fa_[tw1px])], 4 * eidp_px + (vx > vpx))
    VFc = C_V + N1
    ein = eid[4 * x + ((k + 3) & 3)]
    refined = np.stack([vid, VFc + eid, C_V + x, VFc + ein], 1).reshape(-1)
    # C's state
    px, nxx, ntw, ntwp = pv_[x], nx_[x], nx_[tw1x], nx_[tw1px]
    A, B, Cc, D = 4 * x + 1, 4 * tw1x + 1, 4 * nxx + 3, 4 * ntw + 3
    A2, B2, C2, D2 = 4 * px + 1, 4 * tw1px + 1, 4 * x + 3, 4 * ntwp + 3
    bx, bpx = 2 * N1 + 4 * eidp_x, 2 * N1 + 4 * eidp_px
    slot = np.select([k == 0, k == 1, k == 2], [st["slot"][x], bx + rank4(A, B, Cc, D), N1 + x],
                     bpx + rank4(C2, A2, B2, D2))
    tw = np.select([k == 0, k == 1, k == 2], [4 * ntw + 3, 4 * nxx + 2, 4 * px + 1], 4 * tw1px)
    t = np.select([k == 0, k == 1, k == 2], [st["t"][x], bx + rank4(D, A, B, Cc), N1 + nxx],
                  bpx + rank4(A2, B2, C2, D2))
    sc = np.empty(N, np.int64)
    sptr = np.empty(C_V + 1, np.int64)
    # G3: old vertices keep their columns, corners 4x
    sc[:N1] = 4 * st["sc"]
    sptr[:V1] = st["sptr"][:V1]
    # G1: face points
    sc[N1 + np.arange(N1)] = 4 * np.arange(N1) + 2
    sptr[V1:V1 + F1] = N1 + fc.start
    # G2: edge points, sorted {4h+1, 4h2+1, 4nh+3, 4nh2+3}
    h, h2 = st["H"][:, 0], st["H"][:, 1]
    co = np.sort(np.stack([4 * h + 1, 4 * h2 + 1, 4 * nx_[h] + 3, 4 * nx_[h2] + 3], 1), 1)
    sc[2 * N1:] = co.reshape(-1)
    sptr[VF1:VF1 + E1] = 2 * N1 + 4 * np.arange(E1)
    sptr[C_V] = N
    # H of C
    if scheme == SLAK:
        Ha = np.stack([4 * st["sc"], 4 * nx_[st["tw"][st["sc"]]] + 3], 1)     # G3: ids slot1(x)
        Hb = np.stack([4 * np.arange(N1) + 2, 4 * pv_[np.arange(N1)] + 1], 1)  # G1: ids N1 + x
        H = np.concatenate([Ha, Hb])
    else:
        v, u = vid[4 * h], vid[4 * h2]
        fh, fh2 = V1 + fa_[h], V1 + fa_[h2]
        nh, nh2 = nx_[h], nx_[h2]
        Hv = np.stack([4 * h, 4 * nh2 + 3], 1)
        Hu = np.stack([4 * h2, 4 * nh + 3], 1)
        Hf = np.stack([4 * nh + 2, 4 * h + 1], 1)
        Hf2 = np.stack([4 * nh2 + 2, 4 * h2 + 1], 1)
        vu = (v < u)[:, None]
        ff = (fh < fh2)[:, None]
        H = np.stack([np.where(vu, Hv, Hu), np.where(vu, Hu, Hv), np.where(ff, Hf, Hf2), np.where(ff, Hf2, Hf)],
                     1).reshape(-1, 2)
    return refined, dict(sptr=sptr, sc=sc, slot=slot, tw=tw, t=t, H=H)


def _closed_quad(mesh, scheme):
    """A closed quad mesh P: the oracle's one-level refinement of `mesh`."""
    r = oracle.level(mesh, scheme, poly=mesh.type != QUAD)
    m = Mesh(QUAD, r.ids, r.verts, None if scheme == SLAK else r.ptr, None if scheme == SLAK else r.vals,
             r.nfaces, 4, True)
    return m


CASES = [("torus", lambda: meshgen.torus(5, 7, seed=1)),
         ("mixed", lambda: meshgen.mixed_torus(12, 10, 0.1, 0.06, 0.005, seed=5)),
         ("cylinder", lambda: meshgen.capped_cylinder(8, 4, 0.001, seed=6)),
         ("ico", lambda: meshgen.icosphere(2, 0.02, seed=4))]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_closed_form_refinement(name, make, scheme):
    base = make()
    if scheme == LAK and base.ptr is None:
        base = base.with_quad_ptr()
    P = _closed_quad(base, scheme)                       # P: closed quad mesh
    Pm = P if scheme == SLAK else P.with_quad_ptr()
    C = oracle.level(Pm, scheme, poly=False)             # C = refine(P)
    Cm = Mesh(QUAD, C.ids, C.verts, C.ptr, C.vals, C.nfaces, 4, True)
    R = oracle.level(Cm if scheme == LAK else Mesh(QUAD, C.ids, C.verts, None, None, C.nfaces, 4, True),
                     scheme, poly=False)                 # refine(C), the oracle's
    stP = brute_state(P.ids, P.nverts, scheme)
    assert np.array_equal(stP["eid"] + P.nverts + P.nfaces, C.ids[1::4])   # state numbering = oracle's
    refined, stC = emulate(P.ids, P.nverts, C.ids, C.nverts, stP, scheme)
    assert np.array_equal(refined, R.ids)
    bC = brute_state(C.ids, C.nverts, scheme)
    for f in ("sptr", "sc", "slot", "tw", "H"):
        assert np.array_equal(stC[f], bC[f]), f
    if scheme == SLAK:
        assert np.array_equal(stC["t"], bC["t"])


POLY_CASES = [("mixed", lambda: meshgen.mixed_torus(12, 10, 0.1, 0.06, 0.005, seed=5)),
              ("cylinder", lambda: meshgen.capped_cylinder(8, 4, 0.001, seed=6)),
              ("ico", lambda: meshgen.icosphere(2, 0.02, seed=4))]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make", POLY_CASES, ids=[c[0] for c in POLY_CASES])
def test_closed_form_refinement_of_polygon_parent(name, make, scheme):
    """The same formulas when P is the polygon input itself (level 1 of a
    polygon mesh): next / previous / face of P come from its offsets."""
    P = make()
    assert P.type != QUAD
    fc = Faces(P.nnz, P.ptr)
    C = oracle.level(P, scheme, poly=True)               # C = refine(P), all quads
    Cm = Mesh(QUAD, C.ids, C.verts, C.ptr if scheme == LAK else None, C.vals if scheme == LAK else None,
              C.nfaces, 4, True)
    R = oracle.level(Cm, scheme, poly=False)
    stP = brute_state(P.ids, P.nverts, scheme, fc)
    assert np.array_equal(stP["eid"] + P.nverts + P.nfaces, C.ids[1::4])
    refined, stC = emulate(P.ids, P.nverts, C.ids, C.nverts, stP, scheme, fc)
    assert np.array_equal(refined, R.ids)
    bC = brute_state(C.ids, C.nverts, scheme)
    for f in ("sptr", "sc", "slot", "tw", "H"):
        assert np.array_equal(stC[f], bC[f]), f
    if scheme == SLAK:
        assert np.array_equal(stC["t"], bC["t"])
