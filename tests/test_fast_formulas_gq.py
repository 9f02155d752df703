"""CPU check of the grandparent-quad form of the fast path (fast.cuh, k_g1
with GQ): when the level being refined is C = refine(P) and P = refine(PP)
with PP a closed quad mesh, most of P's vertex columns lie inside one 16-lane
group of k_g1 (one PP face: P corners 16g..16g+15) or two (the two faces of a
PP edge).  Their vertex points and SLAK edge points are then computed in
k_g1 from what the lanes hold, instead of from slot records:

* a PP face point g (P vertex V2 + g): its corners 16g + 4j + 2, j = 0..3,
  in column order; C edge (slot N2 + 4g + j) pairs quad j with quad j - 1;
* a PP edge point e (P vertex V2 + F2 + e, half-edges h: v -> u with v < u,
  and h2): its corners {4h+1, 4nh+3, 4h2+1, 4nh2+3}; the lane of 4h+1 has
  the first two, and rebuilds the face points of quads 4h2+1 and 4nh2+3 from
  three gathered positions (P's face points of P faces h2 and nh2, and C's
  vertex on the P edge between them) and two values of its own group; the
  quads of C's edges around it cycle 4h+1 -> 4nh+3 -> 4h2+1 -> 4nh2+3.

Only PP's old vertices keep records (slots below N2).  The numpy restatement
below uses exactly those inputs and that float order, and must reproduce the
oracle's refine(C) bit for bit."""
import numpy as np
import pytest

import oracle
from slak_b200 import meshgen
from slak_b200.mesh import LAK, QUAD, SLAK, Mesh

from test_fast_formulas import _closed_quad, brute_state, qn, qp

f32 = np.float32


def _q(r, scheme):
    return Mesh(QUAD, r.ids, r.verts, r.ptr if scheme == LAK else None, r.vals if scheme == LAK else None,
                r.nfaces, 4, True)


def _fp_slak(c0, c1, c2, c3):
    return ((c0 + c2) + (c1 + c3)) * f32(0.25)


def _fp_lak(c0, c1, c2, c3):
    return ((((f32(0) + c0) + c1) + c2) + c3) / f32(4) + f32(0)


def _vp_slak(Pv, nb, fq):
    acc = np.zeros_like(Pv)
    for t in nb:
        acc = acc + t
    y = acc / f32(16) + (Pv * f32(2)) / f32(4)
    for t in fq:
        y = y + t / f32(16)
    return y


def _vp_lak(Pv, tails, tid, fq):
    acc = np.zeros_like(Pv)
    for t in fq:
        acc = acc + t
    order = np.argsort(np.stack(tid, 1), axis=1, kind="stable")
    T = np.stack(tails, 1)
    for r in range(4):
        acc = acc + np.take_along_axis(T, order[:, r, None, None].repeat(4, 2), 1)[:, 0]
    return ((acc / f32(4) + f32(0)) + Pv * f32(2)) / f32(4) + f32(0)


def _ep(Pv, fq, nb, fr):
    return (f32(0) + (Pv + fq) * f32(0.25)) + (nb + fr) * f32(0.25)


CASES = [("torus", lambda: meshgen.torus(6, 5, seed=1)),
         ("mixed", lambda: meshgen.mixed_torus(12, 10, 0.1, 0.06, 0.005, seed=5)),
         ("cylinder", lambda: meshgen.capped_cylinder(8, 4, 0.001, seed=6)),
         ("ico", lambda: meshgen.icosphere(2, 0.02, seed=4))]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_grandparent_quad_columns(name, make, scheme):
    base = make()
    if scheme == LAK and base.ptr is None:
        base = base.with_quad_ptr()
    PP = _closed_quad(base, scheme)                              # closed quad mesh
    Pr = oracle.level(PP if scheme == SLAK else PP.with_quad_ptr(), scheme, poly=False)
    Cr = oracle.level(_q(Pr, scheme), scheme, poly=False)
    Rr = oracle.level(_q(Cr, scheme), scheme, poly=False)       # refine(C): the oracle's
    N2, V2 = PP.nnz, PP.nverts
    F2, E2 = N2 // 4, N2 // 2
    N1, V1, F1 = Pr.nnz, Pr.nverts, Pr.nfaces
    assert N1 == 4 * N2 and F1 == N2 and V1 == V2 + F2 + E2
    VC, FC = Cr.nverts, Cr.nfaces
    stP = brute_state(Pr.ids, V1, scheme)
    idsP, idsC = Pr.ids.astype(np.int64), Cr.ids.astype(np.int64)
    C = Cr.verts                                                  # C's positions (float32, N x 4)
    R = Rr.verts
    x = np.arange(N1)
    Q = idsC.reshape(N1, 4)
    c0, c1, c2, c3 = C[Q[:, 0]], C[Q[:, 1]], C[Q[:, 2]], C[Q[:, 3]]
    fp = _fp_slak(c0, c1, c2, c3) if scheme == SLAK else _fp_lak(c0, c1, c2, c3)
    assert np.array_equal(fp.view(np.uint32), R[VC + x].view(np.uint32))       # C's face points
    EPb = VC + FC

    # the slot layout the closed form relies on
    assert np.array_equal(stP["sptr"][V2:V2 + F2], N2 + 4 * np.arange(F2))
    assert np.array_equal(stP["sptr"][V2 + F2:V1], 2 * N2 + 4 * np.arange(E2))

    # ---- PP face points: P vertex V2 + g, lanes 16g + 4j + 2
    g = np.arange(F2)
    lane = 16 * g[:, None] + 4 * np.arange(4)[None, :] + 2            # [F2, 4] column order
    assert np.array_equal(stP["sc"][N2:2 * N2].reshape(F2, 4), lane)
    Pv = c0[lane[:, 0]]
    assert (Q[lane, 0] == (V2 + g)[:, None]).all()
    if scheme == SLAK:
        vp = _vp_slak(Pv, [c1[lane[:, j]] for j in range(4)], [fp[lane[:, j]] for j in range(4)])
        for j in range(4):
            ep = _ep(Pv, fp[lane[:, j]], c1[lane[:, j]], fp[lane[:, (j + 3) & 3]])
            assert np.array_equal(ep.view(np.uint32), R[EPb + N2 + 4 * g + j].view(np.uint32))
    else:
        vp = _vp_lak(Pv, [c3[lane[:, j]] for j in range(4)], [Q[lane[:, j], 3] for j in range(4)],
                     [fp[lane[:, j]] for j in range(4)])
    assert np.array_equal(vp.view(np.uint32), R[V2 + g].view(np.uint32))

    # ---- PP edge points: the lane of 4h+1, h the PP half-edge v -> u with v < u
    h = np.arange(N2)
    nh = qn(h)
    own = idsP[4 * h] < idsP[4 * nh]
    h = h[own]
    nh = qn(h)
    e = idsP[4 * h + 1] - V2 - F2                                # the PP edge (P vertex V2 + F2 + e)
    assert np.array_equal(np.sort(e), np.arange(E2))             # each PP edge once
    twP0 = stP["tw"][4 * h]                                       # = 4 nh2 + 3 (lane 4h's state)
    assert ((twP0 & 3) == 3).all()
    nh2 = twP0 >> 2
    h2 = qp(nh2)
    A, B, C2, D2 = 4 * h + 1, 4 * nh + 3, 4 * h2 + 1, 4 * nh2 + 3
    Pv = c0[A]
    # the three gathers, by closed-form ids, and the two values of the own group
    fh2, fnh2 = V1 + h2, V1 + nh2                                 # C vertices: P's face points
    if scheme == SLAK:
        X = V1 + F1 + N2 + nh2                                    # C vertex on P edge (ep(e) -> PP face point)
    else:
        fpp_h, fpp_h2 = h >> 2, h2 >> 2                           # PP faces of h and h2
        X = V1 + F1 + 4 * e + 2 + (fpp_h2 > fpp_h)
    assert np.array_equal(Q[C2, 1], X) and np.array_equal(Q[D2, 3], X)
    assert np.array_equal(Q[C2, 2], fh2) and np.array_equal(Q[D2, 2], fnh2)
    assert np.array_equal(Q[C2, 3], Q[B, 1]) and np.array_equal(Q[D2, 1], Q[4 * h, 1])
    PX, Pf2, Pfn2 = C[X], C[fh2], C[fnh2]
    c1B, c1h0 = c1[B], c1[4 * h]
    if scheme == SLAK:
        fC2 = _fp_slak(Pv, PX, Pf2, c1B)
        fD2 = _fp_slak(Pv, c1h0, Pfn2, PX)
    else:
        fC2 = _fp_lak(Pv, PX, Pf2, c1B)
        fD2 = _fp_lak(Pv, c1h0, Pfn2, PX)
    assert np.array_equal(fC2.view(np.uint32), fp[C2].view(np.uint32))
    assert np.array_equal(fD2.view(np.uint32), fp[D2].view(np.uint32))
    corner = np.stack([A, B, C2, D2], 1)
    nb = np.stack([c1[A], c1B, PX, c1h0], 1)                       # SLAK: e_out of each quad
    tl = np.stack([c3[A], c3[B], c1B, PX], 1)                      # LAK: e_in of each quad
    tid = np.stack([Q[A, 3], Q[B, 3], Q[B, 1], X], 1)
    fq = np.stack([fp[A], fp[B], fC2, fD2], 1)
    order = np.argsort(corner, 1)                                  # column order
    take = lambda a, r: np.take_along_axis(a, order[:, r, None, None].repeat(4, 2), 1)[:, 0] if a.ndim == 3 \
        else np.take_along_axis(a, order[:, r, None], 1)[:, 0]
    v = V2 + F2 + e
    b = 2 * N2 + 4 * e
    assert np.array_equal(stP["sptr"][v], b)
    for r in range(4):
        assert np.array_equal(stP["sc"][b + r], take(corner, r))
    if scheme == SLAK:
        vp = _vp_slak(Pv, [take(nb, r) for r in range(4)], [take(fq, r) for r in range(4)])
        for k in range(4):                                         # quad k's edge pairs it with quad k+1 (cyclic)
            ep = _ep(Pv, fq[:, k], nb[:, k], fq[:, (k + 1) & 3])
            rank = (corner < corner[:, k, None]).sum(1)
            assert np.array_equal(ep.view(np.uint32), R[EPb + b + rank].view(np.uint32))
    else:
        vp = _vp_lak(Pv, [tl[:, k] for k in range(4)], [tid[:, k] for k in range(4)],
                     [take(fq, r) for r in range(4)])
    assert np.array_equal(vp.view(np.uint32), R[v].view(np.uint32))


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_parent_state_from_grandparent(name, make, scheme):
    """The last level's parent state in closed form (k_g1 / k_g3 with SG):
    P = refine(PP), PP a closed quad mesh.  P corner x = 4y + k takes its twin,
    slot and (SLAK) t from PP's twin / slot / t at y and prev(y) and from the
    P vertex at corner x itself (for k = 1, 3 an edge point V2 + F2 + e); P's
    column offsets come from PP's for PP's old vertices and in closed form for
    face points (N2 + 4g) and edge points (2 N2 + 4e)."""
    base = make()
    if scheme == LAK and base.ptr is None:
        base = base.with_quad_ptr()
    PP = _closed_quad(base, scheme)
    Pr = oracle.level(PP if scheme == SLAK else PP.with_quad_ptr(), scheme, poly=False)
    N2, V2 = PP.nnz, PP.nverts
    F2 = N2 // 4
    stPP = brute_state(PP.ids, V2, scheme)
    stP = brute_state(Pr.ids, Pr.nverts, scheme)
    idsP = Pr.ids.astype(np.int64)
    x = np.arange(Pr.nnz)
    y, k = x >> 2, x & 3
    nx, px = qn(y), qp(y)
    tw2, tw2p = stPP["tw"][y], stPP["tw"][px]
    ntw, ntwp = qn(tw2), qn(tw2p)
    eidp = idsP[x] - V2 - F2                              # k = 1: e_out(y); k = 3: e_in(y)
    rk = lambda a, b, c, d: (b < a).astype(np.int64) + (c < a) + (d < a)
    A, B, Cc, D = 4 * y + 1, 4 * tw2 + 1, 4 * nx + 3, 4 * ntw + 3
    A2, B2, C2, D2 = 4 * px + 1, 4 * tw2p + 1, 4 * y + 3, 4 * ntwp + 3
    base_ = 2 * N2 + 4 * eidp
    tw = np.select([k == 0, k == 1, k == 2], [4 * ntw + 3, 4 * nx + 2, 4 * px + 1], 4 * tw2p)
    slot = np.select([k == 0, k == 1, k == 2], [stPP["slot"][y], base_ + rk(A, B, Cc, D), N2 + y],
                     base_ + rk(C2, A2, B2, D2))
    assert np.array_equal(tw, stP["tw"])
    assert np.array_equal(slot, stP["slot"])
    if scheme == SLAK:
        t = np.select([k == 0, k == 1, k == 2], [stPP["t"][y], base_ + rk(D, A, B, Cc), N2 + nx],
                      base_ + rk(A2, B2, C2, D2))
        assert np.array_equal(t, stP["t"])
    v = np.arange(Pr.nverts + 1)
    E2 = N2 // 2
    sptr = np.where(v < V2, stPP["sptr"][np.minimum(v, V2)],
                    np.where(v < V2 + F2, N2 + 4 * (v - V2), 2 * N2 + 4 * (v - V2 - F2)))
    assert np.array_equal(sptr, stP["sptr"])
    assert sptr[-1] == 4 * N2 and Pr.nverts == V2 + F2 + E2
