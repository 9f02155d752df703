// crease.cuh -- semi-sharp creases, applied after each level's smooth
// refinement.
//
// The reference declares this step but does not implement it
// (LibSource/device/CatmullClarkImpl.cu:94-96 and :296-298,
// LibSource/device/LAKCatmullClarkImpl.cu:240-242: "if (has_creases &&
// !creases_decayed) time += handleCreases(...)", commented out).  The rules
// here are the published ones of DeRose, Kass and Truong, "Subdivision Surfaces
// in Character Animation" (SIGGRAPH 1998), with sharpness decaying by one per
// level:
//
//   edge point of a crease edge {a, b} of sharpness s:
//     s >= 1: (p_a + p_b) / 2;  0 < s < 1: smooth (1 - s) + sharp s
//   vertex point of a vertex v with k incident crease edges, w = min(1, mean s):
//     boundary vertex (k >= 1): corner, sharp = p_v
//     k == 1: smooth (a dart)
//     k == 2: sharp = (3/4 p_v + 1/8 p_o1) + 1/8 p_o2 (o1 < o2, the crease's other ends)
//     k >= 3: corner, sharp = p_v
//     result: w >= 1 ? sharp : smooth (1 - w) + sharp w
//   a corner (vertex sharpness s_v, a base vertex): p_v while s_v - level > 0,
//     blended by max(min(1, s_v - level), min(1, mean s of its crease edges))
//   a crease half-edge c (a -> b) of sharpness s > 1 leaves two child
//   half-edges of sharpness s - 1 in the refined mesh: corner 4c (a -> ep) and
//   corner 4 next(c) + 3 (ep -> b).
//
// Smooth values are the ones the level's kernels wrote: the edge and vertex
// rules only read the level's input positions P, and a crease edge point and a
// crease vertex are distinct refined vertices, so the two passes may run in
// either order.  A boundary edge is already sharp (midpoint) and takes no
// crease; a vertex is a boundary vertex at every level iff it is one of the
// base mesh's boundary vertices (edge points of interior creases are interior).
// Sharpness sums run in ascending order of the other end's id, so the results
// are deterministic; arithmetic is IEEE binary32 without contraction.
#pragma once

#include "common.cuh"

namespace slak {

// Where a level's crease vertices find their crease edges, without a sort.
// Crease incidence is inherited from level to level:
//  * a base-mesh vertex v touches, at level 0, the entries j0 listed in its
//    CSR row (inc = j0 << 1 | side; side 0: v is the origin a of the entry's
//    half-edge, side 1: its head b).  At level l that edge's descendant at v is
//    entry (j0 << l) + side (2^l - 1): the child on a's side of entry j is 2j,
//    on b's side 2j + 1;
//  * the edge point ep of entry j of level t (made when its sharpness was
//    > 1) touches exactly the two children of j, and at level l > t their
//    descendants (2j << d) + 2^d - 1 (ep is their head) and (2j + 1) << d (ep
//    is their origin), d = l - t - 1; both carry the same sharpness.
// epid[t][j] is that edge point's vertex id (-1 if j was dead or s <= 1).
constexpr int kMaxCreaseLevels = 30;

struct CreaseEps {
    const int* epid[kMaxCreaseLevels];
};

// Level 0: crease pair (a, b) -> the half-edge min(a,b) -> max(a,b), looked up
// in the level's vertex columns (slot s of vertex v holds corner sc[s], whose
// half-edge goes to snext[s]).  A pair that is not an edge of the mesh, or an
// interior edge named twice, is an error; a boundary edge or sharpness <= 0
// gives a dead entry (cc = -1).  mark[corner] = entry + 1 for live entries.
__global__ void k_crease_resolve(const int* __restrict__ pairs, const float* __restrict__ sharp, int m, int V,
                                 const int* __restrict__ sptr, const int* __restrict__ sc,
                                 const int* __restrict__ snext, int* __restrict__ mark, int* __restrict__ cc,
                                 float* __restrict__ cs, DevStatus* st)
{
    griddep_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int a = __ldg(pairs + 2 * i), b = __ldg(pairs + 2 * i + 1);
    const float s = __ldg(sharp + i);
    cc[i] = -1;
    cs[i] = 0.0f;
    if (a < 0 || b < 0 || a >= V || b >= V || a == b) { set_error(st, 4, 3000000 + i); return; }
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    const auto find = [&](int u, int w) {
        for (int k = __ldg(sptr + u), e = __ldg(sptr + u + 1); k < e; ++k)
            if (__ldg(snext + k) == w) return __ldg(sc + k);
        return -1;
    };
    const int c_up = find(lo, hi), c_dn = find(hi, lo);
    if (c_up < 0 && c_dn < 0) { set_error(st, 4, 3000000 + i); return; }
    if (c_up < 0 || c_dn < 0 || !(s > 0.0f)) return;
    if (atomicCAS(mark + c_up, 0, i + 1) != 0) { set_error(st, 4, 3000000 + i); return; }
    cc[i] = c_up;
    cs[i] = s;
}

// Level 0, per base vertex: live crease edges at v from its column (corner
// sc[s] leaves v, corner sprevc[s] arrives at v), and the boundary flag.
// FILL = false counts into vcnt; FILL = true writes the CSR row.
template <bool FILL>
__global__ void k_crease_vinc(int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                              const int* __restrict__ sprevc, const int* __restrict__ sflag, int bmask,
                              const int* __restrict__ mark, int* __restrict__ vcnt, unsigned char* __restrict__ bnd0,
                              const int* __restrict__ vptr, int* __restrict__ inc)
{
    griddep_enter();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    int k = 0, f = 0;
    const int o = FILL ? __ldg(vptr + v) : 0;
    for (int s = __ldg(sptr + v), e = __ldg(sptr + v + 1); s < e; ++s) {
        const int out = __ldg(mark + __ldg(sc + s)), in = __ldg(mark + __ldg(sprevc + s));
        if (out > 0) { if (FILL) inc[o + k] = (out - 1) << 1; ++k; }
        if (in > 0) { if (FILL) inc[o + k] = ((in - 1) << 1) | 1; ++k; }
        if (!FILL) f |= __ldg(sflag + s);
    }
    if (!FILL) {
        vcnt[v] = k;
        if (bnd0) bnd0[v] = (f & bmask) != 0;
    }
}

// Edge points of the level's crease edges; the next level's crease list and
// the edge points that become crease vertices (ncc == nullptr on the last
// crease level).
template <bool QUAD>
__global__ void k_crease_edges(Faces<QUAD> fc, const int* __restrict__ ids, const int* __restrict__ rids,
                               const float* __restrict__ P, float* __restrict__ R, const int* __restrict__ cc,
                               const float* __restrict__ cs, int n, int* __restrict__ ncc, float* __restrict__ ncs,
                               int* __restrict__ epid)
{
    griddep_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cc[i];
    if (c < 0) {
        if (ncc) { ncc[2 * i] = ncc[2 * i + 1] = -1; epid[i] = -1; }
        return;
    }
    const float s = cs[i];
    const int nc = fc.next(c);
    const int a = __ldg(ids + c), b = __ldg(ids + nc);
    const int ep = __ldg(rids + 4 * (int64_t)c + 1);
    const float4 sharp = f4_mul(f4_add(ldg4(P, a), ldg4(P, b)), 0.5f);
    float4 r = sharp;
    if (!(s >= 1.0f)) r = f4_add(f4_mul(ldg4(R, ep), __fsub_rn(1.0f, s)), f4_mul(sharp, s));
    st4(R, ep, r);
    if (ncc) {
        const bool live = s > 1.0f;
        ncc[2 * i] = live ? 4 * c : -1;
        ncc[2 * i + 1] = live ? 4 * nc + 3 : -1;
        ncs[2 * i] = ncs[2 * i + 1] = live ? __fsub_rn(s, 1.0f) : 0.0f;
        epid[i] = live ? ep : -1;
    }
}

// The vertex rule from a vertex's crease edges (other ends and sharpness).
__device__ __forceinline__ void crease_vertex(const float* __restrict__ P, float* __restrict__ R, int v, int k,
                                              int o1, int o2, float ssum, bool bnd)
{
    float w = __fdiv_rn(ssum, (float)k);
    if (w > 1.0f) w = 1.0f;
    const float4 pv = ldg4(P, v);
    float4 sharp;
    if (bnd || k >= 3) sharp = pv;
    else if (k == 1) return;
    else sharp = f4_add(f4_add(f4_mul(pv, 0.75f), f4_mul(ldg4(P, o1), 0.125f)), f4_mul(ldg4(P, o2), 0.125f));
    float4 r = sharp;
    if (!(w >= 1.0f)) r = f4_add(f4_mul(ldg4(R, v), __fsub_rn(1.0f, w)), f4_mul(sharp, w));
    st4(R, v, r);
}

// Vertex points of the level's crease vertices: threads [0, V0) the base
// vertices (CSR rows), then one thread per entry of every earlier level t < l
// (m 2^t each) for the edge points they made.  Sharpness sums run in ascending
// order of the other end's id.
template <bool QUAD>
__global__ void k_crease_verts(Faces<QUAD> fc, int l, int V0, int64_t m, const int* __restrict__ ids,
                               const int* __restrict__ cc, const float* __restrict__ cs,
                               const int* __restrict__ vcnt, const int* __restrict__ vptr,
                               const int* __restrict__ inc, const unsigned char* __restrict__ bnd0, CreaseEps eps,
                               const float* __restrict__ vcs, const float* __restrict__ P, float* __restrict__ R)
{
    griddep_enter();
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < V0) {
        const int v = (int)idx;
        // corner sharpness left at this level (vertex sharpness decays by one per level)
        const float cv = vcs ? __fsub_rn(__ldg(vcs + v), (float)l) : 0.0f;
        if (__ldg(vcnt + v) == 0 && !(cv > 0.0f)) return;
        const int b = __ldg(vptr + v), e = __ldg(vptr + v + 1);
        const int lm = (1 << l) - 1;
        // the live descendants' other ends, visited in ascending id
        const auto other = [&](int r, float* sr) {
            const int x = __ldg(inc + r), side = x & 1;
            const int jl = ((x >> 1) << l) + (side ? lm : 0);
            const int c = cc[jl];
            if (c < 0) return INT32_MAX;
            *sr = cs[jl];
            return side ? __ldg(ids + c) : __ldg(ids + fc.next(c));
        };
        int k = 0, o[2] = {0, 0}, last = -1;
        float ssum = 0.0f;
        while (true) {
            int best = INT32_MAX;
            float sb = 0.0f;
            for (int r = b; r < e; ++r) {
                float sr;
                const int x = other(r, &sr);
                if (x > last && x < best) { best = x; sb = sr; }
            }
            if (best == INT32_MAX) break;
            if (k < 2) o[k] = best;
            ssum = __fadd_rn(ssum, sb);
            ++k;
            last = best;
        }
        if (cv > 0.0f) {                // a corner: p_v, blended by max(min(1, cv), min(1, mean s))
            float wk = 0.0f;
            if (k > 0) {
                wk = __fdiv_rn(ssum, (float)k);
                if (wk > 1.0f) wk = 1.0f;
            }
            const float wc = cv < 1.0f ? cv : 1.0f;
            const float w = wc > wk ? wc : wk;
            const float4 pv = ldg4(P, v);
            float4 r = pv;
            if (!(w >= 1.0f)) r = f4_add(f4_mul(ldg4(R, v), __fsub_rn(1.0f, w)), f4_mul(pv, w));
            st4(R, v, r);
            return;
        }
        if (k == 0) return;
        crease_vertex(P, R, v, k, o[0], o[1], ssum, bnd0 != nullptr && bnd0[v] != 0);
        return;
    }
    // an edge point made at level t by entry j
    int64_t q = idx - V0;
    int t = 0;
    while (t < l && q >= (m << t)) { q -= m << t; ++t; }
    if (t >= l) return;
    const int ep = __ldg(eps.epid[t] + q);
    if (ep < 0) return;
    const int d = l - t - 1;
    const int jb = (int)((2 * q) << d) + ((1 << d) - 1), ja = (int)((2 * q + 1) << d);
    const int cb = cc[jb];
    if (cb < 0) return;                       // both descendants decayed together
    const int ca = cc[ja];
    const int ob = __ldg(ids + cb), oa = __ldg(ids + fc.next(ca));
    const float s = cs[jb];
    const float ssum = __fadd_rn(__fadd_rn(0.0f, s), s);
    crease_vertex(P, R, ep, 2, ob < oa ? ob : oa, ob < oa ? oa : ob, ssum, false);
}

}  // namespace slak
