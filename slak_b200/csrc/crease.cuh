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

constexpr unsigned long long kCreaseDeadKey = ~0ull;

// Level 0: crease pair (a, b) -> the half-edge min(a,b) -> max(a,b), looked up
// in the level's vertex columns (slot s of vertex v holds corner sc[s], whose
// half-edge goes to snext[s]).  A pair that is not an edge of the mesh, or an
// interior edge named twice, is an error; a boundary edge or sharpness <= 0
// gives a dead entry (cc = -1).
__global__ void k_crease_resolve(const int* __restrict__ pairs, const float* __restrict__ sharp, int m, int V,
                                 const int* __restrict__ sptr, const int* __restrict__ sc,
                                 const int* __restrict__ snext, int* __restrict__ mark, int* __restrict__ cc,
                                 float* __restrict__ cs, DevStatus* st)
{
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
    if (atomicAdd(mark + c_up, 1) != 0) { set_error(st, 4, 3000000 + i); return; }
    cc[i] = c_up;
    cs[i] = s;
}

// Boundary flag of every base vertex (any slot with a boundary half-edge).
__global__ void k_crease_bnd0(int V, const int* __restrict__ sptr, const int* __restrict__ sflag, int mask,
                              unsigned char* __restrict__ bnd0)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    int f = 0;
    for (int k = __ldg(sptr + v), e = __ldg(sptr + v + 1); k < e; ++k) f |= __ldg(sflag + k);
    bnd0[v] = (f & mask) != 0;
}

// Edge points of the level's crease edges; incidence records (v, other) for
// the vertex pass; the next level's crease list (ncc == nullptr on the last
// crease level).
template <bool QUAD>
__global__ void k_crease_edges(Faces<QUAD> fc, const int* __restrict__ ids, const int* __restrict__ rids,
                               const float* __restrict__ P, float* __restrict__ R, const int* __restrict__ cc,
                               const float* __restrict__ cs, int n, unsigned long long* __restrict__ keys,
                               int* __restrict__ vals, int* __restrict__ ncc, float* __restrict__ ncs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cc[i];
    vals[2 * i] = vals[2 * i + 1] = i;
    if (c < 0) {
        keys[2 * i] = keys[2 * i + 1] = kCreaseDeadKey;
        if (ncc) ncc[2 * i] = ncc[2 * i + 1] = -1;
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
    keys[2 * i] = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    keys[2 * i + 1] = ((unsigned long long)(unsigned)b << 32) | (unsigned)a;
    if (ncc) {
        const bool live = s > 1.0f;
        ncc[2 * i] = live ? 4 * c : -1;
        ncc[2 * i + 1] = live ? 4 * nc + 3 : -1;
        ncs[2 * i] = ncs[2 * i + 1] = live ? __fsub_rn(s, 1.0f) : 0.0f;
    }
}

// Vertex points of crease vertices, over the incidence records sorted by
// (vertex, other end): the first record of each vertex evaluates it.
__global__ void k_crease_verts(const unsigned long long* __restrict__ keys, const int* __restrict__ vals, int n2,
                               const float* __restrict__ cs, const unsigned char* __restrict__ bnd0, int V0,
                               const float* __restrict__ P, float* __restrict__ R)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n2) return;
    const unsigned long long key = keys[j];
    if (key == kCreaseDeadKey) return;
    const unsigned v = (unsigned)(key >> 32);
    if (j > 0 && (unsigned)(keys[j - 1] >> 32) == v) return;
    int k = 0, o[2] = {0, 0};
    float ssum = 0.0f;
    for (int t = j; t < n2; ++t) {
        const unsigned long long kt = keys[t];
        if ((unsigned)(kt >> 32) != v || kt == kCreaseDeadKey) break;
        if (k < 2) o[k] = (int)(unsigned)(kt & 0xffffffffu);
        ssum = __fadd_rn(ssum, __ldg(cs + vals[t]));
        ++k;
    }
    float w = __fdiv_rn(ssum, (float)k);
    if (w > 1.0f) w = 1.0f;
    const bool bnd = bnd0 != nullptr && (int)v < V0 && bnd0[v] != 0;
    const float4 pv = ldg4(P, v);
    float4 sharp;
    if (bnd || k >= 3) sharp = pv;
    else if (k == 1) return;
    else sharp = f4_add(f4_add(f4_mul(pv, 0.75f), f4_mul(ldg4(P, o[0]), 0.125f)), f4_mul(ldg4(P, o[1]), 0.125f));
    float4 r = sharp;
    if (!(w >= 1.0f)) r = f4_add(f4_mul(ldg4(R, v), __fsub_rn(1.0f, w)), f4_mul(sharp, w));
    st4(R, v, r);
}

}  // namespace slak
