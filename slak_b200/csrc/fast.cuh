// fast.cuh -- closed-form refinement of an already refined quad mesh.
//
// Let P be a closed quad mesh (N1 corners, V1 vertices, F1 = N1/4 faces,
// E1 = N1/2 edges) and C = refine(P) the level being refined now: quad x of C
// is corner x of P, corner 4x+k of C is corner k of that quad, and C's
// vertices are [V1 old | F1 face points | E1 edge points].  Everything the
// general path rebuilds with atomics, sorting and searching is then known in
// closed form from P's adjacency state:
//
//   sptr1         P's vertex columns (offsets; a column holds its vertex's
//                 corners in corner order)
//   slot1         corner -> its slot in its vertex's column
//   tw1           twin half-edge of each corner of P
//   t1            slot1[tw1[prev(x)]] (SLAK)
//
// C's adjacency: vertex v < V1 keeps its column with corners 4x (x in
// column order), face point V1+g owns corners 4x+2 of g's four corners,
// edge point V1+F1+e owns the sorted corners {4h+1, 4h'+1, 4nh+3, 4nh'+3} of
// e's half-edges (h, h').  C's edge ids (serialized atomics of the reference):
//   SLAK  eid(4x+0) = slot1(x), eid(4x+1) = N1 + next(x), eid(4x+2) = N1 + x,
//         eid(4x+3) = slot1(tw1(prev x))            [owners ranked by (tail, corner)]
//   LAK   edges around edge point e are 4e + {lower end, higher end,
//         lower face point, higher face point}      [ascending (max, min)]
//
// Two kernels per level when P has quad faces, four when P is the polygon
// input; every output is written exactly once:
//   k_g1  per quad of C: C's refined quads, face points of C and the next
//         level's per-corner state; with quad P (4 lanes per face of P) also
//         the vertex points of P's face and edge points, SLAK edge points N1+x
//         and LAK's edge points
//   k_gf  polygon P: per face of P, its face point's vertex point, SLAK N1+x
//   k_g2  polygon P: per edge of P, visited in corner order (the min->max
//         half-edge's lane): vertex points of P's edge points, LAK edge points
//   k_g3  per vertex of P: vertex points of P's vertices and SLAK edge points
//         slot1(x), streamed from slot-ordered records k_g1 scatters
// The float arithmetic and its order are exactly the general path's (and the
// reference's serialized order), so both paths are bit-identical.
#pragma once

#include "common.cuh"

namespace slak {

#ifdef SLAK_FACE_SUM_SHFL
constexpr bool kFaceSumShfl = true;       // comparison builds: the face sums by warp shuffles throughout
#else
constexpr bool kFaceSumShfl = false;
#endif
#ifdef SLAK_NO_TMA_STORE
constexpr bool kTmaQuadStore = false;     // comparison builds: refined quads by coalesced stores
#else
constexpr bool kTmaQuadStore = true;
#endif

__device__ __forceinline__ int qnext(int x) { return (x & ~3) | ((x + 1) & 3); }
__device__ __forceinline__ int qprev(int x) { return (x & ~3) | ((x + 3) & 3); }

// P's adjacency state (read) / C's (written when another level follows)
struct QState {
    int* sptr;
    int* slot;
    int* tw;       // -1: no twin (boundary half-edge)
    int* t;        // -1: the previous corner's half-edge has no twin
    int* brank;    // per edge: boundary edges with a smaller id (meshes with a boundary)
};

struct FastDims {
    int N1, V1, F1, E1;    // P
    int V, N;              // C (F = N1, E = 2 N1 + B1)
    int B1;                // P's boundary edges (0: closed)
    int N2 = 0, V2 = 0, F2 = 0;   // GQ levels: P's parent PP (a closed quad mesh)
};

__device__ __forceinline__ float4 shfl4_xor(float4 v, int m)
{
    return make_float4(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m),
                       __shfl_xor_sync(0xffffffffu, v.z, m), __shfl_xor_sync(0xffffffffu, v.w, m));
}

// A refined position.  At the last level (no STATE) no kernel of the level
// reads it again, so it is stored streaming (measured on B200: the 512x512
// mixed torus takes 1.376 instead of 1.384 ms with LAK, 1.278 instead of
// 1.280 ms with SLAK).
template <bool STATE>
__device__ __forceinline__ void st_pos(float* R, int64_t i, float4 v)
{
    if constexpr (STATE) st4(R, i, v);
    else st4_cs(R, i, v);
}

// A slot record {face point, neighbour} (Z[2s], Z[2s+1]: 32 bytes, 32-byte
// aligned), written by k_g1 and read back once by k_g3, moves as one 256-bit
// access (sm_100's widest vector load / store): one L1 wavefront per lane
// instead of two.  The store carries an L2 evict-last policy (measured on
// B200, 512x512 mixed torus, SLAK: k_g1's last level 641 -> 619 us, k_g3's
// time unchanged); the load is a read-only (non-coherent) one, as __ldg.
__device__ __forceinline__ void st8_keep(float4* p, float4 a, float4 b)
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("st.global.L2::cache_hint.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8}, %9;"
                 :: "l"(p), "f"(a.x), "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w),
                    "l"(pol));
}
__device__ __forceinline__ void ld8_nc(const float4* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// Two refined quads (32 bytes, 32-byte aligned) as one 256-bit streaming
// store: a thread's four quads are 64 contiguous bytes, two full sectors.
__device__ __forceinline__ void st8_cs(int4* p, int4 a, int4 b)
{
    asm volatile("st.global.cs.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
                 :: "l"(p), "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
                 : "memory");
}

// rank of corner `a` among the four corners of an edge point
__device__ __forceinline__ int rank4(int a, int b, int c, int d) { return (b < a) + (c < a) + (d < a); }

// ---------------------------------------------------------------------------------------------
// G1: one thread per quad x of C (= corner x of P); the 4 quads of a face of P
// are 4 consecutive lanes.  Each thread loads its quad {v, e_out, f, e_in} as
// one int4 and the 4 corner positions, so the face point needs no exchange;
// its 4 refined quads are 64 contiguous bytes of the output.
// Slot-ordered records for the per-vertex pass (k_g3): for the corner x of P
// at slot s = slot1(x), Z[2s] = FP(x) and Z[2s+1] = the position of C's next
// (SLAK: e_out(x)) or previous (LAK: e_in(x)) vertex of corner 4x.  LAK:
// T[s] = that vertex id (for the ascending-id order).  SLAK: rot[t1(x)] = s.
// The corner y at slot t1(x) = slot1(tw(prev x)) is x's neighbour around their
// vertex across the edge e_in(x) = e_out(y), so half-edge 4x+3's share of SLAK
// edge point t1(x), (P[e_in(x)] + FP(x)) / 4, is (Z[2 t1(x) + 1] + Z[2 rot]) / 4:
// two records of the same column, which k_g3 has loaded anyway.
// Meshes with a boundary add, per slot: bflag (bit 0: the corner's outgoing
// half-edge has no twin, bit 1: its incoming one), bid (the boundary neighbour
// the records lack: SLAK e_in(x), LAK e_out(x)) and bscan (bit 0 again, the
// input of the scan that ranks C's boundary edges, SLAK).
struct SlotScratch {
    float4* Z;
    int* T;      // LAK
    int* rot;    // SLAK (the same memory as T: one scheme per plan)
    int* bflag;
    int* bid;
    int* bscan;
};

// C's slot / twin / t for its corners 4x+k (the state the next fast level
// reads).  With a boundary, a P edge without a twin gives its edge point 2
// corners instead of 4 (absent corners rank last), its columns start at
// 2 N1 + 4e - 2 brank(e), and C's half-edges along it have no twin.
template <bool LAK>
__device__ __forceinline__ void write_state(const FastDims& d, QState& c, int x, int nxx, int px, int tw1x,
                                            int tw1_px, int ntw, int ntwp, int s1, int t1x, int eidp_x,
                                            int eidp_px, int br_x = 0, int br_px = 0)
{
    const bool tx = tw1x >= 0, tpx = tw1_px >= 0;
    // edge of P through x: corners A=4x+1, B=4tw1x+1, Cc=4nxx+3, D=4ntw+3
    const int A = 4 * x + 1, B = tx ? 4 * tw1x + 1 : INT32_MAX, Cc = 4 * nxx + 3, D = tx ? 4 * ntw + 3 : INT32_MAX;
    // edge of P through prev(x): A'=4px+1, B'=4tw1_px+1, C'=4x+3, D'=4ntwp+3
    const int A2 = 4 * px + 1, B2 = tpx ? 4 * tw1_px + 1 : INT32_MAX, C2 = 4 * x + 3;
    const int D2 = tpx ? 4 * ntwp + 3 : INT32_MAX;
    const int base_x = 2 * d.N1 + 4 * eidp_x - 2 * br_x, base_px = 2 * d.N1 + 4 * eidp_px - 2 * br_px;
    reinterpret_cast<int4*>(c.tw)[x] = make_int4(tx ? 4 * ntw + 3 : -1, 4 * nxx + 2, 4 * px + 1, tpx ? 4 * tw1_px : -1);
    reinterpret_cast<int4*>(c.slot)[x] =
        make_int4(s1, base_x + rank4(A, B, Cc, D), d.N1 + x, base_px + rank4(C2, A2, B2, D2));
    if (!LAK)
        reinterpret_cast<int4*>(c.t)[x] =
            make_int4(t1x, tx ? base_x + rank4(D, A, B, Cc) : -1, d.N1 + nxx, base_px + rank4(A2, B2, C2, D2));
}

// The vertex point of P's edge point ve (edge e = ve - V1 - F1, half-edges
// h: v->u, the min->max one, and h2: u->v) and, for LAK, the four edge points
// 4e..4e+3 of C around it.  Inputs: the positions of v, u, ve and of the two
// face points fh (of h's face), fh2 (of h2's); C's face points of quads h,
// next(h), h2, next(h2).
template <bool LAK, bool STATE, bool BND = false>
__device__ __forceinline__ void edge_point_vertex(const FastDims& d, QState& c, float* __restrict__ R, int h,
                                                  int nh, int h2, int nh2, int ve, int fh, int fh2, float4 Pv,
                                                  float4 Pu, float4 Pe, float4 Pf, float4 Pf2, float4 Fh, float4 Fnh,
                                                  float4 Fh2, float4 Fnh2, int br = 0)
{
    const int e = ve - d.V1 - d.F1;
    const int ce = 4 * e - br;                 // LAK: C's first edge around ve (boundary P edges have 3)
    // corners of the edge point: A=4h+1 (nbr fh, face h), B=4h2+1 (fh2, h2), C=4nh+3 (u, nh), D=4nh2+3 (v, nh2)
    const int A = 4 * h + 1, B = 4 * h2 + 1, Cc = 4 * nh + 3, D = 4 * nh2 + 3;
    const int rA = rank4(A, B, Cc, D), rB = rank4(B, A, Cc, D), rC = rank4(Cc, A, B, D);
    float4 nb[4], fq[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        nb[r] = rA == r ? Pf : rB == r ? Pf2 : rC == r ? Pu : Pv;
        fq[r] = rA == r ? Fh : rB == r ? Fh2 : rC == r ? Fnh : Fnh2;
    }
    float4 yv;
    if (!LAK) {
        float4 acc = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) acc = f4_add(acc, nb[r]);
        yv = f4_add(f4_div(acc, 16.0f), f4_div(f4_mul(Pe, 2.0f), 4.0f));
#pragma unroll
        for (int r = 0; r < 4; ++r) yv = f4_add(yv, f4_div(fq[r], 16.0f));
    } else {
        float4 acc = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) acc = f4_add(acc, fq[r]);
        // tails {v, u, fh, fh2} in ascending id: v < u < V1 <= fh, fh2
        const bool ff = fh < fh2;
        acc = f4_add(acc, Pv);
        acc = f4_add(acc, Pu);
        acc = f4_add(acc, ff ? Pf : Pf2);
        acc = f4_add(acc, ff ? Pf2 : Pf);
        yv = f4_div_z(f4_add(f4_div_z(acc, 4.0f), f4_mul(Pe, 2.0f)), 4.0f);
    }
    st4_cs(R, ve, yv);

    if (LAK) {
        // edges 4e + {lower end, higher end, lower face point, higher face point}; v < u
        const float4 Ev = f4_mul(f4_add(f4_add(f4_add(Pv, Pe), Fh), Fnh2), 0.25f);
        const float4 Eu = f4_mul(f4_add(f4_add(f4_add(Pu, Pe), Fh2), Fnh), 0.25f);
        const float4 Ef = f4_mul(f4_add(f4_add(f4_add(Pf, Pe), Fnh), Fh), 0.25f);
        const float4 Ef2 = f4_mul(f4_add(f4_add(f4_add(Pf2, Pe), Fnh2), Fh2), 0.25f);
        const bool ff = fh < fh2;
        const int64_t base = (int64_t)d.V + d.N1 + ce;
        st4_cs(R, base + 0, Ev);
        st4_cs(R, base + 1, Eu);
        st4_cs(R, base + 2, ff ? Ef : Ef2);
        st4_cs(R, base + 3, ff ? Ef2 : Ef);
        if (STATE && BND)
            for (int k = 0; k < 4; ++k) c.brank[ce + k] = 2 * br;     // ce is not 4-aligned
    }
    if (STATE) c.sptr[ve] = 2 * d.N1 + 4 * e - 2 * br;
}

// A P edge without a twin (half-edge h: v -> u in the face of h): its edge
// point ve is on C's boundary, so its vertex point is 3/4 p + 1/8 of its two
// boundary neighbours (SLAK: u then v, correctBoundaryS2 CatmullClarkKernels.cuh
// :709-740; LAK: ascending edge id, i.e. the lower of v, u first,
// calculateExternalVertexUpdate LAKCatmullClarkKernels.cuh:483-511).  C's
// boundary edges {v, ve} and {ve, u} get midpoints (correctBoundaryS1 :688-707,
// calculateExternalEdgepoints :452-462): SLAK writes {ve, u} (id 2 N1 +
// brank(e)) here and {v, ve} (id slot(h)) in k_g3; LAK writes C's three edges
// around ve, ids 4e - brank(e) + {lower end, higher end, face point}.
template <bool LAK, bool STATE>
__device__ __forceinline__ void boundary_edge(const FastDims& d, QState& c, float* __restrict__ R, int v, int u,
                                              int ve, int br, float4 Pv, float4 Pu, float4 Pe, float4 Pf, float4 Fh,
                                              float4 Fnh)
{
    const int e = ve - d.V1 - d.F1;
    const int64_t EP = (int64_t)d.V + d.N1;
    if (!LAK) {
        st4(R, ve, f4_add(f4_add(f4_mul(Pe, 0.75f), f4_mul(Pu, 0.125f)), f4_mul(Pv, 0.125f)));
        st4_cs(R, EP + 2 * (int64_t)d.N1 + br, f4_mul(f4_add(Pe, Pu), 0.5f));
        if (STATE) c.brank[2 * d.N1 + br] = d.B1 + br;
    } else {
        const bool vu = v < u;
        const float4 Plo = vu ? Pv : Pu, Phi = vu ? Pu : Pv;
        st4(R, ve, f4_add(f4_add(f4_mul(Pe, 0.75f), f4_mul(Plo, 0.125f)), f4_mul(Phi, 0.125f)));
        const int ce = 4 * e - br;
        st4_cs(R, EP + ce + 0, f4_mul(f4_add(Plo, Pe), 0.5f));
        st4_cs(R, EP + ce + 1, f4_mul(f4_add(Phi, Pe), 0.5f));
        st4_cs(R, EP + ce + 2, f4_mul(f4_add(f4_add(f4_add(Pf, Pe), Fnh), Fh), 0.25f));
        if (STATE) { c.brank[ce] = 2 * br; c.brank[ce + 1] = 2 * br + 1; c.brank[ce + 2] = 2 * br + 2; }
    }
    if (STATE) c.sptr[ve] = 2 * d.N1 + 4 * e - 2 * br;
}

// ---------------------------------------------------------------------------------------------
// GQ: P = refine(PP) with PP a closed quad mesh (N2 corners, V2 vertices, F2 =
// N2 / 4 faces), so P corner x = 4y + k is corner k of P face y = PP corner y,
// and the 16 lanes 16g..16g+15 hold the P corners of PP face g.  Two kinds of
// P's vertex columns then lie inside those lanes, and k_g1 computes their
// vertex points (and SLAK edge points) without slot records; k_g3 keeps PP's
// old vertices (slots below N2) only.
//   PP face point V2 + g: corners 16g + 4j + 2 (j = 0..3, column order),
//     slots N2 + 4g + j; SLAK edge slot N2 + 4g + j pairs quad j with quad j-1.
//     The lane of j = 0 sums the column; each of the four lanes its edge point.
//   PP edge point V2 + F2 + e, with PP half-edges h: v -> u (v < u) and h2:
//     corners A = 4h+1 (this lane), B = 4 next(h) + 3 (same group),
//     C2 = 4 h2 + 1, D2 = 4 next(h2) + 3 (the twin's group).  C quads C2 and D2
//     are {ve, X, V1 + h2, e_out(B)} and {ve, e_out(4h), V1 + next(h2), X}: X,
//     C's vertex on the P edge between P faces h2 and next(h2), is V1 + F1 +
//     N2 + next(h2) (SLAK) or V1 + F1 + 4e + 2 + [face(h2) > face(h)] (LAK),
//     and next(h2) comes from P's twin of 4h, 4 next(h2) + 3.  So three gathers
//     (X and two of P's face points) rebuild both face points.  SLAK's four
//     edges around ve pair A-B, B-C2, C2-D2, D2-A; their ids are 2 N2 + 4e +
//     the quad's rank in the column.
// Sums and their order are k_g3's (column order; LAK tails by ascending id).
template <bool LAK, bool STATE>
__device__ __forceinline__ void gq_columns(const FastDims& d, QState& c, const float* __restrict__ P,
                                           float* __restrict__ R, bool valid, int x, int lane, const int4& Q,
                                           int tw1x, float4 c0, float4 c1, float4 c3, float4 fp)
{
    const unsigned full = 0xffffffffu;
    const int k = x & 3, j = (x >> 2) & 3;
    const int g16 = lane & ~15;                    // lane of P corner 16g
    const int l0 = lane & ~3;                      // lane of P corner 4y (y = x >> 2)
    const int ln = g16 | (((j + 1) & 3) << 2);     // lane of P corner 4 next(y)
    const int lB = ln | 3;                         // lane of P corner 4 next(y) + 3
    const int tail = __shfl_sync(full, Q.x, l0);  // PP vertex of corner y
    const int head = __shfl_sync(full, Q.x, ln);  // PP vertex of corner next(y)
    const int tw0 = __shfl_sync(full, tw1x, l0);  // P's twin of 4y: 4 next(h2) + 3
    const bool fw = valid && k == 2 && j == 0;     // sums PP face point (Q.x)'s column
    const bool ew = valid && k == 1 && tail < head;   // sums PP edge point (Q.x)'s column
    // sources of the exchanges, in column order for the face point's lane
    int src[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) src[r] = fw ? g16 | (r << 2) | 2 : lane;
    if (ew) { src[0] = lB; src[1] = l0; }
    if (!fw && !ew && k == 2) src[0] = g16 | (((j + 3) & 3) << 2) | 2;   // the previous quad's face point
    // the values from the edge point's own group: e_out of quads B and 4y, and B's face point
    float4 c1B, c1h0, fpB;
    float4 yv = f4_zero();                         // the face point's vertex point, summed as values arrive
    if (!LAK) {
        float4 acc = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float4 t = shfl4(c1, src[r]);
            acc = f4_add(acc, t);
            if (r == 0) c1B = t;
            if (r == 1) c1h0 = t;
        }
        yv = f4_add(f4_div(acc, 16.0f), f4_div(f4_mul(c0, 2.0f), 4.0f));
        float4 fprev = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float4 t = shfl4(fp, src[r]);
            yv = f4_add(yv, f4_div(t, 16.0f));
            if (r == 0) { fpB = t; fprev = t; }
            if (r == 3 && j == 0) fprev = t;
        }
        if (valid && k == 2) {                     // SLAK edge point of slot N2 + y: quads j and j - 1
            const float4 ta = f4_mul(f4_add(c0, fp), 0.25f);
            st4_cs(R, (int64_t)d.V + d.N1 + d.N2 + (x >> 2),
                   f4_add(f4_add(f4_zero(), ta), f4_mul(f4_add(c1, fprev), 0.25f)));
        }
    } else {
        // the face point's column: face points in column order, then the tails
        // (e_in) in ascending id; the edge point's lane takes B's values
        int tid[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) tid[r] = __shfl_sync(full, Q.w, src[r]);
        const int qyB = __shfl_sync(full, Q.y, lB);
        float4 acc = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float4 t = shfl4(fp, src[r]);
            acc = f4_add(acc, t);
            if (r == 0) fpB = t;
        }
        float4 c3B;
#pragma unroll
        for (int r = 0; r < 4; ++r) {              // source of rank r (the edge point's lane: B)
            int sr = src[0];
#pragma unroll
            for (int i = 1; i < 4; ++i)
                if (rank4(tid[i], tid[(i + 1) & 3], tid[(i + 2) & 3], tid[(i + 3) & 3]) == r) sr = src[i];
            if (rank4(tid[0], tid[1], tid[2], tid[3]) == r) sr = src[0];
            const float4 t = shfl4(c3, fw ? sr : (r == 0 ? lB : lane));
            acc = f4_add(acc, t);
            if (r == 0) c3B = t;
        }
        yv = f4_div_z(f4_add(f4_div_z(acc, 4.0f), f4_mul(c0, 2.0f)), 4.0f);
        c1B = shfl4(c1, lB);
        c1h0 = shfl4(c1, l0);
        if (ew) {
            const int y = x >> 2, nh2 = tw0 >> 2, h2 = qprev(nh2);
            const int e = Q.x - d.V2 - d.F2;
            const int X = d.V1 + d.F1 + 4 * e + 2 + ((h2 >> 2) > (y >> 2));
            const float4 PX = ldg4(P, X), Pf2 = ldg4(P, d.V1 + h2), Pfn2 = ldg4(P, d.V1 + nh2);
            const float4 fC2 = f4_div_z(f4_add(f4_add(f4_add(f4_add(f4_zero(), c0), PX), Pf2), c1B), 4.0f);
            const float4 fD2 = f4_div_z(f4_add(f4_add(f4_add(f4_add(f4_zero(), c0), c1h0), Pfn2), PX), 4.0f);
            const int cA = x, cB = 4 * (y & ~3 | ((y + 1) & 3)) + 3, cC = 4 * h2 + 1, cD = 4 * nh2 + 3;
            const int rA = rank4(cA, cB, cC, cD), rB = rank4(cB, cA, cC, cD), rC = rank4(cC, cA, cB, cD);
            float4 a2 = f4_zero();
#pragma unroll
            for (int r = 0; r < 4; ++r) a2 = f4_add(a2, rA == r ? fp : rB == r ? fpB : rC == r ? fC2 : fD2);
            // tails e_in of A, B, C2, D2 = c3, c3B, c1B, PX with ids Q.w, Q.w(B), Q.y(B), X
            const int tA = Q.w, tB = tid[0], tC = qyB, tD = X;
            const int sA = rank4(tA, tB, tC, tD), sB = rank4(tB, tA, tC, tD), sC = rank4(tC, tA, tB, tD);
#pragma unroll
            for (int r = 0; r < 4; ++r) a2 = f4_add(a2, sA == r ? c3 : sB == r ? c3B : sC == r ? c1B : PX);
            yv = f4_div_z(f4_add(f4_div_z(a2, 4.0f), f4_mul(c0, 2.0f)), 4.0f);
        }
    }
    if (fw || (LAK && ew)) {
        st_pos<STATE>(R, Q.x, yv);
        if (STATE) c.sptr[Q.x] = fw ? d.N2 + (x >> 2) : 2 * d.N2 + 4 * (Q.x - d.V2 - d.F2);
    }
    if (!LAK && ew) {
        const int y = x >> 2, nh2 = tw0 >> 2, h2 = qprev(nh2);
        const int e = Q.x - d.V2 - d.F2;
        const int X = d.V1 + d.F1 + d.N2 + nh2;
        const float4 PX = ldg4(P, X), Pf2 = ldg4(P, d.V1 + h2), Pfn2 = ldg4(P, d.V1 + nh2);
        const float4 fC2 = f4_mul(f4_add(f4_add(c0, Pf2), f4_add(PX, c1B)), 0.25f);
        const float4 fD2 = f4_mul(f4_add(f4_add(c0, Pfn2), f4_add(c1h0, PX)), 0.25f);
        // the column's quads A, B, C2, D2 (neighbour e_out, face point) and their ranks
        const int cA = x, cB = 4 * (y & ~3 | ((y + 1) & 3)) + 3, cC = 4 * h2 + 1, cD = 4 * nh2 + 3;
        const int rA = rank4(cA, cB, cC, cD), rB = rank4(cB, cA, cC, cD), rC = rank4(cC, cA, cB, cD);
        float4 acc = f4_zero();
#pragma unroll
        for (int r = 0; r < 4; ++r) acc = f4_add(acc, rA == r ? c1 : rB == r ? c1B : rC == r ? PX : c1h0);
        float4 ye = f4_add(f4_div(acc, 16.0f), f4_div(f4_mul(c0, 2.0f), 4.0f));
#pragma unroll
        for (int r = 0; r < 4; ++r) ye = f4_add(ye, f4_div(rA == r ? fp : rB == r ? fpB : rC == r ? fC2 : fD2, 16.0f));
        st_pos<STATE>(R, Q.x, ye);
        if (STATE) c.sptr[Q.x] = 2 * d.N2 + 4 * e;
        // edges around ve, at the column's slots: quad A with B, B with C2, C2 with D2, D2 with A
        const int64_t eb = (int64_t)d.V + d.N1 + 2 * (int64_t)d.N2 + 4 * (int64_t)e;
        const auto ep = [&](float4 f, float4 nb, float4 fn) {
            return f4_add(f4_add(f4_zero(), f4_mul(f4_add(c0, f), 0.25f)), f4_mul(f4_add(nb, fn), 0.25f));
        };
        st4_cs(R, eb + rA, ep(fp, c1, fpB));
        st4_cs(R, eb + rB, ep(fpB, c1B, fC2));
        st4_cs(R, eb + rC, ep(fC2, PX, fD2));
        st4_cs(R, eb + (6 - rA - rB - rC), ep(fD2, c1h0, fp));
    }
}

// ---------------------------------------------------------------------------------------------
// SG: the last level with P = refine(PP), PP a closed quad mesh; `pp` is PP's
// state, and the level before writes none.  P's twin, slot and (SLAK) t of
// corner x = 4y + k are what write_state would have stored, from PP's twin of
// y (of prev(y) for k = 3), PP's slot and t of y (k = 0) and, for k = 1, 3,
// the P vertex vx at corner x (PP's edge point V2 + F2 + e, its column at
// 2 N2 + 4e).  Branch-free: every lane loads one twin.
template <bool LAK>
__device__ __forceinline__ void sg_state(const FastDims& d, const QState& pp, int x, int vx, bool valid, int& tw,
                                         int& slot, int& t)
{
    const int y = x >> 2, k = x & 3;
    const int nx = qnext(y), px = qprev(y);
    const int twl = valid ? __ldg(pp.tw + (k == 3 ? px : y)) : 0;
    const int sl = valid && k == 0 ? __ldg(pp.slot + y) : 0;
    const int tl = !LAK && valid && k == 0 ? __ldg(pp.t + y) : 0;
    const int ntw = qnext(twl);
    // the four corners of PP edge point e's column: k = 1 (e = e_out(y)) A, B, C, D;
    // k = 3 (e = e_in(y)) A2, B2, C2, D2 (write_state).  Two of them, p0 and
    // p2, lie in y's PP face (P corners 16 face(y) .. +15), the other two, p1
    // and p3, in the twin's, so their ranks follow from the faces' order and
    // the order within each pair: p0 > p2 when y is corner 3 (k = 1) or
    // corner 0 (k = 3) of its face, p1 > p3 when the twin is corner 3 of its.
    const bool own_first = (y >> 2) < (twl >> 2);
    const int o = own_first ? 0 : 2;
    const int r0 = o + ((y & 3) == (k == 1 ? 3 : 0));
    const int r2 = o + ((y & 3) != (k == 1 ? 3 : 0));
    const int r3 = (2 - o) + ((twl & 3) != 3);
    const int base = 2 * d.N2 + 4 * (vx - d.V2 - d.F2);
    tw = k == 0 ? 4 * ntw + 3 : k == 1 ? 4 * nx + 2 : k == 2 ? 4 * px + 1 : 4 * twl;
    slot = k == 0 ? sl : k == 2 ? d.N2 + y : base + (k == 1 ? r0 : r2);
    t = k == 0 ? tl : k == 2 ? d.N2 + nx : base + (k == 1 ? r3 : r0);
}

// SG: P's column offsets from PP's (old vertices keep their columns; face
// points at N2 + 4g, edge points at 2 N2 + 4e; v = V1 gives N1)
__device__ __forceinline__ int sg_sptr(const FastDims& d, const int* __restrict__ ppsptr, int v)
{
    if (v < d.V2) return __ldg(ppsptr + v);
    if (v < d.V2 + d.F2) return d.N2 + 4 * (v - d.V2);
    return 2 * d.N2 + 4 * (v - d.V2 - d.F2);
}

// P's faces are quads (PQ: the 4 corners of a face are 4 consecutive lanes,
// exchanged by shuffles) or polygons (face offsets and the corner -> face map
// of P, `pf`; a face's corners are consecutive threads, read from memory).
// BND: P has a boundary; tw / t of P are -1 where there is no twin, and P's
// edges carry their boundary ranks.
// optr / ovals (LAK, last level): the refined mesh's ptr[q] = 4q and
// vals[q] = {1, 2, 3, 4}; they depend on q alone, so a block writes the 4 BS
// refined quads of its span with consecutive threads (coalesced).
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false, bool GQ = false, bool SG = false>
__device__ __forceinline__ void k_g1_body(const unsigned bx_, FastDims d, Faces<PQ> pf, const int* __restrict__ ids,
                                          const float* __restrict__ P, QState p, QState c,
                                          int4* __restrict__ out_ids, const CUtensorMap& otm, float* __restrict__ R,
                                          SlotScratch z, int* __restrict__ optr, int4* __restrict__ ovals)
{
    const int x0 = bx_ * blockDim.x;
    const int x = x0 + threadIdx.x;
    const bool valid = x < d.N1;
    const int lane = threadIdx.x & 31, q = x & 3;
    const int gl = lane & ~3;                  // lane of quad 0 of my face of P
    const int VF1 = d.V1 + d.F1;
    const int VFc = d.V + d.N1;                // C: V + F

    const int4 Q = valid ? __ldg(reinterpret_cast<const int4*>(ids) + x) : make_int4(0, 0, 0, 0);
    const float4 c0 = valid ? ldg4(P, Q.x) : f4_zero();
    const float4 c1 = valid ? ldg4(P, Q.y) : f4_zero();
    const float4 c2 = valid ? ldg4(P, Q.z) : f4_zero();
    // with quad P, e_in(x) is e_out(prev x): the previous lane's c1 (a shuffle
    // instead of a fourth scattered gather)
    float4 c3;
    if constexpr (PQ) c3 = shfl4(c1, (threadIdx.x & 31 & ~3) | ((x + 3) & 3));
    else c3 = valid ? ldg4(P, Q.w) : f4_zero();
    int tw1x = 0, s1 = 0, t1x = 0;
    if constexpr (SG) {
        sg_state<LAK>(d, p, x, Q.x, valid, tw1x, s1, t1x);
    } else {
        if (valid && (LAK || STATE || PQ || BND)) tw1x = __ldg(p.tw + x);
        if (valid) s1 = __ldg(p.slot + x);
        if (valid && !LAK) t1x = __ldg(p.t + x);
    }
    const int ln = gl | ((q + 1) & 3), lp = gl | ((q + 3) & 3);
    // next / previous corner of x in its face of P, and the twin of the previous one
    int nxx, px, tw1_px;
    if (PQ) {
        nxx = qnext(x); px = qprev(x);
        tw1_px = __shfl_sync(0xffffffffu, tw1x, lp);
    } else {
        const int f = Q.z - d.V1;              // C's quad x holds P's face point V1 + face(x)
        const int fb = valid ? __ldg(pf.ptr + f) : 0, fe = valid ? __ldg(pf.ptr + f + 1) : 1;
        nxx = x + 1 == fe ? fb : x + 1;
        px = x == fb ? fe - 1 : x - 1;
        tw1_px = valid && (LAK || STATE || BND) ? __ldg(p.tw + px) : 0;
    }
    const int eidp_x = Q.y - VF1, eidp_px = Q.w - VF1;   // P's edge ids of x and prev(x)
    int br_x = 0, br_px = 0;                             // their boundary ranks
    if (BND && valid) { br_x = __ldg(p.brank + eidp_x); br_px = __ldg(p.brank + eidp_px); }
    // quad P: the lane of the min->max half-edge of P's edge through x owns
    // its edge work (below), which gathers three positions of the twin side,
    // two of them behind ids.  The ids depend on Q and tw1x alone; at the last
    // level (no state to write, registers to spare) they are fetched now,
    // beside the quad's own gathers, and the edge work waits for one round
    // trip instead of two.
    bool own = false;
    int ei2 = 0, eo3 = 0;
    if constexpr (PQ && !STATE) {
        const int un = __shfl_sync(0xffffffffu, Q.x, ln);     // every lane takes part
        own = valid && (!BND || tw1x >= 0) && Q.x < un;
        if (own) {
            ei2 = __ldg(ids + 4 * (int64_t)tw1x + 3);
            eo3 = __ldg(ids + 4 * (int64_t)qnext(tw1x) + 1);
        }
    }

    // face point of quad x
    float4 fp;
    if (!LAK) {
        fp = f4_mul(f4_add(f4_add(c0, c2), f4_add(c1, c3)), 0.25f);
    } else {
        fp = f4_div_z(f4_add(f4_add(f4_add(f4_add(f4_zero(), c0), c1), c2), c3), 4.0f);
    }

    // edge ids of C's corners 4x+k
    int e0, e1, e2, e3;
    if (!LAK) {
        // a prev(x) edge without a twin: C's edge {e_in(x), v} is owned by
        // corner 4x+3 itself, ranked after the 2 N1 interior owners
        e0 = s1; e1 = d.N1 + nxx; e2 = d.N1 + x; e3 = (!BND || t1x >= 0) ? t1x : 2 * d.N1 + br_px;
    } else {
        int vnx, vpx, fx, ftw, ftwp;
        if (PQ) {
            vnx = __shfl_sync(0xffffffffu, Q.x, ln); vpx = __shfl_sync(0xffffffffu, Q.x, lp);
            fx = x >> 2; ftw = tw1x >> 2; ftwp = tw1_px >> 2;
        } else {
            vnx = valid ? __ldg(ids + 4 * (int64_t)nxx) : 0;
            vpx = valid ? __ldg(ids + 4 * (int64_t)px) : 0;
            fx = Q.z - d.V1;
            ftw = valid && tw1x >= 0 ? pf.face(tw1x) : 0;        // no face across a boundary
            ftwp = valid && tw1_px >= 0 ? pf.face(tw1_px) : 0;
        }
        // C's edges around P's edge e start at 4e - brank(e); a boundary edge
        // has one face point, ranked 2
        e0 = 4 * eidp_x - br_x + (Q.x > vnx);
        e1 = 4 * eidp_x - br_x + 2 + ((!BND || tw1x >= 0) && fx > ftw);
        e2 = 4 * eidp_px - br_px + 2 + ((!BND || tw1_px >= 0) && fx > ftwp);
        e3 = 4 * eidp_px - br_px + (Q.x > vpx);
    }
    // refined quads {v_k, V+F+e_k, V+x, V+F+e_(k-1)}.  Levels that write the
    // next level's state: the thread's 64 bytes as two 256-bit stores.  Other
    // levels: staged in shared memory, then one coalesced run per block.
    // Measured on B200 (512x512 mixed torus, SLAK): direct stores take a
    // state-writing level 2 from 184 to 180 us and level 1 from 43 to 41 us,
    // but the last level from 596 to 614 us (and a level 2 without state, as SG
    // makes it, from 154 to 166 us).
    const int fpid = d.V + x;
    if constexpr (STATE) {
        if (valid) {
            int4* dst = out_ids + 4 * (int64_t)x;
            st8_cs(dst, make_int4(Q.x, VFc + e0, fpid, VFc + e3), make_int4(Q.y, VFc + e1, fpid, VFc + e0));
            st8_cs(dst + 2, make_int4(Q.z, VFc + e2, fpid, VFc + e1), make_int4(Q.w, VFc + e3, fpid, VFc + e2));
        }
    } else if constexpr (kTmaQuadStore && BS <= 256) {
        // the block's refined quads (row t = thread t's 64 bytes) staged in
        // shared memory in the tensor map's 64-byte swizzle (16-byte chunk k
        // of row t at chunk k ^ (t/2 mod 4): a warp's stores of chunk k fall on
        // all 32 banks), then one TMA tensor store of the block's rows; rows
        // past N1 are clipped by the map.  Replaces the shared-memory round
        // trip and the coalesced stores of the staged layout below.
        __shared__ __align__(1024) int4 sq[4 * BS];
        const int t = threadIdx.x, sw = (t >> 1) & 3;
        sq[4 * t + (0 ^ sw)] = make_int4(Q.x, VFc + e0, fpid, VFc + e3);
        sq[4 * t + (1 ^ sw)] = make_int4(Q.y, VFc + e1, fpid, VFc + e0);
        sq[4 * t + (2 ^ sw)] = make_int4(Q.z, VFc + e2, fpid, VFc + e1);
        sq[4 * t + (3 ^ sw)] = make_int4(Q.w, VFc + e3, fpid, VFc + e2);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                         :: "l"(reinterpret_cast<uint64_t>(&otm)), "r"(0), "r"(x0),
                            "r"((uint32_t)__cvta_generic_to_shared(sq))
                         : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
    } else {
        // refined quad k of thread t at sq[k * (BS + 2) + t]: the stores
        // (consecutive t) and the run-order reads (4 k's of a t, then the next
        // t) are both free of bank conflicts
        constexpr int SQ = BS + 2;
        __shared__ int4 sq[4 * SQ];
        sq[0 * SQ + threadIdx.x] = make_int4(Q.x, VFc + e0, fpid, VFc + e3);
        sq[1 * SQ + threadIdx.x] = make_int4(Q.y, VFc + e1, fpid, VFc + e0);
        sq[2 * SQ + threadIdx.x] = make_int4(Q.z, VFc + e2, fpid, VFc + e1);
        sq[3 * SQ + threadIdx.x] = make_int4(Q.w, VFc + e3, fpid, VFc + e2);
        __syncthreads();
        const int nq = min(BS, d.N1 - x0);
        int4* dst = out_ids + 4 * (int64_t)x0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = i * BS + threadIdx.x;
            if (j < 4 * nq) __stcs(dst + j, sq[(j & 3) * SQ + (j >> 2)]);
        }
    }

    if (valid) {
        st_pos<STATE>(R, (int64_t)d.V + x, fp);
    }
    // records of corner x for its vertex's pass (full 32-byte sectors at slot
    // s1); with GQ only the corners at PP's old vertices (q == 0) have them
    if (valid && (!GQ || q == 0)) {
        st8_keep(z.Z + 2 * (int64_t)s1, fp, LAK ? c3 : c1);
        if (LAK) z.T[s1] = Q.w;
        else if (!BND || t1x >= 0) z.rot[t1x] = s1;
    }
    if (valid) {
        if (BND && !LAK && tw1x < 0) z.rot[s1] = s1;      // no rotation across the boundary: a safe index
        if (BND) {
            z.bflag[s1] = (tw1x < 0) | ((tw1_px < 0) << 1);
            z.bid[s1] = LAK ? Q.y : Q.w;
            if (STATE && !LAK) z.bscan[s1] = tw1x < 0;
        }
    }

    if constexpr (!PQ) {
        // polygon P: P's face points and C's inner edge points are k_gf's
        if (STATE && valid) {
            const int ntw = BND && tw1x < 0 ? 0 : pf.next(tw1x), ntwp = BND && tw1_px < 0 ? 0 : pf.next(tw1_px);
            write_state<LAK>(d, c, x, nxx, px, tw1x, tw1_px, ntw, ntwp, s1, t1x, eidp_x, eidp_px, br_x, br_px);
            if (BND && !LAK) c.brank[d.N1 + x] = d.B1;                 // C's face-point edges are interior
        }
    } else {
        // vertex point of P's face point V1 + (x>>2): corners 4x_j+2 of the face's quads, n = 4
        float4 nb[4], fq[4];
        int tl[4];
        if constexpr (!LAK || BS > 256 || kFaceSumShfl) {
            // SLAK: shuffles (measured on B200, 512x512 mixed torus: the shared
            // memory exchange below took the last level's k_g1 from 596 to
            // 621 us); 512-thread blocks: the staging buffer leaves no room for
            // the exchange under the 48 KB of static shared memory
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                nb[j] = shfl4(LAK ? c1 : c3, gl | j);      // SLAK: e_in(x_j); LAK: tails e_out(x_j)
                fq[j] = shfl4(fp, gl | j);
                tl[j] = __shfl_sync(0xffffffffu, Q.y, gl | j);
            }
        } else {
            // LAK: the group's values pass through shared memory.  Warp
            // shuffles run on the L1 data pipe this kernel is bound by, one
            // wavefront per shuffle for the whole warp, while here only the
            // eight summing lanes (q == 0) read; LAK also ranks the tails by
            // id.  Measured on B200 (512x512 mixed torus): last level's k_g1
            // 769 -> 757 us.  Entry lane + lane / 4 (padded) puts the 16-byte
            // entries those lanes read together on distinct banks.
            __shared__ float4 xs[BS / 32][2][40];
            __shared__ int xt[LAK ? BS / 32 : 1][40];
            const int wv = threadIdx.x >> 5, pl = lane + (lane >> 2);
            xs[wv][0][pl] = LAK ? c1 : c3;             // SLAK: e_in(x_j); LAK: tails e_out(x_j)
            xs[wv][1][pl] = fp;
            if (LAK) xt[wv][pl] = Q.y;
            __syncwarp();
            if (q == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    nb[j] = xs[wv][0][pl + j];
                    fq[j] = xs[wv][1][pl + j];
                    tl[j] = LAK ? xt[wv][pl + j] : 0;
                }
            }
        }
        if (valid && q == 0) {
            float4 yv;
            if (!LAK) {
                float4 acc = f4_zero();
#pragma unroll
                for (int j = 0; j < 4; ++j) acc = f4_add(acc, nb[j]);
                yv = f4_add(f4_div(acc, 16.0f), f4_div(f4_mul(c2, 2.0f), 4.0f));
#pragma unroll
                for (int j = 0; j < 4; ++j) yv = f4_add(yv, f4_div(fq[j], 16.0f));
            } else {
                float4 acc = f4_zero();
#pragma unroll
                for (int j = 0; j < 4; ++j) acc = f4_add(acc, fq[j]);
#pragma unroll
                for (int r = 0; r < 4; ++r) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        int rk = 0;
#pragma unroll
                        for (int i = 0; i < 4; ++i) rk += tl[i] < tl[j];
                        if (rk == r) acc = f4_add(acc, nb[j]);
                    }
                }
                yv = f4_div_z(f4_add(f4_div_z(acc, 4.0f), f4_mul(c2, 2.0f)), 4.0f);
            }
            st_pos<STATE>(R, (int64_t)d.V1 + (x >> 2), yv);
        }

        // SLAK edge point N1 + x: half-edges 4x+2 (tail f, quad x) and 4 prev(x)+1 (tail e_in(x), quad prev x)
        if (!LAK) {
            const float4 fprev = shfl4(fp, lp);
            if (valid) {
                float4 ta = f4_mul(f4_add(c2, fp), 0.25f);
                float4 tb = f4_mul(f4_add(c3, fprev), 0.25f);
                st4_cs(R, (int64_t)VFc + d.N1 + x, f4_add(f4_add(f4_zero(), ta), tb));
            }
        }

        if (STATE && valid) {
            write_state<LAK>(d, c, x, nxx, px, tw1x, tw1_px, BND && tw1x < 0 ? 0 : qnext(tw1x),
                             BND && tw1_px < 0 ? 0 : qnext(tw1_px), s1, t1x, eidp_x, eidp_px, br_x, br_px);
            if (q == 0) c.sptr[d.V1 + (x >> 2)] = d.N1 + x;            // = N1 + 4 * face
            if (BND && !LAK) c.brank[d.N1 + x] = d.B1;                 // C's face-point edges are interior
        }

        // P's edge through x, on the lane of its min->max half-edge: what k_g2
        // does for polygon parents.  Quads h2 = tw(x) and next(h2) of the twin
        // face are {u, ve, fh2, e_in(h2)} and {v, e_out(next h2), fh2, ve}, so
        // their face points are rebuilt from three gathered positions.
        const int u = __shfl_sync(0xffffffffu, Q.x, ln);
        const float4 Pu = shfl4(c0, ln), Fnh = shfl4(fp, ln);
        if (BND && valid && tw1x < 0) {        // the only half-edge of a boundary edge owns it
            boundary_edge<LAK, STATE>(d, c, R, Q.x, u, Q.y, br_x, c0, Pu, c1, c2, fp, Fnh);
        } else if (STATE ? valid && Q.x < u : own) {
            const int h2 = tw1x, nh2 = qnext(h2), fh2 = d.V1 + (h2 >> 2);
            if (STATE) { ei2 = __ldg(ids + 4 * (int64_t)h2 + 3); eo3 = __ldg(ids + 4 * (int64_t)nh2 + 1); }
            const float4 Pf2 = ldg4(P, fh2), Pi2 = ldg4(P, ei2), Po3 = ldg4(P, eo3);
            float4 Fh2, Fnh2;
            if (!LAK) {
                Fh2 = f4_mul(f4_add(f4_add(Pu, Pf2), f4_add(c1, Pi2)), 0.25f);
                Fnh2 = f4_mul(f4_add(f4_add(c0, Pf2), f4_add(Po3, c1)), 0.25f);
            } else {
                Fh2 = f4_div_z(f4_add(f4_add(f4_add(f4_add(f4_zero(), Pu), c1), Pf2), Pi2), 4.0f);
                Fnh2 = f4_div_z(f4_add(f4_add(f4_add(f4_add(f4_zero(), c0), Po3), Pf2), c1), 4.0f);
            }
            edge_point_vertex<LAK, STATE, BND>(d, c, R, x, nxx, h2, nh2, Q.y, Q.z, fh2, c0, Pu, c1, c2, Pf2, fp,
                                               Fnh, Fh2, Fnh2, br_x);
        }
        if constexpr (GQ) gq_columns<LAK, STATE>(d, c, P, R, valid, x, lane, Q, tw1x, c0, c1, c3, fp);
    }
    if (LAK && !STATE && optr != nullptr) {
        const int64_t q0 = 4 * (int64_t)x0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t qq = q0 + threadIdx.x + (int64_t)j * BS;
            if (qq < d.N) {
                __stcs(ovals + qq, make_int4(1, 2, 3, 4));
                __stcs(optr + qq, (int)(4 * qq));
            }
        }
        if (x == 0) optr[d.N] = 4 * d.N;
    }
    if constexpr (!STATE && kTmaQuadStore && BS <= 256) {
        // the tensor store has read the staging buffer and its writes are done
        if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false, bool GQ = false, bool SG = false>
__global__ void __launch_bounds__(BS, (GQ ? 768 : 1024) / BS) k_g1(FastDims d, Faces<PQ> pf, const int* __restrict__ ids,
                                                                   const float* __restrict__ P, QState p, QState c,
                                                                   int4* __restrict__ out_ids,
                                                                   const __grid_constant__ CUtensorMap otm,
                                                                   float* __restrict__ R, SlotScratch z,
                                                                   int* __restrict__ optr, int4* __restrict__ ovals)
{
    griddep_enter();
    k_g1_body<LAK, STATE, PQ, BS, BND, GQ, SG>(blockIdx.x, d, pf, ids, P, p, c, out_ids, otm, R, z, optr, ovals);
}
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false, bool GQ = false, bool SG = false>
struct k_g1_g {
    static constexpr int kBounds = 2, kMaxT = BS, kMinB = (GQ ? 768 : 1024) / BS;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_g1_body<LAK, STATE, PQ, BS, BND, GQ, SG>(bx, a...);
    }
    static constexpr auto kernel() { return &k_g1<LAK, STATE, PQ, BS, BND, GQ, SG>; }
};

// ---------------------------------------------------------------------------------------------
// The vertex point of P's face point with the face's k > 4 corners b..e-1 under
// SLAK_PLAN_COMPENSATED: the same terms in the same order as the general path's
// compensated vertex points (k_vp_slak / k_vp_lak): TwoSum sums, exact-remainder
// quotients, one rounding.  SLAK: e_in(x) then FP(x); LAK: FP(x), then the
// tails e_out(x) in ascending id.
template <bool LAK>
__device__ __noinline__ float4 face_vertex_compensated(const int* __restrict__ ids, const float* __restrict__ P,
                                                       const float* __restrict__ FP, int b, int e, float4 c2)
{
    float4 sh = f4_zero(), sl = f4_zero();
    if (!LAK) {
        for (int x = b; x < e; ++x) dd_acc(sh, sl, ldg4(P, __ldg(ids + 4 * (int64_t)x + 3)));
        for (int x = b; x < e; ++x) dd_acc(sh, sl, ldg4(FP, x));
    } else {
        for (int x = b; x < e; ++x) dd_acc(sh, sl, ldg4(FP, x));
        for (int last = -1;;) {
            int xm = INT32_MAX;
            for (int x = b; x < e; ++x) {
                const int ti = __ldg(ids + 4 * (int64_t)x + 1);
                if (ti > last && ti < xm) xm = ti;
            }
            if (xm == INT32_MAX) break;
            dd_acc(sh, sl, ldg4(P, xm));
            last = xm;
        }
    }
    return vp_finish(sh, sl, c2, e - b);
}

// ---------------------------------------------------------------------------------------------
// GF (polygon P only): one thread per face g of P, with k corners x = ptr[g] ..
// ptr[g+1]-1.  The vertex point of P's face point V1 + g (its column in C is
// corners 4x+2, ascending) and, for SLAK, the edge points N1 + x of C's inner
// edges {face point, e_in(x)}: the work k_g1 does with shuffles when P's faces
// are quads.  Same formulas and order, with n = k.
template <bool LAK, bool STATE>
__device__ __forceinline__ void k_gf_body(const unsigned bx_, FastDims d, const int* __restrict__ pptr, const int* __restrict__ ids,
                                          const float* __restrict__ P, QState c, float* __restrict__ R,
                                          int compensated)
{
    const int g = bx_ * blockDim.x + threadIdx.x;
    if (g >= d.F1) return;
    const int b = __ldg(pptr + g), e = __ldg(pptr + g + 1), k = e - b;
    const float4 c2 = ldg4(P, d.V1 + g);
    const float* FP = R + 4 * (int64_t)d.V;
    const float nn = (float)(k * k);
    float4 yv, acc = f4_zero();
    if (k <= 8) {
        // faces of up to 8 corners: every load issued up front (same arithmetic and order as below)
        int vi[8];
        float4 fq[8], pe[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < k) {
                vi[j] = __ldg(ids + 4 * (int64_t)(b + j) + (LAK ? 1 : 3));    // LAK: e_out; SLAK: e_in
                fq[j] = ldg4(FP, b + j);
            }
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < k) pe[j] = ldg4(P, vi[j]);
        if (!LAK) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < k) acc = f4_add(acc, pe[j]);
            yv = f4_add(f4_div(acc, nn), f4_div(f4_mul(c2, (float)(k - 2)), (float)k));
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < k) yv = f4_add(yv, f4_div(fq[j], nn));
            const int64_t VFc = (int64_t)d.V + d.N1;
            // FP of the last corner (the first corner's prev) loaded again, an L1
            // hit: selecting fq[k-1] would index the array dynamically and put it
            // in local memory
            const float4 flast = ldg4(FP, e - 1);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < k) {
                    const float4 ta = f4_mul(f4_add(c2, fq[j]), 0.25f);
                    const float4 tb = f4_mul(f4_add(pe[j], j == 0 ? flast : fq[j > 0 ? j - 1 : 0]), 0.25f);
                    st4_cs(R, VFc + d.N1 + b + j, f4_add(f4_add(f4_zero(), ta), tb));
                }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < k) acc = f4_add(acc, fq[j]);
            // the tails e_out(x) in ascending id (distinct within a face)
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    int rk = 0;
#pragma unroll
                    for (int i = 0; i < 8; ++i) rk += (i < k && vi[i] < vi[j]);
                    if (j < k && rk == r) acc = f4_add(acc, pe[j]);
                }
            yv = f4_div_z(f4_add(f4_div_z(acc, (float)k), f4_mul(c2, __fadd_rn((float)k, -2.0f))), (float)k);
        }
        if (compensated && k > 4) yv = face_vertex_compensated<LAK>(ids, P, FP, b, e, c2);
        st4(R, (int64_t)d.V1 + g, yv);
        if (STATE) c.sptr[d.V1 + g] = d.N1 + b;
        return;
    }
    if (!LAK) {
        for (int x = b; x < e; ++x) acc = f4_add(acc, ldg4(P, __ldg(ids + 4 * (int64_t)x + 3)));   // e_in(x)
        yv = f4_add(f4_div(acc, nn), f4_div(f4_mul(c2, (float)(k - 2)), (float)k));
        for (int x = b; x < e; ++x) yv = f4_add(yv, f4_div(ldg4(FP, x), nn));
        const int64_t VFc = (int64_t)d.V + d.N1;
        for (int x = b; x < e; ++x) {
            const int px = x == b ? e - 1 : x - 1;
            const float4 ta = f4_mul(f4_add(c2, ldg4(FP, x)), 0.25f);
            const float4 tb = f4_mul(f4_add(ldg4(P, __ldg(ids + 4 * (int64_t)x + 3)), ldg4(FP, px)), 0.25f);
            st4_cs(R, VFc + d.N1 + x, f4_add(f4_add(f4_zero(), ta), tb));
        }
    } else {
        for (int x = b; x < e; ++x) acc = f4_add(acc, ldg4(FP, x));
        // the tails e_out(x) in ascending id
        int last = -1;
        while (true) {
            int xm = INT32_MAX;
            for (int x = b; x < e; ++x) {
                const int ti = __ldg(ids + 4 * (int64_t)x + 1);
                if (ti > last && ti < xm) xm = ti;
            }
            if (xm == INT32_MAX) break;
            acc = f4_add(acc, ldg4(P, xm));
            last = xm;
        }
        yv = f4_div_z(f4_add(f4_div_z(acc, (float)k), f4_mul(c2, __fadd_rn((float)k, -2.0f))), (float)k);
    }
    if (compensated && k > 4) yv = face_vertex_compensated<LAK>(ids, P, FP, b, e, c2);
    st4(R, (int64_t)d.V1 + g, yv);
    if (STATE) c.sptr[d.V1 + g] = d.N1 + b;
}
template <bool LAK, bool STATE>
__global__ void __launch_bounds__(kBlock) k_gf(FastDims d, const int* __restrict__ pptr, const int* __restrict__ ids,
                                               const float* __restrict__ P, QState c, float* __restrict__ R,
                                               int compensated)
{
    griddep_enter();
    k_gf_body<LAK, STATE>(blockIdx.x, d, pptr, ids, P, c, R, compensated);
}
template <bool LAK, bool STATE>
struct k_gf_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_gf_body<LAK, STATE>(bx, a...);
    }
    static constexpr auto kernel() { return &k_gf<LAK, STATE>; }
};

// ---------------------------------------------------------------------------------------------
// G2 (polygon P; with quad P k_g1 does this work): the edges of P, visited in
// corner order.  Thread x is corner x of P (=
// quad x of C); the 4 corners of a face of P are 4 consecutive lanes.  Edge e
// of P with half-edges (h, h2) = (min->max, max->min) is computed by the lane
// x = h, so the quantities of h's face (v, u, P's face point, C's face points
// of quads h and next(h)) are coalesced loads or shuffles, and only the twin
// face's three (its face point, C's face points of quads h2 and next(h2)) are
// gathers.  The edge's outputs land at its id e = e_out(x) - (V1 + F1).
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false>
__device__ __forceinline__ void k_g2_body(const unsigned bx_, FastDims d, Faces<PQ> pf, const int* __restrict__ ids,
                                          const float* __restrict__ P, QState p, QState c, float* __restrict__ R)
{
    const int x = bx_ * blockDim.x + threadIdx.x;
    const bool valid = x < d.N1;
    const int lane = threadIdx.x & 31, q = x & 3;
    const int ln = (lane & ~3) | ((q + 1) & 3);
    const float* FP = R + 4 * (int64_t)d.V;
    // two dependent rounds of loads: the coalesced ones, then every gather at once
    const int4 Q = valid ? __ldg(reinterpret_cast<const int4*>(ids) + x) : make_int4(0, 0, 0, 0);
    const int h2 = valid ? __ldg(p.tw + x) : 0;
    const float4 Fh = valid ? ldg4(FP, x) : f4_zero();
    int u, nh;
    float4 Fnh;
    if (PQ) {
        nh = qnext(x);
        u = __shfl_sync(0xffffffffu, Q.x, ln);
        Fnh = shfl4(Fh, ln);
    } else {
        if (!valid) return;
        const int f = Q.z - d.V1, fb = __ldg(pf.ptr + f), fe = __ldg(pf.ptr + f + 1);
        nh = x + 1 == fe ? fb : x + 1;
        u = __ldg(ids + 4 * (int64_t)nh);
    }
    // the edge's owner: its min->max half-edge, or its only one (BND: no twin)
    if (!valid || (Q.x >= u && !(BND && h2 < 0))) return;
    if (!PQ) Fnh = ldg4(FP, nh);
    const int br = BND ? __ldg(p.brank + (Q.y - d.V1 - d.F1)) : 0;
    if (BND && h2 < 0) {
        boundary_edge<LAK, STATE>(d, c, R, Q.x, u, Q.y, br, ldg4(P, Q.x), ldg4(P, u), ldg4(P, Q.y), ldg4(P, Q.z), Fh,
                                  Fnh);
        return;
    }
    const int h = x, nh2 = pf.next(h2);
    const int ve = Q.y, fh = Q.z, fh2 = d.V1 + pf.face(h2);
    const float4 Pv = ldg4(P, Q.x), Pu = ldg4(P, u);
    const float4 Pe = ldg4(P, ve), Pf = ldg4(P, fh), Pf2 = ldg4(P, fh2);
    const float4 Fh2 = ldg4(FP, h2), Fnh2 = ldg4(FP, nh2);
    edge_point_vertex<LAK, STATE, BND>(d, c, R, h, nh, h2, nh2, ve, fh, fh2, Pv, Pu, Pe, Pf, Pf2, Fh, Fnh, Fh2, Fnh2,
                                       br);
}
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false>
__global__ void __launch_bounds__(BS) k_g2(FastDims d, Faces<PQ> pf, const int* __restrict__ ids,
                                           const float* __restrict__ P, QState p, QState c, float* __restrict__ R)
{
    griddep_enter();
    k_g2_body<LAK, STATE, PQ, BS, BND>(blockIdx.x, d, pf, ids, P, p, c, R);
}
template <bool LAK, bool STATE, bool PQ, int BS, bool BND = false>
struct k_g2_g {
    static constexpr int kBounds = 1, kMaxT = BS, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_g2_body<LAK, STATE, PQ, BS, BND>(bx, a...);
    }
    static constexpr auto kernel() { return &k_g2<LAK, STATE, PQ, BS, BND>; }
};

// ---------------------------------------------------------------------------------------------
// A vertex of P on C's boundary (a slot of its column has a half-edge without
// a twin): 3/4 p + 1/8 of its boundary neighbours, the edge points of the two
// P boundary edges at v.  SLAK: the first out-boundary slot's e_out, then the
// first in-boundary slot's e_in (correctBoundaryS2, CatmullClarkKernels.cuh
// :709-740); LAK: every boundary neighbour once in ascending edge id, which
// for edge points of different P edges is ascending vertex id
// (calculateExternalVertexUpdate, LAKCatmullClarkKernels.cuh:483-511).  yv
// is returned unchanged for an interior vertex.
template <bool LAK>
__device__ __forceinline__ float4 boundary_vertex(const float* __restrict__ P, const SlotScratch& z, int b, int e,
                                                  float4 Pv, float4 yv)
{
    int sb = -1, si = -1;
    for (int s = b; s < e; ++s) {
        const int f = __ldg(z.bflag + s);
        if ((f & 1) && sb < 0) sb = s;
        if ((f & 2) && si < 0) si = s;
    }
    if (sb < 0 && si < 0) return yv;
    if (!LAK) {
        if (sb >= 0) yv = f4_add(f4_mul(Pv, 0.75f), f4_mul(__ldg(z.Z + 2 * (int64_t)sb + 1), 0.125f));
        if (si >= 0) yv = f4_add(yv, f4_mul(ldg4(P, __ldg(z.bid + si)), 0.125f));
        return yv;
    }
    yv = f4_mul(Pv, 0.75f);
    for (int last = -1;;) {            // out-neighbours' ids are in bid, in-neighbours' in T
        int best = INT32_MAX;
        for (int s = b; s < e; ++s) {
            const int f = __ldg(z.bflag + s);
            if (f & 1) { const int o = __ldg(z.bid + s); if (o > last && o < best) best = o; }
            if (f & 2) { const int o = __ldg(z.T + s); if (o > last && o < best) best = o; }
        }
        if (best == INT32_MAX) break;
        yv = f4_add(yv, f4_mul(ldg4(P, best), 0.125f));
        last = best;
    }
    return yv;
}

// ---------------------------------------------------------------------------------------------
// A column of n <= 4 slots from its records in registers: zf / zn the face
// point and neighbour of each slot, tt the LAK tail id or the SLAK rotation
// (rot - b), fl the boundary flags.  Vertex point, then (SLAK) the edge points
// of the column's slots.
template <bool LAK, bool STATE, bool BND>
__device__ __forceinline__ void g3_small(const FastDims& d, const float* __restrict__ P, QState& c,
                                         const SlotScratch& z, float* __restrict__ R, int v, int b, int n,
                                         float4 Pv, const float4 (&zf)[4], const float4 (&zn)[4],
                                         const int (&tt)[4], const int (&fl)[4])
{
    const int e = b + n;
    const float nn = (float)(n * n);
    float4 yv;
    float4 acc = f4_zero();
    if (!LAK) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) acc = f4_add(acc, zn[k]);
        yv = f4_add(f4_div(acc, nn), f4_div(f4_mul(Pv, (float)(n - 2)), (float)n));
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) yv = f4_add(yv, f4_div(zf[k], nn));
        const int64_t EPb = (int64_t)d.V + d.N1;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) {
                if (BND && (fl[k] & 1)) {
                    st4_cs(R, EPb + b + k, f4_mul(f4_add(Pv, zn[k]), 0.5f));
                    continue;
                }
                const int r = tt[k];
                const float4 fr = r == 0 ? zf[0] : r == 1 ? zf[1] : r == 2 ? zf[2] : zf[3];
                const float4 half = f4_mul(f4_add(zn[k], fr), 0.25f);
                st4_cs(R, EPb + b + k, f4_add(f4_add(f4_zero(), f4_mul(f4_add(Pv, zf[k]), 0.25f)), half));
            }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) acc = f4_add(acc, zf[k]);
        // the tails in ascending id (ids in a column are distinct)
        int rk[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            rk[k] = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) rk[k] += (j < n && tt[j] < tt[k]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < n && rk[k] == r) acc = f4_add(acc, zn[k]);
        yv = f4_div_z(f4_add(f4_div_z(acc, (float)n), f4_mul(Pv, __fadd_rn((float)n, -2.0f))), (float)n);
    }
    if (BND && (fl[0] | fl[1] | fl[2] | fl[3])) yv = boundary_vertex<LAK>(P, z, b, e, Pv, yv);
    st_pos<STATE>(R, v, yv);
    if (STATE) c.sptr[v] = b;
}

// ---------------------------------------------------------------------------------------------
// One vertex of P on its own thread (columns of up to kBigCol slots, and
// columns too long for the warp path).
template <bool LAK, bool STATE, bool BND>
__device__ __forceinline__ void g3_vertex(FastDims d, const float* __restrict__ P, QState c, SlotScratch z,
                                          float* __restrict__ R, int compensated, int v, int b, int n)
{
    const int e = b + n;
    const float4 Pv = ldg4(P, v);
    const float nn = (float)(n * n);
    const float4* Z = z.Z;
    float4 yv;
    if (n <= 4) {
        // the common case: every record of the column loaded up front (the
        // arithmetic and its order are the loops' below)
        float4 zf[4], zn[4];
        int tt[4];                             // LAK: tail ids; SLAK: rot - b
        int fl[4] = {0, 0, 0, 0};              // boundary flags
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < n) {
                ld8_nc(Z + 2 * (int64_t)(b + k), zf[k], zn[k]);
                tt[k] = LAK ? __ldg(z.T + b + k) : __ldg(z.rot + b + k) - b;
                if (BND) fl[k] = __ldg(z.bflag + b + k);
            }
        }
        g3_small<LAK, STATE, BND>(d, P, c, z, R, v, b, n, Pv, zf, zn, tt, fl);
        return;
    }
    const bool comp = compensated && n > 4;
    const auto zf = [&](int k) { return __ldg(Z + 2 * (int64_t)(b + k)); };        // FP(x) of slot b+k
    const auto zn = [&](int k) { return __ldg(Z + 2 * (int64_t)(b + k) + 1); };    // its neighbour
    if (!LAK) {
        if (!comp) {
            float4 acc = f4_zero();
            for_each_loaded(n, zn, [&](int, float4 t) { acc = f4_add(acc, t); });
            yv = f4_add(f4_div(acc, nn), f4_div(f4_mul(Pv, (float)(n - 2)), (float)n));
            for_each_loaded(n, zf, [&](int, float4 t) { yv = f4_add(yv, f4_div(t, nn)); });
        } else {
            float4 sh = f4_zero(), sl = f4_zero();
            for_each_loaded(n, zn, [&](int, float4 t) { dd_acc(sh, sl, t); });
            for_each_loaded(n, zf, [&](int, float4 t) { dd_acc(sh, sl, t); });
            yv = vp_finish(sh, sl, Pv, n);
        }
        // edge points of C's edges {v, e_out(x)}, ids b..e-1:
        // 0 + (p_v + FP(x))/4 + (Z[2s+1] + Z[2 rot[s]])/4
        const int64_t EPb = (int64_t)d.V + d.N1;
        for_each_loaded(n, [&](int k) { return f4_add(zn(k), __ldg(Z + 2 * (int64_t)__ldg(z.rot + b + k))); },
                        [&](int k, float4 t) {
                            if (BND && (__ldg(z.bflag + b + k) & 1)) {
                                st4_cs(R, EPb + b + k, f4_mul(f4_add(Pv, zn(k)), 0.5f));
                                return;
                            }
                            const float4 ta = f4_mul(f4_add(Pv, zf(k)), 0.25f);
                            st4_cs(R, EPb + b + k, f4_add(f4_add(f4_zero(), ta), f4_mul(t, 0.25f)));
                        });
    } else {
        // face points in column order, then the tails e_in(x) in ascending id
        float4 acc = f4_zero(), sh = f4_zero(), sl = f4_zero();
        for_each_loaded(n, zf, [&](int, float4 t) { if (comp) dd_acc(sh, sl, t); else acc = f4_add(acc, t); });
        if (n <= kBigCol) {                    // longer columns up to kWarpCol take the warp path
            int perm[kBigCol];
            rank_order(z.T, b, n, perm);
            for_each_loaded(n, [&](int r) { return zn(perm[r]); },
                            [&](int, float4 t) { if (comp) dd_acc(sh, sl, t); else acc = f4_add(acc, t); });
        } else {
            int last = -1;
            while (true) {
                int xm = INT32_MAX, sm = -1;
                for (int s = b; s < e; ++s) {
                    const int ti = __ldg(z.T + s);
                    if (ti > last && ti < xm) { xm = ti; sm = s; }
                }
                if (sm < 0) break;
                const float4 pt = __ldg(Z + 2 * (int64_t)sm + 1);
                if (comp) dd_acc(sh, sl, pt); else acc = f4_add(acc, pt);
                last = xm;
            }
        }
        if (comp) yv = vp_finish(sh, sl, Pv, n);
        else yv = f4_div_z(f4_add(f4_div_z(acc, (float)n), f4_mul(Pv, __fadd_rn((float)n, -2.0f))), (float)n);
    }
    if (BND) yv = boundary_vertex<LAK>(P, z, b, e, Pv, yv);
    st_pos<STATE>(R, v, yv);
    if (STATE) c.sptr[v] = b;
}

// A long column (kBigCol < n <= kWarpCol; the poles of high-valence meshes),
// by the whole warp: each lane loads its (up to two) slots' records, LAK tails
// are ranked by id across the warp, SLAK's edge points are independent per
// slot; the sums run in the order the single-thread path uses, every lane
// fetching slot k (or the tail of rank r) by shuffle, so the result is the
// same bit for bit.  No shared memory: the common path keeps its L1.
template <bool LAK, bool STATE, bool BND>
__device__ __noinline__ void g3_warp_column(FastDims d, const float* __restrict__ P, QState c, SlotScratch z,
                                            float* __restrict__ R, int compensated, int v, int b, int n)
{
    const int lane = threadIdx.x & 31;
    const float4* Z = z.Z;
    const bool h0 = lane < n, h1 = lane + 32 < n;
    const int k0 = b + lane, k1 = b + lane + 32;
    float4 f0 = f4_zero(), f1 = f4_zero(), n0 = f4_zero(), n1 = f4_zero();   // FP(x) and the neighbour
    int t0 = INT32_MAX, t1 = INT32_MAX;
    // two 16-byte loads per record here: ptxas 12.9 fails on the 256-bit load in this function
    if (h0) { f0 = __ldg(Z + 2 * (int64_t)k0); n0 = __ldg(Z + 2 * (int64_t)k0 + 1); if (LAK) t0 = __ldg(z.T + k0); }
    if (h1) { f1 = __ldg(Z + 2 * (int64_t)k1); n1 = __ldg(Z + 2 * (int64_t)k1 + 1); if (LAK) t1 = __ldg(z.T + k1); }
    const float4 Pv = ldg4(P, v);
    if (!LAK) {
        // edge points of C's edges {v, e_out(x)}, ids b..e-1: 0 + (p_v + FP(x))/4 + (Z[2s+1] + Z[2 rot[s]])/4,
        // FP of slot rot[s] from the lane that holds it
        const int64_t EPb = (int64_t)d.V + d.N1;
#pragma unroll
        for (int el = 0; el < 2; ++el) {
            const bool h = el ? h1 : h0;
            const int k = el ? k1 : k0;
            const int q = h ? __ldg(z.rot + k) - b : 0;
            const float4 a = shfl4(f0, q & 31), a1 = shfl4(f1, q & 31);
            if (!h) continue;
            const float4 fr = q < 32 ? a : a1, nk = el ? n1 : n0, fk = el ? f1 : f0;
            if (BND && (__ldg(z.bflag + k) & 1)) {
                st4_cs(R, EPb + k, f4_mul(f4_add(Pv, nk), 0.5f));
                continue;
            }
            const float4 ta = f4_mul(f4_add(Pv, fk), 0.25f);
            st4_cs(R, EPb + k, f4_add(f4_add(f4_zero(), ta), f4_mul(f4_add(nk, fr), 0.25f)));
        }
    }
    // every lane runs the sums (the same values, by shuffle); lane 0 stores
    const bool comp = compensated != 0;
    const float nn = (float)(n * n);
    float4 yv;
    if (!LAK) {
        if (!comp) {
            float4 acc = f4_zero();
            for (int k = 0; k < n; ++k) acc = f4_add(acc, col4(n0, n1, k));
            yv = f4_add(f4_div(acc, nn), f4_div(f4_mul(Pv, (float)(n - 2)), (float)n));
            for (int k = 0; k < n; ++k) yv = f4_add(yv, f4_div(col4(f0, f1, k), nn));
        } else {
            float4 sh = f4_zero(), sl = f4_zero();
            for (int k = 0; k < n; ++k) dd_acc(sh, sl, col4(n0, n1, k));
            for (int k = 0; k < n; ++k) dd_acc(sh, sl, col4(f0, f1, k));
            yv = vp_finish(sh, sl, Pv, n);
        }
    } else {
        int r0, r1;
        rank_of(n, t0, t1, r0, r1);                                  // tails in ascending id
        float4 acc = f4_zero(), sh = f4_zero(), sl = f4_zero();
        for (int k = 0; k < n; ++k) {
            const float4 t = col4(f0, f1, k);
            if (comp) dd_acc(sh, sl, t); else acc = f4_add(acc, t);
        }
        for (int r = 0; r < n; ++r) {
            int src, el;
            slot_of_rank(r, h0, h1, r0, r1, src, el);
            const float4 t = shfl4(el ? n1 : n0, src);
            if (comp) dd_acc(sh, sl, t); else acc = f4_add(acc, t);
        }
        if (comp) yv = vp_finish(sh, sl, Pv, n);
        else yv = f4_div_z(f4_add(f4_div_z(acc, (float)n), f4_mul(Pv, __fadd_rn((float)n, -2.0f))), (float)n);
    }
    if (lane == 0) {
        if (BND) yv = boundary_vertex<LAK>(P, z, b, b + n, Pv, yv);
        st_pos<STATE>(R, v, yv);
        if (STATE) c.sptr[v] = b;
    }
}

// G3: one thread per vertex v of P.  Its column's records (written by k_g1 at
// the column's slots) are contiguous, so the vertex point and, for SLAK, the
// edge points of C's edges {v, e_out(x)} (ids = the slots) stream.  With a
// boundary (BND), an edge {v, e_out(x)} without a twin gets the midpoint.
// Columns longer than kBigCol go to their warp (g3_warp_column).
// `nv`: the vertices of P it covers, V1 (or V2 on a GQ level, whose other
// columns k_g1 sums).
template <bool LAK, bool STATE, int BS, bool BND = false, bool SG = false>
__device__ __forceinline__ void k_g3_body(const unsigned bx_, FastDims d, const float* __restrict__ P, QState p, QState c,
                                          SlotScratch z, float* __restrict__ R, int compensated, int nv)
{
    const int v = bx_ * blockDim.x + threadIdx.x;
    if (STATE && v == nv) c.sptr[d.V] = d.N;
    const bool valid = v < nv;
    int b = 0, n = 0;
    if (valid) {
        if constexpr (SG) { b = sg_sptr(d, p.sptr, v); n = sg_sptr(d, p.sptr, v + 1) - b; }
        else { b = __ldg(p.sptr + v); n = __ldg(p.sptr + v + 1) - b; }
    }
    const bool big = valid && n > kBigCol && n <= kWarpCol;
    if (valid && !big) g3_vertex<LAK, STATE, BND>(d, P, c, z, R, compensated, v, b, n);
    unsigned m = __ballot_sync(0xffffffffu, big);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        g3_warp_column<LAK, STATE, BND>(d, P, c, z, R, compensated, __shfl_sync(0xffffffffu, v, src),
                                        __shfl_sync(0xffffffffu, b, src), __shfl_sync(0xffffffffu, n, src));
    }
}
template <bool LAK, bool STATE, int BS, bool BND = false, bool SG = false>
__global__ void __launch_bounds__(BS) k_g3(FastDims d, const float* __restrict__ P, QState p, QState c,
                                           SlotScratch z, float* __restrict__ R, int compensated, int nv)
{
    griddep_enter();
    k_g3_body<LAK, STATE, BS, BND, SG>(blockIdx.x, d, P, p, c, z, R, compensated, nv);
}
template <bool LAK, bool STATE, int BS, bool BND = false, bool SG = false>
struct k_g3_g {
    static constexpr int kBounds = 1, kMaxT = BS, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_g3_body<LAK, STATE, BS, BND, SG>(bx, a...);
    }
    static constexpr auto kernel() { return &k_g3<LAK, STATE, BS, BND, SG>; }
};

// ---------------------------------------------------------------------------------------------
// k_g3 with its block's slot records staged in shared memory by the bulk-copy
// (TMA) engine.  A block's vertices are consecutive, so their columns are one
// contiguous slot range: thread 0 issues one cp.async.bulk for the range's
// records (32 bytes a slot) and one for its rotation (SLAK) / tail (LAK)
// indices, both completing on an mbarrier; the arithmetic is g3_small's.
// Closed parents only (no boundary records).  Columns of more than 4 slots, and
// blocks whose range exceeds the kBulkSlots staging buffer, read global memory
// as k_g3 does.  The copies read this GPU's own memory, without cluster
// multicast.  The wait is bounded: after `polls` unsuccessful polls the block
// records SLAK_ERR_TIMEOUT, waits (again bounded) for its own copies, which
// write its shared memory, and returns.  128-thread blocks.
constexpr int kBulkBlock = 128;
constexpr int kBulkSlots = 6 * kBulkBlock;
constexpr int kBulkRetire = 1 << 22;      // polls allowed for the copies to land after a timeout

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls)
{
    for (int i = 0; i < polls; ++i) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

template <bool LAK, bool STATE>
__device__ __forceinline__ void k_g3_bulk_body(const unsigned bx_, FastDims d, const float* __restrict__ P, QState p,
                                               QState c, SlotScratch z, float* __restrict__ R,
                                               int compensated, int nv, DevStatus* st, int polls)
{
    __shared__ __align__(128) float4 zs[2 * kBulkSlots];
    __shared__ __align__(16) int rs[kBulkSlots + 8];
    __shared__ __align__(8) unsigned long long bar;
    const int v0 = bx_ * kBulkBlock, v = v0 + threadIdx.x;
    if (STATE && v == nv) c.sptr[d.V] = d.N;
    if (v0 >= nv) return;                                   // the sentinel's block
    const int vl = min(v0 + kBulkBlock, nv);
    const int sb = __ldg(p.sptr + v0), se = __ldg(p.sptr + vl);
    const int rb = sb & ~3, re = (se + 3) & ~3;             // 16-byte aligned index range
    const bool staged = se - sb <= kBulkSlots;              // the same for the whole block
    if (staged) {
        const uint32_t sbar = (uint32_t)__cvta_generic_to_shared(&bar);
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(sbar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t zbytes = 32u * (uint32_t)(se - sb), ibytes = 4u * (uint32_t)(re - rb);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(sbar), "r"(zbytes + ibytes)
                         : "memory");
            if (zbytes)
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             :: "r"((uint32_t)__cvta_generic_to_shared(zs)), "l"(z.Z + 2 * (int64_t)sb),
                                "r"(zbytes), "r"(sbar) : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"((uint32_t)__cvta_generic_to_shared(rs)), "l"((LAK ? z.T : z.rot) + rb),
                            "r"(ibytes), "r"(sbar) : "memory");
        }
        // the warp decides together (the column pass below shuffles across it)
        if (!__all_sync(0xffffffffu, mbar_wait(sbar, 0, polls))) {
            if ((threadIdx.x & 31) == 0) set_error(st, 5, 3000000 + bx_);     // SLAK_ERR_TIMEOUT
            mbar_wait(sbar, 0, kBulkRetire);
            return;
        }
    }
    const bool valid = v < nv;
    int b = 0, n = 0;
    if (valid) { b = __ldg(p.sptr + v); n = __ldg(p.sptr + v + 1) - b; }
    const bool big = valid && n > kBigCol && n <= kWarpCol;
    if (valid && staged && n <= 4) {
        float4 zf[4], zn[4];
        int tt[4], fl[4] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) {
                zf[k] = zs[2 * (b - sb + k)];
                zn[k] = zs[2 * (b - sb + k) + 1];
                tt[k] = LAK ? rs[b + k - rb] : rs[b + k - rb] - b;
            }
        g3_small<LAK, STATE, false>(d, P, c, z, R, v, b, n, ldg4(P, v), zf, zn, tt, fl);
    } else if (valid && !big) {
        g3_vertex<LAK, STATE, false>(d, P, c, z, R, compensated, v, b, n);
    }
    unsigned m = __ballot_sync(0xffffffffu, big);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        g3_warp_column<LAK, STATE, false>(d, P, c, z, R, compensated, __shfl_sync(0xffffffffu, v, src),
                                          __shfl_sync(0xffffffffu, b, src), __shfl_sync(0xffffffffu, n, src));
    }
}
template <bool LAK, bool STATE>
__global__ void __launch_bounds__(kBulkBlock) k_g3_bulk(FastDims d, const float* __restrict__ P, QState p,
                                                        QState c, SlotScratch z, float* __restrict__ R,
                                                        int compensated, int nv, DevStatus* st, int polls)
{
    griddep_enter();
    k_g3_bulk_body<LAK, STATE>(blockIdx.x, d, P, p, c, z, R, compensated, nv, st, polls);
}
template <bool LAK, bool STATE>
struct k_g3_bulk_g {
    static constexpr int kBounds = 1, kMaxT = kBulkBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_g3_bulk_body<LAK, STATE>(bx, a...);
    }
    static constexpr auto kernel() { return &k_g3_bulk<LAK, STATE>; }
};

// ---------------------------------------------------------------------------------------------
// 1 for each edge of a general level without a twin (H holds -1), the input of
// the scan that gives the edges' boundary ranks to the first fast level
__device__ __forceinline__ void k_export_bflag_body(const unsigned bx_, int E, const int2* __restrict__ H, int* __restrict__ isb)
{
    int e = bx_ * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int2 h = H[e];
    isb[e] = (h.x < 0) | (h.y < 0);
}
__global__ void k_export_bflag(int E, const int2* __restrict__ H, int* __restrict__ isb)
{
    griddep_enter();
    k_export_bflag_body(blockIdx.x, E, H, isb);
}
struct k_export_bflag_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_export_bflag_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_export_bflag; }
};

}  // namespace slak
