// general.cuh -- per-level kernels for an arbitrary polygon (or quad) mesh.
//
// One level turns a control mesh (F faces, N corners, V vertices) into an
// all-quad mesh.  The general path rebuilds the vertex adjacency every level:
//
//   k_face_map_valence  corner -> face and corners per vertex (polygon levels)
//                                                         createThreadFaceMapping, CatmullClarkKernels.cuh:189-198,
//                                                         + evaluateValences, :137-145
//   k_valence    corners per vertex (quad levels)         evaluateValences, :137-145
//   scan         adjacency offsets                        cub_wrappers.cuh:30-43
//   k_bucket     corners into their vertex's column       evaluateAdjacencies[Quad], :147-187
//   k_vsort      column sorted by corner index, plus the vertex after / before
//                each slot's corner (S_row_ids of the reference)
//   k_edges_*    twin half-edges, boundary flags, edge-owner counts
//                (SLAK: checkForBoundary*, :200-321; LAK: the M^T M pattern of spgemm.cuh:61-100)
//   scan         edge offsets                             CatmullClarkImpl.cu:209-211
//   k_eids_*     edge id of every half-edge + edge -> half-edge table
//   k_refine     refined quads (+ the fast path's t)      refineTopology*, :405-575; LAKCatmullClarkKernels.cuh:320-431
//
// The reference assigns adjacency slots with atomicAdd, so its edge numbering
// changes from run to run.  Here every column is sorted by corner index, which
// is the numbering a serialized execution of the reference produces; the
// result is deterministic and equals the CPU restatement exactly.
#pragma once

#include "common.cuh"

namespace slak {

enum : int { SF_OWNER = 1, SF_BOUT = 2, SF_BIN = 4 };

// polygon levels: corner -> face (validating ptr) and the valences in one pass
// over the faces
__device__ __forceinline__ void k_face_map_valence_body(const unsigned bx_, const int* __restrict__ ptr, const int* __restrict__ ids, int F, int N, int V,
                                                        int* __restrict__ cface, int* __restrict__ cnt, DevStatus* st)
{
    int f = bx_ * blockDim.x + threadIdx.x;
    if (f == 0 && (ptr[0] != 0 || ptr[F] != N)) set_error(st, 4, -1);
    if (f >= F) return;
    int b = ptr[f], e = ptr[f + 1];
    if (b < 0 || e > N || e - b < 3) { set_error(st, 4, f); return; }
    for (int c = b; c < e; ++c) {
        cface[c] = f;
        const int v = __ldg(ids + c);
        if ((unsigned)v >= (unsigned)V) { set_error(st, 4, c); continue; }
        atomicAdd(cnt + v, 1);
    }
}
__global__ void k_face_map_valence(const int* __restrict__ ptr, const int* __restrict__ ids, int F, int N, int V,
                                   int* __restrict__ cface, int* __restrict__ cnt, DevStatus* st)
{
    griddep_enter();
    k_face_map_valence_body(blockIdx.x, ptr, ids, F, N, V, cface, cnt, st);
}
struct k_face_map_valence_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_face_map_valence_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_face_map_valence; }
};

__device__ __forceinline__ void k_valence_body(const unsigned bx_, const int* __restrict__ ids, int N, int V, int* __restrict__ cnt, DevStatus* st)
{
    int c = bx_ * blockDim.x + threadIdx.x;
    if (c >= N) return;
    int v = ids[c];
    if ((unsigned)v >= (unsigned)V) { set_error(st, 4, c); return; }
    atomicAdd(cnt + v, 1);
}
__global__ void k_valence(const int* __restrict__ ids, int N, int V, int* __restrict__ cnt, DevStatus* st)
{
    griddep_enter();
    k_valence_body(blockIdx.x, ids, N, V, cnt, st);
}
struct k_valence_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_valence_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_valence; }
};

// valence histogram (0..15, 16 or more): the autotuner's key, read with the
// level-0 probe
__device__ __forceinline__ void k_valence_hist_body(const unsigned bx_, int V, const int* __restrict__ sptr, int* __restrict__ hist)
{
    __shared__ int h[17];
    if (threadIdx.x < 17) h[threadIdx.x] = 0;
    __syncthreads();
    const int v = bx_ * blockDim.x + threadIdx.x;
    if (v < V) atomicAdd(&h[min(sptr[v + 1] - sptr[v], 16)], 1);
    __syncthreads();
    if (threadIdx.x < 17 && h[threadIdx.x]) atomicAdd(hist + threadIdx.x, h[threadIdx.x]);
}
__global__ void k_valence_hist(int V, const int* __restrict__ sptr, int* __restrict__ hist)
{
    griddep_enter();
    k_valence_hist_body(blockIdx.x, V, sptr, hist);
}
struct k_valence_hist_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_valence_hist_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_valence_hist; }
};

// slot order from the atomic is arbitrary (the unsorted column goes to
// `loose`); k_vsort makes it canonical.  A malformed polygon mesh (a face the
// valence pass rejected, or corners past ptr[F]) brings more corners to a
// vertex than its column counts: those find no slot (r < 0) and are dropped,
// so nothing is written outside the column; the level fails with BAD_MESH.
__device__ __forceinline__ void k_bucket_body(const unsigned bx_, const int* __restrict__ ids, int N, int V, const int* __restrict__ sptr,
                                              int* __restrict__ fill, int* __restrict__ loose)
{
    int c = bx_ * blockDim.x + threadIdx.x;
    if (c >= N) return;
    int v = ids[c];
    if ((unsigned)v >= (unsigned)V) return;
    int r = atomicSub(fill + v, 1) - 1;
    if (r >= 0) loose[sptr[v] + r] = c;
}
__global__ void k_bucket(const int* __restrict__ ids, int N, int V, const int* __restrict__ sptr,
                         int* __restrict__ fill, int* __restrict__ loose)
{
    griddep_enter();
    k_bucket_body(blockIdx.x, ids, N, V, sptr, fill, loose);
}
struct k_bucket_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_bucket_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_bucket; }
};

// Each column sorted by corner index: a corner's slot is the number of smaller
// corners in its column (corner indices are distinct).  One thread per corner
// (four times the threads of one per vertex, and the corner-indexed reads and
// writes coalesced); a column of up to 8 is read into registers at once.  With
// `xslot` the slot of every corner is exported as well (corner -> slot, for
// the fast path).
template <bool QUAD>
__device__ __forceinline__ void vsort_neighbours(Faces<QUAD> fc, const int* __restrict__ ids, int s, int c,
                                                 int* __restrict__ snext, int* __restrict__ sprev,
                                                 int* __restrict__ sprevc)
{
    const int p = fc.prev(c);
    snext[s] = __ldg(ids + fc.next(c));
    sprev[s] = __ldg(ids + p);
    sprevc[s] = p;
}

template <bool QUAD>
__device__ __forceinline__ void k_vsort_body(const unsigned bx_, Faces<QUAD> fc, const int* __restrict__ ids, int N,
                                             int V, const int* __restrict__ sptr, const int* __restrict__ loose,
                                             int* __restrict__ sc, int* __restrict__ snext, int* __restrict__ sprev,
                                             int* __restrict__ sprevc, int* __restrict__ xslot)
{
    // one thread per corner c: its slot is its rank by corner id within its
    // vertex's column (the column's entries are distinct corner ids)
    const int c = bx_ * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int v = __ldg(ids + c);
    if ((unsigned)v >= (unsigned)V) return;              // flagged by the valence pass
    const int b = __ldg(sptr + v), n = __ldg(sptr + v + 1) - b;
    int r = 0;
    if (n <= 8) {
        int u[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) u[k] = k < n ? __ldg(loose + b + k) : INT32_MAX;
#pragma unroll
        for (int k = 0; k < 8; ++k) r += u[k] < c;
    } else {
        for (int j = 0; j < n; ++j) r += __ldg(loose + b + j) < c;
    }
    // a malformed mesh's dropped corner is not in its column: no slot
    if (r >= n) return;
    sc[b + r] = c;
    if (xslot) xslot[c] = b + r;
    vsort_neighbours(fc, ids, b + r, c, snext, sprev, sprevc);
}
template <bool QUAD>
__global__ void k_vsort(Faces<QUAD> fc, const int* __restrict__ ids, int N, int V, const int* __restrict__ sptr,
                        const int* __restrict__ loose, int* __restrict__ sc, int* __restrict__ snext,
                        int* __restrict__ sprev, int* __restrict__ sprevc, int* __restrict__ xslot)
{
    griddep_enter();
    k_vsort_body<QUAD>(blockIdx.x, fc, ids, N, V, sptr, loose, sc, snext, sprev, sprevc, xslot);
}
template <bool QUAD>
struct k_vsort_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_vsort_body<QUAD>(bx, a...);
    }
    static constexpr auto kernel() { return &k_vsort<QUAD>; }
};

// Twins and boundary flags from the vertex's own column: the outgoing
// half-edge v->w of slot s has a twin iff some corner at v is entered from w.
// SLAK owner: the half-edge min->max, or the only half-edge of a boundary edge
// (epids_tmp = v0 < v1, set to 1 by checkForBoundary*, CatmullClarkKernels.cuh:159,235).
// LAK edges of column v are its distinct neighbours u < v (createEVals, spgemm.cuh:71-100).
//
// One slot's result, given the column as (next vertex, previous vertex,
// previous corner) per slot; NMAX > 0 unrolls over a column held in registers.
template <bool LAK, int NMAX, class Col>
__device__ __forceinline__ void edge_slot(const Col& col, int n, int k, int v, int& tw, int& fl, int& own,
                                          int& bad)
{
    const int w = col.nx(k), u = col.pv(k);
    int in_twin = 0;
    tw = -1;
    bool dn = w < v, dp = u < v && u != w;
#pragma unroll
    for (int t = 0; t < (NMAX > 0 ? NMAX : n); ++t) {
        if (NMAX > 0 && t >= n) break;
        const int nt = col.nx(t), pt = col.pv(t);
        if (pt == w) { if (tw < 0) tw = col.pc(t); else bad = 1; }
        if (nt == u) in_twin = 1;
        if (t < k) {
            if (nt == w) bad = 1;
            if (LAK) {
                if (nt == w || pt == w) dn = false;
                if (nt == u || pt == u) dp = false;
            }
        }
    }
    if (w == v || u == v) bad = 1;
    fl = (tw < 0 ? SF_BOUT : 0) | (in_twin ? 0 : SF_BIN);
    own = 0;
    if (!LAK) {
        if (v < w || tw < 0) { fl |= SF_OWNER; own = 1; }
    } else {
        own = (int)dn + (int)dp;            // enumerated as snext[0], sprev[0], snext[1], ...
    }
}

struct ColGlobal {       // column slots b.. in global memory
    const int *snext, *sprev, *sprevc;
    int b;
    __device__ int nx(int t) const { return __ldg(snext + b + t); }
    __device__ int pv(int t) const { return __ldg(sprev + b + t); }
    __device__ int pc(int t) const { return __ldg(sprevc + b + t); }
};
struct ColRegs {         // a column of at most 8 slots in registers
    int n_[8], p_[8], c_[8];
    __device__ int nx(int t) const { return n_[t]; }
    __device__ int pv(int t) const { return p_[t]; }
    __device__ int pc(int t) const { return c_[t]; }
};

// Columns of up to 8 slots are handled by their own thread from registers; a
// longer column (a high-valence vertex) is shared by its warp's 32 lanes, one
// slot per lane, so no thread walks n^2 pairs alone.
// With `xtw` the twin of every corner is exported as well (corner -> twin).
template <bool LAK>
__device__ __forceinline__ void k_edges_body(const unsigned bx_, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                                             const int* __restrict__ snext, const int* __restrict__ sprev,
                                             const int* __restrict__ sprevc, int* __restrict__ stw, int* __restrict__ sflag,
                                             int* __restrict__ ecnt, int* __restrict__ bcount, int* __restrict__ xtw, DevStatus* st)
{
    const int v = bx_ * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int nb = 0, b = 0, n = 0;
    if (v < V) { b = sptr[v]; n = sptr[v + 1] - b; }
    if (v < V && n <= 8) {
        ColRegs col;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            col.n_[k] = k < n ? __ldg(snext + b + k) : -1;
            col.p_[k] = k < n ? __ldg(sprev + b + k) : -1;
            col.c_[k] = k < n ? __ldg(sprevc + b + k) : -1;
        }
        int own = 0, bad = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k < n) {
                int tw, fl, o;
                edge_slot<LAK, 8>(col, n, k, v, tw, fl, o, bad);
                own += o;
                nb += tw < 0;
                stw[b + k] = tw;
                sflag[b + k] = fl;
                if (xtw) xtw[__ldg(sc + b + k)] = tw;
            }
        }
        ecnt[v] = own;
        if (bad) set_error(st, 4, v);
    }
    unsigned big = __ballot_sync(0xffffffffu, v < V && n > 8);
    while (big) {
        const int src = __ffs(big) - 1;
        big &= big - 1;
        const int bv = __shfl_sync(0xffffffffu, v, src), bb = __shfl_sync(0xffffffffu, b, src);
        const int bn = __shfl_sync(0xffffffffu, n, src);
        const ColGlobal col{snext, sprev, sprevc, bb};
        int own = 0, bad = 0;
        for (int k = lane; k < bn; k += 32) {
            int tw, fl, o;
            edge_slot<LAK, 0>(col, bn, k, bv, tw, fl, o, bad);
            own += o;
            nb += tw < 0;
            stw[bb + k] = tw;
            sflag[bb + k] = fl;
            if (xtw) xtw[__ldg(sc + bb + k)] = tw;
        }
        for (int o = 16; o > 0; o >>= 1) own += __shfl_down_sync(0xffffffffu, own, o);
        bad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
            ecnt[bv] = own;
            if (bad) set_error(st, 4, bv);
        }
    }
    // boundary half-edge count of the level
    for (int o = 16; o > 0; o >>= 1) nb += __shfl_down_sync(0xffffffffu, nb, o);
    if (lane == 0 && nb) atomicAdd(bcount, nb);
}
template <bool LAK>
__global__ void k_edges(int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                        const int* __restrict__ snext, const int* __restrict__ sprev,
                        const int* __restrict__ sprevc, int* __restrict__ stw, int* __restrict__ sflag,
                        int* __restrict__ ecnt, int* __restrict__ bcount, int* __restrict__ xtw, DevStatus* st)
{
    griddep_enter();
    k_edges_body<LAK>(blockIdx.x, V, sptr, sc, snext, sprev, sprevc, stw, sflag, ecnt, bcount, xtw, st);
}
template <bool LAK>
struct k_edges_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_edges_body<LAK>(bx, a...);
    }
    static constexpr auto kernel() { return &k_edges<LAK>; }
};

// SLAK edge ids: owners in slot order get eptr[v] + rank; the twin shares it.
// Thread 0 of k_eids_* also checks the level's edge and boundary counts
// against the sizes the plan was made for (a topology change since creation).
__device__ __forceinline__ void check_level(int v, const int* eptr, int V, int E, const int* bcount, int B,
                                            DevStatus* st, int li)
{
    if (v == 0 && (eptr[V] != E || *bcount != B)) set_error(st, 4, 1000 + li);
}

__device__ __forceinline__ void k_eids_slak_body(const unsigned bx_, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                                                 const int* __restrict__ stw, const int* __restrict__ sflag,
                                                 const int* __restrict__ eptr, int Ecap, int* __restrict__ eid,
                                                 int2* __restrict__ H, DevStatus* st, const int* bcount, int B, int li)
{
    int v = bx_ * blockDim.x + threadIdx.x;
    check_level(v, eptr, V, Ecap, bcount, B, st, li);
    if (v >= V) return;
    int id = eptr[v];
    for (int s = sptr[v]; s < sptr[v + 1]; ++s) {
        if (!(sflag[s] & SF_OWNER)) continue;
        if (id >= Ecap) { set_error(st, 4, v); return; }
        int c = sc[s], t = stw[s];
        eid[c] = id;
        if (t >= 0) eid[t] = id;
        H[id] = make_int2(c, t);
        ++id;
    }
}
__global__ void k_eids_slak(int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                            const int* __restrict__ stw, const int* __restrict__ sflag,
                            const int* __restrict__ eptr, int Ecap, int* __restrict__ eid,
                            int2* __restrict__ H, DevStatus* st, const int* bcount, int B, int li)
{
    griddep_enter();
    k_eids_slak_body(blockIdx.x, V, sptr, sc, stw, sflag, eptr, Ecap, eid, H, st, bcount, B, li);
}
struct k_eids_slak_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_eids_slak_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_eids_slak; }
};

// LAK edge ids of one vertex's column on its own thread
__device__ __forceinline__ void eids_lak_vertex(const int* __restrict__ sc, const int* __restrict__ snext,
                                                const int* __restrict__ sprev, const int* __restrict__ sprevc,
                                                const int* __restrict__ eptr, int Ecap, int* __restrict__ eid,
                                                int2* __restrict__ H, DevStatus* st, int v, int b, int e)
{
    int id = eptr[v], last = -1;
    while (true) {
        int x = INT32_MAX, s = b;
        for (; s + 4 <= e; s += 4) {          // the column's loads issued four slots at a time
            int w[4], u[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { w[i] = __ldg(snext + s + i); u[i] = __ldg(sprev + s + i); }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (w[i] > last && w[i] < v && w[i] < x) x = w[i];
                if (u[i] > last && u[i] < v && u[i] < x) x = u[i];
            }
        }
        for (; s < e; ++s) {
            int w = snext[s], u = sprev[s];
            if (w > last && w < v && w < x) x = w;
            if (u > last && u < v && u < x) x = u;
        }
        if (x == INT32_MAX) break;
        if (id >= Ecap) { set_error(st, 4, v); return; }
        int cvx = -1, cxv = -1;
        for (int s = b; s < e; ++s) {
            if (snext[s] == x && cvx < 0) cvx = sc[s];
            if (sprev[s] == x && cxv < 0) cxv = sprevc[s];
        }
        if (cvx >= 0) eid[cvx] = id;
        if (cxv >= 0) eid[cxv] = id;
        H[id] = make_int2(cxv, cvx);
        ++id;
        last = x;
    }
}

// a long column (kBigCol < n <= kWarpCol) by its warp.  The distinct smaller
// neighbours are the snext values < v (distinct) plus the sprev values < v not
// among them; each of a lane's (up to two) slots ranks its values among those,
// reading the column by shuffle, then writes its own corners' edge ids and
// their halves of H (-1 for the half whose half-edge is missing) -- the ids
// and H the serial ascending walk assigns.
__device__ __noinline__ void eids_lak_warp(const int* __restrict__ sc, const int* __restrict__ snext,
                                           const int* __restrict__ sprev, const int* __restrict__ sprevc,
                                           const int* __restrict__ eptr, int Ecap, int* __restrict__ eid,
                                           int2* __restrict__ H, DevStatus* st, int v, int b, int n)
{
    const int lane = threadIdx.x & 31;
    const bool h0 = lane < n, h1 = lane + 32 < n;
    const int sn0 = h0 ? __ldg(snext + b + lane) : INT32_MAX, sn1 = h1 ? __ldg(snext + b + lane + 32) : INT32_MAX;
    const int sp0 = h0 ? __ldg(sprev + b + lane) : INT32_MAX, sp1 = h1 ? __ldg(sprev + b + lane + 32) : INT32_MAX;
    // fn: my snext value is also a prev; fp: my prev value is also a next
    int fn0 = 0, fn1 = 0, fp0 = 0, fp1 = 0;
    for (int j = 0; j < n; ++j) {
        const int y = col1(sp0, sp1, j), x = col1(sn0, sn1, j);
        fn0 |= y == sn0; fn1 |= y == sn1;
        fp0 |= x == sp0; fp1 |= x == sp1;
    }
    // rank of value u among the distinct values < v: next values below u, and
    // prev values below u that are not next values
    int rn0 = 0, rn1 = 0, rp0 = 0, rp1 = 0;
    for (int j = 0; j < n; ++j) {
        const int x = col1(sn0, sn1, j), y = col1(sp0, sp1, j);
        const int only = !__shfl_sync(0xffffffffu, j < 32 ? fp0 : fp1, j & 31);
        rn0 += (x < sn0) + ((y < sn0) & only); rn1 += (x < sn1) + ((y < sn1) & only);
        rp0 += (x < sp0) + ((y < sp0) & only); rp1 += (x < sp1) + ((y < sp1) & only);
    }
    const int base = eptr[v];
    int* Hi = reinterpret_cast<int*>(H);
#pragma unroll
    for (int el = 0; el < 2; ++el) {
        if (!(el ? h1 : h0)) continue;
        const int k = b + lane + 32 * el;
        const int u = el ? sn1 : sn0, w = el ? sp1 : sp0;
        if (u < v) {
            const int id = base + (el ? rn1 : rn0);
            if (id >= Ecap) set_error(st, 4, v);
            else {
                const int c = __ldg(sc + k);
                eid[c] = id;
                Hi[2 * id + 1] = c;
                if (!(el ? fn1 : fn0)) Hi[2 * id] = -1;
            }
        }
        if (w < v) {
            const int id = base + (el ? rp1 : rp0);
            if (id >= Ecap) set_error(st, 4, v);
            else {
                const int c = __ldg(sprevc + k);
                eid[c] = id;
                Hi[2 * id] = c;
                if (!(el ? fp1 : fp0)) Hi[2 * id + 1] = -1;
            }
        }
    }
}

// LAK edge ids: ascending (max, min); H = (half-edge min->max, half-edge
// max->min), -1 where one is missing.  Columns longer than kBigCol go to
// their warp.
__device__ __forceinline__ void k_eids_lak_body(const unsigned bx_, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                                                const int* __restrict__ snext, const int* __restrict__ sprev,
                                                const int* __restrict__ sprevc, const int* __restrict__ eptr, int Ecap,
                                                int* __restrict__ eid, int2* __restrict__ H, DevStatus* st, const int* bcount, int B,
                                                int li)
{
    const int v = bx_ * blockDim.x + threadIdx.x;
    check_level(v, eptr, V, Ecap, bcount, B, st, li);
    const bool valid = v < V;
    int b = 0, n = 0;
    if (valid) { b = sptr[v]; n = sptr[v + 1] - b; }
    const bool big = valid && n > kBigCol && n <= kWarpCol;
    if (valid && !big) eids_lak_vertex(sc, snext, sprev, sprevc, eptr, Ecap, eid, H, st, v, b, b + n);
    unsigned m = __ballot_sync(0xffffffffu, big);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        eids_lak_warp(sc, snext, sprev, sprevc, eptr, Ecap, eid, H, st, __shfl_sync(0xffffffffu, v, src),
                      __shfl_sync(0xffffffffu, b, src), __shfl_sync(0xffffffffu, n, src));
    }
}
__global__ void k_eids_lak(int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                           const int* __restrict__ snext, const int* __restrict__ sprev,
                           const int* __restrict__ sprevc, const int* __restrict__ eptr, int Ecap,
                           int* __restrict__ eid, int2* __restrict__ H, DevStatus* st, const int* bcount, int B,
                           int li)
{
    griddep_enter();
    k_eids_lak_body(blockIdx.x, V, sptr, sc, snext, sprev, sprevc, eptr, Ecap, eid, H, st, bcount, B, li);
}
struct k_eids_lak_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_eids_lak_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_eids_lak; }
};

// refined quad of corner c: {v, V+F+e_out, V+face, V+F+e_in}
// With `xt` (a SLAK level whose state feeds the fast path) it also exports
// t[c] = slot[twin(prev c)], -1 where prev(c) has no twin.
template <bool QUAD, bool LAK>
__device__ __forceinline__ void k_refine_body(const unsigned bx_, Faces<QUAD> fc, const int* __restrict__ ids, const int* __restrict__ eid, int N,
                                              int V, int F, int4* __restrict__ out_ids, int* __restrict__ out_ptr,
                                              int4* __restrict__ out_vals, const int* __restrict__ xslot, const int* __restrict__ xtw,
                                              int* __restrict__ xt)
{
    int c = bx_ * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int VF = V + F;
    const int p = fc.prev(c);
    int4 q = make_int4(__ldg(ids + c), VF + __ldg(eid + c), V + fc.face(c), VF + __ldg(eid + p));
    __stcs(out_ids + c, q);
    if (xt) {
        const int tp = __ldg(xtw + p);
        xt[c] = tp >= 0 ? __ldg(xslot + tp) : -1;
    }
    if (LAK && out_vals != nullptr) {          // only the final level stores ptr / vals
        __stcs(out_vals + c, make_int4(1, 2, 3, 4));
        out_ptr[c] = 4 * c;
        if (c == N - 1) out_ptr[N] = 4 * N;
    }
}
template <bool QUAD, bool LAK>
__global__ void k_refine(Faces<QUAD> fc, const int* __restrict__ ids, const int* __restrict__ eid, int N,
                         int V, int F, int4* __restrict__ out_ids, int* __restrict__ out_ptr,
                         int4* __restrict__ out_vals, const int* __restrict__ xslot, const int* __restrict__ xtw,
                         int* __restrict__ xt)
{
    griddep_enter();
    k_refine_body<QUAD, LAK>(blockIdx.x, fc, ids, eid, N, V, F, out_ids, out_ptr, out_vals, xslot, xtw, xt);
}
template <bool QUAD, bool LAK>
struct k_refine_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_refine_body<QUAD, LAK>(bx, a...);
    }
    static constexpr auto kernel() { return &k_refine<QUAD, LAK>; }
};

// ------------------------------------------------------------------ positions

// SLAK quad face point: ((c0 + c2) + (c1 + c3)) * 1/4, the pairing of the
// width-16 shuffles in calculateFaceEdgepointsQuad (CatmullClarkKernels.cuh:586-594)
__device__ __forceinline__ void k_fp_slak_quad_body(const unsigned bx_, const int4* __restrict__ ids4, const float* __restrict__ P, int F,
                                                    float* __restrict__ FP)
{
    int f = bx_ * blockDim.x + threadIdx.x;
    if (f >= F) return;
    int4 q = __ldg(ids4 + f);
    float4 a = ldg4(P, q.x), b = ldg4(P, q.y), c = ldg4(P, q.z), d = ldg4(P, q.w);
    st4(FP, f, f4_mul(f4_add(f4_add(a, c), f4_add(b, d)), 0.25f));
}
__global__ void k_fp_slak_quad(const int4* __restrict__ ids4, const float* __restrict__ P, int F,
                               float* __restrict__ FP)
{
    griddep_enter();
    k_fp_slak_quad_body(blockIdx.x, ids4, P, F, FP);
}
struct k_fp_slak_quad_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_fp_slak_quad_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_fp_slak_quad; }
};

// polygon face point: sum from zero in corner order, then
//   SLAK: times the rounded reciprocal of the order (calculateFacepoints, :602-618)
//   LAK:  divided by the order, plus 0 (spmv_left_mapped_f4 + divElementWise,
//         LAKCatmullClarkImpl.cu:175-178)
template <bool QUAD, bool LAK>
__device__ __forceinline__ void k_fp_seq_body(const unsigned bx_, const int* __restrict__ ptr, const int* __restrict__ ids, const float* __restrict__ P,
                                              int F, float* __restrict__ FP)
{
    int f = bx_ * blockDim.x + threadIdx.x;
    if (f >= F) return;
    int b = QUAD ? 4 * f : ptr[f], e = QUAD ? 4 * f + 4 : ptr[f + 1];
    float4 acc = f4_zero();
    for (int c = b; c < e; ++c) acc = f4_add(acc, ldg4(P, __ldg(ids + c)));
    float n = (float)(e - b);
    st4(FP, f, LAK ? f4_div_z(acc, n) : f4_mul(acc, __fdiv_rn(1.0f, n)));
}
template <bool QUAD, bool LAK>
__global__ void k_fp_seq(const int* __restrict__ ptr, const int* __restrict__ ids, const float* __restrict__ P,
                         int F, float* __restrict__ FP)
{
    griddep_enter();
    k_fp_seq_body<QUAD, LAK>(blockIdx.x, ptr, ids, P, F, FP);
}
template <bool QUAD, bool LAK>
struct k_fp_seq_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_fp_seq_body<QUAD, LAK>(bx, a...);
    }
    static constexpr auto kernel() { return &k_fp_seq<QUAD, LAK>; }
};

// edge points.  SLAK: 0 + (p_a + fp_a)/4 + (p_b + fp_b)/4 over the two
// half-edges (calculateFaceEdgepointsQuad :597-599, calculateEdgepoints
// :620-632); a boundary edge becomes the midpoint (correctBoundaryS1 :713).
// LAK: (((p_min + p_max) + fp(min->max)) + fp(max->min)) / 4, boundary midpoint
// (calculateInternal/ExternalEdgepoints, LAKCatmullClarkKernels.cuh:437-462).
template <bool QUAD, bool LAK>
__device__ __forceinline__ void k_ep_body(const unsigned bx_, Faces<QUAD> fc, const int* __restrict__ ids, const int2* __restrict__ H, int E,
                                          const float* __restrict__ P, const float* __restrict__ FP, float* __restrict__ EP)
{
    int e = bx_ * blockDim.x + threadIdx.x;
    if (e >= E) return;
    int2 h = __ldg(H + e);
    float4 r;
    if (h.x >= 0 && h.y >= 0) {
        if (!LAK) {
            float4 ta = f4_mul(f4_add(ldg4(P, __ldg(ids + h.x)), ldg4(FP, fc.face(h.x))), 0.25f);
            float4 tb = f4_mul(f4_add(ldg4(P, __ldg(ids + h.y)), ldg4(FP, fc.face(h.y))), 0.25f);
            r = f4_add(f4_add(f4_zero(), ta), tb);
        } else {
            float4 s = f4_add(ldg4(P, __ldg(ids + h.x)), ldg4(P, __ldg(ids + h.y)));
            s = f4_add(f4_add(s, ldg4(FP, fc.face(h.x))), ldg4(FP, fc.face(h.y)));
            r = f4_mul(s, 0.25f);
        }
    } else {
        int a = h.x >= 0 ? h.x : h.y;
        int t = __ldg(ids + a), hd = __ldg(ids + fc.next(a));
        int lo = t < hd ? t : hd, hi = t < hd ? hd : t;
        r = LAK ? f4_mul(f4_add(ldg4(P, lo), ldg4(P, hi)), 0.5f)
                : f4_mul(f4_add(ldg4(P, t), ldg4(P, hd)), 0.5f);
    }
    st4_cs(EP, e, r);
}
template <bool QUAD, bool LAK>
__global__ void k_ep(Faces<QUAD> fc, const int* __restrict__ ids, const int2* __restrict__ H, int E,
                     const float* __restrict__ P, const float* __restrict__ FP, float* __restrict__ EP)
{
    griddep_enter();
    k_ep_body<QUAD, LAK>(blockIdx.x, fc, ids, H, E, P, FP, EP);
}
template <bool QUAD, bool LAK>
struct k_ep_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_ep_body<QUAD, LAK>(bx, a...);
    }
    static constexpr auto kernel() { return &k_ep<QUAD, LAK>; }
};

// SLAK boundary vertex: 3/4 p + 1/8 next (first out-boundary slot) + 1/8 prev
// (first in-boundary slot); y unchanged when v has no boundary slot
__device__ __forceinline__ float4 vp_slak_boundary(const int* __restrict__ snext, const int* __restrict__ sprev,
                                                   const int* __restrict__ sflag, const float* __restrict__ P,
                                                   int v, int b, int e, float4 y)
{
    int sb = -1, si = -1;
    for (int s = b; s < e; ++s) {
        int f = sflag[s];
        if ((f & SF_BOUT) && sb < 0) sb = s;
        if ((f & SF_BIN) && si < 0) si = s;
    }
    if (sb >= 0) y = f4_add(f4_mul(ldg4(P, v), 0.75f), f4_mul(ldg4(P, snext[sb]), 0.125f));
    if (si >= 0) y = f4_add(y, f4_mul(ldg4(P, sprev[si]), 0.125f));
    return y;
}

// SLAK vertex point of one vertex on its own thread
template <bool QUAD>
__device__ __forceinline__ void vp_slak_vertex(Faces<QUAD> fc, const int* __restrict__ sc,
                                               const int* __restrict__ snext, const int* __restrict__ sprev,
                                               const int* __restrict__ sflag, int boundary,
                                               const float* __restrict__ P, const float* __restrict__ FP,
                                               float* __restrict__ R, int compensated, int v, int b, int n)
{
    const int e = b + n;
    const float nn = (float)(n * n);
    float4 y;
    const auto nbr = [&](int k) { return ldg4(P, __ldg(snext + b + k)); };
    const auto fpt = [&](int k) { return ldg4(FP, fc.face(__ldg(sc + b + k))); };
    if (!compensated || n <= 4) {
        float4 acc = f4_zero();
        for_each_loaded(n, nbr, [&](int, float4 t) { acc = f4_add(acc, t); });
        float4 orig = f4_div(f4_mul(ldg4(P, v), (float)(n - 2)), (float)n);
        y = f4_add(f4_div(acc, nn), orig);
        for_each_loaded(n, fpt, [&](int, float4 t) { y = f4_add(y, f4_div(t, nn)); });
    } else {
        // compensated: the 2n neighbour and face terms are summed as an unevaluated
        // float pair (TwoSum), divided by n^2 with an exact remainder, and added to
        // p (n-2)/n evaluated the same way; one rounding at the end
        float4 sh = f4_zero(), sl = f4_zero();
        for_each_loaded(n, nbr, [&](int, float4 t) { dd_acc(sh, sl, t); });
        for_each_loaded(n, fpt, [&](int, float4 t) { dd_acc(sh, sl, t); });
        y = vp_finish(sh, sl, ldg4(P, v), n);
    }
    if (boundary) y = vp_slak_boundary(snext, sprev, sflag, P, v, b, e, y);
    st4(R, v, y);
}

// a long column (kBigCol < n <= kWarpCol) by its warp: each lane loads its (up
// to two) slots; the sums run in column order with every lane fetching slot k
// by shuffle; lane 0 stores
template <bool QUAD>
__device__ __noinline__ void vp_slak_warp(Faces<QUAD> fc, const int* __restrict__ sc,
                                          const int* __restrict__ snext, const int* __restrict__ sprev,
                                          const int* __restrict__ sflag, int boundary, const float* __restrict__ P,
                                          const float* __restrict__ FP, float* __restrict__ R, int compensated,
                                          int v, int b, int n)
{
    const int lane = threadIdx.x & 31;
    float4 a0 = f4_zero(), a1 = f4_zero(), f0 = f4_zero(), f1 = f4_zero();    // neighbour, face point
    if (lane < n) { a0 = ldg4(P, __ldg(snext + b + lane)); f0 = ldg4(FP, fc.face(__ldg(sc + b + lane))); }
    if (lane + 32 < n) { a1 = ldg4(P, __ldg(snext + b + lane + 32)); f1 = ldg4(FP, fc.face(__ldg(sc + b + lane + 32))); }
    const float nn = (float)(n * n);
    float4 y;
    if (!compensated) {
        float4 acc = f4_zero();
        for (int k = 0; k < n; ++k) acc = f4_add(acc, col4(a0, a1, k));
        y = f4_add(f4_div(acc, nn), f4_div(f4_mul(ldg4(P, v), (float)(n - 2)), (float)n));
        for (int k = 0; k < n; ++k) y = f4_add(y, f4_div(col4(f0, f1, k), nn));
    } else {
        float4 sh = f4_zero(), sl = f4_zero();
        for (int k = 0; k < n; ++k) dd_acc(sh, sl, col4(a0, a1, k));
        for (int k = 0; k < n; ++k) dd_acc(sh, sl, col4(f0, f1, k));
        y = vp_finish(sh, sl, ldg4(P, v), n);
    }
    if (lane == 0) {
        if (boundary) y = vp_slak_boundary(snext, sprev, sflag, P, v, b, b + n, y);
        st4(R, v, y);
    }
}

// SLAK vertex point: vertexSum (:634-652) then the face-point scatter of
// facepointSum[Quad] (:654-686) in ascending corner order; a boundary vertex
// becomes 3/4 p + 1/8 next + 1/8 prev (correctBoundaryS1/S2, :688-740).
// Columns longer than kBigCol go to their warp.
template <bool QUAD>
__device__ __forceinline__ void k_vp_slak_body(const unsigned bx_, Faces<QUAD> fc, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                                               const int* __restrict__ snext, const int* __restrict__ sprev,
                                               const int* __restrict__ sflag, int boundary, const float* __restrict__ P,
                                               const float* __restrict__ FP, float* __restrict__ R, int compensated)
{
    const int v = bx_ * blockDim.x + threadIdx.x;
    const bool valid = v < V;
    int b = 0, n = 0;
    if (valid) { b = sptr[v]; n = sptr[v + 1] - b; }
    const bool big = valid && n > kBigCol && n <= kWarpCol;
    if (valid && !big) vp_slak_vertex<QUAD>(fc, sc, snext, sprev, sflag, boundary, P, FP, R, compensated, v, b, n);
    unsigned m = __ballot_sync(0xffffffffu, big);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        vp_slak_warp<QUAD>(fc, sc, snext, sprev, sflag, boundary, P, FP, R, compensated,
                           __shfl_sync(0xffffffffu, v, src), __shfl_sync(0xffffffffu, b, src),
                           __shfl_sync(0xffffffffu, n, src));
    }
}
template <bool QUAD>
__global__ void k_vp_slak(Faces<QUAD> fc, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                          const int* __restrict__ snext, const int* __restrict__ sprev,
                          const int* __restrict__ sflag, int boundary, const float* __restrict__ P,
                          const float* __restrict__ FP, float* __restrict__ R, int compensated)
{
    griddep_enter();
    k_vp_slak_body<QUAD>(blockIdx.x, fc, V, sptr, sc, snext, sprev, sflag, boundary, P, FP, R, compensated);
}
template <bool QUAD>
struct k_vp_slak_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_vp_slak_body<QUAD>(bx, a...);
    }
    static constexpr auto kernel() { return &k_vp_slak<QUAD>; }
};

// LAK boundary vertex: 3/4 p + 1/8 p_other per boundary edge in edge-id order;
// y unchanged when v has no boundary slot
__device__ __forceinline__ float4 vp_lak_boundary(const int* __restrict__ sc, const int* __restrict__ snext,
                                                  const int* __restrict__ sprev, const int* __restrict__ sprevc,
                                                  const int* __restrict__ sflag, const int* __restrict__ eid,
                                                  const float* __restrict__ P, int v, int b, int e, float4 y)
{
    bool any = false;
    for (int s = b; s < e; ++s) any |= (sflag[s] & (SF_BOUT | SF_BIN)) != 0;
    if (!any) return y;
    y = f4_mul(ldg4(P, v), 0.75f);
    int lastid = -1;
    while (true) {
        int best = INT32_MAX, other = -1;
        for (int s = b; s < e; ++s) {
            int f = sflag[s];
            if (f & SF_BOUT) { int id = eid[sc[s]]; if (id > lastid && id < best) { best = id; other = snext[s]; } }
            if (f & SF_BIN) { int id = eid[sprevc[s]]; if (id > lastid && id < best) { best = id; other = sprev[s]; } }
        }
        if (best == INT32_MAX) break;
        y = f4_add(y, f4_mul(ldg4(P, other), 0.125f));
        lastid = best;
    }
    return y;
}

// LAK vertex point of one vertex on its own thread
template <bool QUAD>
__device__ __forceinline__ void vp_lak_vertex(Faces<QUAD> fc, const int* __restrict__ sc,
                                              const int* __restrict__ snext, const int* __restrict__ sprev,
                                              const int* __restrict__ sprevc, const int* __restrict__ sflag,
                                              const int* __restrict__ eid, int boundary, const float* __restrict__ P,
                                              const float* __restrict__ FP, float* __restrict__ R, int compensated,
                                              int v, int b, int n)
{
    const int e = b + n;
    const auto fpt = [&](int k) { return ldg4(FP, fc.face(__ldg(sc + b + k))); };
    float4 acc = f4_zero();
    for_each_loaded(n, fpt, [&](int, float4 t) { acc = f4_add(acc, t); });
    // the tails (distinct neighbours) in ascending id
    int perm[kBigCol];
    const bool ranked = n <= kBigCol;      // longer columns up to kWarpCol take the warp path
    if (ranked) rank_order(sprev, b, n, perm);
    const auto tail = [&](int r) { return ldg4(P, __ldg(sprev + b + perm[r])); };
    if (ranked) {
        for_each_loaded(n, tail, [&](int, float4 t) { acc = f4_add(acc, t); });
    } else {
        int last = -1;
        while (true) {
            int x = INT32_MAX;
            for (int s = b; s < e; ++s) { int u = sprev[s]; if (u > last && u < x) x = u; }
            if (x == INT32_MAX) break;
            acc = f4_add(acc, ldg4(P, x));
            last = x;
        }
    }
    float4 y;
    if (!compensated || n <= 4) {
        float4 pn = f4_mul(ldg4(P, v), __fadd_rn((float)n, -2.0f));
        y = f4_div_z(f4_add(f4_div_z(acc, (float)n), pn), (float)n);
    } else {
        // same terms, summed with TwoSum and finished with exact remainders
        float4 sh = f4_zero(), sl = f4_zero();
        for_each_loaded(n, fpt, [&](int, float4 t) { dd_acc(sh, sl, t); });
        if (ranked) {
            for_each_loaded(n, tail, [&](int, float4 t) { dd_acc(sh, sl, t); });
        } else {
            for (int l2 = -1;;) {
                int x = INT32_MAX;
                for (int s = b; s < e; ++s) { int u = sprev[s]; if (u > l2 && u < x) x = u; }
                if (x == INT32_MAX) break;
                dd_acc(sh, sl, ldg4(P, x));
                l2 = x;
            }
        }
        y = vp_finish(sh, sl, ldg4(P, v), n);
    }
    if (boundary) y = vp_lak_boundary(sc, snext, sprev, sprevc, sflag, eid, P, v, b, e, y);
    st4(R, v, y);
}

// a long column (kBigCol < n <= kWarpCol) by its warp: each lane loads its (up
// to two) slots, the tails are ranked by id across the warp, and the sums run
// in the fixed order with every lane fetching by shuffle; lane 0 stores
template <bool QUAD>
__device__ __noinline__ void vp_lak_warp(Faces<QUAD> fc, const int* __restrict__ sc,
                                         const int* __restrict__ snext, const int* __restrict__ sprev,
                                         const int* __restrict__ sprevc, const int* __restrict__ sflag,
                                         const int* __restrict__ eid, int boundary, const float* __restrict__ P,
                                         const float* __restrict__ FP, float* __restrict__ R, int compensated,
                                         int v, int b, int n)
{
    const int lane = threadIdx.x & 31;
    const bool h0 = lane < n, h1 = lane + 32 < n;
    float4 f0 = f4_zero(), f1 = f4_zero(), p0 = f4_zero(), p1 = f4_zero();    // face point, tail position
    int t0 = INT32_MAX, t1 = INT32_MAX;                                     // tail ids
    if (h0) { f0 = ldg4(FP, fc.face(__ldg(sc + b + lane))); t0 = __ldg(sprev + b + lane); p0 = ldg4(P, t0); }
    if (h1) { f1 = ldg4(FP, fc.face(__ldg(sc + b + lane + 32))); t1 = __ldg(sprev + b + lane + 32); p1 = ldg4(P, t1); }
    int r0, r1;
    rank_of(n, t0, t1, r0, r1);
    float4 y;
    if (!compensated) {
        float4 acc = f4_zero();
        for (int k = 0; k < n; ++k) acc = f4_add(acc, col4(f0, f1, k));
        for (int r = 0; r < n; ++r) {
            int src, el;
            slot_of_rank(r, h0, h1, r0, r1, src, el);
            acc = f4_add(acc, shfl4(el ? p1 : p0, src));
        }
        float4 pn = f4_mul(ldg4(P, v), __fadd_rn((float)n, -2.0f));
        y = f4_div_z(f4_add(f4_div_z(acc, (float)n), pn), (float)n);
    } else {
        float4 sh = f4_zero(), sl = f4_zero();
        for (int k = 0; k < n; ++k) dd_acc(sh, sl, col4(f0, f1, k));
        for (int r = 0; r < n; ++r) {
            int src, el;
            slot_of_rank(r, h0, h1, r0, r1, src, el);
            dd_acc(sh, sl, shfl4(el ? p1 : p0, src));
        }
        y = vp_finish(sh, sl, ldg4(P, v), n);
    }
    if (lane == 0) {
        if (boundary) y = vp_lak_boundary(sc, snext, sprev, sprevc, sflag, eid, P, v, b, b + n, y);
        st4(R, v, y);
    }
}

// LAK vertex point ((sum fp + sum p_tail) / n + p (n - 2)) / n with the face
// points in corner order and the incoming tails in ascending vertex id
// (spmv_right_mapped_f4 over M then over F, LAKCatmullClarkImpl.cu:200-221);
// boundary vertex 3/4 p + 1/8 p_other per boundary edge in edge-id order
// (prepare/calculateExternalVertexUpdate, LAKCatmullClarkKernels.cuh:464-511).
// Columns longer than kBigCol go to their warp.
template <bool QUAD>
__device__ __forceinline__ void k_vp_lak_body(const unsigned bx_, Faces<QUAD> fc, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                                              const int* __restrict__ snext, const int* __restrict__ sprev,
                                              const int* __restrict__ sprevc, const int* __restrict__ sflag,
                                              const int* __restrict__ eid, int boundary, const float* __restrict__ P,
                                              const float* __restrict__ FP, float* __restrict__ R, int compensated)
{
    const int v = bx_ * blockDim.x + threadIdx.x;
    const bool valid = v < V;
    int b = 0, n = 0;
    if (valid) { b = sptr[v]; n = sptr[v + 1] - b; }
    const bool big = valid && n > kBigCol && n <= kWarpCol;
    if (valid && !big)
        vp_lak_vertex<QUAD>(fc, sc, snext, sprev, sprevc, sflag, eid, boundary, P, FP, R, compensated, v, b, n);
    unsigned m = __ballot_sync(0xffffffffu, big);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        vp_lak_warp<QUAD>(fc, sc, snext, sprev, sprevc, sflag, eid, boundary, P, FP, R, compensated,
                          __shfl_sync(0xffffffffu, v, src), __shfl_sync(0xffffffffu, b, src),
                          __shfl_sync(0xffffffffu, n, src));
    }
}
template <bool QUAD>
__global__ void k_vp_lak(Faces<QUAD> fc, int V, const int* __restrict__ sptr, const int* __restrict__ sc,
                         const int* __restrict__ snext, const int* __restrict__ sprev,
                         const int* __restrict__ sprevc, const int* __restrict__ sflag,
                         const int* __restrict__ eid, int boundary, const float* __restrict__ P,
                         const float* __restrict__ FP, float* __restrict__ R, int compensated)
{
    griddep_enter();
    k_vp_lak_body<QUAD>(blockIdx.x, fc, V, sptr, sc, snext, sprev, sprevc, sflag, eid, boundary, P, FP, R, compensated);
}
template <bool QUAD>
struct k_vp_lak_g {
    static constexpr int kBounds = 0, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_vp_lak_body<QUAD>(bx, a...);
    }
    static constexpr auto kernel() { return &k_vp_lak<QUAD>; }
};

}  // namespace slak
