// slak_abi.cu -- host driver and C ABI (include/slak_b200.h).
//
// A plan fixes every level's size when it is created: only level 0 is read
// back (one stream sync for its boundary and edge counts); afterwards
//   N' = 4N (quads = coarse corners), F' = N, B' = 2B,
//   E = (N - B)/2 + B, V' = V + F + E
// (CatmullClarkImpl.cu:118-120, LAKCatmullClarkImpl.cu:94-96).  All scratch is
// one arena allocated at creation; an execution only launches kernels, so it
// can be captured as a CUDA graph.
#include "slak_b200.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <cstdlib>
#include <new>
#include <vector>
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <type_traits>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "general.cuh"
#include "fast.cuh"
#include "scan.cuh"
#include "crease.cuh"

using namespace slak;

namespace {

struct Level {
    int64_t F = 0, V = 0, N = 0, B = 0, E = 0;
    int64_t Fo = 0, Vo = 0, No = 0;
    bool quad = true;       // implicit 4-corner faces
    bool poly_fn = false;   // the reference's first-level (polygon) functions
    bool fast = false;      // closed-form refinement from the parent level's state
    bool export_state = false;   // general level whose state feeds a fast level
    bool make_state = false;     // fast level whose state feeds the next fast level
    // fast level whose parent's parent is a closed quad mesh (GQ, fast.cuh):
    // k_g1 sums most of the parent's vertex columns; that mesh's sizes
    bool gq = false;
    int64_t gN = 0, gV = 0, gF = 0;
    // the last level, when its parent's parent is a closed quad mesh (SG,
    // fast.cuh): it takes its parent's state in closed form from the
    // grandparent's, so the level before writes none
    bool sg = false;
    // k_g3 with bulk-copied slot records (SLAK_PLAN_BULK_RECORDS, closed parents)
    bool bulk3 = false;
    int bulk_polls = 0;
    DevStatus* st = nullptr;
    QState in_state{}, out_state{};
    SlotScratch slots{};    // fast level: slot-ordered records from k_g1 to k_g3
    const int* ptr = nullptr;
    const int* ids = nullptr;
    const float* verts = nullptr;
    int* o_ids = nullptr;
    float* o_verts = nullptr;
    int* o_ptr = nullptr;
    int* o_vals = nullptr;
    int* scan_tmp = nullptr;       // fast level with a boundary (SLAK, state): scan of C's boundary edges
    // fast level: block size of k_g1, k_g2, k_g3 (chosen by the autotuner)
    int bs[3] = {256, 256, 256};
    int tuned = 0;                 // 0 default, 1 measured now, 2 from the tuning cache
    float tune_ms[3][3] = {};      // measured ms of each kernel at block 128 / 256 / 512
    std::string tune_key;
};

constexpr int kTuneBlocks[3] = {128, 256, 512};

// Calls f with the block size as a compile-time constant.
template <class F>
void with_block(int bs, F&& f)
{
    if (bs == 128) f(std::integral_constant<int, 128>{});
    else if (bs == 512) f(std::integral_constant<int, 512>{});
    else f(std::integral_constant<int, 256>{});
}

struct Scratch {
    int *cface = nullptr, *cnt = nullptr, *sptr = nullptr, *sc = nullptr, *snext = nullptr, *sprev = nullptr,
        *sprevc = nullptr, *stw = nullptr, *sflag = nullptr, *eid = nullptr, *ecnt = nullptr, *eptr = nullptr,
        *tmp = nullptr;
    int2* H = nullptr;
    int *xslot = nullptr, *xtw = nullptr, *xt = nullptr;   // state export of a general quad level
    int *xbrank = nullptr, *xisb = nullptr;                // ... with a boundary: edges' boundary ranks
};

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct Carver {
    char* base;
    size_t off = 0;
    bool dry;
    explicit Carver(char* b) : base(b), dry(b == nullptr) {}
    template <class T>
    T* take(int64_t count)
    {
        size_t bytes = align_up(sizeof(T) * (size_t)(count > 0 ? count : 1));
        T* p = dry ? nullptr : reinterpret_cast<T*>(base + off);
        off += bytes;
        return p;
    }
};

// Launch bookkeeping: counts launches and, in debug mode (SLAK_DEBUG_SYNC=1 in
// the environment when the plan is created), synchronises after every launch
// and records which kernel failed.
thread_local std::string g_detail;

struct KernelRec {
    const char* name;
    int level;
    int64_t bytes;
};

struct Lc {
    cudaStream_t s;
    int64_t* nl;
    bool debug;
    int level;
    int err = 0;
    std::vector<cudaEvent_t>* ev = nullptr;   // timing: one event after every launch (ev[0] before the first)
    std::vector<KernelRec>* recs = nullptr;
    // independent kernels of a level on side streams (fork / join by events);
    // off while timing (per-launch events need one stream) and when debugging
    bool conc = false;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t cev[4] = {nullptr, nullptr, nullptr, nullptr};
    // side stream k waits for the work enqueued so far on s
    void fork(int k)
    {
        cudaEventRecord(cev[k], s);
        cudaStreamWaitEvent(side[k], cev[k], 0);
    }
    // s waits for side stream k
    void join(int k)
    {
        cudaEventRecord(cev[2 + k], side[k]);
        cudaStreamWaitEvent(s, cev[2 + k], 0);
    }
    void after(const char* name, int n = 1, int64_t bytes = 0)
    {
        *nl += n;
        if (ev && recs->size() + 1 < ev->size()) {
            cudaEventRecord((*ev)[recs->size() + 1], s);
            recs->push_back(KernelRec{name, level, bytes});
        }
        if (!debug || err) return;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            err = e == cudaErrorMemoryAllocation ? SLAK_ERR_OOM : SLAK_ERR_CUDA;
            g_detail = std::string(name) + " (level " + std::to_string(level) + "): " + cudaGetErrorString(e);
        }
    }
};

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return SLAK_OK;
    if (e == cudaErrorMemoryAllocation) return SLAK_ERR_OOM;
    return SLAK_ERR_CUDA;
}

}  // namespace

struct slak_plan {
    int scheme = SLAK_SCHEME_SLAK;
    int flags = 0;
    slak_mesh in{};
    slak_mesh out{};
    bool out_owned = true;
    std::vector<Level> lv;
    // device memory
    void* arena = nullptr;
    Scratch s;
    int* ping_ids[2] = {nullptr, nullptr};
    float* ping_verts[2] = {nullptr, nullptr};
    DevStatus* st = nullptr;
    DevStatus* h_st = nullptr;       // pinned
    bool h_st_owned = true;
    int64_t maxN = 0, maxV = 0, maxE = 0;
    bool any_poly = false;
    int64_t exN = 0, stN = 0, stV = 0, slN = 0, mid_ids = 0, mid_verts = 0;
    int64_t exE = 0, stE = 0;        // edges of the exported / state levels (boundary ranks)
    bool bnd_fast = false;           // some fast level has a parent with a boundary
    int* bnd_tmp = nullptr;          // scan tiles for C's boundary ranks
    bool arena_owned = true;
    QState qs[2]{};
    SlotScratch slots{};
    // graph
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t gstream = nullptr;
    int64_t launches = 0;
    int executed = 0;
    bool debug = false;
    int vhist[17] = {};              // level 0's valence histogram (probe)
    // per-launch timing (SLAK_PLAN_TIMING)
    std::vector<cudaEvent_t> ev;
    std::vector<KernelRec> recs;
    // side streams and fork / join events for a level's independent kernels
    // (a standalone plan owns them; a batch lends its stream slot's)
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t cev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool side_owned = true;
    // creases (slak_plan_create_creased): a snapshot of the pairs and
    // sharpness, the crease list of each level that has a live crease
    // (ncrease << level entries), the base vertices' crease edges (CSR) and
    // the edge points made on live creases
    int64_t ncrease = 0;
    int crease_levels = 0;           // ceil(largest sharpness), at most the level count
    int* c_pairs = nullptr;
    float* c_sharp = nullptr;
    float* c_vcs = nullptr;          // corner sharpness of the base vertices (with corners)
    std::vector<float> h_vcs;        // its host copy, uploaded at creation
    int* c_mark = nullptr;           // level-0 corner -> live crease entry + 1
    unsigned char* c_bnd0 = nullptr; // base vertices on the boundary (open meshes)
    int *c_vcnt = nullptr, *c_vptr = nullptr, *c_inc = nullptr;
    std::vector<int*> c_cc;
    std::vector<float*> c_cs;
    std::vector<int*> c_ep;          // per level t < crease_levels - 1: edge point of entry j, or -1
};

namespace {

// scratch for one level of at most N corners, V vertices, E edges
void carve_scratch(Carver& cv, Scratch& s, int64_t N, int64_t V, int64_t E, bool poly)
{
    s.cface = poly ? cv.take<int>(N) : nullptr;
    s.cnt = cv.take<int>(V);
    s.sptr = cv.take<int>(V + 1);
    s.sc = cv.take<int>(N);
    s.snext = cv.take<int>(N);
    s.sprev = cv.take<int>(N);
    s.sprevc = cv.take<int>(N);
    s.stw = cv.take<int>(N);
    s.sflag = cv.take<int>(N);
    s.eid = cv.take<int>(N);
    s.ecnt = cv.take<int>(V);
    s.eptr = cv.take<int>(V + 1);
    s.tmp = cv.take<int>(scan_tiles(N > V ? N : V) + 2);
    s.H = cv.take<int2>(E);
}

// E > 0: the exported level has a boundary, so its edges' boundary ranks go too
void carve_export(Carver& cv, Scratch& s, int64_t N, int64_t E)
{
    s.xslot = cv.take<int>(N);
    s.xtw = cv.take<int>(N);
    s.xt = cv.take<int>(N);
    s.xbrank = E ? cv.take<int>(E + 1) : nullptr;
    s.xisb = E ? cv.take<int>(E) : nullptr;
}

void carve_state(Carver& cv, QState& q, int64_t N, int64_t V, int64_t E)
{
    q.sptr = cv.take<int>(V + 1);
    q.slot = cv.take<int>(N);
    q.tw = cv.take<int>(N);
    q.t = cv.take<int>(N);
    q.brank = E ? cv.take<int>(E + 1) : nullptr;
}

// Topology of a level up to the edge-offset scan (needs no output buffers).
void launch_topology_a(const Level& L, int li, int scheme, Scratch& s, DevStatus* st, Lc& lc)
{
    const int F = (int)L.F, V = (int)L.V, N = (int)L.N;
    cudaStream_t str = lc.s;
    zero_async(s.cnt, sizeof(int) * (size_t)V, str);
    if (!L.quad) {
        zero_async(s.cface, sizeof(int) * (size_t)N, str);
        launch_g<k_face_map_valence_g>(grid_for(F), kBlock, str, L.ptr, L.ids, F, N, V, s.cface, s.cnt, st);
        lc.after("k_face_map_valence");
    } else {
        launch_g<k_valence_g>(grid_for(N), kBlock, str, L.ids, N, V, s.cnt, st);
        lc.after("k_valence");
    }
    int64_t dummy = 0;
    scan_exclusive(s.cnt, s.sptr, V, s.tmp, str, &dummy);
    lc.after("scan(valence)", 3);
    // the unsorted columns live in sflag until k_edges writes the flags
    launch_g<k_bucket_g>(grid_for(N), kBlock, str, L.ids, N, V, s.sptr, s.cnt, s.sflag);
    lc.after("k_bucket");
    int* bcount = &st->bcount[li];
    // a general quad level feeding the fast path exports corner -> slot / twin
    int* xslot = L.export_state ? s.xslot : nullptr;
    int* xtw = L.export_state ? s.xtw : nullptr;
    if (L.quad) {
        Faces<true> fc{L.ptr, s.cface};
        launch_g<k_vsort_g<true>>(grid_for(N), kBlock, str, fc, L.ids, N, V, s.sptr, s.sflag, s.sc, s.snext, s.sprev,
                                  s.sprevc, xslot);
    } else {
        Faces<false> fc{L.ptr, s.cface};
        launch_g<k_vsort_g<false>>(grid_for(N), kBlock, str, fc, L.ids, N, V, s.sptr, s.sflag, s.sc, s.snext, s.sprev,
                                   s.sprevc, xslot);
    }
    lc.after("k_vsort");
    if (scheme == SLAK_SCHEME_LAK)
        launch_g<k_edges_g<true>>(grid_for(V), kBlock, str, V, s.sptr, s.sc, s.snext, s.sprev, s.sprevc, s.stw,
                                  s.sflag, s.ecnt, bcount, xtw, st);
    else
        launch_g<k_edges_g<false>>(grid_for(V), kBlock, str, V, s.sptr, s.sc, s.snext, s.sprev, s.sprevc, s.stw,
                                   s.sflag, s.ecnt, bcount, xtw, st);
    lc.after("k_edges");
    scan_exclusive(s.ecnt, s.eptr, V, s.tmp, str, &dummy);
    lc.after("scan(edges)", 3);
}


// The rest of a general level, after launch_topology_a: edge ids (with the
// check of the level's counts), refined quads (and, for a SLAK level feeding
// the fast path, t), face, edge and vertex points.
template <bool QUAD>
void launch_rest(const Level& L, int li, int scheme, bool compensated, Scratch& s, DevStatus* st, Lc& lc)
{
    const int F = (int)L.F, V = (int)L.V, N = (int)L.N, E = (int)L.E;
    const bool lak = scheme == SLAK_SCHEME_LAK;
    cudaStream_t str = lc.s;
    Faces<QUAD> fc{L.ptr, s.cface};
    const int* bcount = &st->bcount[li];
    if (lak)
        launch_g<k_eids_lak_g>(grid_for(V), kBlock, str, V, s.sptr, s.sc, s.snext, s.sprev, s.sprevc, s.eptr, E, s.eid,
                               s.H, st, bcount, (int)L.B, li);
    else
        launch_g<k_eids_slak_g>(grid_for(V), kBlock, str, V, s.sptr, s.sc, s.stw, s.sflag, s.eptr, E, s.eid, s.H, st,
                                bcount, (int)L.B, li);
    lc.after("k_eids");
    // the refined quads (side stream 0) need only the edge ids; the positions
    // (k_fp, then k_ep on side stream 1 beside k_vp) need the face points
    if (lc.conc) lc.fork(0);
    cudaStream_t s_ref = lc.conc ? lc.side[0] : str;
    if (lak)
        launch_g<k_refine_g<QUAD, true>>(grid_for(N), kBlock, s_ref, fc, L.ids, s.eid, N, V, F,
                                         reinterpret_cast<int4*>(L.o_ids), L.o_ptr,
                                         reinterpret_cast<int4*>(L.o_vals), nullptr, nullptr,
                                         nullptr);
    else
        launch_g<k_refine_g<QUAD, false>>(grid_for(N), kBlock, s_ref, fc, L.ids, s.eid, N, V, F,
                                          reinterpret_cast<int4*>(L.o_ids), nullptr, nullptr,
                                          s.xslot, s.xtw, L.export_state ? s.xt : nullptr);
    lc.after("k_refine");
    float* R = L.o_verts;
    float* FPo = R + 4 * (size_t)V;
    float* EPo = R + 4 * ((size_t)V + (size_t)F);
    if (!lak && QUAD && !L.poly_fn)
        launch_g<k_fp_slak_quad_g>(grid_for(F), kBlock, str, reinterpret_cast<const int4*>(L.ids), L.verts, F, FPo);
    else if (lak)
        launch_g<k_fp_seq_g<QUAD, true>>(grid_for(F), kBlock, str, L.ptr, L.ids, L.verts, F, FPo);
    else
        launch_g<k_fp_seq_g<QUAD, false>>(grid_for(F), kBlock, str, L.ptr, L.ids, L.verts, F, FPo);
    lc.after("k_fp");
    if (lc.conc) lc.fork(1);
    cudaStream_t s_ep = lc.conc ? lc.side[1] : str;
    if (lak)
        launch_g<k_ep_g<QUAD, true>>(grid_for(E), kBlock, s_ep, fc, L.ids, s.H, E, L.verts, FPo, EPo);
    else
        launch_g<k_ep_g<QUAD, false>>(grid_for(E), kBlock, s_ep, fc, L.ids, s.H, E, L.verts, FPo, EPo);
    lc.after("k_ep");
    const int bnd = L.B > 0;
    if (lak)
        launch_g<k_vp_lak_g<QUAD>>(grid_for(V), kBlock, str, fc, V, s.sptr, s.sc, s.snext, s.sprev, s.sprevc, s.sflag,
                                   s.eid, bnd, L.verts, FPo, R, compensated);
    else
        launch_g<k_vp_slak_g<QUAD>>(grid_for(V), kBlock, str, fc, V, s.sptr, s.sc, s.snext, s.sprev, s.sflag, bnd,
                                    L.verts, FPo, R, compensated);
    lc.after("k_vp");
    if (lc.conc) { lc.join(0); lc.join(1); }
}

// The tensor map of a level's refined quads for k_g1's tensor store: `rows`
// rows of 16 int32 (thread x's four quads at out + 16 x), boxes of `bs` rows,
// 64-byte swizzle (the layout k_g1 stages them in).  A null `out` (a launch
// sequence recorded before any memory exists) leaves the map zeroed.
bool quad_store_map(CUtensorMap& m, int* out, int64_t rows, int bs)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    if (out == nullptr) return true;
    if (enc == nullptr || rows < 1) {
        g_detail = "cuTensorMapEncodeTiled unavailable";
        return false;
    }
    const cuuint64_t dims[2] = {16, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {64};
    const cuuint32_t box[2] = {16, (cuuint32_t)bs};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_INT32, 2, out, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) g_detail = "cuTensorMapEncodeTiled: error " + std::to_string((int)r);
    return r == CUDA_SUCCESS;
}

// One fast level: C = L (refined from its parent level Pl, whose state is
// L.in_state).  BND: Pl has a boundary (quad faces only).
template <bool LAK, bool STATE, bool PQ, bool BND, bool GQ = false, bool SG = false>
void launch_fast_t(const Level& Pl, const Level& L, Faces<PQ> pf, bool comp, Lc& lc)
{
    FastDims d{(int)Pl.N, (int)Pl.V, (int)Pl.F, (int)Pl.E, (int)L.V, (int)L.N, (int)Pl.B};
    if (GQ || SG) { d.N2 = (int)L.gN; d.V2 = (int)L.gV; d.F2 = (int)L.gF; }
    const int nv3 = GQ ? (int)L.gV : (int)Pl.V;      // k_g3's vertices
    cudaStream_t str = lc.s;
    // compulsory bytes of each kernel: the level's corner ids and positions it
    // must read once, and the refined ids / positions it alone writes
    const int64_t g1b = 4 * L.N + 16 * L.V + 16 * L.N + 16 * L.F + 16 * Pl.F + (LAK ? 0 : 16 * L.F);
    const int64_t g2b = 16 * Pl.E + (LAK ? 16 * 2 * L.F : 0);
    // LAK's last level: the refined ptr / vals come from k_g1 too
    int* optr = LAK && !STATE ? L.o_ptr : nullptr;
    int4* ovals = LAK && !STATE ? reinterpret_cast<int4*>(L.o_vals) : nullptr;
    bool mapped = true;
    with_block(L.bs[0], [&](auto b) {
        constexpr int BS = decltype(b)::value;
        CUtensorMap otm;
        std::memset(&otm, 0, sizeof otm);
        if constexpr (!STATE && kTmaQuadStore && BS <= 256) mapped = quad_store_map(otm, L.o_ids, Pl.N, BS);
        if (!mapped) return;            // nothing of the level is launched
        launch_g<k_g1_g<LAK, STATE, PQ, BS, BND, GQ, SG>>(grid_for(L.F, BS), BS, str, d, pf, L.ids, L.verts, L.in_state,
                                                          L.out_state, reinterpret_cast<int4*>(L.o_ids), otm, L.o_verts,
                                                          L.slots, optr, ovals);
    });
    if (!mapped) {
        if (!lc.err) lc.err = SLAK_ERR_CUDA;
        return;
    }
    // GQ: k_g1 also writes the vertex points of P's vertices past V2 (and SLAK their slots' edge points)
    const int64_t gqb = GQ ? 16 * (Pl.V - L.gV) + (LAK ? 0 : 16 * (L.F - L.gN)) : 0;
    lc.after("k_g1", 1, (PQ ? g1b + g2b : g1b) + (optr ? 4 * (L.N + 1) + 16 * L.N : 0) + gqb);
    if (!PQ) {      // with quad faces, k_g1 also does k_gf's and k_g2's work
        // k_gf, k_g2 and k_g3 read only k_g1's records and the level's inputs and
        // write disjoint outputs: with side streams they run side by side
        if (lc.conc) { lc.fork(0); lc.fork(1); }
        launch_g<k_gf_g<LAK, STATE>>(grid_for(Pl.F), kBlock, lc.conc ? lc.side[0] : str, d, Pl.ptr, L.ids, L.verts, L.out_state, L.o_verts, comp ? 1 : 0);
        lc.after("k_gf");
        with_block(L.bs[1], [&](auto b) {
            constexpr int BS = decltype(b)::value;
            launch_g<k_g2_g<LAK, STATE, PQ, BS, BND>>(grid_for(L.F, BS), BS, lc.conc ? lc.side[1] : str, d, pf, L.ids, L.verts, L.in_state, L.out_state, L.o_verts);
        });
        lc.after("k_g2", 1, g2b);
    }
    if (!BND && !SG && L.bulk3) {
        launch_g<k_g3_bulk_g<LAK, STATE>>(grid_for(nv3 + 1, kBulkBlock), kBulkBlock, str, d, L.verts, L.in_state, L.out_state, L.slots, L.o_verts, comp ? 1 : 0, nv3, L.st, L.bulk_polls);
    } else {
        with_block(L.bs[2], [&](auto b) {
            constexpr int BS = decltype(b)::value;
            launch_g<k_g3_g<LAK, STATE, BS, BND, SG>>(grid_for(nv3 + 1, BS), BS, str, d, L.verts, L.in_state, L.out_state, L.slots, L.o_verts, comp ? 1 : 0, nv3);
        });
    }
    // compulsory bytes: the vertex points of its vertices, SLAK the edge points of their slots
    const int64_t ns3 = GQ ? L.gN : L.F;
    lc.after("k_g3", 1, 16 * (int64_t)nv3 + (LAK ? 0 : 16 * ns3));
    if (BND && STATE && !LAK) {    // C's edges 0..N1-1 (P's slots): boundary ranks by a scan
        int64_t nl = 0;
        scan_exclusive(L.slots.bscan, L.out_state.brank, Pl.N, L.scan_tmp, str, &nl);
        lc.after("scan(boundary)", (int)nl);
    }
    if (!PQ && lc.conc) { lc.join(0); lc.join(1); }
}

template <bool PQ, bool BND, bool GQ = false>
void launch_fast_p(const Level& Pl, const Level& L, Faces<PQ> pf, bool lak, bool comp, Lc& lc)
{
    if constexpr (PQ && !BND) {
        if (L.sg) {             // the last level: no state to write
            if (lak) launch_fast_t<true, false, PQ, BND, GQ, true>(Pl, L, pf, comp, lc);
            else launch_fast_t<false, false, PQ, BND, GQ, true>(Pl, L, pf, comp, lc);
            return;
        }
    }
    if (lak) {
        if (L.make_state) launch_fast_t<true, true, PQ, BND, GQ>(Pl, L, pf, comp, lc);
        else launch_fast_t<true, false, PQ, BND, GQ>(Pl, L, pf, comp, lc);
    } else {
        if (L.make_state) launch_fast_t<false, true, PQ, BND, GQ>(Pl, L, pf, comp, lc);
        else launch_fast_t<false, false, PQ, BND, GQ>(Pl, L, pf, comp, lc);
    }
}

// `cface` is the parent's corner -> face map when the parent is a polygon level
void launch_fast(const Level& Pl, const Level& L, const int* cface, int scheme, bool comp, Lc& lc)
{
    const bool lak = scheme == SLAK_SCHEME_LAK;
    if (L.gq) launch_fast_p<true, false, true>(Pl, L, Faces<true>{nullptr, nullptr}, lak, comp, lc);
    else if (L.sg) launch_fast_p<true, false>(Pl, L, Faces<true>{nullptr, nullptr}, lak, comp, lc);
    else if (Pl.quad && Pl.B > 0) launch_fast_p<true, true>(Pl, L, Faces<true>{nullptr, nullptr}, lak, comp, lc);
    else if (Pl.quad) launch_fast_p<true, false>(Pl, L, Faces<true>{nullptr, nullptr}, lak, comp, lc);
    else if (Pl.B > 0) launch_fast_p<false, true>(Pl, L, Faces<false>{Pl.ptr, cface}, lak, comp, lc);
    else launch_fast_p<false, false>(Pl, L, Faces<false>{Pl.ptr, cface}, lak, comp, lc);
}

// The crease pass of level li (after the level's own kernels): level 0 first
// resolves the crease pairs on its vertex columns and lists each base
// vertex's crease edges.
template <bool QUAD>
void launch_creases_t(slak_plan* p, int li, Faces<QUAD> fc, Lc& lc)
{
    const Level& L = p->lv[li];
    const Level& L0 = p->lv[0];
    cudaStream_t str = lc.s;
    const int64_t m = p->ncrease, n = m << li;
    const int V0 = (int)L0.V;
    if (li == 0) {
        cudaMemsetAsync(p->c_mark, 0, sizeof(int) * (size_t)L0.N, str);
        launch_k(k_crease_resolve, grid_for(m), kBlock, str, p->c_pairs, p->c_sharp, (int)m, V0, p->s.sptr, p->s.sc,
                                                          p->s.snext, p->c_mark, p->c_cc[0], p->c_cs[0], p->st);
        lc.after("k_crease_resolve");
        launch_k(k_crease_vinc<false>, grid_for(V0), kBlock, str, V0, p->s.sptr, p->s.sc, p->s.sprevc, p->s.sflag,
                                                               SF_BOUT | SF_BIN, p->c_mark, p->c_vcnt, p->c_bnd0,
                                                               nullptr, nullptr);
        lc.after("k_crease_vinc");
        int64_t ns = 0;
        scan_exclusive(p->c_vcnt, p->c_vptr, V0, p->s.tmp, str, &ns);
        lc.after("scan(crease vertices)", (int)ns);
        launch_k(k_crease_vinc<true>, grid_for(V0), kBlock, str, V0, p->s.sptr, p->s.sc, p->s.sprevc, p->s.sflag,
                                                              SF_BOUT | SF_BIN, p->c_mark, nullptr, nullptr,
                                                              p->c_vptr, p->c_inc);
        lc.after("k_crease_vinc");
    }
    const bool more = li + 1 < p->crease_levels;
    launch_k(k_crease_edges<QUAD>, grid_for(n), kBlock, str, fc, L.ids, L.o_ids, L.verts, L.o_verts, p->c_cc[li],
                                                          p->c_cs[li], (int)n, more ? p->c_cc[li + 1] : nullptr,
                                                          more ? p->c_cs[li + 1] : nullptr,
                                                          more ? p->c_ep[li] : nullptr);
    lc.after("k_crease_edges");
    CreaseEps eps{};
    for (int t = 0; t < li; ++t) eps.epid[t] = p->c_ep[t];
    const int64_t nv = (int64_t)V0 + m * ((1ll << li) - 1);
    launch_k(k_crease_verts<QUAD>, grid_for(nv), kBlock, str, fc, li, V0, m, L.ids, p->c_cc[li], p->c_cs[li],
                                                           p->c_vcnt, p->c_vptr, p->c_inc, p->c_bnd0, eps, p->c_vcs, L.verts,
                                                           L.o_verts);
    lc.after("k_crease_verts");
}

void launch_creases(slak_plan* p, int li, Lc& lc)
{
    const Level& L = p->lv[li];
    if (L.quad) launch_creases_t<true>(p, li, Faces<true>{nullptr, nullptr}, lc);
    else launch_creases_t<false>(p, li, Faces<false>{L.ptr, p->s.cface}, lc);
}

int enqueue_all(slak_plan* p, cudaStream_t str)
{
    int64_t nl = 0;
    Lc lc{str, &nl, p->debug, 0};
    if (p->side[0] && !(p->flags & SLAK_PLAN_TIMING) && !p->debug && !g_record) {
        lc.conc = true;
        for (int k = 0; k < 2; ++k) lc.side[k] = p->side[k];
        for (int k = 0; k < 4; ++k) lc.cev[k] = p->cev[k];
    }
    if (p->flags & SLAK_PLAN_TIMING) {
        if (p->ev.empty()) {
            p->ev.resize(512);
            for (auto& e : p->ev) cudaEventCreate(&e);
        }
        p->recs.clear();
        lc.ev = &p->ev;
        lc.recs = &p->recs;
        cudaEventRecord(p->ev[0], str);
    }
    zero_async(p->st, sizeof(DevStatus), str);
    const bool comp = (p->flags & SLAK_PLAN_COMPENSATED) != 0;
    for (size_t li = 0; li < p->lv.size(); ++li) {
        const Level& L = p->lv[li];
        lc.level = (int)li;
        if (L.fast) {
            launch_fast(p->lv[li - 1], L, p->s.cface, p->scheme, comp, lc);
            if (lc.err) break;          // a level that could not be launched stops the plan
            if ((int)li < p->crease_levels) launch_creases(p, (int)li, lc);
            continue;
        }
        launch_topology_a(L, (int)li, p->scheme, p->s, p->st, lc);
        // slot / twin of an exported SLAK state come from k_vsort / k_edges, t from k_refine
        if (L.quad) launch_rest<true>(L, (int)li, p->scheme, comp, p->s, p->st, lc);
        else launch_rest<false>(L, (int)li, p->scheme, comp, p->s, p->st, lc);
        if (L.export_state && L.B > 0) {     // the edges' boundary ranks
            launch_g<k_export_bflag_g>(grid_for(L.E), kBlock, str, (int)L.E, p->s.H, p->s.xisb);
            lc.after("k_export_bflag");
            int64_t n3 = 0;
            scan_exclusive(p->s.xisb, p->s.xbrank, L.E, p->s.tmp, str, &n3);
            lc.after("scan(boundary)", (int)n3);
        }
        if ((int)li < p->crease_levels) launch_creases(p, (int)li, lc);
    }
    p->launches = nl;
    if (lc.err) return lc.err;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) g_detail = std::string("launch: ") + cudaGetErrorString(e);
    return cuda_status(e);
}

void free_plan_memory(slak_plan* p)
{
    for (auto& e : p->ev) cudaEventDestroy(e);
    p->ev.clear();
    for (auto& e : p->cev) {
        if (e && p->side_owned) cudaEventDestroy(e);
        e = nullptr;
    }
    for (auto& st : p->side) {
        if (st && p->side_owned) cudaStreamDestroy(st);
        st = nullptr;
    }
    if (p->gexec) cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
    if (p->arena && p->arena_owned) cudaFree(p->arena);
    p->arena = nullptr;
    if (p->h_st && p->h_st_owned) cudaFreeHost(p->h_st);
    p->h_st = nullptr;
    if (p->out_owned) {
        if (p->out.ids) cudaFree(p->out.ids);
        if (p->out.verts) cudaFree(p->out.verts);
        if (p->out.ptr) cudaFree(p->out.ptr);
        if (p->out.vals) cudaFree(p->out.vals);
    }
    std::memset(&p->out, 0, sizeof(p->out));
}

// Reads level 0's topology once to size the whole plan.
size_t probe_bytes(const Level& L0)
{
    Carver dry(nullptr);
    Scratch s;
    carve_scratch(dry, s, L0.N, L0.V, 1, !L0.quad);
    dry.take<DevStatus>(1);
    return dry.off;
}

// `given` (at least probe_bytes) is used when non-null; else the probe allocates.
int probe_level0(slak_plan* p, Level& L0, cudaStream_t str, void* given = nullptr)
{
    Scratch s;
    void* mem = given;
    cudaError_t e = cudaSuccess;
    if (!given) {
        e = cudaMalloc(&mem, probe_bytes(L0));
        if (e != cudaSuccess) return cuda_status(e);
    }
    Carver cv((char*)mem);
    carve_scratch(cv, s, L0.N, L0.V, 1, !L0.quad);
    DevStatus* st = cv.take<DevStatus>(1);
    int64_t nl = 0;
    Lc lc{str, &nl, p->debug, 0};
    cudaMemsetAsync(st, 0, sizeof(DevStatus), str);
    launch_topology_a(L0, 0, p->scheme, s, st, lc);
    launch_g<k_valence_hist_g>(grid_for(L0.V), kBlock, str, (int)L0.V, s.sptr, st->vhist);
    cudaMemcpyAsync(p->h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
    cudaMemcpyAsync(&p->h_st->nedges, s.eptr + L0.V, sizeof(int), cudaMemcpyDeviceToHost, str);
    e = cudaStreamSynchronize(str);
    if (!given) cudaFree(mem);
    if (lc.err) return lc.err;
    if (e != cudaSuccess) { g_detail = std::string("level-0 probe: ") + cudaGetErrorString(e); return cuda_status(e); }
    if (p->h_st->err) { g_detail = "level-0 probe: device detail " + std::to_string(p->h_st->detail); return p->h_st->err; }
    L0.B = p->h_st->bcount[0];
    L0.E = p->h_st->nedges;
    std::memcpy(p->vhist, p->h_st->vhist, sizeof(p->vhist));
    if (L0.E != (L0.N - L0.B) / 2 + L0.B) return SLAK_ERR_BAD_MESH;   // not a 2-manifold
    return SLAK_OK;
}


int validate_mesh(const slak_mesh* cm, int scheme)
{
    if (scheme != SLAK_SCHEME_LAK && scheme != SLAK_SCHEME_SLAK) return SLAK_ERR_INVALID_ARG;
    if (cm->nfaces < 0 || cm->nverts < 0 || cm->nnz < 0) return SLAK_ERR_INVALID_ARG;
    if (cm->type < SLAK_MESH_TRI || cm->type > SLAK_MESH_POLY) return SLAK_ERR_INVALID_ARG;
    const bool quad_in = cm->type == SLAK_MESH_QUAD;
    if (cm->nfaces > 0 && (!cm->ids || !cm->verts)) return SLAK_ERR_INVALID_ARG;
    if (!quad_in && cm->nfaces > 0 && !cm->ptr) return SLAK_ERR_INVALID_ARG;
    if (quad_in && cm->nnz != 4 * cm->nfaces) return SLAK_ERR_BAD_MESH;
    if (cm->nnz >= (1ll << 31) || cm->nverts >= (1ll << 31)) return SLAK_ERR_UNSUPPORTED;
    return SLAK_OK;
}

// Level count and level-0 description (subdivideIteratively's rule: a
// non-QUAD input always runs one polygon level).
int plan_init(slak_plan* p, const slak_mesh* cm, int target_level, int scheme, int flags)
{
    p->scheme = scheme;
    p->flags = flags;
    const char* dbg = std::getenv("SLAK_DEBUG_SYNC");
    p->debug = dbg && dbg[0] == '1';
    p->in = *cm;
    const bool quad_in = cm->type == SLAK_MESH_QUAD;
    int nlev = quad_in ? 0 : 1;
    if (target_level > nlev) nlev = target_level;
    if (cm->nfaces == 0) nlev = 0;
    p->lv.assign(nlev, Level{});
    if (nlev) {
        Level& L0 = p->lv[0];
        L0.F = cm->nfaces; L0.V = cm->nverts; L0.N = cm->nnz;
        L0.quad = quad_in;
        L0.poly_fn = !quad_in;
        L0.ptr = cm->ptr; L0.ids = cm->ids; L0.verts = cm->verts;
    }
    return nlev;
}

// All level sizes from level 0's boundary and edge counts; which levels run
// closed-form; the maxima the arena is carved for.
int plan_levels(slak_plan* p)
{
    const int nlev = (int)p->lv.size();
    const bool force_general = (p->flags & SLAK_PLAN_GENERAL) != 0;
    for (int i = 0; i < nlev; ++i) {
        Level& L = p->lv[i];
        if (i > 0) {
            const Level& P = p->lv[i - 1];
            L.F = P.Fo; L.V = P.Vo; L.N = P.No; L.B = 2 * P.B;
            L.E = (L.N - L.B) / 2 + L.B;
            L.quad = true; L.poly_fn = false;
            L.fast = !force_general;     // any parent: closed or open, quad or polygon faces
        }
        L.Fo = L.N; L.No = 4 * L.N; L.Vo = L.V + L.F + L.E;
        if (L.No >= (1ll << 31) || L.Vo >= (1ll << 31)) return SLAK_ERR_UNSUPPORTED;
        // the parent is refine(PP) with PP a closed quad mesh: GQ on request; SG
        // on the last level (SLAK_NO_SG builds: off, for comparisons)
        const bool gq_parent = L.fast && i >= 2 && p->lv[i - 2].quad && p->lv[i - 2].B == 0;
        if (gq_parent && (p->flags & SLAK_PLAN_GQ)) L.gq = true;
#ifndef SLAK_NO_SG
        if (gq_parent && i == nlev - 1 && p->lv[i - 1].fast) L.sg = true;
#endif
        if (L.gq || L.sg) { L.gN = p->lv[i - 2].N; L.gV = p->lv[i - 2].V; L.gF = p->lv[i - 2].F; }
        if (!L.fast) {
            if (L.N > p->maxN) p->maxN = L.N;
            if (L.V > p->maxV) p->maxV = L.V;
            if (L.E > p->maxE) p->maxE = L.E;
            if (!L.quad) p->any_poly = true;
        }
    }
    for (int i = 0; i < nlev; ++i) {
        Level& L = p->lv[i];
        if (L.fast && p->lv[i - 1].B == 0 && (p->flags & SLAK_PLAN_BULK_RECORDS)) {
            L.bulk3 = true;
            const char* e = std::getenv("SLAK_BULK_WAIT_POLLS");      // tests: 0 forces the timeout path
            L.bulk_polls = e ? std::atoi(e) : (1 << 20);
        }
        if (L.fast && p->lv[i - 1].N > p->slN) p->slN = p->lv[i - 1].N;
        if (L.fast && p->lv[i - 1].B > 0) p->bnd_fast = true;
        if (i + 1 < nlev && p->lv[i + 1].fast && !L.fast) {
            L.export_state = true;
            if (L.N > p->exN) p->exN = L.N;
            if (L.B > 0 && L.E > p->exE) p->exE = L.E;
        }
        if (L.fast && i + 1 < nlev && p->lv[i + 1].fast && !p->lv[i + 1].sg) {
            L.make_state = true;
            if (L.N > p->stN) p->stN = L.N;
            if (L.V > p->stV) p->stV = L.V;
            if (L.B > 0 && L.E > p->stE) p->stE = L.E;
        }
    }
    for (int i = 0; i + 1 < nlev; ++i) {
        if (p->lv[i].No > p->mid_ids) p->mid_ids = p->lv[i].No;
        if (p->lv[i].Vo > p->mid_verts) p->mid_verts = p->lv[i].Vo;
    }
    return SLAK_OK;
}

// Arena layout: general scratch, state export, fast-path states, slot records,
// ping-pong intermediate meshes, status.  A dry Carver (null base) measures it.
void plan_carve(slak_plan* p, Carver& cv)
{
    const int nlev = (int)p->lv.size();
    carve_scratch(cv, p->s, p->maxN, p->maxV, p->maxE, p->any_poly);
    if (p->exN) carve_export(cv, p->s, p->exN, p->exE);
    if (p->stN) {
        carve_state(cv, p->qs[0], p->stN, p->stV, p->stE);
        carve_state(cv, p->qs[1], p->stN, p->stV, p->stE);
    }
    if (p->slN) {
        p->slots.Z = cv.take<float4>(2 * p->slN);
        p->slots.T = p->slots.rot = cv.take<int>(p->slN + 8);     // bulk copies read whole 16-byte groups
        if (p->bnd_fast) {
            p->slots.bflag = cv.take<int>(p->slN);
            p->slots.bid = cv.take<int>(p->slN);
            p->slots.bscan = cv.take<int>(p->slN);
            p->bnd_tmp = cv.take<int>(scan_tiles(p->slN) + 2);
        }
    }
    for (int k = 0; k < 2; ++k) {
        p->ping_ids[k] = nlev > 1 ? cv.take<int>(p->mid_ids) : nullptr;
        p->ping_verts[k] = nlev > 1 ? cv.take<float>(4 * p->mid_verts) : nullptr;
    }
    p->st = cv.take<DevStatus>(1);
    if (p->crease_levels > 0) {
        const int64_t m = p->ncrease;
        p->c_pairs = cv.take<int>(2 * m);
        p->c_sharp = cv.take<float>(m);
        p->c_mark = cv.take<int>(p->lv[0].N);
        p->c_bnd0 = p->lv[0].B > 0 ? cv.take<unsigned char>(p->lv[0].V) : nullptr;
        p->c_vcs = p->h_vcs.empty() ? nullptr : cv.take<float>(p->lv[0].V);
        p->c_vcnt = cv.take<int>(p->lv[0].V);
        p->c_vptr = cv.take<int>(p->lv[0].V + 1);
        p->c_inc = cv.take<int>(2 * m);
        p->c_cc.assign(p->crease_levels, nullptr);
        p->c_cs.assign(p->crease_levels, nullptr);
        p->c_ep.assign(p->crease_levels, nullptr);
        for (int l = 0; l < p->crease_levels; ++l) {
            p->c_cc[l] = cv.take<int>(m << l);
            p->c_cs[l] = cv.take<float>(m << l);
            if (l + 1 < p->crease_levels) p->c_ep[l] = cv.take<int>(m << l);
        }
    }
}

// Counts and flags of the refined mesh (arrays not set).
slak_mesh plan_output_shape(const slak_plan* p)
{
    slak_mesh o{};
    const Level& LL = p->lv.back();
    o.type = SLAK_MESH_QUAD;
    o.nfaces = LL.Fo; o.nnz = LL.No; o.nverts = LL.Vo;
    if (p->scheme == SLAK_SCHEME_LAK) { o.max_face_order = 4; o.is_reduced = 0; }
    else { o.max_face_order = 0; o.is_reduced = 1; }
    return o;
}

// Level inputs/outputs and fast-path state wiring, once p->out holds the final arrays.
void plan_wire(slak_plan* p)
{
    const int nlev = (int)p->lv.size();
    for (int i = 0; i < nlev; ++i) {
        Level& L = p->lv[i];
        if (i > 0) {
            L.ids = p->lv[i - 1].o_ids;
            L.verts = p->lv[i - 1].o_verts;
            L.ptr = nullptr;
        }
        if (i == nlev - 1) {
            L.o_ids = p->out.ids; L.o_verts = p->out.verts;
            L.o_ptr = p->out.ptr; L.o_vals = p->out.vals;
        } else {
            L.o_ids = p->ping_ids[i & 1]; L.o_verts = p->ping_verts[i & 1];
        }
    }
    int qi = 0;
    for (int i = 1; i < nlev; ++i) {
        Level& L = p->lv[i];
        if (!L.fast) continue;
        const Level& P = p->lv[i - 1];
        if (L.sg) L.in_state = P.in_state;      // the grandparent's state: the parent's own input
        else if (P.export_state) L.in_state = QState{p->s.sptr, p->s.xslot, p->s.xtw, p->s.xt, p->s.xbrank};
        else L.in_state = P.out_state;
        if (L.make_state) { L.out_state = p->qs[qi]; qi ^= 1; }
        L.slots = p->slots;
        L.scan_tmp = p->bnd_tmp;
        L.st = p->st;
    }
}

// One-shot calls (slak_subdivide) reuse a per-device workspace: the arena of
// intermediate levels and the pinned status word stay allocated between calls
// instead of a cudaMalloc / cudaFree pair per call.  A call takes the
// workspace exclusively (a concurrent call on the same device allocates its
// own) and returns it only after its stream has synchronized, so the next call
// on any stream finds it idle.  slak_workspace_release frees it;
// SLAK_WORKSPACE_CACHE=0 disables the cache.
struct Workspace {
    void* mem = nullptr;
    size_t bytes = 0;
    DevStatus* h_st = nullptr;
    bool busy = false;
};
constexpr int kWsMaxDevices = 64;
std::mutex g_ws_mu;
Workspace g_ws[kWsMaxDevices];

Workspace* workspace_acquire()
{
    const char* env = std::getenv("SLAK_WORKSPACE_CACHE");
    if (env && env[0] == '0') return nullptr;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kWsMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    Workspace* w = &g_ws[dev];
    if (w->busy) return nullptr;
    if (!w->h_st && cudaMallocHost(&w->h_st, sizeof(DevStatus)) != cudaSuccess) { w->h_st = nullptr; return nullptr; }
    w->busy = true;
    return w;
}

void workspace_return(Workspace* w)
{
    if (!w) return;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    w->busy = false;
}

// grows (never shrinks) the workspace to `bytes`
cudaError_t workspace_reserve(Workspace* w, size_t bytes)
{
    if (w->bytes >= bytes) return cudaSuccess;
    if (w->mem) cudaFree(w->mem);
    w->mem = nullptr;
    w->bytes = 0;
    cudaError_t e = cudaMalloc(&w->mem, bytes);
    if (e == cudaSuccess) w->bytes = bytes;
    return e;
}

}  // namespace

// ------------------------------------------------------------------ autotuner
// The block sizes of k_g1 / k_g2 / k_g3 of every fast level are chosen by
// measurement.  The key is what sets them: the scheme, the parent's face type,
// whether the level writes the next level's state, the level's size (log2 of
// its quads) and the input's valence histogram (largest valence class; share
// of valence-4 vertices).  Choices are cached per process and, with
// SLAK_TUNE_FILE set, in that text file (a key and three block sizes a line).
// Every plan applies cached choices; SLAK_PLAN_AUTOTUNE measures missing keys.
std::mutex g_tune_mu;
std::map<std::string, std::array<int, 3>> g_tune;
bool g_tune_loaded = false;
const char* const kTuneKernels[3] = {"k_g1", "k_g2", "k_g3"};

std::string tune_key(const slak_plan* p, int li)
{
    const Level& L = p->lv[li];
    const Level& P = p->lv[li - 1];
    int vmax = 0;
    int64_t tot = 0;
    for (int k = 0; k < 17; ++k) {
        if (p->vhist[k]) vmax = k;
        tot += p->vhist[k];
    }
    const double share4 = tot ? (double)p->vhist[4] / (double)tot : 0.0;
    const int vclass = vmax <= 4 ? 4 : vmax <= 8 ? 8 : vmax < 16 ? 15 : 16;
    const int sclass = share4 < 0.5 ? 0 : share4 < 0.9 ? 50 : 90;
    const int fb = (int)std::floor(std::log2((double)std::max<int64_t>(L.F, 1)));
    char buf[96];
    std::snprintf(buf, sizeof buf, "%s/%s%s/%s/q2^%d/vmax%d/v4_%d", p->scheme == SLAK_SCHEME_LAK ? "lak" : "slak",
                  L.gq ? "gquad" : P.quad ? "quad" : "poly", P.B > 0 ? "-open" : "",
                  L.make_state ? "state" : L.sg ? "last-sg" : "last",
                  fb, vclass, sclass);
    return buf;
}

bool valid_block(int b) { return b == 128 || b == 256 || b == 512; }

void tune_load_locked()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("SLAK_TUNE_FILE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[128];
    int a, b, c;
    while (std::fscanf(f, "%127s %d %d %d", key, &a, &b, &c) == 4)
        if (valid_block(a) && valid_block(b) && valid_block(c)) g_tune[key] = {a, b, c};
    std::fclose(f);
}

void tune_save_locked()
{
    const char* path = std::getenv("SLAK_TUNE_FILE");
    if (!path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (const auto& kv : g_tune) std::fprintf(f, "%s %d %d %d\n", kv.first.c_str(), kv.second[0], kv.second[1], kv.second[2]);
    std::fclose(f);
}

// cached choices for every fast level; returns the fast levels still untuned
std::vector<int> apply_tuning(slak_plan* p)
{
    std::vector<int> todo;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    for (int i = 1; i < (int)p->lv.size(); ++i) {
        Level& L = p->lv[i];
        if (!L.fast) continue;
        L.tune_key = tune_key(p, i);
        auto it = g_tune.find(L.tune_key);
        if (it != g_tune.end()) {
            for (int k = 0; k < 3; ++k) L.bs[k] = it->second[k];
            L.tuned = 2;
        } else {
            todo.push_back(i);
        }
    }
    return todo;
}

// device ms of kernel `name` of level `li` in the last timed execution
float kernel_ms(slak_plan* p, int li, const char* name)
{
    for (size_t i = 0; i < p->recs.size(); ++i)
        if (p->recs[i].level == li && std::strcmp(p->recs[i].name, name) == 0) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p->ev[i], p->ev[i + 1]);
            return ms;
        }
    return 0.f;
}

// Measures every candidate block size of each kernel of the untuned fast
// levels (median of 3 timed executions each; the other kernels keep their
// current choice) and keeps the fastest.  Runs the plan eagerly several
// times; its outputs are rewritten by the next execution.
int plan_autotune(slak_plan* p, cudaStream_t str)
{
    std::vector<int> todo = apply_tuning(p);
    if (todo.empty()) return SLAK_OK;
    const int saved = p->flags;
    p->flags |= SLAK_PLAN_TIMING;
    int rc = enqueue_all(p, str);                          // warm-up
    if (rc == SLAK_OK) rc = cuda_status(cudaStreamSynchronize(str));
    for (int li : todo) {
        Level& L = p->lv[li];
        for (int k = 0; k < 3 && rc == SLAK_OK; ++k) {
            if (k == 1 && p->lv[li - 1].quad) continue;    // k_g2 runs for polygon parents only
            for (int ci = 0; ci < 3 && rc == SLAK_OK; ++ci) {
                L.bs[k] = kTuneBlocks[ci];
                float t[3] = {0.f, 0.f, 0.f};
                for (int r = 0; r < 3 && rc == SLAK_OK; ++r) {
                    rc = enqueue_all(p, str);
                    if (rc == SLAK_OK) rc = cuda_status(cudaStreamSynchronize(str));
                    t[r] = kernel_ms(p, li, kTuneKernels[k]);
                }
                std::sort(t, t + 3);
                L.tune_ms[k][ci] = t[1];
            }
            int best = 1;                                   // ties keep the default
            for (int ci = 0; ci < 3; ++ci)
                if (L.tune_ms[k][ci] < L.tune_ms[k][best]) best = ci;
            L.bs[k] = kTuneBlocks[best];
        }
        L.tuned = 1;
    }
    p->flags = saved;
    if (rc != SLAK_OK) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int li : todo) g_tune[p->lv[li].tune_key] = {p->lv[li].bs[0], p->lv[li].bs[1], p->lv[li].bs[2]};
    tune_save_locked();
    return SLAK_OK;
}

// Plan creation; with `ws`, the arena and the status word come from the
// workspace (the plan does not own them).
// Crease list sizing from a host copy of the sharpness (one sync): the levels
// with a live crease.
static int plan_crease_setup(slak_plan* p, const float* sharp, int64_t m, const int32_t* cverts,
                             const float* csharp, int64_t nc, cudaStream_t str)
{
    std::vector<float> h((size_t)m), hc((size_t)nc);
    std::vector<int32_t> hv((size_t)nc);
    cudaError_t e = cudaSuccess;
    if (m) e = cudaMemcpyAsync(h.data(), sharp, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost, str);
    if (nc && e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), csharp, sizeof(float) * (size_t)nc, cudaMemcpyDeviceToHost, str);
    if (nc && e == cudaSuccess) e = cudaMemcpyAsync(hv.data(), cverts, sizeof(int32_t) * (size_t)nc, cudaMemcpyDeviceToHost, str);
    if (e == cudaSuccess) e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) { g_detail = std::string("crease sharpness: ") + cudaGetErrorString(e); return cuda_status(e); }
    float smax = 0.0f;
    for (float x : h) {
        if (!std::isfinite(x)) { g_detail = "crease sharpness is not finite"; return SLAK_ERR_INVALID_ARG; }
        smax = std::max(smax, x);
    }
    if (nc) {                        // corners: a dense sharpness per base vertex, checked here
        const int64_t V0 = p->lv[0].V;
        p->h_vcs.assign((size_t)V0, 0.0f);
        std::vector<char> seen((size_t)V0, 0);
        for (int64_t i = 0; i < nc; ++i) {
            const int32_t v = hv[(size_t)i];
            const float x = hc[(size_t)i];
            if (!std::isfinite(x)) { g_detail = "corner sharpness is not finite"; return SLAK_ERR_INVALID_ARG; }
            if (v < 0 || v >= V0 || seen[(size_t)v]) {
                g_detail = "corner " + std::to_string(i) + ": vertex out of range or named twice";
                return SLAK_ERR_BAD_MESH;
            }
            seen[(size_t)v] = 1;
            p->h_vcs[(size_t)v] = std::max(x, 0.0f);
            smax = std::max(smax, x);
        }
    }
    const int nlev = (int)p->lv.size();
    int cl = smax > 0.0f ? (int)std::ceil((double)smax) : 0;
    p->ncrease = m;
    p->crease_levels = std::min(std::min(cl, nlev), kMaxCreaseLevels);
    if (p->crease_levels == 0) return SLAK_OK;
    if ((m << p->crease_levels) >= (1ll << 30) || m >= (1ll << 29)) return SLAK_ERR_UNSUPPORTED;
    return SLAK_OK;
}

static int plan_create_impl(const slak_mesh* cm, int target_level, int scheme, int flags, cudaStream_t str,
                            Workspace* ws, slak_plan** out_plan, const int* cpairs = nullptr,
                            const float* csharp = nullptr, int64_t ncrease = 0, const int32_t* kverts = nullptr,
                            const float* ksharp = nullptr, int64_t ncorner = 0)
{
    *out_plan = nullptr;
    int rc = validate_mesh(cm, scheme);
    if (rc != SLAK_OK) return rc;
    slak_plan* p = new (std::nothrow) slak_plan();
    if (!p) return SLAK_ERR_OOM;
    const int nlev = plan_init(p, cm, target_level, scheme, flags);
    cudaError_t ce = cudaSuccess;
    if (ws) { p->h_st = ws->h_st; p->h_st_owned = false; }
    else ce = cudaMallocHost(&p->h_st, sizeof(DevStatus));
    if (ce != cudaSuccess) { p->h_st = nullptr; delete p; return cuda_status(ce); }
    if (nlev == 0) { *out_plan = p; return SLAK_OK; }
    void* probe_mem = nullptr;
    if (ws) {
        ce = workspace_reserve(ws, probe_bytes(p->lv[0]));
        if (ce != cudaSuccess) { free_plan_memory(p); delete p; return cuda_status(ce); }
        probe_mem = ws->mem;
    }
    rc = probe_level0(p, p->lv[0], str, probe_mem);
    if (rc == SLAK_OK) rc = plan_levels(p);
    if (rc == SLAK_OK) {              // side streams for the levels' independent kernels
        for (int k = 0; k < 2 && ce == cudaSuccess; ++k) ce = cudaStreamCreateWithFlags(&p->side[k], cudaStreamNonBlocking);
        for (int k = 0; k < 4 && ce == cudaSuccess; ++k) ce = cudaEventCreateWithFlags(&p->cev[k], cudaEventDisableTiming);
        if (ce != cudaSuccess) rc = cuda_status(ce);
    }
    if (rc == SLAK_OK && (ncrease > 0 || ncorner > 0))
        rc = plan_crease_setup(p, csharp, ncrease, kverts, ksharp, ncorner, str);
    if (rc != SLAK_OK) { free_plan_memory(p); delete p; return rc; }
    Carver dry(nullptr);
    plan_carve(p, dry);
    if (ws) {
        ce = workspace_reserve(ws, dry.off);
        p->arena = ws->mem;
        p->arena_owned = false;
    } else {
        ce = cudaMalloc(&p->arena, dry.off);
    }
    if (ce != cudaSuccess) { free_plan_memory(p); delete p; return cuda_status(ce); }
    Carver cv((char*)p->arena);
    plan_carve(p, cv);
    // final outputs (caller-ownable, one allocation each)
    slak_mesh o = plan_output_shape(p);
    ce = cudaMalloc(&o.ids, sizeof(int) * (size_t)o.nnz);
    if (ce == cudaSuccess) ce = cudaMalloc(&o.verts, sizeof(float) * 4 * (size_t)o.nverts);
    if (ce == cudaSuccess && scheme == SLAK_SCHEME_LAK) {
        ce = cudaMalloc(&o.ptr, sizeof(int) * (size_t)(o.nfaces + 1));
        if (ce == cudaSuccess) ce = cudaMalloc(&o.vals, sizeof(int) * (size_t)o.nnz);
    }
    p->out = o;
    if (ce == cudaSuccess && p->crease_levels > 0) {   // the plan keeps its own copy of the creases
        if (ncrease > 0) {
            ce = cudaMemcpyAsync(p->c_pairs, cpairs, sizeof(int) * 2 * (size_t)ncrease, cudaMemcpyDeviceToDevice, str);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(p->c_sharp, csharp, sizeof(float) * (size_t)ncrease, cudaMemcpyDeviceToDevice,
                                     str);
        }
        if (ce == cudaSuccess && p->c_vcs)
            ce = cudaMemcpyAsync(p->c_vcs, p->h_vcs.data(), sizeof(float) * p->h_vcs.size(), cudaMemcpyHostToDevice,
                                 str);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(str);
    }
    if (ce != cudaSuccess) { free_plan_memory(p); delete p; return cuda_status(ce); }
    plan_wire(p);
    if (flags & SLAK_PLAN_AUTOTUNE) rc = plan_autotune(p, str);
    else apply_tuning(p);
    if (rc != SLAK_OK) { free_plan_memory(p); delete p; return rc; }
    *out_plan = p;
    return SLAK_OK;
}

extern "C" {

const char* slak_status_string(int status)
{
    switch (status) {
    case SLAK_OK: return "ok";
    case SLAK_ERR_INVALID_ARG: return "invalid argument";
    case SLAK_ERR_CUDA: return "CUDA runtime error";
    case SLAK_ERR_OOM: return "device out of memory";
    case SLAK_ERR_BAD_MESH: return "malformed mesh (index out of range, face order < 3 or non-manifold edge)";
    case SLAK_ERR_TIMEOUT: return "bounded device wait timed out";
    case SLAK_ERR_UNSUPPORTED: return "mesh too large for 32-bit indices";
    case SLAK_ERR_NOT_READY: return "plan has not been executed";
    default: return "unknown status";
    }
}

int slak_abi_version(void) { return SLAK_B200_ABI_VERSION; }

const char* slak_last_error_detail(void) { return g_detail.c_str(); }

int slak_plan_create(const slak_mesh* cm, int target_level, int scheme, int flags, slak_stream_t stream,
                     slak_plan** out_plan)
{
    if (!cm || !out_plan) return SLAK_ERR_INVALID_ARG;
    return plan_create_impl(cm, target_level, scheme, flags, reinterpret_cast<cudaStream_t>(stream), nullptr,
                            out_plan);
}

int slak_plan_create_sharp(const slak_mesh* cm, int target_level, int scheme, int flags,
                           const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                           const int32_t* corner_verts, const float* corner_sharpness, int64_t ncorners,
                           slak_stream_t stream, slak_plan** out_plan)
{
    if (!cm || !out_plan || ncreases < 0 || ncorners < 0) return SLAK_ERR_INVALID_ARG;
    if (ncreases > 0 && (!crease_verts || !crease_sharpness)) return SLAK_ERR_INVALID_ARG;
    if (ncorners > 0 && (!corner_verts || !corner_sharpness)) return SLAK_ERR_INVALID_ARG;
    return plan_create_impl(cm, target_level, scheme, flags, reinterpret_cast<cudaStream_t>(stream), nullptr,
                            out_plan, crease_verts, crease_sharpness, ncreases, corner_verts, corner_sharpness,
                            ncorners);
}

int slak_plan_create_creased(const slak_mesh* cm, int target_level, int scheme, int flags,
                             const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                             slak_stream_t stream, slak_plan** out_plan)
{
    return slak_plan_create_sharp(cm, target_level, scheme, flags, crease_verts, crease_sharpness, ncreases,
                                  nullptr, nullptr, 0, stream, out_plan);
}

int slak_subdivide_sharp(const slak_mesh* cm, slak_mesh* rm, int target_level, int scheme,
                         const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                         const int32_t* corner_verts, const float* corner_sharpness, int64_t ncorners,
                         slak_stream_t stream)
{
    if (!cm || !rm) return SLAK_ERR_INVALID_ARG;
    std::memset(rm, 0, sizeof(*rm));
    slak_plan* p = nullptr;
    int rc = slak_plan_create_sharp(cm, target_level, scheme, 0, crease_verts, crease_sharpness, ncreases,
                                    corner_verts, corner_sharpness, ncorners, stream, &p);
    if (rc != SLAK_OK) return rc;
    rc = slak_plan_execute(p, stream);
    if (rc == SLAK_OK) rc = slak_plan_status(p, stream);
    if (rc == SLAK_OK) rc = slak_plan_release_output(p, rm);
    slak_plan_destroy(p);
    return rc;
}

int slak_subdivide_creased(const slak_mesh* cm, slak_mesh* rm, int target_level, int scheme,
                           const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                           slak_stream_t stream)
{
    return slak_subdivide_sharp(cm, rm, target_level, scheme, crease_verts, crease_sharpness, ncreases, nullptr,
                                nullptr, 0, stream);
}

int slak_plan_execute(slak_plan* p, slak_stream_t stream)
{
    if (!p) return SLAK_ERR_INVALID_ARG;
    if (p->lv.empty()) { p->executed = 1; return SLAK_OK; }
    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    int rc;
    if ((p->flags & SLAK_PLAN_GRAPH) && str != nullptr) {
        if (!p->gexec) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(str, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_status(e);
            rc = enqueue_all(p, str);
            e = cudaStreamEndCapture(str, &g);
            if (rc != SLAK_OK) { if (g) cudaGraphDestroy(g); return rc; }
            if (e != cudaSuccess) return cuda_status(e);
            e = cudaGraphInstantiate(&p->gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_status(e);
        }
        rc = cuda_status(cudaGraphLaunch(p->gexec, str));
    } else {
        rc = enqueue_all(p, str);
    }
    p->executed = 1;
    return rc;
}

int slak_plan_status(slak_plan* p, slak_stream_t stream)
{
    if (!p) return SLAK_ERR_INVALID_ARG;
    if (!p->executed) return SLAK_ERR_NOT_READY;
    if (p->lv.empty()) return SLAK_OK;
    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(p->h_st, p->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
    if (e == cudaSuccess) e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) { g_detail = std::string("status: ") + cudaGetErrorString(e); return cuda_status(e); }
    if (p->h_st->err) g_detail = "device detail " + std::to_string(p->h_st->detail);
    return p->h_st->err;
}

int slak_plan_output(const slak_plan* p, slak_mesh* r)
{
    if (!p || !r) return SLAK_ERR_INVALID_ARG;
    if (p->lv.empty()) return SLAK_OK;
    *r = p->out;
    return SLAK_OK;
}

int slak_plan_release_output(slak_plan* p, slak_mesh* r)
{
    if (!p || !r) return SLAK_ERR_INVALID_ARG;
    if (p->lv.empty()) return SLAK_OK;
    if (!p->out_owned) return SLAK_ERR_INVALID_ARG;
    *r = p->out;
    p->out_owned = false;
    return SLAK_OK;
}

int slak_plan_num_levels(const slak_plan* p) { return p ? (int)p->lv.size() : 0; }

int slak_plan_level_stats(const slak_plan* p, int level, slak_level_stats* s)
{
    if (!p || !s || level < 0 || level >= (int)p->lv.size()) return SLAK_ERR_INVALID_ARG;
    const Level& L = p->lv[level];
    s->nfaces = L.F; s->nverts = L.V; s->nnz = L.N; s->nedges = L.E; s->nboundary = L.B;
    s->out_faces = L.Fo; s->out_verts = L.Vo;
    // compulsory bytes: ids in, positions in, refined ids out, refined positions out
    int64_t b = 4 * L.N + 16 * L.V + 4 * L.No + 16 * L.Vo;
    if (!L.quad) b += 4 * (L.F + 1);
    if (p->scheme == SLAK_SCHEME_LAK) b += 4 * (L.F + 1) + 4 * L.N + 4 * (L.Fo + 1) + 4 * L.No;
    s->algorithmic_bytes = b;
    return SLAK_OK;
}

int64_t slak_plan_launches(const slak_plan* p) { return p ? p->launches : 0; }

int slak_plan_kernel_timings(slak_plan* p, slak_kernel_timing* out, int capacity)
{
    if (!p || (capacity > 0 && !out)) return -SLAK_ERR_INVALID_ARG;
    if (!(p->flags & SLAK_PLAN_TIMING) || !p->executed) return -SLAK_ERR_NOT_READY;
    if (cudaEventSynchronize(p->ev[p->recs.size()]) != cudaSuccess) return -SLAK_ERR_CUDA;
    const int n = (int)p->recs.size();
    for (int i = 0; i < n && i < capacity; ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p->ev[i], p->ev[i + 1]);
        out[i].name = p->recs[i].name;
        out[i].level = p->recs[i].level;
        out[i].ms = ms;
        out[i].algorithmic_bytes = p->recs[i].bytes;
    }
    return n;
}

int slak_plan_tuning(const slak_plan* p, int level, slak_tuning* out)
{
    if (!p || !out || level < 0 || level >= (int)p->lv.size()) return SLAK_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    const Level& L = p->lv[level];
    out->state = L.fast ? L.tuned : -1;
    for (int k = 0; k < 3; ++k) {
        out->block[k] = L.bs[k];
        for (int c = 0; c < 3; ++c) out->ms[k][c] = L.tune_ms[k][c];
    }
    std::snprintf(out->key, sizeof out->key, "%s", L.tune_key.c_str());
    return SLAK_OK;
}

int slak_autotune_reset(void)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    g_tune_loaded = true;     // the file is not read again
    return SLAK_OK;
}

int slak_plan_destroy(slak_plan* p)
{
    if (!p) return SLAK_OK;
    free_plan_memory(p);
    delete p;
    return SLAK_OK;
}

int slak_subdivide(const slak_mesh* cm, slak_mesh* rm, int target_level, int scheme, slak_stream_t stream)
{
    if (!cm || !rm) return SLAK_ERR_INVALID_ARG;
    slak_plan* p = nullptr;
    Workspace* ws = workspace_acquire();
    int rc = plan_create_impl(cm, target_level, scheme, 0, reinterpret_cast<cudaStream_t>(stream), ws, &p);
    if (rc != SLAK_OK) { workspace_return(ws); return rc; }
    struct Return {      // the workspace goes back after the plan's last stream sync
        Workspace* w;
        ~Return() { workspace_return(w); }
    } ret{ws};
    if (p->lv.empty()) { slak_plan_destroy(p); return SLAK_OK; }   // rmesh left untouched
    rc = slak_plan_execute(p, stream);
    if (rc == SLAK_OK) rc = slak_plan_status(p, stream);
    if (rc == SLAK_OK) {
        slak_mesh o;
        slak_plan_release_output(p, &o);
        int64_t mfo = rm->max_face_order;
        *rm = o;
        if (scheme == SLAK_SCHEME_SLAK) rm->max_face_order = mfo;   // SLAK never assigns it
    }
    slak_plan_destroy(p);
    return rc;
}

int slak_workspace_release(void)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= kWsMaxDevices) return SLAK_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    Workspace* w = &g_ws[dev];
    if (w->busy) return SLAK_ERR_NOT_READY;
    if (w->mem) e = cudaFree(w->mem);
    if (w->h_st) cudaFreeHost(w->h_st);
    *w = Workspace{};
    return cuda_status(e);
}

int slak_mesh_free(slak_mesh* m)
{
    if (!m) return SLAK_ERR_INVALID_ARG;
    cudaError_t e = cudaSuccess, t;
    if (m->ptr) { t = cudaFree(m->ptr); if (t != cudaSuccess) e = t; }
    if (m->ids) { t = cudaFree(m->ids); if (t != cudaSuccess) e = t; }
    if (m->vals) { t = cudaFree(m->vals); if (t != cudaSuccess) e = t; }
    if (m->verts) { t = cudaFree(m->verts); if (t != cudaSuccess) e = t; }
    std::memset(m, 0, sizeof(*m));
    return cuda_status(e);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Batches: many meshes, each with its own level count, refined by one call.
//
// Every mesh gets its own plan (so each mesh's numbering and float results are
// exactly those of slak_subdivide on it alone), but all plans are sized up
// front and write straight into one batch output buffer.  Meshes are dealt to
// kBatchStreams chains, longest predicted time first, each to the chain with
// the least predicted time so far; a chain runs its meshes one after another
// (in mesh order, so large and small ones alternate) on its own stream and
// reuses one slice of the arena sized to its largest mesh.  The chains run
// concurrently and join once.  Only when the chains' slices do not fit the
// memory budget does the batch fall back to several such waves, joined in
// turn.  With SLAK_PLAN_GRAPH the whole batch (every wave, mesh and level) is
// captured as one CUDA graph whose branches are the chains.
struct slak_batch {
    int scheme = SLAK_SCHEME_SLAK;
    int flags = 0;
    std::vector<slak_plan*> plans;              // nullptr where the mesh is not refined
    std::vector<slak_mesh> outs;
    std::vector<std::vector<int64_t>> waves;    // mesh indices per wave, in enqueue order
    std::vector<int> chain;                     // per mesh: its chain (stream) within its wave
    void* out_mem = nullptr;
    void* arena = nullptr;
    size_t out_bytes = 0, arena_bytes = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> fork, join;
    // per stream slot: two side streams and four events lent to the plans it
    // runs (a plan records each event and waits on it at once, so plans that
    // follow one another on a slot can share them)
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> sev;
    cudaGraphExec_t gexec = nullptr;
    DevStatus* h_st = nullptr;                  // pinned, one per mesh
    DevStatus* d_st = nullptr;                  // device, one per mesh (outlives the waves' arenas)
    int64_t launches = 0;
    int executed = 0;
    bool per_mesh_out = false;                  // outputs allocated per mesh (slak_subdivide_batched)
    std::vector<char> out_given;                // per mesh: arrays handed to the caller
    // small meshes run in groups: meshes whose plans launch the same kernels
    // in the same order, each step one grouped launch over all of them
    struct GroupStep {
        GroupLaunchFn fn;
        unsigned grid, block;
        size_t args_off, bstart_off;            // in gmem
    };
    struct Group {
        std::vector<int64_t> meshes;
        std::vector<GroupStep> steps;
        double cost = 0.0;
    };
    std::vector<Group> groups;
    std::vector<char> grouped;                  // per mesh
    void* gmem = nullptr;                       // device: the groups' argument packs and block offsets
    std::vector<cudaStream_t> gstreams;
    std::vector<int> gstream_of;                // per group
    cudaEvent_t gfork = nullptr;
    std::vector<cudaEvent_t> gjoin;
};

namespace {

constexpr int kBatchStreams = 16;
constexpr int kGroupStreams = 4;
// meshes refined to fewer quads than this run in groups;
// SLAK_BATCH_GROUP_QUADS overrides it (0: no groups)
constexpr int64_t kGroupQuads = int64_t(1) << 19;
constexpr size_t kGroupSliceBytes = size_t(1) << 30;       // scratch of one group, at most

void batch_free(slak_batch* b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    for (auto* p : b->plans)
        if (p) { free_plan_memory(p); delete p; }
    for (auto s : b->streams) cudaStreamDestroy(s);
    for (auto s : b->side) cudaStreamDestroy(s);
    for (auto e : b->sev) cudaEventDestroy(e);
    for (auto e : b->fork) cudaEventDestroy(e);
    for (auto e : b->join) cudaEventDestroy(e);
    if (b->out_mem) cudaFree(b->out_mem);
    if (b->per_mesh_out)
        for (size_t i = 0; i < b->outs.size(); ++i)
            if (!b->out_given[i]) {
                slak_mesh& m = b->outs[i];
                if (m.ids) cudaFree(m.ids);
                if (m.verts) cudaFree(m.verts);
                if (m.ptr) cudaFree(m.ptr);
                if (m.vals) cudaFree(m.vals);
            }
    if (b->arena) cudaFree(b->arena);
    if (b->gmem) cudaFree(b->gmem);
    for (auto s : b->gstreams) cudaStreamDestroy(s);
    if (b->gfork) cudaEventDestroy(b->gfork);
    for (auto e : b->gjoin) cudaEventDestroy(e);
    if (b->d_st) cudaFree(b->d_st);
    if (b->h_st) cudaFreeHost(b->h_st);
    delete b;
}

size_t out_bytes_of(const slak_mesh& o, bool lak)
{
    size_t b = align_up(sizeof(int) * (size_t)o.nnz) + align_up(sizeof(float) * 4 * (size_t)o.nverts);
    if (lak) b += align_up(sizeof(int) * (size_t)(o.nfaces + 1)) + align_up(sizeof(int) * (size_t)o.nnz);
    return b;
}

// Predicted device time of one mesh's plan while kBatchStreams chains share
// the GPU: its levels' refined quads at 1/kBatchStreams of a measured
// 55 G quads/s, plus the dependent launches' latency (level 0 about 45 us,
// each later level about 12 us), which concurrency does not divide.
double batch_cost_us(const slak_plan* p)
{
    double quads = 0.0;
    for (const Level& L : p->lv) quads += (double)L.Fo;
    return quads * kBatchStreams / 55.0e3 + 45.0 + 12.0 * (double)(p->lv.size() - 1);
}

int batch_enqueue(slak_batch* b, cudaStream_t str)
{
    int64_t nl = 0;
    // the groups, on their own streams beside the chains
    if (!b->groups.empty()) {
        cudaEventRecord(b->gfork, str);
        for (auto gs : b->gstreams) cudaStreamWaitEvent(gs, b->gfork, 0);
        char* gm = static_cast<char*>(b->gmem);
        for (size_t g = 0; g < b->groups.size(); ++g) {
            const auto& G = b->groups[g];
            cudaStream_t gs = b->gstreams[b->gstream_of[g]];
            for (const auto& st : G.steps) {
                st.fn(gm + st.args_off, reinterpret_cast<const unsigned*>(gm + st.bstart_off), (int)G.meshes.size(),
                      st.grid, st.block, gs);
                ++nl;
            }
        }
    }
    for (size_t w = 0; w < b->waves.size(); ++w) {
        const auto& wave = b->waves[w];
        int nb = 0;
        for (int64_t i : wave) nb = std::max(nb, b->chain[i] + 1);
        cudaEventRecord(b->fork[w], str);
        for (int k = 0; k < nb; ++k) cudaStreamWaitEvent(b->streams[k], b->fork[w], 0);
        for (size_t j = 0; j < wave.size(); ++j) {
            slak_plan* p = b->plans[wave[j]];
            const int k = b->chain[wave[j]];
            if (!b->side.empty()) {
                p->side[0] = b->side[2 * k];
                p->side[1] = b->side[2 * k + 1];
                for (int i = 0; i < 4; ++i) p->cev[i] = b->sev[4 * k + i];
                p->side_owned = false;
            }
            int rc = enqueue_all(p, b->streams[k]);
            if (rc != SLAK_OK) return rc;
            nl += p->launches;
        }
        for (int k = 0; k < nb; ++k) {
            cudaEventRecord(b->join[w * kBatchStreams + k], b->streams[k]);
            cudaStreamWaitEvent(str, b->join[w * kBatchStreams + k], 0);
        }
    }
    if (!b->groups.empty())
        for (size_t k = 0; k < b->gstreams.size(); ++k) {
            cudaEventRecord(b->gjoin[k], b->gstreams[k]);
            cudaStreamWaitEvent(str, b->gjoin[k], 0);
        }
    b->launches = nl;
    return cuda_status(cudaGetLastError());
}

// Records the launches one execution of plan p makes, without launching.
int record_plan(slak_plan* p, std::vector<RecLaunch>& r, cudaStream_t str)
{
    g_record = &r;
    const int rc = enqueue_all(p, str);
    g_record = nullptr;
    return rc;
}

// The groups of small meshes, before any memory exists.  Each candidate's
// plan is wired to null scratch and its launch sequence recorded (the
// sequence does not depend on addresses); meshes with the same sequence form
// a kind, and each kind is cut into groups of at most `slice` bytes of
// scratch.  Groups go to kGroupStreams streams (longest predicted first, to
// the least loaded); a stream's groups run one after another in one region
// of the arena sized to its largest group.  Sets b->groups, b->gstream_of,
// b->grouped, each grouped mesh's offset in `aoff` (from the start of the
// groups' part of the arena) and returns that part's size.
size_t batch_plan_groups(slak_batch* b, const std::vector<int64_t>& cand, const std::vector<size_t>& ab,
                         const std::vector<double>& cost, size_t slice, std::vector<size_t>& aoff, cudaStream_t str,
                         int* rc)
{
    std::map<std::vector<std::pair<uintptr_t, unsigned>>, std::vector<int64_t>> kinds;
    for (int64_t i : cand) {
        slak_plan* p = b->plans[i];
        if (ab[i] > slice) continue;
        p->arena = nullptr;
        Carver dry(nullptr);
        plan_carve(p, dry);
        p->st = nullptr;
        p->out = b->outs[i];
        plan_wire(p);
        std::vector<RecLaunch> r;
        *rc = record_plan(p, r, str);
        if (*rc != SLAK_OK) return 0;
        std::vector<std::pair<uintptr_t, unsigned>> key;
        for (const auto& x : r) key.emplace_back(reinterpret_cast<uintptr_t>(x.fn), x.block);
        kinds[key].push_back(i);
    }
    std::vector<size_t> gbytes;
    for (auto& kv : kinds) {
        size_t used = slice;
        for (int64_t i : kv.second) {
            if (used + ab[i] > slice) {
                b->groups.emplace_back();
                gbytes.push_back(0);
                used = 0;
            }
            slak_batch::Group& G = b->groups.back();
            aoff[i] = used;                 // within the group, for now
            G.meshes.push_back(i);
            G.cost += cost[i];
            used += ab[i];
            gbytes.back() = used;
            b->grouped[i] = 1;
        }
    }
    const int ns = (int)std::min<size_t>(kGroupStreams, b->groups.size());
    if (ns == 0) return 0;
    std::vector<size_t> ord(b->groups.size());
    for (size_t g = 0; g < ord.size(); ++g) ord[g] = g;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return b->groups[x].cost > b->groups[y].cost; });
    std::vector<double> load(ns, 0.0);
    std::vector<size_t> region(ns, 0);
    b->gstream_of.assign(b->groups.size(), 0);
    for (size_t g : ord) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->gstream_of[g] = k;
        load[k] += b->groups[g].cost;
        region[k] = std::max(region[k], gbytes[g]);
    }
    std::vector<size_t> base(ns, 0);
    size_t tot = 0;
    for (int k = 0; k < ns; ++k) { base[k] = tot; tot += region[k]; }
    for (size_t g = 0; g < b->groups.size(); ++g)
        for (int64_t i : b->groups[g].meshes) aoff[i] += base[b->gstream_of[g]];
    return tot;
}

// Records every grouped mesh's launches again, now with its real scratch and
// outputs, and uploads each group step's argument packs and block offsets.
int batch_upload_groups(slak_batch* b, cudaStream_t str)
{
    if (b->groups.empty()) return SLAK_OK;
    std::vector<std::vector<RecLaunch>> rec(b->plans.size());
    for (const auto& G : b->groups)
        for (int64_t i : G.meshes) {
            const int rc = record_plan(b->plans[i], rec[i], str);
            if (rc != SLAK_OK) return rc;
        }
    size_t off = 0;
    for (auto& G : b->groups) {
        const auto& r0 = rec[G.meshes[0]];
        const size_t nm = G.meshes.size();
        for (size_t j = 0; j < r0.size(); ++j) {
            slak_batch::GroupStep st{r0[j].fn, 0u, r0[j].block, off, 0};
            off += align_up(nm * r0[j].pack.size());
            st.bstart_off = off;
            off += align_up(sizeof(unsigned) * (nm + 1));
            G.steps.push_back(st);
        }
    }
    std::vector<unsigned char> hb(off, 0);
    for (auto& G : b->groups) {
        const size_t nm = G.meshes.size();
        for (size_t j = 0; j < G.steps.size(); ++j) {
            auto& st = G.steps[j];
            unsigned* bs = reinterpret_cast<unsigned*>(hb.data() + st.bstart_off);
            uint64_t tot = 0;
            for (size_t m = 0; m < nm; ++m) {
                const auto& rm = rec[G.meshes[m]];
                // the same launcher (kernel and argument types) in every mesh of the group
                if (rm.size() != G.steps.size() || rm[j].fn != st.fn || rm[j].block != st.block) {
                    g_detail = "grouped launch: launch sequences differ";
                    return SLAK_ERR_INVALID_ARG;
                }
                std::memcpy(hb.data() + st.args_off + m * rm[j].pack.size(), rm[j].pack.data(), rm[j].pack.size());
                bs[m] = (unsigned)tot;
                tot += rm[j].grid;
            }
            bs[nm] = (unsigned)tot;
            if (tot >= (uint64_t(1) << 31)) return SLAK_ERR_UNSUPPORTED;
            st.grid = (unsigned)tot;
        }
    }
    cudaError_t ce = cudaMalloc(&b->gmem, off);
    if (ce == cudaSuccess) ce = cudaMemcpy(b->gmem, hb.data(), off, cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return cuda_status(ce);
    const int ns = *std::max_element(b->gstream_of.begin(), b->gstream_of.end()) + 1;
    b->gstreams.resize(ns);
    for (auto& gs : b->gstreams) cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&b->gfork, cudaEventDisableTiming);
    b->gjoin.resize(ns);
    for (auto& e : b->gjoin) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return cuda_status(cudaGetLastError());
}

}  // namespace

extern "C" {

}  // extern "C"

// per_mesh_out: every mesh's output arrays come from their own cudaMalloc, so
// they can be handed to the caller (slak_subdivide_batched)
static int batch_create_impl(const slak_mesh* meshes, const int* levels, int64_t count, int scheme, int flags,
                             slak_stream_t stream, slak_batch** out_batch, bool per_mesh_out)
{
    if (!meshes || !levels || count < 0 || !out_batch) return SLAK_ERR_INVALID_ARG;
    *out_batch = nullptr;
    slak_batch* b = new (std::nothrow) slak_batch();
    if (!b) return SLAK_ERR_OOM;
    b->scheme = scheme;
    b->flags = flags;
    b->per_mesh_out = per_mesh_out;
    b->plans.assign(count, nullptr);
    b->outs.assign(count, slak_mesh{});
    b->out_given.assign(count, 0);
    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    int rc = SLAK_OK;
    int64_t maxN = 0, maxV = 0;
    bool any_poly = false;
    for (int64_t i = 0; i < count && rc == SLAK_OK; ++i) {
        rc = validate_mesh(&meshes[i], scheme);
        if (rc != SLAK_OK) break;
        slak_plan* p = new (std::nothrow) slak_plan();
        if (!p) { rc = SLAK_ERR_OOM; break; }
        p->arena_owned = false;
        p->out_owned = false;
        b->plans[i] = p;
        if (plan_init(p, &meshes[i], levels[i], scheme, flags & ~SLAK_PLAN_GRAPH) == 0) {
            delete p;
            b->plans[i] = nullptr;
            continue;
        }
        maxN = std::max(maxN, meshes[i].nnz);
        maxV = std::max(maxV, meshes[i].nverts);
        any_poly |= meshes[i].type != SLAK_MESH_QUAD;
    }
    cudaError_t ce = cudaSuccess;
    if (rc == SLAK_OK) ce = cudaMallocHost(&b->h_st, sizeof(DevStatus) * (size_t)(count > 0 ? count : 1));
    if (rc == SLAK_OK && ce != cudaSuccess) rc = cuda_status(ce);
    // level-0 topology of every mesh: one scratch, results copied back in stream order, one sync
    if (rc == SLAK_OK && maxN > 0) {
        Carver dry(nullptr);
        Scratch sc;
        carve_scratch(dry, sc, maxN, maxV, 1, any_poly);
        DevStatus* st = dry.take<DevStatus>(1);
        void* mem = nullptr;
        ce = cudaMalloc(&mem, dry.off);
        if (ce != cudaSuccess) rc = cuda_status(ce);
        else {
            Carver cv((char*)mem);
            carve_scratch(cv, sc, maxN, maxV, 1, any_poly);
            st = cv.take<DevStatus>(1);
            int64_t nl = 0;
            Lc lc{str, &nl, false, 0};
            for (int64_t i = 0; i < count; ++i) {
                slak_plan* p = b->plans[i];
                if (!p) continue;
                cudaMemsetAsync(st, 0, sizeof(DevStatus), str);
                launch_topology_a(p->lv[0], 0, scheme, sc, st, lc);
                launch_g<k_valence_hist_g>(grid_for(p->lv[0].V), kBlock, str, (int)p->lv[0].V, sc.sptr, st->vhist);
                cudaMemcpyAsync(&b->h_st[i], st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
                cudaMemcpyAsync(&b->h_st[i].nedges, sc.eptr + p->lv[0].V, sizeof(int), cudaMemcpyDeviceToHost, str);
            }
            ce = cudaStreamSynchronize(str);
            cudaFree(mem);
            if (ce != cudaSuccess) rc = cuda_status(ce);
        }
        for (int64_t i = 0; i < count && rc == SLAK_OK; ++i) {
            slak_plan* p = b->plans[i];
            if (!p) continue;
            if (b->h_st[i].err) {
                g_detail = "mesh " + std::to_string(i) + ": device detail " + std::to_string(b->h_st[i].detail);
                rc = b->h_st[i].err;
                break;
            }
            Level& L0 = p->lv[0];
            L0.B = b->h_st[i].bcount[0];
            L0.E = b->h_st[i].nedges;
            std::memcpy(p->vhist, b->h_st[i].vhist, sizeof(p->vhist));
            if (L0.E != (L0.N - L0.B) / 2 + L0.B) { g_detail = "mesh " + std::to_string(i); rc = SLAK_ERR_BAD_MESH; }
            else rc = plan_levels(p);
        }
    }
    // memory: every mesh's output in one buffer; chains of plans, each chain
    // reusing one arena slice
    std::vector<size_t> ab(count, 0), ob(count, 0), aoff(count, 0);
    std::vector<double> cost(count, 0.0);
    b->chain.assign(count, 0);
    size_t total_out = 0;
    for (int64_t i = 0; i < count && rc == SLAK_OK; ++i) {
        slak_plan* p = b->plans[i];
        if (!p) continue;
        Carver dry(nullptr);
        plan_carve(p, dry);
        ab[i] = dry.off;
        b->outs[i] = plan_output_shape(p);
        ob[i] = out_bytes_of(b->outs[i], scheme == SLAK_SCHEME_LAK);
        total_out += ob[i];
        cost[i] = batch_cost_us(p);
    }
    if (rc == SLAK_OK) {
        size_t freeb = 0, totalb = 0;
        cudaMemGetInfo(&freeb, &totalb);
        const size_t margin = size_t(2) << 30;
        if (total_out + margin > freeb) { g_detail = "batch outputs exceed device memory"; rc = SLAK_ERR_OOM; }
        size_t budget = rc == SLAK_OK ? (freeb - total_out - margin) * 3 / 4 : 0;
        size_t cap = size_t(24) << 30;
        if (const char* wb = std::getenv("SLAK_BATCH_WAVE_BYTES")) cap = (size_t)std::strtoull(wb, nullptr, 10);
        if (budget > cap) budget = cap;
        // small meshes run in groups (kinds of identical launch sequences cut
        // into groups of at most `slice` bytes of scratch); the groups' part
        // of the arena takes at most half the budget
        b->grouped.assign(count, 0);
        int64_t gq = kGroupQuads;
        if (const char* e = std::getenv("SLAK_BATCH_GROUP_QUADS")) gq = std::atoll(e);
        size_t gbytes = 0;
        if (rc == SLAK_OK && gq > 0 && !(flags & SLAK_PLAN_TIMING)) {
            std::vector<int64_t> cand;
            for (int64_t i = 0; i < count; ++i) {
                slak_plan* p = b->plans[i];
                if (p && !p->debug && p->lv.back().Fo < gq) cand.push_back(i);
            }
            const size_t slice = std::min(kGroupSliceBytes, budget / (2 * kGroupStreams));
            gbytes = batch_plan_groups(b, cand, ab, cost, slice, aoff, str, &rc);
        }
        budget -= std::min(budget, gbytes);
        // meshes by predicted time, longest first; each goes to the chain with
        // the least predicted time so far, unless the chains' slices would
        // outgrow the budget, which closes the wave.  A mesh above the budget
        // (but within free memory) runs in a wave of its own.
        const size_t hard = rc == SLAK_OK ? (freeb - total_out - margin) * 3 / 4 : 0;
        std::vector<int64_t> order;
        for (int64_t i = 0; i < count && rc == SLAK_OK; ++i) {
            if (!b->plans[i] || b->grouped[i]) continue;
            if (ab[i] > hard) { g_detail = "mesh " + std::to_string(i) + " needs more scratch than is free"; rc = SLAK_ERR_OOM; break; }
            order.push_back(i);
        }
        std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return cost[x] > cost[y]; });
        std::vector<std::vector<int64_t>> chains(kBatchStreams);
        std::vector<size_t> slice(kBatchStreams, 0);
        std::vector<double> load(kBatchStreams, 0.0);
        size_t used = 0;
        auto close_wave = [&]() {
            size_t off = 0;
            std::vector<int64_t> wave;
            for (int k = 0; k < kBatchStreams; ++k) {
                std::sort(chains[k].begin(), chains[k].end());
                for (int64_t i : chains[k]) aoff[i] = off;
                off += slice[k];
            }
            // enqueue order: the chains' first meshes, then their second ones, ...
            for (size_t j = 0;; ++j) {
                bool any = false;
                for (int k = 0; k < kBatchStreams; ++k)
                    if (j < chains[k].size()) { wave.push_back(chains[k][j]); any = true; }
                if (!any) break;
            }
            if (!wave.empty()) b->waves.push_back(wave);
            b->arena_bytes = std::max(b->arena_bytes, off);
            for (int k = 0; k < kBatchStreams; ++k) { chains[k].clear(); slice[k] = 0; load[k] = 0.0; }
            used = 0;
        };
        for (int64_t i : order) {
            int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            size_t grow = ab[i] > slice[k] ? ab[i] - slice[k] : 0;
            if (used + grow > budget && used > 0) {
                // the chain whose slice already holds it, else a new wave
                int fit = -1;
                for (int c = 0; c < kBatchStreams; ++c)
                    if (slice[c] >= ab[i] && (fit < 0 || load[c] < load[fit])) fit = c;
                if (fit >= 0) { k = fit; grow = 0; }
                else { close_wave(); k = 0; grow = ab[i]; }
            }
            chains[k].push_back(i);
            b->chain[i] = k;
            slice[k] += grow;
            used += grow;
            load[k] += cost[i];
        }
        close_wave();
        // the groups' part after the chains' region
        const size_t goff = b->arena_bytes;
        for (int64_t i = 0; i < count; ++i)
            if (b->grouped[i]) aoff[i] += goff;
        b->arena_bytes = goff + gbytes;
    }
    if (rc == SLAK_OK && total_out) {
        if (!b->per_mesh_out) ce = cudaMalloc(&b->out_mem, total_out);
        if (ce == cudaSuccess && b->arena_bytes) ce = cudaMalloc(&b->arena, b->arena_bytes);
        if (ce == cudaSuccess) ce = cudaMalloc(&b->d_st, sizeof(DevStatus) * (size_t)count);
        if (ce != cudaSuccess) rc = cuda_status(ce);
    }
    if (rc == SLAK_OK && b->per_mesh_out) {
        for (int64_t i = 0; i < count && ce == cudaSuccess; ++i) {
            if (!b->plans[i]) continue;
            slak_mesh& m = b->outs[i];
            ce = cudaMalloc(&m.ids, sizeof(int) * (size_t)m.nnz);
            if (ce == cudaSuccess) ce = cudaMalloc(&m.verts, sizeof(float) * 4 * (size_t)m.nverts);
            if (ce == cudaSuccess && scheme == SLAK_SCHEME_LAK) {
                ce = cudaMalloc(&m.ptr, sizeof(int) * (size_t)(m.nfaces + 1));
                if (ce == cudaSuccess) ce = cudaMalloc(&m.vals, sizeof(int) * (size_t)m.nnz);
            }
        }
        if (ce != cudaSuccess) rc = cuda_status(ce);
    }
    if (rc == SLAK_OK) {
        char* o = static_cast<char*>(b->out_mem);
        for (int64_t i = 0; i < count && !b->per_mesh_out; ++i) {
            if (!b->plans[i]) continue;
            slak_mesh& m = b->outs[i];
            m.ids = reinterpret_cast<int*>(o); o += align_up(sizeof(int) * (size_t)m.nnz);
            m.verts = reinterpret_cast<float*>(o); o += align_up(sizeof(float) * 4 * (size_t)m.nverts);
            if (scheme == SLAK_SCHEME_LAK) {
                m.ptr = reinterpret_cast<int*>(o); o += align_up(sizeof(int) * (size_t)(m.nfaces + 1));
                m.vals = reinterpret_cast<int*>(o); o += align_up(sizeof(int) * (size_t)m.nnz);
            }
        }
        for (int64_t i = 0; i < count; ++i) {
            slak_plan* p = b->plans[i];
            if (!p) continue;
            p->arena = static_cast<char*>(b->arena) + aoff[i];
            Carver cv(static_cast<char*>(p->arena));
            plan_carve(p, cv);
            p->st = b->d_st + i;               // a chain's slice is reused by its later meshes
            p->out = b->outs[i];
            plan_wire(p);
        }
        b->fork.resize(b->waves.size());
        b->join.resize(b->waves.size() * kBatchStreams);
        for (auto& e : b->fork) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        for (auto& e : b->join) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        b->streams.resize(kBatchStreams);
        for (auto& st2 : b->streams) cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking);
        b->side.resize(2 * kBatchStreams);
        for (auto& st2 : b->side) cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking);
        b->sev.resize(4 * kBatchStreams);
        for (auto& e : b->sev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        ce = cudaGetLastError();
        if (ce != cudaSuccess) rc = cuda_status(ce);
    }
    // launch shapes: cached choices, or (SLAK_PLAN_AUTOTUNE) measured on the
    // first mesh of each key, alone on `stream`, before any batch execution
    // (grouped meshes keep the default shapes, so that more of them share a
    // launch sequence)
    for (int64_t i = 0; i < count && rc == SLAK_OK; ++i) {
        slak_plan* p = b->plans[i];
        if (!p || b->grouped[i]) continue;
        if (flags & SLAK_PLAN_AUTOTUNE) rc = plan_autotune(p, str);
        else apply_tuning(p);
    }
    if (rc == SLAK_OK) rc = batch_upload_groups(b, str);
    if (rc != SLAK_OK) { batch_free(b); return rc; }
    *out_batch = b;
    return SLAK_OK;
}

extern "C" {

int slak_batch_create(const slak_mesh* meshes, const int* levels, int64_t count, int scheme, int flags,
                      slak_stream_t stream, slak_batch** out_batch)
{
    return batch_create_impl(meshes, levels, count, scheme, flags, stream, out_batch, false);
}

int slak_subdivide_batched(const slak_mesh* meshes, const int* levels, int64_t count, int scheme,
                           slak_mesh* rmeshes, slak_stream_t stream)
{
    if (!rmeshes || count < 0) return SLAK_ERR_INVALID_ARG;
    for (int64_t i = 0; i < count; ++i) std::memset(&rmeshes[i], 0, sizeof(slak_mesh));
    slak_batch* b = nullptr;
    int rc = batch_create_impl(meshes, levels, count, scheme, 0, stream, &b, true);   // one execution: eager
    if (rc != SLAK_OK) return rc;
    rc = slak_batch_execute(b, stream);
    if (rc == SLAK_OK) rc = slak_batch_status(b, stream);
    if (rc == SLAK_OK)
        for (int64_t i = 0; i < count; ++i) {
            if (!b->plans[i]) continue;
            rmeshes[i] = b->outs[i];
            b->out_given[i] = 1;
        }
    batch_free(b);
    return rc;
}

int slak_batch_execute(slak_batch* b, slak_stream_t stream)
{
    if (!b) return SLAK_ERR_INVALID_ARG;
    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    int rc;
    if ((b->flags & SLAK_PLAN_GRAPH) && str != nullptr) {
        if (!b->gexec) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(str, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_status(e);
            rc = batch_enqueue(b, str);
            e = cudaStreamEndCapture(str, &g);
            if (rc != SLAK_OK) { if (g) cudaGraphDestroy(g); return rc; }
            if (e != cudaSuccess) return cuda_status(e);
            e = cudaGraphInstantiate(&b->gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_status(e);
        }
        rc = cuda_status(cudaGraphLaunch(b->gexec, str));
    } else {
        rc = batch_enqueue(b, str);
    }
    b->executed = 1;
    for (auto* p : b->plans) if (p) p->executed = 1;
    return rc;
}

int slak_batch_status(slak_batch* b, slak_stream_t stream)
{
    if (!b) return SLAK_ERR_INVALID_ARG;
    if (!b->executed) return SLAK_ERR_NOT_READY;
    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) { g_detail = std::string("batch: ") + cudaGetErrorString(e); return cuda_status(e); }
    for (size_t i = 0; i < b->plans.size(); ++i)
        if (b->plans[i]) cudaMemcpyAsync(&b->h_st[i], b->plans[i]->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
    e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) return cuda_status(e);
    for (size_t i = 0; i < b->plans.size(); ++i)
        if (b->plans[i] && b->h_st[i].err) {
            g_detail = "mesh " + std::to_string(i) + ": device detail " + std::to_string(b->h_st[i].detail);
            return b->h_st[i].err;
        }
    return SLAK_OK;
}

int slak_batch_output(const slak_batch* b, int64_t index, slak_mesh* rmesh)
{
    if (!b || !rmesh || index < 0 || index >= (int64_t)b->outs.size()) return SLAK_ERR_INVALID_ARG;
    if (!b->plans[index]) return SLAK_OK;     // nothing refined: *rmesh untouched
    *rmesh = b->outs[index];
    return SLAK_OK;
}

int slak_batch_num_waves(const slak_batch* b) { return b ? (int)b->waves.size() : 0; }

int slak_batch_num_groups(const slak_batch* b) { return b ? (int)b->groups.size() : 0; }

int64_t slak_batch_launches(const slak_batch* b) { return b ? b->launches : 0; }

int slak_batch_destroy(slak_batch* b)
{
    if (b) batch_free(b);
    return SLAK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// One subdivision level that allocates nothing.  Some callers cannot call
// cudaMalloc: an application whose device memory is owned by its own pool
// allocator, or a latency-critical loop that must not hit cudaMalloc/cudaFree
// (which can synchronise the device and take unbounded time).  For them the
// scratch of one general level lives in a fixed, file-scope device array of
// kNoAllocScratchBytes; the caller passes the input mesh and the output
// buffers.  Every GPU that loads this library holds the array until exit.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;     // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

}  // namespace

extern "C" int slak_subdivide_level_noalloc(const slak_mesh* cm, slak_mesh* rm, int scheme, slak_stream_t stream)
{
    if (!cm || !rm) return SLAK_ERR_INVALID_ARG;
    if (scheme != SLAK_SCHEME_LAK && scheme != SLAK_SCHEME_SLAK) return SLAK_ERR_INVALID_ARG;
    if (cm->type < SLAK_MESH_TRI || cm->type > SLAK_MESH_POLY) return SLAK_ERR_INVALID_ARG;
    if (cm->nfaces <= 0 || cm->nverts <= 0 || cm->nnz <= 0 || !cm->ids || !cm->verts) return SLAK_ERR_INVALID_ARG;
    const bool quad = cm->type == SLAK_MESH_QUAD, lak = scheme == SLAK_SCHEME_LAK;
    if (quad && cm->nnz != 4 * cm->nfaces) return SLAK_ERR_BAD_MESH;
    if (!quad && !cm->ptr) return SLAK_ERR_INVALID_ARG;
    if (!rm->ids || !rm->verts || (lak && (!rm->ptr || !rm->vals))) return SLAK_ERR_INVALID_ARG;
    if (4 * cm->nnz >= (1ll << 31) || cm->nverts >= (1ll << 31)) return SLAK_ERR_UNSUPPORTED;

    // the scratch of one general level (edges <= corners), checked against the fixed array
    const int64_t N = cm->nnz, V = cm->nverts, F = cm->nfaces;
    Scratch s;
    Carver dry(nullptr);
    carve_scratch(dry, s, N, V, N, !quad);
    dry.take<DevStatus>(1);
    if (dry.off > kNoAllocScratchBytes) {
        g_detail = "mesh needs " + std::to_string(dry.off) + " bytes of scratch; the allocation-free entry point has " +
                   std::to_string(kNoAllocScratchBytes);
        return SLAK_ERR_UNSUPPORTED;
    }

    // device address of the array, looked up once per device with that device current
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= kMaxDevices) return SLAK_ERR_UNSUPPORTED;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                g_detail = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return cuda_status(e);
            }
        }
        base = g_noalloc_addr[dev];
    }
    Carver cv(static_cast<char*>(base));
    carve_scratch(cv, s, N, V, N, !quad);
    DevStatus* st = cv.take<DevStatus>(1);

    cudaStream_t str = reinterpret_cast<cudaStream_t>(stream);
    Level L;
    L.F = F; L.V = V; L.N = N;
    L.quad = quad; L.poly_fn = !quad;
    L.ptr = cm->ptr; L.ids = cm->ids; L.verts = cm->verts;
    int64_t nl = 0;
    Lc lc{str, &nl, false, 0};
    cudaMemsetAsync(st, 0, sizeof(DevStatus), str);              // the array keeps the last call's contents
    launch_topology_a(L, 0, scheme, s, st, lc);
    DevStatus h;
    int nedges = 0;
    cudaMemcpyAsync(&h, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
    cudaMemcpyAsync(&nedges, s.eptr + V, sizeof(int), cudaMemcpyDeviceToHost, str);
    e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) return cuda_status(e);
    if (h.err) {
        g_detail = "level 0 topology: detail " + std::to_string(h.detail);
        return h.err;
    }
    L.B = h.bcount[0];
    L.E = nedges;
    if (L.E != (N - L.B) / 2 + L.B) {
        g_detail = "level 0 has " + std::to_string(L.E) + " edges and " + std::to_string(L.B) +
                   " boundary half-edges: not a manifold mesh";
        return SLAK_ERR_BAD_MESH;
    }
    L.Fo = N; L.No = 4 * N; L.Vo = V + F + L.E;
    if (rm->nverts < L.Vo) {      // rm->nverts carries the capacity of rm->verts, in vertices
        g_detail = "output positions need " + std::to_string(L.Vo) + " vertices";
        return SLAK_ERR_INVALID_ARG;
    }
    L.o_ids = rm->ids; L.o_verts = rm->verts;
    L.o_ptr = lak ? rm->ptr : nullptr;
    L.o_vals = lak ? rm->vals : nullptr;
    if (quad) launch_rest<true>(L, 0, scheme, false, s, st, lc);
    else launch_rest<false>(L, 0, scheme, false, s, st, lc);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        // kernels of this call that did launch may still use the array: the
        // call returns only once the stream is idle, so the next call cannot race them
        cudaStreamSynchronize(str);
        g_detail = std::string("launch: ") + cudaGetErrorString(e);
        return cuda_status(e);
    }
    cudaMemcpyAsync(&h, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, str);
    e = cudaStreamSynchronize(str);
    if (e != cudaSuccess) return cuda_status(e);
    if (h.err) {
        g_detail = "level 0: detail " + std::to_string(h.detail);
        return h.err;
    }
    rm->type = SLAK_MESH_QUAD;
    rm->nfaces = L.Fo; rm->nnz = L.No; rm->nverts = L.Vo;
    rm->is_reduced = lak ? 0 : 1;
    if (lak) rm->max_face_order = 4;
    return SLAK_OK;
}
