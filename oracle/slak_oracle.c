/*
 * slak_oracle.c -- CPU restatement of GPUPeople/SLAK's Catmull-Clark schemes.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Loaded by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
 *
 * All reference citations are path:line inside the GPUPeople/SLAK project.
 *
 * Serialization rule.  The reference computes several results with atomics:
 *   - CCKernels::evaluateValences (LibInclude/device/CatmullClarkKernels.cuh:137-145)
 *     hands each corner a slot in its vertex's adjacency column by atomicAdd;
 *   - createEVals (LibInclude/device/math/spgemm.cuh:71-100) numbers LAK edges
 *     with a global atomicAdd;
 *   - facepoint/edgepoint/vertex scatters use float atomicAdd
 *     (CatmullClarkKernels.cuh:577-686, spmv.cuh:83-121, LAKCatmullClarkKernels.cuh:483-511).
 * The oracle executes each such kernel as if its threads ran one after the
 * other in ascending thread index.  Consequences used throughout:
 *   - the corners of vertex v appear in its adjacency column in ascending
 *     corner order (a stable counting sort);
 *   - float scatters into one address are summed in ascending thread order.
 * Everything else (face order, face-point ids, original vertex ids) is
 * already deterministic in the reference and is restated as is.
 *
 * Floating point: IEEE binary32 with round-to-nearest and no contraction
 * (build with -ffp-contract=off); x/4 and x*0.25 are identical in IEEE, so
 * divisions by powers of two are written as multiplications where the
 * reference's compiler does the same.
 */
#include "slak_oracle.h"

#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Thread count of the following calls (n <= 0: the OpenMP default); returns
 * the count now in effect.  Used to time the single-thread baseline. */
int or_set_threads(int n)
{
#ifdef _OPENMP
    static int dflt = 0;
    if (!dflt) dflt = omp_get_max_threads();
    omp_set_num_threads(n > 0 ? n : dflt);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* small helpers                                                              */

typedef struct { float x, y, z, w; } f4;
typedef struct { double x, y, z, w; } d4;

static inline f4 ld4(const float* p, int64_t i) { f4 r = { p[4*i], p[4*i+1], p[4*i+2], p[4*i+3] }; return r; }
static inline void st4(float* p, int64_t i, f4 v) { p[4*i] = v.x; p[4*i+1] = v.y; p[4*i+2] = v.z; p[4*i+3] = v.w; }
static inline f4 add4(f4 a, f4 b) { f4 r = { a.x+b.x, a.y+b.y, a.z+b.z, a.w+b.w }; return r; }
static inline f4 mul4(f4 a, float s) { f4 r = { a.x*s, a.y*s, a.z*s, a.w*s }; return r; }
static inline f4 div4(f4 a, float s) { f4 r = { a.x/s, a.y/s, a.z/s, a.w/s }; return r; }
/* x / s + 0.0f : LAKHelperKernels::divElementWise_d adds `add` (= 0) after the
 * division (LAKCatmullClarkKernels.cuh:108), which turns -0.0 into +0.0 */
static inline f4 div4z(f4 a, float s) { f4 r = { a.x/s + 0.0f, a.y/s + 0.0f, a.z/s + 0.0f, a.w/s + 0.0f }; return r; }

static inline d4 ld4d(const double* p, int64_t i) { d4 r = { p[4*i], p[4*i+1], p[4*i+2], p[4*i+3] }; return r; }
static inline void st4d(double* p, int64_t i, d4 v) { p[4*i] = v.x; p[4*i+1] = v.y; p[4*i+2] = v.z; p[4*i+3] = v.w; }
static inline d4 add4d(d4 a, d4 b) { d4 r = { a.x+b.x, a.y+b.y, a.z+b.z, a.w+b.w }; return r; }
static inline d4 mul4d(d4 a, double s) { d4 r = { a.x*s, a.y*s, a.z*s, a.w*s }; return r; }
static inline d4 div4d(d4 a, double s) { d4 r = { a.x/s, a.y/s, a.z/s, a.w/s }; return r; }

static void* xcalloc(int64_t n, int64_t sz) { return calloc((size_t)(n > 0 ? n : 1), (size_t)sz); }
static void* xmalloc(int64_t n, int64_t sz) { return malloc((size_t)(n > 0 ? n : 1) * (size_t)sz); }

void or_mesh_free(or_mesh* m)
{
    if (!m) return;
    free(m->ptr); free(m->ids); free(m->vals); free(m->verts); free(m->verts64);
    memset(m, 0, sizeof(*m));
}

/* ------------------------------------------------------------------------- */
/* per-level topology shared by both schemes                                  */

typedef struct {
    int64_t F, V, N;
    const int32_t* ids;
    int32_t* fstart;   /* F+1 : first corner of each face                       */
    int32_t* cface;    /* N   : face of each corner (createThreadFaceMapping)   */
    int32_t* nextc;    /* N   : next corner in the face                          */
    int32_t* prevc;    /* N   : previous corner in the face                      */
    int32_t* val;      /* V   : number of corners at each vertex (valence)       */
    int64_t* sptr;     /* V+1 : adjacency column offsets (S_col_ptr)             */
    int32_t* sc;       /* N   : corner held in each adjacency slot               */
    int32_t* sids;     /* N   : S_row_ids: vertex after the slot's corner        */
} topo_t;

static void topo_free(topo_t* t)
{
    free(t->fstart); free(t->cface); free(t->nextc); free(t->prevc);
    free(t->val); free(t->sptr); free(t->sc); free(t->sids);
    memset(t, 0, sizeof(*t));
}

/* Builds the corner/face maps and the vertex adjacency S with the slot order of
 * serialized evaluateValences + evaluateAdjacencies[Quad]
 * (CatmullClarkKernels.cuh:137-187, scan CatmullClarkImpl.cu:179-181,395-397).
 * quad!=0 uses the implicit 4-corner faces of the quad functions
 * (`threadId / 4 * 4 + (threadId + 1) % 4`, CatmullClarkKernels.cuh:155). */
static int topo_build(topo_t* t, const or_mesh* m, int quad)
{
    memset(t, 0, sizeof(*t));
    t->F = m->nfaces; t->V = m->nverts; t->N = m->nnz; t->ids = m->ids;
    const int64_t F = t->F, V = t->V, N = t->N;
    if (quad && N != 4 * F) return 1;
    if (!quad && !m->ptr) return 1;
    t->fstart = (int32_t*)xmalloc(F + 1, 4);
    t->cface  = (int32_t*)xmalloc(N, 4);
    t->nextc  = (int32_t*)xmalloc(N, 4);
    t->prevc  = (int32_t*)xmalloc(N, 4);
    t->val    = (int32_t*)xcalloc(V, 4);
    t->sptr   = (int64_t*)xmalloc(V + 1, 8);
    t->sc     = (int32_t*)xmalloc(N, 4);
    t->sids   = (int32_t*)xmalloc(N, 4);
    for (int64_t f = 0; f <= F; ++f) t->fstart[f] = quad ? (int32_t)(4 * f) : m->ptr[f];
    if (t->fstart[0] != 0 || t->fstart[F] != N) return 1;
    for (int64_t f = 0; f < F; ++f) {
        int64_t b = t->fstart[f], e = t->fstart[f + 1];
        if (e - b < 1) return 1;
        for (int64_t c = b; c < e; ++c) {
            t->cface[c] = (int32_t)f;
            t->nextc[c] = (int32_t)(c + 1 < e ? c + 1 : b);
            t->prevc[c] = (int32_t)(c > b ? c - 1 : e - 1);
        }
    }
    for (int64_t c = 0; c < N; ++c) {
        int32_t v = m->ids[c];
        if (v < 0 || v >= V) return 1;
        t->val[v]++;
    }
    t->sptr[0] = 0;
    for (int64_t v = 0; v < V; ++v) t->sptr[v + 1] = t->sptr[v] + t->val[v];
    int32_t* fill = (int32_t*)xcalloc(V, 4);
    for (int64_t c = 0; c < N; ++c) {          /* serialized atomicAdd slot order */
        int32_t v = m->ids[c];
        int64_t s = t->sptr[v] + fill[v]++;
        t->sc[s] = (int32_t)c;
        t->sids[s] = m->ids[t->nextc[c]];
    }
    free(fill);
    return 0;
}

/* first slot in column `col` whose S_row_ids equals `row`; -1 if none */
static inline int64_t col_find(const topo_t* t, int64_t col, int32_t row)
{
    for (int64_t s = t->sptr[col]; s < t->sptr[col + 1]; ++s)
        if (t->sids[s] == row) return s;
    return -1;
}

/* ------------------------------------------------------------------------- */
/* SLAK                                                                      */

/* One SLAK level.  Restates
 *   initQuadMesh / initPolyMesh           CatmullClarkImpl.cu:151-226 / 360-452
 *   subdivideTopology{Quad,Poly}Mesh      CatmullClarkImpl.cu:107-149 / 311-358
 *   subdivideVertexData{Quad,Poly}Mesh    CatmullClarkImpl.cu:37-105  / 231-309
 * `has_boundary` is Context::has_boundary (CatmullClark.h:55): the quad
 * functions only look for boundary edges while it is set; it latches to false
 * after a closed level (CatmullClarkImpl.cu:197-206). */
static int slak_level(const or_mesh* in, or_mesh* out, int poly, int* has_boundary, int fp64)
{
    topo_t T;
    memset(out, 0, sizeof(*out));
    if (topo_build(&T, in, !poly)) { topo_free(&T); return 1; }
    const int64_t F = T.F, V = T.V, N = T.N;
    const int32_t* ids = in->ids;

    /* evaluateAdjacencies: S_epids_lt = v0 < v1 (CatmullClarkKernels.cuh:158-159,184-185) */
    int32_t* ep_tmp = (int32_t*)xmalloc(N, 4);
    for (int64_t s = 0; s < N; ++s) ep_tmp[s] = ids[T.sc[s]] < T.sids[s];

    /* boundary detection: checkForBoundaryQuad (:200-236) / checkForBoundaryFillFaceAdjacency (:280-321) */
    int check = poly ? 1 : *has_boundary;
    int64_t nextern = 0;
    uint8_t* ext = (uint8_t*)xcalloc(N, 1);
    int64_t* eslot = (int64_t*)xcalloc(N, 8);
    if (check) {
        for (int64_t c = 0; c < N; ++c) {
            int32_t v0 = ids[c], vout = ids[T.nextc[c]];
            int64_t e = col_find(&T, v0, vout);
            eslot[c] = e < 0 ? 0 : e;
            if (col_find(&T, vout, v0) >= 0) continue;
            ext[c] = 1; nextern++;
            ep_tmp[eslot[c]] = 1;
        }
        *has_boundary = nextern != 0;      /* CatmullClarkImpl.cu:197-206, 421-430 */
    }

    /* exclusive scan of the edge-owner flags -> edge ids (CatmullClarkImpl.cu:209-211) */
    int32_t* sep = (int32_t*)xmalloc(N, 4);
    { int64_t acc = 0; for (int64_t s = 0; s < N; ++s) { sep[s] = (int32_t)acc; acc += ep_tmp[s]; } }

    /* markBoundary[Quad] (:324-403): serialized atomic decrement fills everts from the back */
    int32_t* everts = (int32_t*)xmalloc(nextern, 4);
    if (nextern) {
        int64_t cnt = nextern;
        for (int64_t c = 0; c < N; ++c) {
            if (!ext[c]) continue;
            everts[--cnt] = ids[c];
            sep[eslot[c]] = -(sep[eslot[c]] + 1);
        }
    }

    const int64_t nedges = (N - nextern) / 2 + nextern;     /* CatmullClarkImpl.cu:120,326 */
    const int64_t Vn = V + F + nedges;
    out->type = OR_QUAD; out->is_reduced = 1;
    out->nfaces = N; out->nnz = 4 * N; out->nverts = Vn;
    out->max_face_order = 0;   /* SLAK never assigns it: a fresh MeshInfo keeps 0 */
    out->ptr = NULL; out->vals = NULL;
    out->ids = (int32_t*)xmalloc(4 * N, 4);
    const int ext_variant = check && nextern != 0;          /* which refine kernel runs */

    /* edge id of the edge {a,b}: refineTopology[Quad][Extern] (:405-575) */
    #define SLAK_EDGE(a, b, res) do {                                                  \
        int32_t mn_ = (a) < (b) ? (a) : (b), mx_ = (a) < (b) ? (b) : (a);               \
        int64_t sl_ = col_find(&T, mn_, mx_);                                            \
        if (sl_ < 0 && ext_variant) sl_ = col_find(&T, mx_, mn_);                        \
        if (sl_ < 0) sl_ = 0;                                                            \
        int32_t se_ = sep[sl_];                                                          \
        if (poly && !ext_variant) (res) = (int32_t)(se_ + V + F);                        \
        else (res) = (int32_t)(se_ >= 0 ? se_ + V + F : -se_ + V + F - 1);               \
    } while (0)

    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        int32_t v0 = ids[c];
        int32_t eo, ei;
        SLAK_EDGE(v0, ids[T.nextc[c]], eo);
        SLAK_EDGE(v0, ids[T.prevc[c]], ei);
        out->ids[4*c + 0] = v0;
        out->ids[4*c + 1] = eo;
        out->ids[4*c + 2] = (int32_t)(V + T.cface[c]);
        out->ids[4*c + 3] = ei;
    }
    #undef SLAK_EDGE

    /* ---- positions ---- */
    const float* P = in->verts;
    float* R = (float*)xcalloc(4 * Vn, 4);      /* edge points start zeroed (cudaMemset :60, :254) */
    float* FP = R + 4 * V;
    float* EP = R + 4 * (V + F);
    const double* P64 = fp64 ? in->verts64 : NULL;
    double* R64 = fp64 ? (double*)xcalloc(4 * Vn, 8) : NULL;
    double* FP64 = R64 ? R64 + 4 * V : NULL;
    double* EP64 = R64 ? R64 + 4 * (V + F) : NULL;

    /* face points */
    #pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        int64_t b = T.fstart[f], e = T.fstart[f + 1];
        if (!poly) {
            /* calculateFaceEdgepointsQuad (:577-600): width-16 shuffles give ((c0+c2)+(c1+c3))*(1/4) */
            f4 c0 = ld4(P, ids[b]), c1 = ld4(P, ids[b+1]), c2 = ld4(P, ids[b+2]), c3 = ld4(P, ids[b+3]);
            st4(FP, f, mul4(add4(add4(c0, c2), add4(c1, c3)), 0.25f));
            if (P64) {
                d4 d0 = ld4d(P64, ids[b]), d1 = ld4d(P64, ids[b+1]), d2 = ld4d(P64, ids[b+2]), d3 = ld4d(P64, ids[b+3]);
                st4d(FP64, f, mul4d(add4d(add4d(d0, d2), add4d(d1, d3)), 0.25));
            }
        } else {
            /* calculateFacepoints (:602-618): sum from zero, times 1/order */
            float rcp = 1.0f / (float)(e - b);
            f4 acc = { 0.f, 0.f, 0.f, 0.f };
            for (int64_t c = b; c < e; ++c) acc = add4(acc, ld4(P, ids[c]));
            st4(FP, f, mul4(acc, rcp));
            if (P64) {
                d4 a = { 0, 0, 0, 0 };
                for (int64_t c = b; c < e; ++c) a = add4d(a, ld4d(P64, ids[c]));
                st4d(FP64, f, mul4d(a, 1.0 / (double)(e - b)));
            }
        }
    }

    /* edge points: eps[e_out] += (fp + p)/4 per corner, serialized ascending
     * (quad :597-599, poly calculateEdgepoints :620-632).  Two terms per edge,
     * so the sum is order-independent anyway. */
    for (int64_t c = 0; c < N; ++c) {
        int64_t e = out->ids[4*c + 1] - V - F;
        f4 t = mul4(add4(ld4(P, ids[c]), ld4(FP, T.cface[c])), 0.25f);
        st4(EP, e, add4(ld4(EP, e), t));
        if (R64) {
            d4 td = mul4d(add4d(ld4d(P64, ids[c]), ld4d(FP64, T.cface[c])), 0.25);
            st4d(EP64, e, add4d(ld4d(EP64, e), td));
        }
    }

    /* vertex points: vertexSum (:634-652) then facepointSum[Quad] (:654-686),
     * the latter restated as a gather in ascending corner order */
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < V; ++v) {
        int32_t n = T.val[v];
        f4 acc = { 0.f, 0.f, 0.f, 0.f };
        for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s) acc = add4(acc, ld4(P, T.sids[s]));
        f4 orig = div4(mul4(ld4(P, v), (float)(n - 2)), (float)n);
        f4 y = add4(div4(acc, (float)(n * n)), orig);
        for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s)
            y = add4(y, div4(ld4(FP, T.cface[T.sc[s]]), (float)(n * n)));
        st4(R, v, y);
        if (R64) {
            d4 a = { 0, 0, 0, 0 };
            for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s) a = add4d(a, ld4d(P64, T.sids[s]));
            d4 o = div4d(mul4d(ld4d(P64, v), (double)(n - 2)), (double)n);
            d4 yd = add4d(div4d(a, (double)n * (double)n), o);
            for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s)
                yd = add4d(yd, div4d(ld4d(FP64, T.cface[T.sc[s]]), (double)n * (double)n));
            st4d(R64, v, yd);
        }
    }

    /* boundary: correctBoundaryS1 then correctBoundaryS2 (:688-740); the
     * 3/4 p + 1/8 q product pair is evaluated without contraction */
    if (*has_boundary && nextern) {
        int64_t* e0 = (int64_t*)xmalloc(nextern, 8);
        for (int64_t i = 0; i < nextern; ++i) {
            int32_t ev = everts[i];
            int64_t loc = 0;
            for (int64_t s = T.sptr[ev]; s < T.sptr[ev + 1]; ++s) if (sep[s] < 0) { loc = s; break; }
            e0[i] = loc;
            int64_t ep = -(int64_t)sep[loc] + V + F - 1;
            int32_t w = T.sids[loc];
            st4(R, ep, mul4(add4(ld4(P, ev), ld4(P, w)), 0.5f));
            st4(R, ev, add4(mul4(ld4(P, ev), 0.75f), mul4(ld4(P, w), 0.125f)));
            if (R64) {
                st4d(R64, ep, mul4d(add4d(ld4d(P64, ev), ld4d(P64, w)), 0.5));
                st4d(R64, ev, add4d(mul4d(ld4d(P64, ev), 0.75), mul4d(ld4d(P64, w), 0.125)));
            }
        }
        for (int64_t i = 0; i < nextern; ++i) {
            int32_t ev = everts[i];
            int32_t w = T.sids[e0[i]];
            st4(R, w, add4(ld4(R, w), mul4(ld4(P, ev), 0.125f)));
            if (R64) st4d(R64, w, add4d(ld4d(R64, w), mul4d(ld4d(P64, ev), 0.125)));
        }
        free(e0);
    }

    out->verts = R;
    out->verts64 = R64;
    free(ep_tmp); free(ext); free(eslot); free(sep); free(everts);
    topo_free(&T);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* LAK                                                                       */

static int cmp_i32(const void* a, const void* b)
{
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* One LAK level.  Restates
 *   initPolyMesh (run for every level)   LAKCatmullClarkImpl.cu:309-507
 *   subdivideTopology{Poly,Quad}Mesh     LAKCatmullClarkImpl.cu:255-307 / 79-130
 *   subdivideVertexDataPolyMesh          LAKCatmullClarkImpl.cu:150-253
 * Topology: the mapped SpGEMM M^T M (spgemm.cuh:61-69,102-309) yields, per
 * vertex pair {w<v} sharing a face, F (face of v->w) and F^T (face of w->v);
 * createEVals (spgemm.cuh:71-100), serialized by column v ascending then row
 * w ascending, numbers every pair with a half-edge in either direction:
 * edges are numbered in ascending (max, min) order, 1-based, -id interior and
 * +id boundary.  The per-face sort by vertex id and the sort back by vals
 * (LAKCatmullClarkImpl.cu:101,277,326) leave valid input (vals = 1..k in
 * storage order) unchanged, so storage order is the cyclic order here. */
static int lak_level(const or_mesh* in, or_mesh* out, int poly, int fp64)
{
    topo_t T;
    memset(out, 0, sizeof(*out));
    if (!in->ptr) return 1;
    if (topo_build(&T, in, 0)) { topo_free(&T); return 1; }
    const int64_t F = T.F, V = T.V, N = T.N;
    const int32_t* ids = in->ids;
    (void)poly;

    /* smaller neighbours of each vertex (row w < column v with F or F^T nonzero) */
    int64_t* nptr = (int64_t*)xmalloc(V + 1, 8);
    int32_t* nb = (int32_t*)xmalloc(2 * N, 4);
    int64_t fill = 0;
    for (int64_t v = 0; v < V; ++v) {
        nptr[v] = fill;
        int64_t b = fill;
        for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s) {
            int32_t c = T.sc[s];
            int32_t wo = ids[T.nextc[c]], wi = ids[T.prevc[c]];
            if (wo < v) nb[fill++] = wo;
            if (wi < v) nb[fill++] = wi;
        }
        qsort(nb + b, (size_t)(fill - b), 4, cmp_i32);
        int64_t u = b;
        for (int64_t k = b; k < fill; ++k) if (k == b || nb[k] != nb[k - 1]) nb[u++] = nb[k];
        fill = u;
    }
    nptr[V] = fill;
    const int64_t nedges = fill;

    /* E values: -id for an edge with both half-edges, +id for a boundary edge */
    int32_t* eval = (int32_t*)xmalloc(nedges, 4);
    int64_t nextern = 0;
    for (int64_t v = 0; v < V; ++v) {
        for (int64_t k = nptr[v]; k < nptr[v + 1]; ++k) {
            int32_t w = nb[k];
            int have_vw = col_find(&T, v, w) >= 0;   /* F(w,v) != 0 : half-edge v->w */
            int have_wv = col_find(&T, w, (int32_t)v) >= 0;
            int32_t id = (int32_t)(k + 1);
            if (have_vw && have_wv) eval[k] = -id;
            else { eval[k] = id; nextern++; }
        }
    }

    /* refineTopology / refineTopologyHomogeneous (LAKCatmullClarkKernels.cuh:320-411):
     * look E up at column max, row min; edge point = |E| - 1 + V + F */
    #define LAK_EDGE(a, b, res) do {                                                    \
        int32_t mn_ = (a) < (b) ? (a) : (b), mx_ = (a) < (b) ? (b) : (a);                 \
        int64_t k_ = nptr[mx_];                                                            \
        while (k_ < nptr[mx_ + 1] && nb[k_] != mn_) ++k_;                                  \
        int32_t ev_ = k_ < nptr[mx_ + 1] ? eval[k_] : 0;                                   \
        (res) = (int32_t)((ev_ < 0 ? -ev_ : ev_) - 1 + V + F);                              \
    } while (0)

    const int64_t Vn = V + F + (N - nextern) / 2 + nextern;   /* LAKCatmullClarkImpl.cu:96,272 */
    out->type = OR_QUAD; out->is_reduced = 0;
    out->nfaces = N; out->nnz = 4 * N; out->nverts = Vn; out->max_face_order = 4;
    out->ids = (int32_t*)xmalloc(4 * N, 4);
    out->ptr = (int32_t*)xmalloc(N + 1, 4);
    out->vals = (int32_t*)xmalloc(4 * N, 4);
    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        int32_t v0 = ids[c], eo, ei;
        LAK_EDGE(v0, ids[T.nextc[c]], eo);
        LAK_EDGE(v0, ids[T.prevc[c]], ei);
        out->ids[4*c + 0] = v0;
        out->ids[4*c + 1] = eo;
        out->ids[4*c + 2] = (int32_t)(V + T.cface[c]);
        out->ids[4*c + 3] = ei;
    }
    #undef LAK_EDGE
    for (int64_t q = 0; q <= N; ++q) out->ptr[q] = (int32_t)(4 * q);      /* createQuadColPtr :413-421 */
    for (int64_t i = 0; i < 4 * N; ++i) out->vals[i] = (int32_t)(i % 4 + 1); /* createQuadVals :423-431 */

    /* ---- positions ---- */
    const float* P = in->verts;
    float* R = (float*)xcalloc(4 * Vn, 4);
    float* FP = R + 4 * V;
    float* EP = R + 4 * (V + F);
    const double* P64 = fp64 ? in->verts64 : NULL;
    double* R64 = fp64 ? (double*)xcalloc(4 * Vn, 8) : NULL;
    double* FP64 = R64 ? R64 + 4 * V : NULL;
    double* EP64 = R64 ? R64 + 4 * (V + F) : NULL;

    /* face points: spmv_left_mapped_f4 (spmv.cuh:64-81; map is all ones) then
     * divElementWise by the face order (LAKCatmullClarkImpl.cu:175-178) */
    #pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        int64_t b = T.fstart[f], e = T.fstart[f + 1];
        f4 acc = { 0.f, 0.f, 0.f, 0.f };
        for (int64_t c = b; c < e; ++c) acc = add4(acc, ld4(P, ids[c]));
        st4(FP, f, div4z(acc, (float)(e - b)));
        if (P64) {
            d4 a = { 0, 0, 0, 0 };
            for (int64_t c = b; c < e; ++c) a = add4d(a, ld4d(P64, ids[c]));
            st4d(FP64, f, div4d(a, (double)(e - b)));
        }
    }

    /* edge points: calculateInternalEdgepoints / calculateExternalEdgepoints
     * (LAKCatmullClarkKernels.cuh:437-462): (((p_min + p_max) + fp0) + fp1)/4 with
     * fp0 the face of min->max and fp1 the face of max->min; boundary midpoint */
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < V; ++v) {
        for (int64_t k = nptr[v]; k < nptr[v + 1]; ++k) {
            int32_t w = nb[k];            /* w = min, v = max */
            int64_t id = (eval[k] < 0 ? -eval[k] : eval[k]) - 1;
            if (eval[k] < 0) {
                int64_t s0 = col_find(&T, w, (int32_t)v);  /* half-edge min->max */
                int64_t s1 = col_find(&T, v, w);            /* half-edge max->min */
                int32_t f0 = T.cface[T.sc[s0]], f1 = T.cface[T.sc[s1]];
                f4 a = add4(add4(add4(ld4(P, w), ld4(P, v)), ld4(FP, f0)), ld4(FP, f1));
                st4(EP, id, mul4(a, 0.25f));
                if (R64) {
                    d4 ad = add4d(add4d(add4d(ld4d(P64, w), ld4d(P64, v)), ld4d(FP64, f0)), ld4d(FP64, f1));
                    st4d(EP64, id, mul4d(ad, 0.25));
                }
            } else {
                st4(EP, id, mul4(add4(ld4(P, w), ld4(P, v)), 0.5f));
                if (R64) st4d(EP64, id, mul4d(add4d(ld4d(P64, w), ld4d(P64, v)), 0.5));
            }
        }
    }

    /* vertex points (LAKCatmullClarkImpl.cu:200-221):
     *   pn  = p * (n + (-2))                     multElementWise
     *   acc = sum fp over corners, face order    spmv_right_mapped_f4 over M
     *       + sum p[u] over incoming tails u,     spmv_right_mapped_f4 over F
     *         ascending u (F column u, row v)
     *   v'  = ((acc / n) + pn) / n               divElementWise, addElementWise, divElementWise */
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < V; ++v) {
        int32_t n = T.val[v];
        f4 acc = { 0.f, 0.f, 0.f, 0.f };
        d4 accd = { 0, 0, 0, 0 };
        int32_t tails[64];
        int32_t* tl = tails;
        int64_t deg = T.sptr[v + 1] - T.sptr[v];
        if (deg > 64) tl = (int32_t*)xmalloc(deg, 4);
        int64_t nt = 0;
        for (int64_t s = T.sptr[v]; s < T.sptr[v + 1]; ++s) {
            int32_t c = T.sc[s];
            acc = add4(acc, ld4(FP, T.cface[c]));
            if (R64) accd = add4d(accd, ld4d(FP64, T.cface[c]));
            tl[nt++] = ids[T.prevc[c]];
        }
        qsort(tl, (size_t)nt, 4, cmp_i32);
        for (int64_t k = 0; k < nt; ++k) {
            if (k > 0 && tl[k] == tl[k - 1]) continue;
            acc = add4(acc, ld4(P, tl[k]));
            if (R64) accd = add4d(accd, ld4d(P64, tl[k]));
        }
        if (tl != tails) free(tl);
        f4 pn = mul4(ld4(P, v), (float)n + (-2.0f));
        st4(R, v, div4z(add4(div4z(acc, (float)n), pn), (float)n));
        if (R64) {
            d4 pnd = mul4d(ld4d(P64, v), (double)n - 2.0);
            st4d(R64, v, div4d(add4d(div4d(accd, (double)n), pnd), (double)n));
        }
    }

    /* boundary vertices: prepareExternalVertexUpdate then
     * calculateExternalVertexUpdate (LAKCatmullClarkKernels.cuh:464-511), the
     * boundary list in ascending edge id (serialized extractEdgeInfoFromE) */
    if (nextern) {
        for (int64_t v = 0; v < V; ++v)
            for (int64_t k = nptr[v]; k < nptr[v + 1]; ++k) if (eval[k] > 0) {
                int32_t a = nb[k];
                st4(R, a, mul4(ld4(P, a), 0.75f));
                st4(R, v, mul4(ld4(P, v), 0.75f));
                if (R64) { st4d(R64, a, mul4d(ld4d(P64, a), 0.75)); st4d(R64, v, mul4d(ld4d(P64, v), 0.75)); }
            }
        for (int64_t v = 0; v < V; ++v)
            for (int64_t k = nptr[v]; k < nptr[v + 1]; ++k) if (eval[k] > 0) {
                int32_t a = nb[k];         /* v0 = a (min), v1 = v (max) */
                st4(R, v, add4(ld4(R, v), mul4(ld4(P, a), 0.125f)));
                st4(R, a, add4(ld4(R, a), mul4(ld4(P, v), 0.125f)));
                if (R64) {
                    st4d(R64, v, add4d(ld4d(R64, v), mul4d(ld4d(P64, a), 0.125)));
                    st4d(R64, a, add4d(ld4d(R64, a), mul4d(ld4d(P64, v), 0.125)));
                }
            }
    }

    out->verts = R;
    out->verts64 = R64;
    free(nptr); free(nb); free(eval);
    topo_free(&T);
    return 0;
}

/* ------------------------------------------------------------------------- */

int or_level(const or_mesh* in, or_mesh* out, int scheme, int poly, int with_fp64)
{
    if (scheme == OR_SLAK) { int hb = 1; return slak_level(in, out, poly, &hb, with_fp64); }
    return lak_level(in, out, poly, with_fp64);
}

int or_subdivide(const or_mesh* in, or_mesh* out, int target_level, int scheme, int with_fp64)
{
    memset(out, 0, sizeof(*out));
    or_mesh cur = *in;          /* shallow: the input is never freed (CatmullClarkImpl.cu:469) */
    int owned = 0, level = 0, has_boundary = 1, rc = 0;
    if (with_fp64 && !in->verts64) {
        cur.verts64 = (double*)xmalloc(4 * in->nverts, 8);
        for (int64_t i = 0; i < 4 * in->nverts; ++i) cur.verts64[i] = (double)in->verts[i];
        owned = 2;              /* only the fp64 shadow is ours */
    }
    if (cur.type != OR_QUAD) {
        or_mesh r;
        rc = scheme == OR_SLAK ? slak_level(&cur, &r, 1, &has_boundary, with_fp64)
                               : lak_level(&cur, &r, 1, with_fp64);
        if (rc) goto done;
        if (owned == 2) free(cur.verts64); else if (owned) or_mesh_free(&cur);
        cur = r; owned = 1; level = 1;
    }
    for (; level < target_level; ++level) {
        or_mesh r;
        rc = scheme == OR_SLAK ? slak_level(&cur, &r, 0, &has_boundary, with_fp64)
                               : lak_level(&cur, &r, 0, with_fp64);
        if (rc) goto done;
        if (owned == 2) free(cur.verts64); else if (owned) or_mesh_free(&cur);
        cur = r; owned = 1;
    }
    if (owned == 1) { *out = cur; return 0; }
done:
    if (owned == 2) free(cur.verts64); else if (owned == 1) or_mesh_free(&cur);
    return rc;
}
