// common.cuh -- shared device helpers for the subdivision kernels.
//
// Position arithmetic is IEEE binary32 round-to-nearest with no FMA
// contraction (explicit __f*_rn intrinsics, and the library is built with
// -fmad=false), so every float result is reproducible and equals the CPU
// restatement bit for bit.
#pragma once

#include <cstdint>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

namespace slak {

constexpr int kBlock = 256;

// ------------------------------------------------------- dependent launches
// Programmatic dependent launch: every kernel is launched with the
// programmatic-serialization attribute and starts with griddep_enter(): it
// waits until the grid before it in the stream has completed and its memory
// is visible (griddepcontrol.wait returns at once when there is none), then
// allows the grid after it to begin launching.  So each launch overlaps the
// tail of the grid before it instead of following its end, while no thread
// touches memory before its predecessor is done.  SLAK_NO_PDL builds launch
// plainly, for comparisons.
__device__ __forceinline__ void griddep_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

#ifdef SLAK_NO_PDL
constexpr bool kUsePdl = false;
#else
constexpr bool kUsePdl = true;
#endif

template <class... KArgs, class... Args>
inline void launch_k(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = kUsePdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------- grouped launches
// Every kernel a plan launches is written as a body, a __device__ function of
// its block index (k_*_body); a __global__ wrapper (k_*) runs it for
// blockIdx.x, and a group functor (k_*_g) names it for grouped launches.  A
// grouped launch runs one kernel for many meshes at once: its grid is the
// meshes' grids end to end, and each block finds its mesh in a table of block
// offsets (binary search) and its arguments in an array of argument packs.
// A batch records the launches of its small meshes' plans (launch_g with
// g_record set) and replays each step of a group of plans with identical
// launch sequences as one grouped launch.

// The arguments of one launch, trivially copyable, in one block of bytes.
template <size_t I, class T> struct PackLeaf { T v; };
template <class Seq, class... A> struct PackImpl;
template <size_t... I, class... A>
struct PackImpl<std::index_sequence<I...>, A...> : PackLeaf<I, A>... {
    PackImpl() = default;
    explicit PackImpl(const A&... a) : PackLeaf<I, A>{a}... {}
};
template <class... A> using Pack = PackImpl<std::index_sequence_for<A...>, A...>;

template <class G, size_t... I, class... A>
__device__ __forceinline__ void run_pack(unsigned bx, const PackImpl<std::index_sequence<I...>, A...>& p)
{
    G{}(bx, static_cast<const PackLeaf<I, A>&>(p).v...);
}

// the mesh whose block range [bstart[m], bstart[m+1]) holds this block
__device__ __forceinline__ int group_mesh(const unsigned* __restrict__ bstart, int nm)
{
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(bstart + mid) <= blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// G::kBounds: the launch bounds of the kernel's own wrapper (0 none, 1 the
// block size, 2 the block size and blocks per SM), repeated here
template <class G, class P>
__global__ void k_group(const P* __restrict__ args, const unsigned* __restrict__ bstart, int nm)
{
    griddep_enter();
    const int m = group_mesh(bstart, nm);
    run_pack<G>(blockIdx.x - __ldg(bstart + m), args[m]);
}
template <class G, class P>
__global__ void __launch_bounds__(G::kMaxT) k_group_t(const P* __restrict__ args, const unsigned* __restrict__ bstart,
                                                      int nm)
{
    griddep_enter();
    const int m = group_mesh(bstart, nm);
    run_pack<G>(blockIdx.x - __ldg(bstart + m), args[m]);
}
template <class G, class P>
__global__ void __launch_bounds__(G::kMaxT, G::kMinB) k_group_b(const P* __restrict__ args,
                                                                const unsigned* __restrict__ bstart, int nm)
{
    griddep_enter();
    const int m = group_mesh(bstart, nm);
    run_pack<G>(blockIdx.x - __ldg(bstart + m), args[m]);
}

using GroupLaunchFn = void (*)(const void* args, const unsigned* bstart, int nm, unsigned grid, unsigned block,
                               cudaStream_t s);

template <class G, class P>
void group_launch(const void* args, const unsigned* bstart, int nm, unsigned grid, unsigned block, cudaStream_t s)
{
    const P* a = static_cast<const P*>(args);
    if constexpr (G::kBounds == 2) launch_k(k_group_b<G, P>, grid, block, s, a, bstart, nm);
    else if constexpr (G::kBounds == 1) launch_k(k_group_t<G, P>, grid, block, s, a, bstart, nm);
    else launch_k(k_group<G, P>, grid, block, s, a, bstart, nm);
}

// One recorded launch: the grouped launcher of its kernel and argument types
// (which identifies it), its shape and its argument pack.
struct RecLaunch {
    GroupLaunchFn fn = nullptr;
    unsigned grid = 0, block = 0;
    size_t align = 0;
    std::vector<unsigned char> pack;
};
inline thread_local std::vector<RecLaunch>* g_record = nullptr;

template <class G, class... Args>
inline void launch_g(unsigned grid, unsigned block, cudaStream_t s, Args&&... args)
{
    if (g_record) {
        using P = Pack<std::decay_t<Args>...>;
        static_assert(std::is_trivially_copyable<P>::value, "launch arguments must be trivially copyable");
        const P pk(args...);
        RecLaunch r;
        r.fn = &group_launch<G, P>;
        r.grid = grid;
        r.block = block;
        r.align = alignof(P);
        r.pack.resize(sizeof(P));
        std::memcpy(r.pack.data(), &pk, sizeof(P));
        g_record->push_back(std::move(r));
        return;
    }
    launch_k(G::kernel(), grid, block, s, std::forward<Args>(args)...);
}

// n int32 words set to 0 (the plans' status words and counters)
__device__ __forceinline__ void k_zero_body(const unsigned bx_, int* __restrict__ p, int64_t n)
{
    const int64_t i = (int64_t)bx_ * kBlock + threadIdx.x;
    if (i < n) p[i] = 0;
}
__global__ void __launch_bounds__(kBlock) k_zero(int* __restrict__ p, int64_t n)
{
    griddep_enter();
    k_zero_body(blockIdx.x, p, n);
}
struct k_zero_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const { k_zero_body(bx, a...); }
    static constexpr auto kernel() { return &k_zero; }
};

// cudaMemsetAsync to 0 of `bytes` (a multiple of 4), or its grouped form
inline void zero_async(void* p, size_t bytes, cudaStream_t s)
{
    if (g_record) {
        const int64_t n = (int64_t)(bytes / 4);
        launch_g<k_zero_g>((unsigned)((n + kBlock - 1) / kBlock > 0 ? (n + kBlock - 1) / kBlock : 1), kBlock, s,
                           static_cast<int*>(p), n);
        return;
    }
    cudaMemsetAsync(p, 0, bytes, s);
}

// ---------------------------------------------------------------- float4 ops
__device__ __forceinline__ float4 f4_add(float4 a, float4 b)
{
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 f4_mul(float4 a, float s)
{
    return make_float4(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s), __fmul_rn(a.w, s));
}
// x / s.  When s is a normal power of two the quotient is an exact scaling, so
// the product with the exact reciprocal 2^-e is the same correctly rounded
// number (also under overflow / underflow) and avoids the IEEE divide sequence.
__device__ __forceinline__ bool pow2_recip(float s, float& r)
{
    const unsigned u = __float_as_uint(s), ex = u & 0x7f800000u;
    if ((u & 0x007fffffu) != 0u || ex == 0u || ex >= 0x7f000000u) return false;
    r = __uint_as_float((0x7f000000u - ex) | (u & 0x80000000u));
    return true;
}
__device__ __forceinline__ float4 f4_div(float4 a, float s)
{
    float r;
    if (pow2_recip(s, r)) return f4_mul(a, r);
    return make_float4(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s), __fdiv_rn(a.w, s));
}
// x / s + 0.0f (turns -0 into +0, as an element-wise divide-then-add does)
__device__ __forceinline__ float4 f4_div_z(float4 a, float s)
{
    float4 q = f4_div(a, s);
    return make_float4(__fadd_rn(q.x, 0.0f), __fadd_rn(q.y, 0.0f), __fadd_rn(q.z, 0.0f), __fadd_rn(q.w, 0.0f));
}
__device__ __forceinline__ float4 f4_zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }

__device__ __forceinline__ float4 ldg4(const float* p, int64_t i)
{
    return __ldg(reinterpret_cast<const float4*>(p) + i);
}
__device__ __forceinline__ void st4(float* p, int64_t i, float4 v)
{
    reinterpret_cast<float4*>(p)[i] = v;
}
// streaming store for outputs that are not read again by this level
__device__ __forceinline__ void st4_cs(float* p, int64_t i, float4 v)
{
    __stcs(reinterpret_cast<float4*>(p) + i, v);
}

// TwoSum (Knuth): s + e == a + b exactly
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// (hi, lo) += x, componentwise, with TwoSum: hi + lo carries the sum to about
// twice the working precision
__device__ __forceinline__ void dd_acc1(float& hi, float& lo, float x)
{
    float s, e;
    two_sum(hi, x, s, e);
    hi = s;
    lo = __fadd_rn(lo, e);
}
__device__ __forceinline__ void dd_acc(float4& hi, float4& lo, float4 x)
{
    dd_acc1(hi.x, lo.x, x.x); dd_acc1(hi.y, lo.y, x.y);
    dd_acc1(hi.z, lo.z, x.z); dd_acc1(hi.w, lo.w, x.w);
}

// (sh + sl) / n^2 + p (n-2) / n with exact remainders (fmaf) for both quotients
// and for the product, then a TwoSum of the two quotients; rounded once.
__device__ __forceinline__ float vp_finish1(float sh, float sl, float p, int n)
{
    const float nn = (float)(n * n), fn = (float)n, k = (float)(n - 2);
    float q = __fdiv_rn(sh, nn);
    float ql = __fdiv_rn(__fadd_rn(fmaf(-q, nn, sh), sl), nn);
    float oh = __fmul_rn(p, k);
    float ol = fmaf(p, k, -oh);
    float o = __fdiv_rn(oh, fn);
    float olo = __fdiv_rn(__fadd_rn(fmaf(-o, fn, oh), ol), fn);
    float hi, lo;
    two_sum(q, o, hi, lo);
    return __fadd_rn(hi, __fadd_rn(lo, __fadd_rn(ql, olo)));
}
__device__ __forceinline__ float4 vp_finish(float4 sh, float4 sl, float4 p, int n)
{
    return make_float4(vp_finish1(sh.x, sl.x, p.x, n), vp_finish1(sh.y, sl.y, p.y, n),
                       vp_finish1(sh.z, sl.z, p.z, n), vp_finish1(sh.w, sl.w, p.w, n));
}

// ---------------------------------------------------------------- in-order sums
// add(load(k)) for k = 0..n-1, in that order, with W loads in flight: a
// long column's records come from L2, and a loop that waited for each one
// would pay the full latency per slot.
template <int W = 4, class Load, class Add>
__device__ __forceinline__ void for_each_loaded(int n, Load load, Add add)
{
    for (int k0 = 0; k0 < n; k0 += W) {
        float4 t[W];
#pragma unroll
        for (int i = 0; i < W; ++i)
            if (k0 + i < n) t[i] = load(k0 + i);
#pragma unroll
        for (int i = 0; i < W; ++i)
            if (k0 + i < n) add(k0 + i, t[i]);
    }
}

// ---------------------------------------------------------------- ordering
// Columns longer than kBigCol slots (and up to kWarpCol) are taken by their
// whole warp: each lane holds two slots, ranks and loads run in parallel, and
// the sums run in the fixed order by shuffle (same bits as the single-thread
// paths, no shared memory).  Shorter columns, and longer ones, stay on one
// thread.
constexpr int kBigCol = 16;
constexpr int kWarpCol = 64;

__device__ __forceinline__ float4 shfl4(float4 v, int src)
{
    return make_float4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                       __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

// A long column's slots in its warp: slot k is element k >> 5 of lane k & 31
// (two per lane for up to kWarpCol = 64 slots).  col4 / col1 fetch slot k
// (k the same on every lane) from its lane; rank_of gives each of a lane's
// keys its rank in ascending key order, ties by slot.
__device__ __forceinline__ float4 col4(float4 e0, float4 e1, int k) { return shfl4(k < 32 ? e0 : e1, k & 31); }
__device__ __forceinline__ int col1(int e0, int e1, int k) { return __shfl_sync(0xffffffffu, k < 32 ? e0 : e1, k & 31); }
__device__ __forceinline__ void rank_of(int n, int key0, int key1, int& r0, int& r1)
{
    const int lane = threadIdx.x & 31;
    r0 = 0;
    r1 = 0;
    for (int j = 0; j < n; ++j) {
        const int y = col1(key0, key1, j);
        r0 += (y < key0) | ((y == key0) & (j < lane));
        r1 += (y < key1) | ((y == key1) & (j < lane + 32));
    }
}
// The slot of rank r (r the same on every lane), as (lane, element).
__device__ __forceinline__ void slot_of_rank(int r, bool h0, bool h1, int r0, int r1, int& src, int& el)
{
    const unsigned m0 = __ballot_sync(0xffffffffu, h0 && r0 == r);
    const unsigned m1 = __ballot_sync(0xffffffffu, h1 && r1 == r);
    el = m0 ? 0 : 1;
    src = __ffs(m0 ? m0 : m1) - 1;
}
// The slots k = 0..n-1 of key[b..b+n) in ascending key order (equal keys by
// slot): perm[r] = the slot of rank r.  n^2 independent compares, instead of
// n selection passes that each wait for the previous minimum; for one thread's
// columns of 5 to kBigCol slots (shorter ones are ranked in registers).
__device__ __forceinline__ void rank_order(const int* __restrict__ key, int b, int n, int* perm)
{
    for (int k = 0; k < n; ++k) {
        const int x = __ldg(key + b + k);
        int r = 0, j = 0;
        for (; j + 8 <= n; j += 8) {          // eight loads in flight before the compares
            int y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) y[i] = __ldg(key + b + j + i);
#pragma unroll
            for (int i = 0; i < 8; ++i) r += (y[i] < x) | ((y[i] == x) & (j + i < k));
        }
        for (; j < n; ++j) {
            const int y = __ldg(key + b + j);
            r += (y < x) | ((y == x) & (j < k));
        }
        perm[r] = k;
    }
}

// ---------------------------------------------------------------- status
// Device-side status written by kernels; the host reads it after a sync.
struct DevStatus {
    int err;          // first error code (slak_status), 0 = ok
    int detail;       // kernel-specific detail (e.g. offending index)
    int nextern;      // boundary half-edges of level 0
    int nedges;       // edges of level 0
    int bcount[32];   // boundary half-edges counted per level
    int vhist[17];    // level 0: vertices of valence 0..15, and 16 or more
};

__device__ __forceinline__ void set_error(DevStatus* st, int code, int detail)
{
    if (atomicCAS(&st->err, 0, code) == 0) st->detail = detail;
}

// ---------------------------------------------------------------- faces
// Corner navigation: QUAD uses the implicit 4-corner faces of the reference's
// quad functions (`threadId / 4 * 4 + (threadId + 1) % 4`,
// CatmullClarkKernels.cuh:155); otherwise face offsets + a corner->face map.
template <bool QUAD>
struct Faces {
    const int* __restrict__ ptr;
    const int* __restrict__ cface;
    __device__ __forceinline__ int face(int c) const { return QUAD ? (c >> 2) : __ldg(cface + c); }
    __device__ __forceinline__ int next(int c) const
    {
        if (QUAD) return (c & ~3) | ((c + 1) & 3);
        int f = __ldg(cface + c);
        return c + 1 < __ldg(ptr + f + 1) ? c + 1 : __ldg(ptr + f);
    }
    __device__ __forceinline__ int prev(int c) const
    {
        if (QUAD) return (c & ~3) | ((c + 3) & 3);
        int f = __ldg(cface + c);
        int b = __ldg(ptr + f);
        return c > b ? c - 1 : __ldg(ptr + f + 1) - 1;
    }
};

inline unsigned grid_for(int64_t n, int block = kBlock)
{
    int64_t g = (n + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace slak
