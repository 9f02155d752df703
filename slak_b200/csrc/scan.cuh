// scan.cuh -- device-wide exclusive prefix sum of int32 counts.
//
// Replaces CubFunctions::scan_exclusive (LibInclude/device/cub_wrappers.cuh:30-43):
// out[0] = 0, out[i+1] = in[0] + ... + in[i], out has n+1 entries, so out[n] is
// the total.  Reduce-then-scan over tiles of 2048 items: tile sums, one block
// scanning the tile sums, then a tile scan with the tile's carry (up to 2048
// tiles, each tile's block sums the tile sums before it instead).  Integer and
// deterministic.
#pragma once

#include "common.cuh"

namespace slak {

constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// exclusive scan of one value per thread across the block; returns the block total in *total
__device__ __forceinline__ int block_excl_scan(int x, int* total)
{
    __shared__ int warp_tot[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = warp_incl_scan(x);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int t = lane < kBlock / 32 ? warp_tot[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < kBlock / 32) warp_tot[lane] = ti - t;
        if (lane == kBlock / 32 - 1) *total = ti;
    }
    __syncthreads();
    int r = warp_tot[warp] + incl - x;
    __syncthreads();
    return r;
}

__device__ __forceinline__ void k_scan_reduce_body(const unsigned bx_, const int* __restrict__ in, int64_t n, int* __restrict__ tsum)
{
    const int64_t base = (int64_t)bx_ * kScanTile;
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int64_t k = base + (int64_t)i * kBlock + threadIdx.x;
        if (k < n) s += in[k];
    }
    __shared__ int tot;
    block_excl_scan(s, &tot);
    __syncthreads();
    if (threadIdx.x == 0) tsum[bx_] = tot;
}
__global__ void __launch_bounds__(kBlock) k_scan_reduce(const int* __restrict__ in, int64_t n, int* __restrict__ tsum)
{
    griddep_enter();
    k_scan_reduce_body(blockIdx.x, in, n, tsum);
}
struct k_scan_reduce_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_scan_reduce_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_scan_reduce; }
};

// one block: exclusive scan of the tile sums in place, tsum[nt] = grand total
__device__ __forceinline__ void k_scan_tiles_body(const unsigned bx_, int* __restrict__ tsum, int nt)
{
    __shared__ int tot;
    int carry = 0;
    for (int base = 0; base < nt; base += kBlock) {
        int k = base + threadIdx.x;
        int x = k < nt ? tsum[k] : 0;
        int e = block_excl_scan(x, &tot);
        __syncthreads();
        if (k < nt) tsum[k] = carry + e;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) tsum[nt] = carry;
}
__global__ void __launch_bounds__(kBlock) k_scan_tiles(int* __restrict__ tsum, int nt)
{
    griddep_enter();
    k_scan_tiles_body(blockIdx.x, tsum, nt);
}
struct k_scan_tiles_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_scan_tiles_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_scan_tiles; }
};

__device__ __forceinline__ void k_scan_final_body(const unsigned bx_, const int* __restrict__ in, int64_t n,
                                                  const int* __restrict__ tsum, int nt, int* __restrict__ out)
{
    __shared__ int tile[kScanTile];
    __shared__ int tot;
    const int64_t base = (int64_t)bx_ * kScanTile;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int j = i * kBlock + threadIdx.x;
        int64_t k = base + j;
        tile[j] = k < n ? in[k] : 0;
    }
    __syncthreads();
    int loc[kScanItems];
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) { loc[i] = s; s += tile[threadIdx.x * kScanItems + i]; }
    int e = block_excl_scan(s, &tot) + tsum[bx_];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) tile[threadIdx.x * kScanItems + i] = e + loc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int j = i * kBlock + threadIdx.x;
        int64_t k = base + j;
        if (k < n) out[k] = tile[j];
    }
    if (bx_ == 0 && threadIdx.x == 0) out[n] = tsum[nt];
}
__global__ void __launch_bounds__(kBlock) k_scan_final(const int* __restrict__ in, int64_t n,
                                                       const int* __restrict__ tsum, int nt, int* __restrict__ out)
{
    griddep_enter();
    k_scan_final_body(blockIdx.x, in, n, tsum, nt, out);
}
struct k_scan_final_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_scan_final_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_scan_final; }
};

// Up to kScanSmallTiles tiles: no separate scan of the tile sums; each block
// adds up the sums of the tiles before it (and all of them, for out[n]).
constexpr int kScanSmallTiles = 2048;

__device__ __forceinline__ void k_scan_final_small_body(const unsigned bx_, const int* __restrict__ in, int64_t n,
                                                        const int* __restrict__ tsum, int nt,
                                                        int* __restrict__ out)
{
    __shared__ int tile[kScanTile];
    __shared__ int tot;
    int before = 0, all = 0;
    for (int k = threadIdx.x; k < nt; k += kBlock) {
        const int x = tsum[k];
        all += x;
        if (k < (int)bx_) before += x;
    }
    block_excl_scan(before, &tot);
    __syncthreads();
    const int carry = tot;
    __syncthreads();
    block_excl_scan(all, &tot);
    __syncthreads();
    const int total = tot;
    const int64_t base = (int64_t)bx_ * kScanTile;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int j = i * kBlock + threadIdx.x;
        int64_t k = base + j;
        tile[j] = k < n ? in[k] : 0;
    }
    __syncthreads();
    int loc[kScanItems];
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) { loc[i] = s; s += tile[threadIdx.x * kScanItems + i]; }
    int e = block_excl_scan(s, &tot) + carry;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) tile[threadIdx.x * kScanItems + i] = e + loc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int j = i * kBlock + threadIdx.x;
        int64_t k = base + j;
        if (k < n) out[k] = tile[j];
    }
    if (bx_ == 0 && threadIdx.x == 0) out[n] = total;
}
__global__ void __launch_bounds__(kBlock) k_scan_final_small(const int* __restrict__ in, int64_t n,
                                                             const int* __restrict__ tsum, int nt,
                                                             int* __restrict__ out)
{
    griddep_enter();
    k_scan_final_small_body(blockIdx.x, in, n, tsum, nt, out);
}
struct k_scan_final_small_g {
    static constexpr int kBounds = 1, kMaxT = kBlock, kMinB = 0;
    template <class... A> __device__ __forceinline__ void operator()(unsigned bx, const A&... a) const
    {
        k_scan_final_small_body(bx, a...);
    }
    static constexpr auto kernel() { return &k_scan_final_small; }
};

inline int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

// tmp must hold scan_tiles(n) + 1 ints
inline void scan_exclusive(const int* in, int* out, int64_t n, int* tmp, cudaStream_t s, int64_t* launches)
{
    int64_t nt = scan_tiles(n);
    if (nt < 1) nt = 1;
    launch_g<k_scan_reduce_g>((unsigned)nt, kBlock, s, in, n, tmp);
    if (nt <= kScanSmallTiles) {
        launch_g<k_scan_final_small_g>((unsigned)nt, kBlock, s, in, n, tmp, (int)nt, out);
        if (launches) *launches += 2;
        return;
    }
    launch_g<k_scan_tiles_g>(1, kBlock, s, tmp, (int)nt);
    launch_g<k_scan_final_g>((unsigned)nt, kBlock, s, in, n, tmp, (int)nt, out);
    if (launches) *launches += 3;
}

}  // namespace slak
