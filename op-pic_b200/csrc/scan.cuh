// Block- and device-wide exclusive prefix sums of int32 used by the hole fill and
// the radix sort.  Scratch comes from the caller's workspace.
#pragma once

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanBlock * kScanItems;

// Exclusive scan of one value per thread across a block of kScanBlock threads.
// Returns the exclusive prefix; *total receives the block sum.  smem needs
// kScanBlock/32 + 1 ints.
__device__ __forceinline__ int block_exclusive_scan(int v, int* smem, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < kScanBlock / 32) ? smem[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFullMask, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kScanBlock / 32) smem[lane] = wi - w;
        if (lane == kScanBlock / 32 - 1) smem[kScanBlock / 32] = wi;
    }
    __syncthreads();
    const int res = smem[warp] + incl - v;
    *total = smem[kScanBlock / 32];
    __syncthreads();
    return res;
}

// Per-tile sums of in[0,n).
__global__ void __launch_bounds__(kScanBlock) scan_tile_sums_kernel(const int* __restrict__ in, int64_t n,
                                                                   int* __restrict__ tile_sums) {
    __shared__ int sm[kScanBlock / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int64_t j = base + (int64_t)k * kScanBlock + threadIdx.x;
        if (j < n) s += in[j];
    }
    int total;
    block_exclusive_scan(s, sm, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// In-place exclusive scan of a[0,n) by one block, kScanTile values a pass (coalesced loads into
// shared memory, kScanItems consecutive values a thread); a[n] receives the total.
__global__ void __launch_bounds__(kScanBlock) scan_single_block_kernel(int* a, int n) {
    __shared__ int tile[kScanTile];
    __shared__ int sm[kScanBlock / 32 + 1];
    int carry = 0;
    for (int base = 0; base < n; base += kScanTile) {
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const int j = base + k * kScanBlock + threadIdx.x;
            tile[k * kScanBlock + threadIdx.x] = (j < n) ? a[j] : 0;
        }
        __syncthreads();
        int vals[kScanItems];
        int s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            vals[k] = tile[threadIdx.x * kScanItems + k];
            s += vals[k];
        }
        int total;
        int run = block_exclusive_scan(s, sm, &total) + carry;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            tile[threadIdx.x * kScanItems + k] = run;
            run += vals[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const int j = base + k * kScanBlock + threadIdx.x;
            if (j < n) a[j] = tile[k * kScanBlock + threadIdx.x];
        }
        carry += total;
        __syncthreads();  // the next pass overwrites the tile
    }
    if (threadIdx.x == 0) a[n] = carry;
}

// out[j] = tile_prefix[tile] + exclusive prefix of in within the tile (in-place allowed).
__global__ void __launch_bounds__(kScanBlock) scan_apply_kernel(const int* in, int* out, int64_t n,
                                                               const int* __restrict__ tile_prefix) {
    __shared__ int tile[kScanTile];
    __shared__ int sm[kScanBlock / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int64_t j = base + (int64_t)k * kScanBlock + threadIdx.x;
        tile[k * kScanBlock + threadIdx.x] = (j < n) ? in[j] : 0;
    }
    __syncthreads();
    int vals[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        vals[k] = tile[threadIdx.x * kScanItems + k];
        s += vals[k];
    }
    int total;
    int run = block_exclusive_scan(s, sm, &total) + tile_prefix[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        tile[threadIdx.x * kScanItems + k] = run;
        run += vals[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int64_t j = base + (int64_t)k * kScanBlock + threadIdx.x;
        if (j < n) out[j] = tile[k * kScanBlock + threadIdx.x];
    }
}

// Scratch ints a device-wide scan of n values needs (tile sums + total).
inline size_t scan_scratch_ints(int64_t n) { return (size_t)ceil_div(n, kScanTile) + 1; }

// Exclusive scan of in[0,n) into out[0,n) (in-place allowed); scratch[num_tiles] = total.
inline void device_exclusive_scan(const int* in, int* out, int64_t n, int* scratch, cudaStream_t s) {
    const int tiles = ceil_div(n, kScanTile);
    if (tiles == 0) return;
    scan_tile_sums_kernel<<<tiles, kScanBlock, 0, s>>>(in, n, scratch);
    scan_single_block_kernel<<<1, kScanBlock, 0, s>>>(scratch, tiles);
    scan_apply_kernel<<<tiles, kScanBlock, 0, s>>>(in, out, n, scratch);
    count_launches(3);
}

}  // namespace
}  // namespace oppb
