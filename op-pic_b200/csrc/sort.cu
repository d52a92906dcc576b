// Stable cell sort of particles: hand-written LSD radix sort (8-bit digits) of the
// cell keys with the particle index as value, then one gather of every dat.
//
// Key of particle i: p2c[i], or n_cells for a removed particle (so removed particles
// sort last, as MAX_CELL_INDEX does in sort_iota_by_key, opp_lib/include/opp_util.h:211-221).
// Each pass: (1) per-tile digit histogram, (2) exclusive scan of the digit-major
// histogram table, (3) per tile a stable rank of every key among equal digits
// (warp match + per-warp digit counters, warps in index order), staging in shared
// memory so each digit run is written out contiguously.  The last pass writes the
// sorted keys straight into the p2c swap buffer and the source indices (the
// permutation) for the gather.

#include "oppb_graph.h"
#include "scan.cuh"

namespace oppb {
namespace {

// The particle count of a sort: the host's, or (dev != nullptr) the device count plus `add`
// capped by the host's value, which is then an upper bound (include/oppb_graph.h).  With
// remove_dev, a zero remove count turns the sort into a plain copy into the swap buffers.
struct SortCount {
    int32_t host;
    const int32_t* dev;
    int32_t add;
    const int32_t* remove_dev;
};

__device__ __forceinline__ int32_t sort_size(const SortCount& c) {
    if (!c.dev) return c.host;
    const int32_t v = *c.dev + c.add;
    return v < 0 ? 0 : (v < c.host ? v : c.host);
}

__device__ __forceinline__ bool sort_is_copy(const SortCount& c) { return c.remove_dev && *c.remove_dev == 0; }

constexpr int kSortBlock = 256;
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortBlock * kSortItems;  // 2048 keys
constexpr int kScatterMinBlocks = 5;  // 48 registers: the scatter is latency-bound, occupancy pays
constexpr int kRadix = 256;
constexpr int kMaxDats = 16;

__device__ __forceinline__ uint32_t cell_key(int32_t c, int32_t n_cells) {
    return ((uint32_t)c < (uint32_t)n_cells) ? (uint32_t)c : (uint32_t)n_cells;
}

// Shuffle key of particle j (Shuffle_All / Shuffle_Periodic): 30 random bits from a
// splitmix64 hash of (seed, j) for a particle with a valid cell, 2^30 for a removed one, so
// that removed particles still sort last.  The reference draws its keys with Thrust's
// default engine seeded 123 (opp_lib/src/cuda/opp_particle_sorter.cu:40-54,195-201); only the
// rule (random keys, removed last, stable sort) is kept, not the draws.
constexpr uint32_t kShuffleRemoved = 1u << 30;

__device__ __forceinline__ uint32_t shuffle_key(uint64_t seed, int64_t j, int32_t c, int32_t n_cells) {
    if ((uint32_t)c >= (uint32_t)n_cells) return kShuffleRemoved;
    uint64_t z = seed + 0x9e3779b97f4a7c15ull * (uint64_t)(j + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (uint32_t)(z >> 34);
}

// Pass input: either raw p2c (first pass) or keys from the previous pass.
struct PassIn {
    const int32_t* p2c;     // first pass only
    const uint32_t* keys;   // later passes
    const int32_t* vals;    // later passes (first pass: value = index)
    uint64_t shuffle_seed;  // first pass: 0 = cell keys, else shuffle keys
};

__device__ __forceinline__ uint32_t load_key(const PassIn& in, int64_t j, int32_t n_cells) {
    if (!in.p2c) return in.keys[j];
    const int32_t c = in.p2c[j];
    return in.shuffle_seed ? shuffle_key(in.shuffle_seed, j, c, n_cells) : cell_key(c, n_cells);
}

__global__ void __launch_bounds__(kSortBlock) radix_hist_kernel(PassIn in, SortCount cnt, int32_t n_cells,
                                                                int shift, int n_tiles, int* __restrict__ hist) {
    __shared__ int h[kRadix];
    const int32_t size = sort_size(cnt);
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; k++) {
        const int64_t j = base + (int64_t)k * kSortBlock + threadIdx.x;
        if (j < size) atomicAdd(&h[(load_key(in, j, n_cells) >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// offsets: exclusive scan of hist (digit-major), i.e. the first output slot of
// (digit, tile).  keys_out/vals_out receive the pass result.  On the last pass
// keys_out is the p2c swap buffer (removed key mapped back to the removed cell).
__global__ void __launch_bounds__(kSortBlock, kScatterMinBlocks) radix_scatter_kernel(PassIn in, SortCount count, int32_t n_cells,
                                                                   int shift, int n_tiles,
                                                                   const int* __restrict__ offsets,
                                                                   uint32_t* __restrict__ keys_out,
                                                                   int32_t* __restrict__ vals_out, int last,
                                                                   int32_t* __restrict__ inv_out) {
    const int32_t size = sort_size(count);
    if (sort_is_copy(count) || (int64_t)blockIdx.x * kSortTile >= size) return;  // whole block
    __shared__ int cnt[kSortWarps][kRadix];
    __shared__ int tile_base[kRadix];
    __shared__ int scan_sm[kSortBlock / 32 + 1];
    __shared__ uint32_t sk[kSortTile];
    __shared__ int32_t sv[kSortTile];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kSortWarps * kRadix; d += kSortBlock) (&cnt[0][0])[d] = 0;
    __syncthreads();

    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    const int tile_n = ((int64_t)size - base) < kSortTile ? (int)((int64_t)size - base) : kSortTile;
    uint32_t key[kSortItems];
    int32_t val[kSortItems];
    int off[kSortItems];
    const unsigned lt = lanemask_lt();
    // Warp w ranks tile items [w*256, w*256+256) in 8 rounds of 32, in index order.
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
        const int t = warp * (kSortItems * 32) + r * 32 + lane;
        const int64_t j = base + t;
        const bool ok = t < tile_n;
        key[r] = ok ? load_key(in, j, n_cells) : 0xffffffffu;
        val[r] = ok ? (in.p2c ? (int32_t)j : in.vals[j]) : 0;
        const int d = ok ? (int)((key[r] >> shift) & (kRadix - 1)) : kRadix;
        const unsigned peers = __match_any_sync(kFullMask, d);
        const int leader = __ffs(peers) - 1;
        int b = 0;
        if (lane == leader && ok) b = cnt[warp][d];
        b = __shfl_sync(kFullMask, b, leader);
        off[r] = b + __popc(peers & lt);
        __syncwarp();
        if (lane == leader && ok) cnt[warp][d] = b + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // Per digit: exclusive prefix over warps, then the tile-local digit base.
    {
        const int d = threadIdx.x;
        int run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) {
            const int c = cnt[w][d];
            cnt[w][d] = run;
            run += c;
        }
        int total;
        tile_base[d] = block_exclusive_scan(run, scan_sm, &total);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
        const int t = warp * (kSortItems * 32) + r * 32 + lane;
        if (t < tile_n) {
            const int d = (int)((key[r] >> shift) & (kRadix - 1));
            const int pos = tile_base[d] + cnt[warp][d] + off[r];
            sk[pos] = key[r];
            sv[pos] = val[r];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < tile_n; t += kSortBlock) {
        const uint32_t k = sk[t];
        const int d = (int)((k >> shift) & (kRadix - 1));
        const int64_t dest = (int64_t)offsets[(int64_t)d * n_tiles + blockIdx.x] + (t - tile_base[d]);
        if (last)
            reinterpret_cast<int32_t*>(keys_out)[dest] = (k >= (uint32_t)n_cells) ? kRemoved : (int32_t)k;
        else
            keys_out[dest] = k;
        vals_out[dest] = sv[t];
        if (inv_out) inv_out[sv[t]] = (int32_t)dest;  // the scatter form's destination of each source
    }
}

constexpr int kMaxCols = 16;  // gathered columns per launch

// One column of a dat: element j of column c lives at src + (c * stride + j) * bytes.
struct GatherCols {
    int32_t n;
    const char* src[kMaxCols];
    char* dst[kMaxCols];
    int32_t bytes[kMaxCols];
};

// L2 eviction policies (createpolicy, sm_80+): the gathered sources are reused by neighbouring
// destinations (a 32-B sector holds four particles of one column that end up within a few
// hundred thousand destinations of each other), so their lines are kept in L2 ahead of the
// streaming destination writes and the permutation, which are touched once.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ long long ld_keep(const long long* p, uint64_t pol) {
    long long v;
    asm("ld.global.nc.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_keep(const int* p, uint64_t pol) {
    int v;
    asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// dst[c][j] = src[c][perm[j]] for every column of every dat other than the key dat.
// All loads of a particle are issued before its stores, so each thread keeps up to
// kMaxCols loads in flight.  When the sort is a copy (device count, no removal), perm is
// not read (from = j) and the key column (key_src -> key_dst) is copied too.
__global__ void __launch_bounds__(256) gather_kernel(SortCount cnt, const int32_t* __restrict__ perm, GatherCols g,
                                                     const int32_t* __restrict__ key_src, int32_t* __restrict__ key_dst) {
    const int32_t size = sort_size(cnt);
    const int64_t j = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (j >= size) return;
    const bool copy = sort_is_copy(cnt);
    const int64_t from = copy ? j : __ldcs(perm + j);
    if (copy && key_src) key_dst[j] = key_src[j];
    const uint64_t keep = l2_policy_evict_last();
    uint64_t v[kMaxCols];
#pragma unroll
    for (int c = 0; c < kMaxCols; c++) {
        if (c < g.n) {
            if (g.bytes[c] == 8)
                v[c] = (uint64_t)ld_keep(reinterpret_cast<const long long*>(g.src[c]) + from, keep);
            else
                v[c] = (uint32_t)ld_keep(reinterpret_cast<const int*>(g.src[c]) + from, keep);
        }
    }
#pragma unroll
    for (int c = 0; c < kMaxCols; c++) {
        if (c < g.n) {
            if (g.bytes[c] == 8)
                __stcs(reinterpret_cast<long long*>(g.dst[c]) + j, (long long)v[c]);
            else
                __stcs(reinterpret_cast<int*>(g.dst[c]) + j, (int)v[c]);
        }
    }
}

// The scatter form of the dat move (oppb_tuning.sort_scatter): thread i reads every column of
// source particle i (coalesced) and writes it to its destination inv[i] (scattered 8-B and 4-B
// stores, merged into whole sectors in L2 when neighbouring destinations arrive close in time);
// the gather form reads scattered and writes coalesced.  Same result.
__global__ void __launch_bounds__(256) scatter_cols_kernel(SortCount cnt, const int32_t* __restrict__ inv, GatherCols g,
                                                           const int32_t* __restrict__ key_src,
                                                           int32_t* __restrict__ key_dst) {
    const int32_t size = sort_size(cnt);
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= size) return;
    const bool copy = sort_is_copy(cnt);
    const int64_t to = copy ? i : inv[i];
    if (copy && key_src) key_dst[i] = key_src[i];
    uint64_t v[kMaxCols];
#pragma unroll
    for (int c = 0; c < kMaxCols; c++) {
        if (c < g.n) {
            if (g.bytes[c] == 8)
                v[c] = (uint64_t)__ldcs(reinterpret_cast<const long long*>(g.src[c]) + i);
            else
                v[c] = (uint32_t)__ldcs(reinterpret_cast<const int*>(g.src[c]) + i);
        }
    }
#pragma unroll
    for (int c = 0; c < kMaxCols; c++) {
        if (c < g.n) {
            if (g.bytes[c] == 8)
                reinterpret_cast<long long*>(g.dst[c])[to] = (long long)v[c];
            else
                reinterpret_cast<int*>(g.dst[c])[to] = (int)v[c];
        }
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

int key_bits(int32_t n_cells) {
    int b = 0;
    while (b < 31 && ((uint32_t)n_cells >> b) != 0) b++;
    return b > 0 ? b : 1;
}

struct SortLayout {
    size_t keys_a, vals_a, keys_b, vals_b, perm, inv, hist, scan, total;
};

SortLayout sort_layout(int32_t size) {
    SortLayout L{};
    const size_t n = (size_t)(size > 0 ? size : 1);
    const int n_tiles = ceil_div(size > 0 ? size : 1, kSortTile);
    const size_t hist_n = (size_t)kRadix * n_tiles;
    size_t o = 0;
    L.keys_a = o; o += align256(4 * n);
    L.vals_a = o; o += align256(4 * n);
    L.keys_b = o; o += align256(4 * n);
    L.vals_b = o; o += align256(4 * n);
    L.perm = o;   o += align256(4 * n);
    L.inv = o;    o += align256(4 * n);
    L.hist = o;   o += align256(4 * hist_n);
    L.scan = o;   o += align256(4 * scan_scratch_ints((int64_t)hist_n));
    L.total = o;
    return L;
}

}  // namespace
}  // namespace oppb

extern "C" size_t oppb_sort_workspace_bytes(int32_t size, int32_t n_cells) {
    (void)n_cells;
    if (size < 0) return 0;
    return oppb::sort_layout(size).total;
}

namespace oppb {
namespace {

// The sort's launches for `size` particles (the host count, or the bound in device-count mode).
// shuffle_seed != 0: sort by shuffle keys instead of cells; the key dat is then gathered like
// the others.
int launch_sort(const SortCount& cnt, int32_t size, int32_t n_cells, int32_t stride, int32_t n_dats,
                const oppb_dat* dats, int32_t key_dat, int32_t* perm_out, void* workspace, cudaStream_t s,
                uint64_t shuffle_seed = 0) {
    const oppb_dat& kd = dats[key_dat];
    const SortLayout L = sort_layout(size);
    char* ws = static_cast<char*>(workspace);
    uint32_t* keys[2] = {reinterpret_cast<uint32_t*>(ws + L.keys_a), reinterpret_cast<uint32_t*>(ws + L.keys_b)};
    int32_t* vals[2] = {reinterpret_cast<int32_t*>(ws + L.vals_a), reinterpret_cast<int32_t*>(ws + L.vals_b)};
    int32_t* perm = perm_out ? perm_out : reinterpret_cast<int32_t*>(ws + L.perm);
    const bool scatter = tuning().sort_scatter != 0;
    int32_t* inv = scatter ? reinterpret_cast<int32_t*>(ws + L.inv) : nullptr;
    int* hist = reinterpret_cast<int*>(ws + L.hist);
    int* scan_tmp = reinterpret_cast<int*>(ws + L.scan);

    const int n_tiles = ceil_div(size, kSortTile);
    const bool shuffle = shuffle_seed != 0;
    const int passes = shuffle ? 4 : (key_bits(n_cells) + 7) / 8;  // shuffle keys: 31 bits
    PassIn in{static_cast<const int32_t*>(kd.data), nullptr, nullptr, shuffle_seed};
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        const bool last = (p == passes - 1);
        uint32_t* ko = (last && !shuffle) ? static_cast<uint32_t*>(kd.swap) : keys[p & 1];
        int32_t* vo = last ? perm : vals[p & 1];
        radix_hist_kernel<<<n_tiles, kSortBlock, 0, s>>>(in, cnt, n_cells, shift, n_tiles, hist);
        device_exclusive_scan(hist, hist, (int64_t)kRadix * n_tiles, scan_tmp, s);
        radix_scatter_kernel<<<n_tiles, kSortBlock, 0, s>>>(in, cnt, n_cells, shift, n_tiles, hist, ko, vo,
                                                            (last && !shuffle) ? 1 : 0, last ? inv : nullptr);
        count_launches(2);
        in = PassIn{nullptr, keys[p & 1], vals[p & 1], 0};
    }
    GatherCols g{};
    const int group = tuning().sort_gather_cols < kMaxCols ? tuning().sort_gather_cols : kMaxCols;
    // The key column rides with the first gather launch (used only when the sort is a copy).
    const int32_t* key_src = (cnt.remove_dev && !shuffle) ? static_cast<const int32_t*>(kd.data) : nullptr;
    int32_t* key_dst = static_cast<int32_t*>(kd.swap);
    for (int d = 0; d < n_dats; d++) {
        if (d == key_dat && !shuffle) continue;
        for (int c = 0; c < dats[d].dim; c++) {
            const size_t off = (size_t)c * stride * dats[d].elem_bytes;
            g.src[g.n] = static_cast<const char*>(dats[d].data) + off;
            g.dst[g.n] = static_cast<char*>(dats[d].swap) + off;
            g.bytes[g.n] = dats[d].elem_bytes;
            if (++g.n == group) {
                if (scatter)
                    scatter_cols_kernel<<<ceil_div(size, 256), 256, 0, s>>>(cnt, inv, g, key_src, key_dst);
                else
                    gather_kernel<<<ceil_div(size, 256), 256, 0, s>>>(cnt, perm, g, key_src, key_dst);
                count_launches(1);
                g.n = 0;
                key_src = nullptr;
            }
        }
    }
    if (g.n > 0 || key_src) {
        if (scatter)
            scatter_cols_kernel<<<ceil_div(size, 256), 256, 0, s>>>(cnt, inv, g, key_src, key_dst);
        else
            gather_kernel<<<ceil_div(size, 256), 256, 0, s>>>(cnt, perm, g, key_src, key_dst);
        count_launches(1);
    }
    return launch_status();
}

int check_sort_args(int32_t size, int32_t n_cells, int32_t stride, int32_t n_dats, const oppb_dat* dats,
                    int32_t key_dat) {
    if (size < 0 || n_cells <= 0 || n_cells >= kRemoved || stride < size || n_dats <= 0 || n_dats > kMaxDats ||
        !dats || key_dat < 0 || key_dat >= n_dats)
        return OPPB_ERR_ARG;
    const oppb_dat& kd = dats[key_dat];
    if (!kd.data || !kd.swap || kd.dim != 1 || kd.elem_bytes != 4) return OPPB_ERR_ARG;
    for (int d = 0; d < n_dats; d++)
        if (!dats[d].data || !dats[d].swap || dats[d].dim <= 0 || (dats[d].elem_bytes != 4 && dats[d].elem_bytes != 8))
            return OPPB_ERR_ARG;
    return OPPB_OK;
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_sort_by_cell(int32_t size, int32_t n_cells, int32_t stride, int32_t n_dats, const oppb_dat* dats,
                                 int32_t key_dat, int32_t* perm_out, void* workspace, size_t workspace_bytes,
                                 void* stream) {
    using namespace oppb;
    const int rc = check_sort_args(size, n_cells, stride, n_dats, dats, key_dat);
    if (rc) return rc;
    if (size == 0) return OPPB_OK;
    if (!workspace || workspace_bytes < oppb_sort_workspace_bytes(size, n_cells)) return OPPB_ERR_WORKSPACE;
    return launch_sort(SortCount{size, nullptr, 0, nullptr}, size, n_cells, stride, n_dats, dats, key_dat, perm_out,
                       workspace, as_stream(stream));
}

extern "C" size_t oppb_sort_dev_workspace_bytes(int32_t size_bound) {
    if (size_bound < 0) return 0;
    return oppb::sort_layout(size_bound).total;
}

extern "C" int oppb_sort_by_cell_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                                     const oppb_move_status* status, int32_t n_cells, int32_t stride, int32_t n_dats,
                                     const oppb_dat* dats, int32_t key_dat, void* workspace, size_t workspace_bytes,
                                     void* stream) {
    using namespace oppb;
    const int rc = check_sort_args(size_bound, n_cells, stride, n_dats, dats, key_dat);
    if (rc) return rc;
    if (!count || !status || pending < 0) return OPPB_ERR_ARG;
    if (size_bound == 0) return OPPB_OK;
    if (!workspace || workspace_bytes < oppb_sort_dev_workspace_bytes(size_bound)) return OPPB_ERR_WORKSPACE;
    const SortCount cnt{size_bound, &count->size, pending, &status->remove_count};
    return launch_sort(cnt, size_bound, n_cells, stride, n_dats, dats, key_dat, nullptr, workspace,
                       as_stream(stream));
}

extern "C" int oppb_shuffle(int32_t size, int32_t n_cells, int32_t stride, int32_t n_dats, const oppb_dat* dats,
                            int32_t key_dat, uint64_t seed, int32_t* perm_out, void* workspace,
                            size_t workspace_bytes, void* stream) {
    using namespace oppb;
    const int rc = check_sort_args(size, n_cells, stride, n_dats, dats, key_dat);
    if (rc) return rc;
    if (seed == 0) return OPPB_ERR_ARG;
    if (size == 0) return OPPB_OK;
    if (!workspace || workspace_bytes < oppb_sort_workspace_bytes(size, n_cells)) return OPPB_ERR_WORKSPACE;
    return launch_sort(SortCount{size, nullptr, 0, nullptr}, size, n_cells, stride, n_dats, dats, key_dat, perm_out,
                       workspace, as_stream(stream), seed);
}

extern "C" int oppb_shuffle_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                                const oppb_move_status* status, int32_t n_cells, int32_t stride, int32_t n_dats,
                                const oppb_dat* dats, int32_t key_dat, uint64_t seed, void* workspace,
                                size_t workspace_bytes, void* stream) {
    using namespace oppb;
    const int rc = check_sort_args(size_bound, n_cells, stride, n_dats, dats, key_dat);
    if (rc) return rc;
    if (!count || !status || pending < 0 || seed == 0) return OPPB_ERR_ARG;
    if (size_bound == 0) return OPPB_OK;
    if (!workspace || workspace_bytes < oppb_sort_dev_workspace_bytes(size_bound)) return OPPB_ERR_WORKSPACE;
    const SortCount cnt{size_bound, &count->size, pending, &status->remove_count};
    return launch_sort(cnt, size_bound, n_cells, stride, n_dats, dats, key_dat, nullptr, workspace,
                       as_stream(stream), seed);
}
