// Hole fill after a move (removal compaction).
//
// Holes are the set bits of the removal bitmap the move kernels write (one 32-bit
// word per warp of particles).  The k-th hole in ascending order is paired with the
// k-th live particle counted from the back; pairs are kept while the live particle
// lies behind the hole and k < remove_count.  Both sequences are monotone, so the
// kept pairs are a prefix: exactly the pairs of the reference's sequential loop
// (opp_lib/src/core/opp_particle_organize_core.cpp:124-218).
//   1. per-block hole counts over the bitmap,
//   2. exclusive scan of the block counts,
//   3. emit hole[k] and mover[k] for k < remove_count (ranks from the scan),
//   4. copy every dat element mover[k] -> hole[k] for the kept pairs.

#include <climits>
#include <mutex>

#include "oppb_graph.h"
#include "scan.cuh"

namespace oppb {
namespace {

constexpr int kHfBlock = 256;
// Two bitmap words (64 particles) a thread: the threads over the last live particles emit the
// movers bit by bit, so this bounds the longest thread of the emit kernel.
constexpr int kHfWordsPerThread = 2;
constexpr int kHfWords = kHfBlock * kHfWordsPerThread;  // words per block (16,384 particles)
constexpr int kMaxDats = 16;

struct DatList {
    int32_t n;
    int32_t total_cols;
    void* data[kMaxDats];
    int32_t dim[kMaxDats];
    int32_t bytes[kMaxDats];
};

// A count of a launch: the host's value, or (dev != nullptr) the value in device memory plus
// `add`, capped by the host's value, which is then its upper bound (include/oppb_graph.h).
struct CountArg {
    int32_t host;
    const int32_t* dev;
    int32_t add;
};

__device__ __forceinline__ int32_t resolve(const CountArg& c) {
    if (!c.dev) return c.host;
    const int32_t v = *c.dev + c.add;
    return v < 0 ? 0 : (v < c.host ? v : c.host);
}

// Bitmap word w restricted to particles < size.
__device__ __forceinline__ uint32_t hole_word(const uint32_t* bits, int64_t w, int32_t size) {
    const int64_t first = w * 32;
    if (first >= size) return 0u;
    uint32_t v = bits[w];
    const int64_t valid = size - first;
    if (valid < 32) v &= (1u << valid) - 1u;
    return v;
}

__global__ void __launch_bounds__(kHfBlock) hf_count_kernel(const uint32_t* __restrict__ bits, CountArg size_arg,
                                                            int64_t n_words, int* __restrict__ block_holes) {
    __shared__ int sm[kHfBlock / 32 + 1];
    const int32_t size = resolve(size_arg);
    const int64_t w0 = (int64_t)blockIdx.x * kHfWords;
    int c = 0;
#pragma unroll
    for (int k = 0; k < kHfWordsPerThread; k++) {
        const int64_t w = w0 + (int64_t)k * kHfBlock + threadIdx.x;
        if (w < n_words) c += __popc(hole_word(bits, w, size));
    }
    int total;
    block_exclusive_scan(c, sm, &total);
    if (threadIdx.x == 0) block_holes[blockIdx.x] = total;
}

// block_base: exclusive hole prefix per block, block_base[n_blocks] = total holes H.
__global__ void __launch_bounds__(kHfBlock) hf_emit_kernel(const uint32_t* __restrict__ bits, CountArg size_arg,
                                                           int64_t n_words, const int* __restrict__ block_base,
                                                           int n_blocks, CountArg remove_arg,
                                                           int32_t* __restrict__ hole_list,
                                                           int32_t* __restrict__ mover_list) {
    __shared__ int sm[kHfBlock / 32 + 1];
    const int32_t size = resolve(size_arg);
    const int32_t remove_count = resolve(remove_arg);
    // Thread t owns words [w0 + t*8, w0 + t*8 + 8) (blocked, so ranks follow index order).
    const int64_t wt = (int64_t)blockIdx.x * kHfWords + (int64_t)threadIdx.x * kHfWordsPerThread;
    uint32_t w[kHfWordsPerThread];
    int c = 0;
#pragma unroll
    for (int k = 0; k < kHfWordsPerThread; k++) {
        w[k] = (wt + k < n_words) ? hole_word(bits, wt + k, size) : 0u;
        c += __popc(w[k]);
    }
    int total;
    int holes_before = block_exclusive_scan(c, sm, &total) + block_base[blockIdx.x];
    const int64_t H = block_base[n_blocks];
    const int64_t live_total = (int64_t)size - H;
#pragma unroll 1
    for (int k = 0; k < kHfWordsPerThread; k++) {
        const int64_t word = wt + k;
        const int64_t first = word * 32;
        if (first >= size) break;
        const int n_valid = (size - first) < 32 ? (int)(size - first) : 32;
        uint32_t hw = w[k];
        // Holes: ascending rank holes_before, holes_before+1, ...
        if (holes_before < remove_count) {
            uint32_t m = hw;
            int h = holes_before;
            while (m && h < remove_count) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                hole_list[h++] = (int32_t)(first + b);
            }
        }
        // Live particles: back rank = live_total - 1 - (index - holes before index).
        // The largest live index of this word has the smallest back rank.
        const int64_t live_first_rank = first - holes_before;  // front rank of first live in word
        const int n_live = n_valid - __popc(hw);
        if (n_live > 0) {
            const int64_t min_back = live_total - 1 - (live_first_rank + n_live - 1);
            if (min_back < remove_count) {
                int64_t front = live_first_rank;
                for (int b = 0; b < n_valid; b++) {
                    if (hw & (1u << b)) continue;
                    const int64_t back = live_total - 1 - front;
                    if (back < remove_count) mover_list[back] = (int32_t)(first + b);
                    front++;
                }
            }
        }
        holes_before += __popc(hw);
    }
}

// One (pair, column) per thread and pass of a grid-stride loop: copies the element of column
// col of the mover to the hole.  The pair index runs fastest, so a warp reads consecutive
// entries of the two lists and, the movers being the last live particles in descending order,
// neighbouring elements of one column; only the writes to the holes scatter.
__global__ void hf_copy_kernel(CountArg pairs_arg, const int32_t* __restrict__ hole_list,
                               const int32_t* __restrict__ mover_list, const int* __restrict__ totals,
                               CountArg size_arg, int32_t stride, DatList dats) {
    const int64_t n_pairs_max = resolve(pairs_arg);
    const int64_t size = resolve(size_arg);
    const int64_t H = totals[0];
    const int64_t n_items = n_pairs_max * dats.total_cols;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_items;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int col = (int)(t / n_pairs_max);
        const int64_t k = t - (int64_t)col * n_pairs_max;
        if (k >= H || k >= size - H) continue;
        const int32_t to = hole_list[k], from = mover_list[k];
        if (from <= to) continue;
        int d = 0, c = col;
        while (d < dats.n && c >= dats.dim[d]) {
            c -= dats.dim[d];
            d++;
        }
        if (d >= dats.n) continue;
        const int64_t off = (int64_t)c * stride;
        if (dats.bytes[d] == 8) {
            int64_t* a = reinterpret_cast<int64_t*>(dats.data[d]) + off;
            a[to] = a[from];
        } else {
            int32_t* a = reinterpret_cast<int32_t*>(dats.data[d]) + off;
            a[to] = a[from];
        }
    }
}

// Closes a device-sized step (one thread): the step record, the first error, the new count.
__global__ void step_end_kernel(oppb_set_count* cnt, int32_t pending, const oppb_move_status* st,
                                oppb_step_record* records, int32_t n_records) {
    const int32_t n = cnt->size + pending;
    const int32_t removed = st->remove_count;
    oppb_step_record r;
    r.size_before_move = n;
    r.removed = removed;
    r.size = n - removed;
    r.max_visits = st->max_visits;
    r.total_visits = st->total_visits;
    r.recheck_count = st->recheck_count;
    r.error = st->error;
    const int32_t step = cnt->steps;
    if (records && n_records > 0) records[step % n_records] = r;
    if (st->error && !cnt->error) {
        cnt->error = st->error;
        cnt->error_step = step;
    }
    cnt->size = n - removed;
    cnt->steps = step + 1;
}

// bits[w] bit b = (p2c[32 w + b] == removed) over [0, size); a warp writes one word, bits past
// size are 0.
__global__ void __launch_bounds__(256) removal_bits_kernel(const int32_t* __restrict__ p2c, int32_t size,
                                                           uint32_t* __restrict__ bits) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const bool gone = i < size && __ldg(p2c + i) == kRemoved;
    const uint32_t w = __ballot_sync(kFullMask, gone);
    if ((threadIdx.x & 31) == 0 && i < size) bits[i >> 5] = w;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace
}  // namespace oppb

extern "C" int oppb_removal_bits(const int32_t* p2c, int32_t size, uint32_t* remove_bits, void* stream) {
    using namespace oppb;
    if (size < 0 || (size > 0 && (!p2c || !remove_bits))) return OPPB_ERR_ARG;
    if (size == 0) return OPPB_OK;
    removal_bits_kernel<<<ceil_div(size, 256), 256, 0, as_stream(stream)>>>(p2c, size, remove_bits);
    count_launches(1);
    return launch_status();
}

extern "C" size_t oppb_hole_fill_workspace_bytes(int32_t size, int32_t remove_count) {
    using namespace oppb;
    if (size < 0 || remove_count < 0) return 0;
    const int64_t n_words = ceil_div(size, 32);
    const int n_blocks = ceil_div(n_words, kHfWords);
    return align256(sizeof(int) * (size_t)(n_blocks + 1)) + align256(sizeof(int) * scan_scratch_ints(n_blocks)) +
           2 * align256(sizeof(int32_t) * (size_t)(remove_count > 0 ? remove_count : 1));
}

extern "C" int oppb_hole_fill(int32_t size, int32_t remove_count, const uint32_t* remove_bits, int32_t stride,
                              int32_t n_dats, const oppb_dat* dats, void* workspace, size_t workspace_bytes,
                              void* stream) {
    using namespace oppb;
    if (size < 0 || remove_count < 0 || stride < size || n_dats < 0 || n_dats > kMaxDats) return OPPB_ERR_ARG;
    if (remove_count == 0 || size == 0) return OPPB_OK;
    if (!remove_bits || !dats || !workspace) return OPPB_ERR_ARG;
    if (workspace_bytes < oppb_hole_fill_workspace_bytes(size, remove_count)) return OPPB_ERR_WORKSPACE;
    DatList dl{};
    dl.n = n_dats;
    dl.total_cols = 0;
    for (int d = 0; d < n_dats; d++) {
        if (!dats[d].data || dats[d].dim <= 0 || (dats[d].elem_bytes != 4 && dats[d].elem_bytes != 8))
            return OPPB_ERR_ARG;
        dl.data[d] = dats[d].data;
        dl.dim[d] = dats[d].dim;
        dl.bytes[d] = dats[d].elem_bytes;
        dl.total_cols += dats[d].dim;
    }
    cudaStream_t s = as_stream(stream);
    const int64_t n_words = ceil_div(size, 32);
    const int n_blocks = ceil_div(n_words, kHfWords);
    char* ws = static_cast<char*>(workspace);
    int* block_base = reinterpret_cast<int*>(ws);
    ws += align256(sizeof(int) * (size_t)(n_blocks + 1));
    int* scan_tmp = reinterpret_cast<int*>(ws);
    ws += align256(sizeof(int) * scan_scratch_ints(n_blocks));
    int32_t* hole_list = reinterpret_cast<int32_t*>(ws);
    ws += align256(sizeof(int32_t) * (size_t)remove_count);
    int32_t* mover_list = reinterpret_cast<int32_t*>(ws);

    const CountArg sz{size, nullptr, 0}, rc{remove_count, nullptr, 0};
    hf_count_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base);
    // block_base[0..n_blocks) exclusive, block_base[n_blocks] = total holes.
    scan_single_block_kernel<<<1, kScanBlock, 0, s>>>(block_base, n_blocks);
    (void)scan_tmp;
    hf_emit_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base, n_blocks, rc, hole_list,
                                                 mover_list);
    count_launches(3);
    if (dl.total_cols > 0) {
        const int64_t threads = (int64_t)remove_count * dl.total_cols;
        hf_copy_kernel<<<ceil_div(threads, 256), 256, 0, s>>>(rc, hole_list, mover_list, block_base + n_blocks, sz,
                                                             stride, dl);
        count_launches(1);
    }
    return launch_status();
}

extern "C" size_t oppb_hole_fill_dev_workspace_bytes(int32_t size_bound) {
    return oppb_hole_fill_workspace_bytes(size_bound, size_bound);
}

extern "C" int oppb_hole_fill_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                                  const oppb_move_status* status, const uint32_t* remove_bits, int32_t stride,
                                  int32_t n_dats, const oppb_dat* dats, void* workspace, size_t workspace_bytes,
                                  void* stream) {
    using namespace oppb;
    if (size_bound < 0 || pending < 0 || stride < size_bound || n_dats < 0 || n_dats > kMaxDats) return OPPB_ERR_ARG;
    if (!count || !status) return OPPB_ERR_ARG;
    if (size_bound == 0) return OPPB_OK;
    if (!remove_bits || !dats || !workspace) return OPPB_ERR_ARG;
    if (workspace_bytes < oppb_hole_fill_dev_workspace_bytes(size_bound)) return OPPB_ERR_WORKSPACE;
    DatList dl{};
    dl.n = n_dats;
    dl.total_cols = 0;
    for (int d = 0; d < n_dats; d++) {
        if (!dats[d].data || dats[d].dim <= 0 || (dats[d].elem_bytes != 4 && dats[d].elem_bytes != 8))
            return OPPB_ERR_ARG;
        dl.data[d] = dats[d].data;
        dl.dim[d] = dats[d].dim;
        dl.bytes[d] = dats[d].elem_bytes;
        dl.total_cols += dats[d].dim;
    }
    cudaStream_t s = as_stream(stream);
    const int64_t n_words = ceil_div(size_bound, 32);
    const int n_blocks = ceil_div(n_words, kHfWords);
    char* ws = static_cast<char*>(workspace);
    int* block_base = reinterpret_cast<int*>(ws);
    ws += align256(sizeof(int) * (size_t)(n_blocks + 1));
    ws += align256(sizeof(int) * scan_scratch_ints(n_blocks));
    int32_t* hole_list = reinterpret_cast<int32_t*>(ws);
    ws += align256(sizeof(int32_t) * (size_t)size_bound);
    int32_t* mover_list = reinterpret_cast<int32_t*>(ws);
    // The count and the move's remove count are read on the device; the lists hold up to
    // size_bound pairs, and no more than the count can be removed.
    const CountArg sz{size_bound, &count->size, pending};
    const CountArg rc{size_bound, &status->remove_count, 0};
    hf_count_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base);
    scan_single_block_kernel<<<1, kScanBlock, 0, s>>>(block_base, n_blocks);
    hf_emit_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base, n_blocks, rc, hole_list,
                                                 mover_list);
    count_launches(3);
    if (dl.total_cols > 0) {
        const int64_t items = (int64_t)size_bound * dl.total_cols;
        const int grid = ceil_div(items, 256) < 148 * 16 ? ceil_div(items, 256) : 148 * 16;
        hf_copy_kernel<<<grid, 256, 0, s>>>(rc, hole_list, mover_list, block_base + n_blocks, sz, stride, dl);
        count_launches(1);
    }
    return launch_status();
}

extern "C" int oppb_step_end_dev(oppb_set_count* count, int32_t pending, const oppb_move_status* status,
                                 oppb_step_record* records, int32_t n_records, void* stream) {
    using namespace oppb;
    if (!count || !status || pending < 0 || n_records < 0 || (n_records > 0 && !records)) return OPPB_ERR_ARG;
    step_end_kernel<<<1, 1, 0, as_stream(stream)>>>(count, pending, status, records, n_records);
    count_launches(1);
    return launch_status();
}

// ------------------------------------------------------- allocation-free hole fill
//
// oppb_hole_fill_static runs the same four kernels as oppb_hole_fill with its scratch in
// a fixed array of this library instead of a caller workspace, for callers that cannot
// allocate device memory where they move particles (a plugin that sees only the dats'
// device pointers while another runtime owns the memory, or a loop that cannot afford
// the device-wide synchronisation of cudaMalloc / cudaFree).
//
// Layout of the array (int32 words): per-block hole counts for the largest possible
// particle count (their scan leaves the total at [n_blocks]), then the hole list and the
// mover list of OPPB_HOLE_FILL_STATIC_MAX_REMOVES entries each.  Every word a call reads
// was written earlier in the same call, so nothing has to start at zero and the contents
// left by the previous call are harmless.  All calls on a device share the array: calls
// that overlap on the GPU race.

namespace oppb {
namespace {

constexpr int64_t kStaticMaxBlocks = (((int64_t)INT_MAX + 31) / 32 + kHfWords - 1) / kHfWords;  // 131,072
constexpr int64_t kStaticBaseWords = (kStaticMaxBlocks + 1 + 63) / 64 * 64;  // whole 256-B lines
constexpr int64_t kStaticListWords = OPPB_HOLE_FILL_STATIC_MAX_REMOVES;
constexpr int64_t kStaticWords = kStaticBaseWords + 2 * kStaticListWords;  // about 8.5 MiB

}  // namespace

// Held by every GPU that loads the library, until the process exits.
static __device__ __align__(256) int32_t g_hole_fill_scratch[kStaticWords];

namespace {

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
int32_t* g_static_addr[kStaticMaxDevices];  // device address of g_hole_fill_scratch, per device

// Device address of the scratch array on the current device.  In host code the array's name
// only stands in for the symbol; a kernel must be given this address instead.  It is looked
// up again on every call made outside a stream capture (cheap once the module is loaded), so
// that a device reset, which unloads the module and may place the array elsewhere when it is
// loaded again, never leaves a stale address behind; a call inside a capture uses the address
// found by the last call outside one.
int static_scratch(cudaStream_t stream, int32_t** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return OPPB_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kStaticMaxDevices) return OPPB_ERR_NO_DEVICE;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
        cudaGetLastError();
        return OPPB_ERR_LAUNCH;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev] || cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_hole_fill_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return OPPB_ERR_LAUNCH;
        }
        g_static_addr[dev] = static_cast<int32_t*>(p);
    }
    *out = g_static_addr[dev];
    return OPPB_OK;
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_hole_fill_static(int32_t size, int32_t remove_count, const uint32_t* remove_bits,
                                     int32_t stride, int32_t n_dats, const oppb_dat* dats, void* stream) {
    using namespace oppb;
    if (size < 0 || remove_count < 0 || stride < size || n_dats < 0 || n_dats > kMaxDats) return OPPB_ERR_ARG;
    if (remove_count > OPPB_HOLE_FILL_STATIC_MAX_REMOVES) return OPPB_ERR_SCRATCH_LIMIT;
    if (remove_count == 0 || size == 0) return OPPB_OK;
    if (!remove_bits || !dats) return OPPB_ERR_ARG;
    DatList dl{};
    dl.n = n_dats;
    dl.total_cols = 0;
    for (int d = 0; d < n_dats; d++) {
        if (!dats[d].data || dats[d].dim <= 0 || (dats[d].elem_bytes != 4 && dats[d].elem_bytes != 8))
            return OPPB_ERR_ARG;
        dl.data[d] = dats[d].data;
        dl.dim[d] = dats[d].dim;
        dl.bytes[d] = dats[d].elem_bytes;
        dl.total_cols += dats[d].dim;
    }
    cudaStream_t s = as_stream(stream);
    int32_t* scratch = nullptr;
    const int lookup = static_scratch(s, &scratch);
    if (lookup != OPPB_OK) return lookup;
    const int64_t n_words = ceil_div(size, 32);
    const int n_blocks = ceil_div(n_words, kHfWords);  // <= kStaticMaxBlocks for any int32 size
    int* block_base = scratch;
    int32_t* hole_list = scratch + kStaticBaseWords;
    int32_t* mover_list = hole_list + kStaticListWords;

    const CountArg sz{size, nullptr, 0}, rc{remove_count, nullptr, 0};
    hf_count_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base);
    scan_single_block_kernel<<<1, kScanBlock, 0, s>>>(block_base, n_blocks);
    hf_emit_kernel<<<n_blocks, kHfBlock, 0, s>>>(remove_bits, sz, n_words, block_base, n_blocks, rc, hole_list,
                                                 mover_list);
    count_launches(3);
    if (dl.total_cols > 0) {
        const int64_t threads = (int64_t)remove_count * dl.total_cols;
        hf_copy_kernel<<<ceil_div(threads, 256), 256, 0, s>>>(rc, hole_list, mover_list, block_base + n_blocks, sz,
                                                             stride, dl);
        count_launches(1);
    }
    return launch_status();
}
