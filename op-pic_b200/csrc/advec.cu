// NESO-advection particle path: periodic position update and axis-wise multi-hop move, for a
// batch of independent instances (different meshes, particle counts and constants) in one
// persistent launch.
//
// Work is cut into 256-particle items that never straddle two instances (tile_prefix); a
// grid sized to the resident capacity of the GPU loops over the items, so instances of
// uneven size share the SMs without a launch per instance.  One thread per particle of an
// item: update_pos (apps_codegen/app_neso_advection_mdir_cg/kernels.h update_pos_kernel) in
// registers, then the hops of move_kernel (the direction chosen on the first call, x first,
// then y), reading one 32-byte cell record {c_pos_ll, c2c} per call.  This file is compiled
// with -fmad=false and the periodic wrap uses the library's FMOD (a - b * trunc(a / b),
// opp_lib/include/opp_util.h:48) with a correctly rounded divide, so positions, directions and
// cells are bit-identical to the seq backend.

#include "oppb_advec.h"
#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kAdvBlock = 256;  // = particles per work item
constexpr int kAdvWarps = kAdvBlock / 32;
enum AdvMode { kStep = 0, kUpdateOnly = 1, kMoveOnly = 2 };

// Work item w belongs to the instance i with prefix[i] <= w < prefix[i + 1].
__device__ __forceinline__ int find_instance(const int32_t* __restrict__ prefix, int n, int w) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= w)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// update_pos_kernel for one axis: x += v dt, then the periodic wrap.
__device__ __forceinline__ double update_axis(double x, double v, double dt, double extent) {
    const double offset = v * dt;
    x += offset;
    const int n_extent_offset_int = __double2int_rz(fabs(x) + 2.0);
    const double temp_pos = x + (double)n_extent_offset_int * extent;
    return temp_pos - extent * trunc(__ddiv_rn(temp_pos, extent));
}

// move_kernel's hops for one particle; returns the number of calls, sets *err on failure.
__device__ __forceinline__ int move_particle(const double* __restrict__ cells, int32_t cell_offset, int32_t n_cells,
                                             double x, double y, int& mx, int& my, int32_t& cell, double cw,
                                             double ex, double ey, int32_t max_hops, int& err) {
    int calls = 0;
    for (;;) {
        if ((uint32_t)cell >= (uint32_t)n_cells) {
            err = OPPB_ERR_CELL_RANGE;
            return calls;
        }
        calls++;
        double llx, lly, n01, n23;
        ldg256(cells + ((int64_t)cell_offset + cell) * 4, llx, lly, n01, n23);
        const double dx = x - llx;
        const double dy = y - lly;
        if (calls == 1) {  // OPP_DO_ONCE
            const bool xp = ((dx > cw) && (ex > 2 * dx - cw)) || ((dx < 0) && (ex < cw - 2 * dx));
            const bool yp = ((dy > cw) && (ey > 2 * dy - cw)) || ((dy < 0) && (ey < cw - 2 * dy));
            mx = xp ? 1 : -1;
            my = yp ? 1 : -1;
        }
        const long long a = __double_as_longlong(n01), b = __double_as_longlong(n23);
        int32_t next = -1;
        bool hop = false;
        if ((dx >= 0.0) && (dx <= cw)) {
            mx = 0;
        } else if (mx != 0) {
            next = mx > 0 ? (int32_t)(a >> 32) : (int32_t)(a & 0xffffffffll);  // xu_y : xd_y
            hop = true;
        }
        if (!hop) {
            if ((dy >= 0.0) && (dy <= cw)) {
                my = 0;
            } else if (my != 0) {
                next = my > 0 ? (int32_t)(b >> 32) : (int32_t)(b & 0xffffffffll);  // x_yu : x_yd
                hop = true;
            }
        }
        if (!hop) return calls;
        cell = next;
        if (calls >= max_hops) {
            err = OPPB_ERR_HOP_LIMIT;
            return calls;
        }
    }
}

template <int kMode>
__global__ void __launch_bounds__(kAdvBlock) advec_kernel(oppb_advec_batch b, oppb_move_status* st,
                                                          int32_t max_hops) {
    unsigned long long my_calls = 0;
    int my_max = 0;
    const int64_t sd = b.stride;
    for (int w = blockIdx.x; w < b.n_work; w += gridDim.x) {
        const int inst = find_instance(b.tile_prefix, b.n_instances, w);
        const oppb_advec_instance& I = b.instances[inst];
        const int32_t local = (w - __ldg(b.tile_prefix + inst)) * kAdvBlock + threadIdx.x;
        const int32_t n_parts = __ldg(&I.n_parts);
        if (local >= n_parts) continue;
        const int64_t i = __ldg(&I.part_offset) + local;
        double x = ld_stream(b.pos + i), y = ld_stream(b.pos + sd + i);
        const double ex = __ldg(&I.extents[0]), ey = __ldg(&I.extents[1]);
        if (kMode != kMoveOnly) {
            const double dt = __ldg(&I.dt);
            x = update_axis(x, __ldg(b.vel + i), dt, ex);
            y = update_axis(y, __ldg(b.vel + sd + i), dt, ey);
            st_stream(b.pos + i, x);
            st_stream(b.pos + sd + i, y);
        }
        if (kMode != kUpdateOnly) {
            int32_t cell = ld_stream(b.p2c + i);
            if (cell == kRemoved) continue;
            const int32_t cell0 = cell;
            int mx = ld_stream(b.mdir + i), my = ld_stream(b.mdir + sd + i);
            int err = 0;
            const int calls = move_particle(b.cells, __ldg(&I.cell_offset), __ldg(&I.n_cells), x, y, mx, my, cell,
                                            __ldg(&I.cell_width), ex, ey, max_hops, err);
            if (err) raise_error(st, err, (int32_t)i);
            st_stream(b.mdir + i, mx);
            st_stream(b.mdir + sd + i, my);
            if (cell != cell0) st_stream(b.p2c + i, cell);
            my_calls += (unsigned long long)calls;
            my_max = max(my_max, calls);
        }
    }
    if (kMode == kUpdateOnly) return;
    // One atomic per counter per block: the grid is persistent, so this is a few hundred.
    __shared__ unsigned long long s_calls[kAdvWarps];
    __shared__ int s_max[kAdvWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_calls += __shfl_xor_sync(kFullMask, my_calls, o);
    my_max = (int)__reduce_max_sync(kFullMask, (unsigned)my_max);
    if (lane == 0) {
        s_calls[warp] = my_calls;
        s_max[warp] = my_max;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long c = 0;
        int m = 0;
        for (int k = 0; k < kAdvWarps; k++) {
            c += s_calls[k];
            m = max(m, s_max[k]);
        }
        if (c) atomicAdd(reinterpret_cast<unsigned long long*>(&st->total_visits), c);
        if (m) atomicMax(&st->max_visits, m);
    }
}

__global__ void __launch_bounds__(256) advec_pack_kernel(double* cells, int32_t cell_offset, int32_t n_cells, int32_t ld,
                                                         const double* c_pos_ll, const int32_t* c2c) {
    const int64_t c = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (c >= n_cells) return;
    int32_t nb[4];
#pragma unroll
    for (int k = 0; k < 4; k++) nb[k] = c2c[(int64_t)k * ld + c];
    double4 r;
    r.x = c_pos_ll[c];
    r.y = c_pos_ll[(int64_t)ld + c];
    r.z = __longlong_as_double(((long long)(uint32_t)nb[1] << 32) | (uint32_t)nb[0]);
    r.w = __longlong_as_double(((long long)(uint32_t)nb[3] << 32) | (uint32_t)nb[2]);
    reinterpret_cast<double4*>(cells)[(int64_t)cell_offset + c] = r;
}

// Persistent grid: resident blocks of the kernel on every SM (cached per device and mode).
template <int kMode>
int persistent_grid(int n_work) {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return n_work;
    if (!cached[dev]) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, advec_kernel<kMode>, kAdvBlock, 0);
        cached[dev] = sms * (per_sm > 0 ? per_sm : 1);
    }
    return n_work < cached[dev] ? n_work : cached[dev];
}

int check_batch(const oppb_advec_batch* b) {
    if (!b || b->n_instances <= 0 || b->n_work < 0 || !b->instances || !b->tile_prefix) return OPPB_ERR_ARG;
    if (!b->pos || !b->vel || !b->mdir || !b->p2c || !b->cells || !aligned(b->cells, 32) || b->stride <= 0)
        return OPPB_ERR_ARG;
    return OPPB_OK;
}

template <int kMode>
int launch_advec(const oppb_advec_batch* b, oppb_move_status* status, int32_t max_hops, void* stream) {
    const int rc = check_batch(b);
    if (rc) return rc;
    if (kMode != kUpdateOnly && (!status || max_hops <= 0)) return OPPB_ERR_ARG;
    if (b->n_work == 0) return OPPB_OK;
    advec_kernel<kMode><<<persistent_grid<kMode>(b->n_work), kAdvBlock, 0, as_stream(stream)>>>(*b, status, max_hops);
    count_launches(1);
    return launch_status();
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_advec_pack_cells(double* cells, int32_t cell_offset, int32_t n_cells, int32_t ld,
                                     const double* c_pos_ll, const int32_t* c2c, void* stream) {
    using namespace oppb;
    if (!cells || !aligned(cells, 32) || cell_offset < 0 || n_cells <= 0 || ld < n_cells || !c_pos_ll || !c2c)
        return OPPB_ERR_ARG;
    advec_pack_kernel<<<ceil_div(n_cells, 256), 256, 0, as_stream(stream)>>>(cells, cell_offset, n_cells, ld,
                                                                             c_pos_ll, c2c);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_advec_step(const oppb_advec_batch* batch, oppb_move_status* status, int32_t max_hops,
                               void* stream) {
    return oppb::launch_advec<oppb::kStep>(batch, status, max_hops, stream);
}

extern "C" int oppb_advec_update_pos(const oppb_advec_batch* batch, void* stream) {
    return oppb::launch_advec<oppb::kUpdateOnly>(batch, nullptr, 1, stream);
}

extern "C" int oppb_advec_move(const oppb_advec_batch* batch, oppb_move_status* status, int32_t max_hops,
                               void* stream) {
    return oppb::launch_advec<oppb::kMoveOnly>(batch, status, max_hops, stream);
}
