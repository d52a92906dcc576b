// NESO-advection particle path: periodic position update and axis-wise multi-hop move, for a
// batch of independent instances (different meshes, particle counts and constants) in one
// persistent launch.
//
// Work is cut into 256-particle items that never straddle two instances (tile_prefix); a
// grid sized to the resident capacity of the GPU takes the items in order from a counter, so
// instances of uneven size share the SMs without a launch per instance and the items in
// flight stay within one or two instances.  One thread per particle of an
// item: update_pos (apps_codegen/app_neso_advection_mdir_cg/kernels.h update_pos_kernel) in
// registers, then the hops of move_kernel (the direction chosen on the first call, x first,
// then y), reading one 32-byte cell record {c_pos_ll, c2c} per call.  This file is compiled
// with -fmad=false and the periodic wrap uses the library's FMOD (a - b * trunc(a / b),
// opp_lib/include/opp_util.h:48) with a correctly rounded divide, so positions, directions and
// cells are bit-identical to the seq backend.  With the global move on (batch.dh), each walk
// starts from the cell of the direct-hop grid box holding the updated position.

#include "oppb_advec.h"
#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kAdvBlock = 256;  // = particles per work item
constexpr int kAdvWarps = kAdvBlock / 32;
enum AdvMode { kStep = 0, kUpdateOnly = 1, kMoveOnly = 2 };

// Work item w belongs to the instance i with prefix[i] <= w < prefix[i + 1].  A block's items
// only increase, so the search moves a cursor forward from the previous answer: usually one
// comparison per item instead of a dependent binary search.
__device__ __forceinline__ int find_instance(const int32_t* __restrict__ prefix, int n, int w, int& cursor) {
    while (cursor + 1 < n && __ldg(prefix + cursor + 1) <= w) cursor++;
    return cursor;
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

// move_kernel's hops on an instance whose cells are the periodic nx x ny grid of the app's
// init_mesh (apps_codegen/app_neso_advection_mdir_cg/advec_misc.h:115-141): the corner
// (ix w, iy w) and the VOXEL_MAP neighbours (advec_defs.h:46-54) computed from the cell
// index instead of read from the record, which oppb_advec_check_grid found equal to them bit
// for bit.  The walk keeps (ix, iy) and steps them with the periodic wrap; the arithmetic
// and the decisions are move_particle's.
__device__ __forceinline__ int move_particle_grid(int32_t nx, int32_t n_cells, double x, double y, int& mx, int& my,
                                                  int32_t& cell, double cw, double ex, double ey, int32_t max_hops,
                                                  int& err) {
    if ((uint32_t)cell >= (uint32_t)n_cells) {
        err = OPPB_ERR_CELL_RANGE;
        return 0;
    }
    const int32_t ny = n_cells / nx;
    int32_t iy = cell / nx;
    int32_t ix = cell - iy * nx;
    int calls = 0;
    for (;;) {
        calls++;
        const double dx = x - (double)ix * cw;  // c_pos_ll = (x * cell_width, y * cell_width)
        const double dy = y - (double)iy * cw;
        if (calls == 1) {  // OPP_DO_ONCE
            const bool xp = ((dx > cw) && (ex > 2 * dx - cw)) || ((dx < 0) && (ex < cw - 2 * dx));
            const bool yp = ((dy > cw) && (ey > 2 * dy - cw)) || ((dy < 0) && (ey < cw - 2 * dy));
            mx = xp ? 1 : -1;
            my = yp ? 1 : -1;
        }
        bool hop = false;
        if ((dx >= 0.0) && (dx <= cw)) {
            mx = 0;
        } else if (mx != 0) {
            ix = mx > 0 ? (ix + 1 >= nx ? 0 : ix + 1) : (ix - 1 < 0 ? nx - 1 : ix - 1);  // xu_y : xd_y
            hop = true;
        }
        if (!hop) {
            if ((dy >= 0.0) && (dy <= cw)) {
                my = 0;
            } else if (my != 0) {
                iy = my > 0 ? (iy + 1 >= ny ? 0 : iy + 1) : (iy - 1 < 0 ? ny - 1 : iy - 1);  // x_yu : x_yd
                hop = true;
            }
        }
        if (!hop) break;
        if (calls >= max_hops) {
            err = OPPB_ERR_HOP_LIMIT;
            break;
        }
    }
    cell = ix + nx * iy;
    return calls;
}

constexpr int kChunkItems = 8;  // work items a block takes from the counter at once

// Direct-hop seed (oppb_advec_dh): the cell of the grid box holding (x, y), or kRemoved
// outside the grid or in a box without a cell.  Each box coordinate is (pos - min) * (1/h)
// truncated by a round-toward-zero conversion that saturates (negative and NaN give 0), the
// conversion the reference's (size_t) cast compiles to.
__device__ __forceinline__ int32_t dh_seed_2d(const oppb_advec_dh& g, double x, double y) {
    const unsigned long long ix = __double2ull_rz(__dmul_rn(__dsub_rn(x, __ldg(&g.min[0])), __ldg(&g.inv_spacing)));
    const unsigned long long iy = __double2ull_rz(__dmul_rn(__dsub_rn(y, __ldg(&g.min[1])), __ldg(&g.inv_spacing)));
    const unsigned long long dx = (unsigned long long)__ldg(&g.dims[0]), dy = (unsigned long long)__ldg(&g.dims[1]);
    if (ix >= dx || iy >= dy) return kRemoved;
    return __ldg(g.map + (int64_t)(ix + dx * iy));
}

// A block takes a chunk of work items from the batch's counter (so items are processed in
// order across the whole GPU) and walks it kItems items per pass (one particle of each per
// thread), so every thread has kItems independent particles' loads in flight.
template <int kMode, int kItems, bool kSeed>
__global__ void __launch_bounds__(kAdvBlock) advec_kernel(oppb_advec_batch b, oppb_move_status* st,
                                                          int32_t max_hops) {
    static_assert(kChunkItems % kItems == 0, "a chunk is a whole number of passes");
    static_assert(!kSeed || kMode != kUpdateOnly, "the seed belongs to the move");
    __shared__ int s_chunk;
    unsigned long long my_calls = 0;
    int my_max = 0;
    int my_removed = 0;
    int cursor = 0;
    const int64_t sd = b.stride;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(b.work_counter, kChunkItems);
        __syncthreads();
        const int chunk = s_chunk;
        __syncthreads();
        if (chunk >= b.n_work) break;
        for (int w0 = chunk; w0 < chunk + kChunkItems && w0 < b.n_work; w0 += kItems) {
            double x[kItems], y[kItems], vx[kItems], vy[kItems];
            int32_t cell[kItems], mx[kItems], my[kItems];
            int64_t idx[kItems];
            int inst[kItems];
            bool ok[kItems];
    #pragma unroll
            for (int k = 0; k < kItems; k++) {  // all loads first
                const int w = w0 + k;
                ok[k] = false;
                if (w >= b.n_work) continue;
                inst[k] = find_instance(b.tile_prefix, b.n_instances, w, cursor);
                const oppb_advec_instance& I = b.instances[inst[k]];
                const int32_t local = (w - __ldg(b.tile_prefix + inst[k])) * kAdvBlock + threadIdx.x;
                if (local >= __ldg(&I.n_parts)) continue;
                ok[k] = true;
                const int64_t i = __ldg(&I.part_offset) + local;
                idx[k] = i;
                x[k] = ld_stream(b.pos + i);
                y[k] = ld_stream(b.pos + sd + i);
                if (kMode != kMoveOnly) {
                    vx[k] = __ldg(b.vel + i);
                    vy[k] = __ldg(b.vel + sd + i);
                }
                if (kMode != kUpdateOnly) {
                    cell[k] = ld_stream(b.p2c + i);
                    mx[k] = ld_stream(b.mdir + i);
                    my[k] = ld_stream(b.mdir + sd + i);
                }
            }
    #pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (!ok[k]) continue;
                const oppb_advec_instance& I = b.instances[inst[k]];
                const int64_t i = idx[k];
                const double ex = __ldg(&I.extents[0]), ey = __ldg(&I.extents[1]);
                if (kMode != kMoveOnly) {
                    const double dt = __ldg(&I.dt);
                    x[k] = update_axis(x[k], vx[k], dt, ex);
                    y[k] = update_axis(y[k], vy[k], dt, ey);
                    st_stream(b.pos + i, x[k]);
                    st_stream(b.pos + sd + i, y[k]);
                }
                if (kMode != kUpdateOnly) {
                    if (cell[k] == kRemoved) continue;
                    if (kSeed) {  // the global-move pre-pass, after the update as in the reference
                        cell[k] = dh_seed_2d(b.dh[inst[k]], x[k], y[k]);
                        if (cell[k] == kRemoved) {
                            st_stream(b.p2c + i, kRemoved);
                            my_removed++;
                            continue;
                        }
                    }
                    int err = 0;
                    const int32_t gnx = __ldg(&I.grid_nx);
                    const int calls =
                        gnx > 0 ? move_particle_grid(gnx, __ldg(&I.n_cells), x[k], y[k], mx[k], my[k], cell[k],
                                                     __ldg(&I.cell_width), ex, ey, max_hops, err)
                                : move_particle(b.cells, __ldg(&I.cell_offset), __ldg(&I.n_cells), x[k], y[k], mx[k],
                                                my[k], cell[k], __ldg(&I.cell_width), ex, ey, max_hops, err);
                    if (err) raise_error(st, err, (int32_t)i);
                    st_stream(b.mdir + i, mx[k]);
                    st_stream(b.mdir + sd + i, my[k]);
                    // Every processed particle's cell is stored, changed or not: a warp then
                    // writes whole sectors of p2c, which DRAM takes without reading them first.
                    st_stream(b.p2c + i, cell[k]);
                    my_calls += (unsigned long long)calls;
                    my_max = max(my_max, calls);
                }
            }
        }
    }
    if (kMode == kUpdateOnly) return;
    // One atomic per counter per block: the grid is persistent, so this is a few hundred.
    __shared__ unsigned long long s_calls[kAdvWarps];
    __shared__ int s_max[kAdvWarps];
    __shared__ int s_removed[kAdvWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_calls += __shfl_xor_sync(kFullMask, my_calls, o);
    my_max = (int)__reduce_max_sync(kFullMask, (unsigned)my_max);
    if (kSeed) my_removed = (int)__reduce_add_sync(kFullMask, (unsigned)my_removed);
    if (lane == 0) {
        s_calls[warp] = my_calls;
        s_max[warp] = my_max;
        s_removed[warp] = my_removed;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long c = 0;
        int m = 0, r = 0;
        for (int k = 0; k < kAdvWarps; k++) {
            c += s_calls[k];
            m = max(m, s_max[k]);
            r += s_removed[k];
        }
        if (c) atomicAdd(reinterpret_cast<unsigned long long*>(&st->total_visits), c);
        if (m) atomicMax(&st->max_visits, m);
        if (kSeed && r) atomicAdd(&st->remove_count, r);
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

// Counts the cells whose packed record differs, in any bit, from the periodic grid's corner and
// neighbours (move_particle_grid).
__global__ void __launch_bounds__(256) advec_check_grid_kernel(const double* cells, int32_t n_cells, int32_t nx,
                                                               double cw, int32_t* mismatches) {
    const int32_t c = (int32_t)(blockIdx.x * 256 + threadIdx.x);
    if (c >= n_cells) return;
    const int32_t ny = n_cells / nx, iy = c / nx, ix = c - iy * nx;
    const int32_t xd = (ix - 1 < 0 ? nx - 1 : ix - 1) + nx * iy, xu = (ix + 1 >= nx ? 0 : ix + 1) + nx * iy;
    const int32_t yd = ix + nx * (iy - 1 < 0 ? ny - 1 : iy - 1), yu = ix + nx * (iy + 1 >= ny ? 0 : iy + 1);
    double llx, lly, n01, n23;
    ldg256(cells + (int64_t)c * 4, llx, lly, n01, n23);
    const bool same = __double_as_longlong(llx) == __double_as_longlong((double)ix * cw) &&
                      __double_as_longlong(lly) == __double_as_longlong((double)iy * cw) &&
                      __double_as_longlong(n01) == (long long)(((unsigned long long)(uint32_t)xu << 32) | (uint32_t)xd) &&
                      __double_as_longlong(n23) == (long long)(((unsigned long long)(uint32_t)yu << 32) | (uint32_t)yd);
    if (!same) atomicAdd(mismatches, 1);
}

// Persistent grid: resident blocks of the kernel on every SM (cached per device and variant).
template <int kMode, int kItems, bool kSeed>
int persistent_grid(int n_blocks_needed) {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return n_blocks_needed;
    if (!cached[dev]) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, advec_kernel<kMode, kItems, kSeed>, kAdvBlock, 0);
        cached[dev] = sms * (per_sm > 0 ? per_sm : 1);
    }
    return n_blocks_needed < cached[dev] ? n_blocks_needed : cached[dev];
}

template <int kMode, int kItems, bool kSeed>
void launch_items(const oppb_advec_batch* b, oppb_move_status* status, int32_t max_hops, cudaStream_t s) {
    const int grid = persistent_grid<kMode, kItems, kSeed>(ceil_div(b->n_work, kChunkItems));
    advec_kernel<kMode, kItems, kSeed><<<grid, kAdvBlock, 0, s>>>(*b, status, max_hops);
}

template <int kMode, bool kSeed>
void launch_seeded(const oppb_advec_batch* b, oppb_move_status* status, int32_t max_hops, cudaStream_t s) {
    const int items = tuning().advec_items;
    if (items == 4)
        launch_items<kMode, 4, kSeed>(b, status, max_hops, s);
    else if (items == 1)
        launch_items<kMode, 1, kSeed>(b, status, max_hops, s);
    else
        launch_items<kMode, 2, kSeed>(b, status, max_hops, s);
}

// The pointers a launch reads or writes must be set: pos always, vel unless the launch only
// moves, mdir, p2c and the 32-byte-aligned cells unless it only updates positions.
template <int kMode>
int check_batch(const oppb_advec_batch* b) {
    if (!b || b->n_instances <= 0 || b->n_work < 0 || !b->instances || !b->tile_prefix) return OPPB_ERR_ARG;
    if (!b->pos || b->stride <= 0 || !b->work_counter) return OPPB_ERR_ARG;
    if (kMode != kMoveOnly && !b->vel) return OPPB_ERR_ARG;
    if (kMode != kUpdateOnly && (!b->mdir || !b->p2c || !b->cells || !aligned(b->cells, 32))) return OPPB_ERR_ARG;
    return OPPB_OK;
}

// verify_kernel (apps/app_neso_advection/kernels.h:115-151): a particle is incorrect when its
// cell's global index g gives ix = g - (g / nx) nx < 0 or iy = g / nx < 0, or when its position
// lies outside the closed box [ix w, ix w + w] x [iy w, iy w + w] (the products and sums rounded
// on their own, as there; this file is compiled with -fmad=false).  Block counts are added
// into *incorrect.
__global__ void __launch_bounds__(256) advec_verify_kernel(const double* __restrict__ pos, int64_t stride,
                                                           const int32_t* __restrict__ p2c,
                                                           const int32_t* __restrict__ c_gbl_idx, int32_t n,
                                                           int32_t nx, double w, int32_t* incorrect) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    int bad = 0;
    if (i < n) {
        const int32_t g = __ldg(c_gbl_idx + __ldg(p2c + i));
        const int32_t iy = g / nx, ix = g - iy * nx;
        if (ix < 0 || iy < 0) {
            bad = 1;
        } else {
            const double llx = ix * w, lly = iy * w;
            const double x = __ldg(pos + i), y = __ldg(pos + stride + i);
            bad = (x < llx || x > llx + w || y < lly || y > lly + w) ? 1 : 0;
        }
    }
    const int warp_bad = __popc(__ballot_sync(kFullMask, bad));
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && warp_bad) atomicAdd(&s_bad, warp_bad);
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) atomicAdd(incorrect, s_bad);
}

template <int kMode>
int launch_advec(const oppb_advec_batch* b, oppb_move_status* status, int32_t max_hops, void* stream) {
    const int rc = check_batch<kMode>(b);
    if (rc) return rc;
    if (kMode != kUpdateOnly && (!status || max_hops <= 0)) return OPPB_ERR_ARG;
    if (b->n_work == 0) return OPPB_OK;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(b->work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    if constexpr (kMode != kUpdateOnly) {
        if (b->dh)
            launch_seeded<kMode, true>(b, status, max_hops, s);
        else
            launch_seeded<kMode, false>(b, status, max_hops, s);
    } else {
        launch_seeded<kMode, false>(b, status, max_hops, s);
    }
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

extern "C" int oppb_advec_check_grid(const double* cells, int32_t cell_offset, int32_t n_cells, int32_t nx,
                                     double cell_width, int32_t* mismatches, void* stream) {
    using namespace oppb;
    if (!cells || !aligned(cells, 32) || cell_offset < 0 || n_cells <= 0 || nx <= 0 || n_cells % nx != 0 ||
        !mismatches)
        return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(mismatches, 0, sizeof(int32_t), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    advec_check_grid_kernel<<<ceil_div(n_cells, 256), 256, 0, s>>>(cells + (int64_t)cell_offset * 4, n_cells, nx,
                                                                   cell_width, mismatches);
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

extern "C" int oppb_advec_verify(const double* pos, int64_t stride, const int32_t* p2c, const int32_t* c_gbl_idx,
                                 int32_t n_parts, int32_t nx, double cell_width, int32_t* incorrect, void* stream) {
    using namespace oppb;
    if (n_parts < 0 || nx <= 0 || !incorrect || (n_parts > 0 && (!pos || !p2c || !c_gbl_idx || stride < n_parts)))
        return OPPB_ERR_ARG;
    if (n_parts == 0) return OPPB_OK;
    advec_verify_kernel<<<ceil_div(n_parts, 256), 256, 0, as_stream(stream)>>>(pos, stride, p2c, c_gbl_idx, n_parts,
                                                                              nx, cell_width, incorrect);
    count_launches(1);
    return launch_status();
}
