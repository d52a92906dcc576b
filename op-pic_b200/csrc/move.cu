// Particle move (multi-hop barycentric cell location) and node-charge deposit for
// tetrahedral meshes, FP64 and mixed FP32/FP64.
//
// One thread per particle, particles in SoA (stride = capacity), cells in packed
// records (det: 128 B, conn: 32 B, coef: 8 B) read through the read-only path.
// The FP64 arithmetic uses explicit round-to-nearest intrinsics so nothing is
// contracted into FMAs: each lambda_i is bit-identical to the reference expression
//   coef * (((d0 - d1*x) + d2*y) - d3*z)          (apps/app_fempic/kernels.h:110-117)
// and the inside test / argmin follow kernels.h:121-146 exactly.

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kMoveBlock = 256;
constexpr double kTol = 1e-10;  // KERNEL_TOLERENCE, apps/app_fempic/kernels.h:44

enum : int { kDone = 0, kNeedMove = 1, kNeedRemove = 2, kFailed = 3 };

struct MeshArgs {
    int32_t n_cells;
    int32_t n_nodes;
    const double* det;
    const double* coef;
    const int32_t* conn;
    const float* geo32;
    const float* org32;
};

struct PartArgs {
    int32_t size;
    int32_t stride;
    const double* pos;
    double* lc;
    int32_t* p2c;
    uint32_t* remove_bits;
};

// lambda_0..3 of point (x,y,z) in cell c, evaluated exactly as the FP64 reference.
__device__ __forceinline__ void lambda_f64(const MeshArgs& m, int32_t c, double x, double y, double z,
                                           double l[4]) {
    const double* d = m.det + (int64_t)c * 16;
    const double coef = __ldg(m.coef + c);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const double2 ab = ldg_d2(d + 4 * i);
        const double2 gd = ldg_d2(d + 4 * i + 2);
        double t = __dsub_rn(ab.x, __dmul_rn(ab.y, x));
        t = __dadd_rn(t, __dmul_rn(gd.x, y));
        t = __dsub_rn(t, __dmul_rn(gd.y, z));
        l[i] = __dmul_rn(coef, t);
    }
}

// Inside test of kernels.h:121-124 and first-index argmin of kernels.h:139-146.
__device__ __forceinline__ bool inside_f64(const double l[4]) {
    bool in = true;
#pragma unroll
    for (int i = 0; i < 4; i++) in = in && (l[i] > -kTol) && (__dsub_rn(l[i], 1.0) < kTol);
    return in;
}
__device__ __forceinline__ int argmin4(const double l[4]) {
    int mi = 0;
    double mv = l[0];
#pragma unroll
    for (int i = 1; i < 4; i++)
        if (l[i] < mv) {
            mv = l[i];
            mi = i;
        }
    return mi;
}

// Warp-level bookkeeping shared by all move variants: removal bitmap word, remove
// count, visit statistics.  Every lane of the warp must call it.
__device__ __forceinline__ void warp_account(const PartArgs& p, oppb_move_status* st, int64_t i, bool active,
                                             int32_t final_cell, bool newly_removed, int visits,
                                             int rechecks) {
    const int lane = threadIdx.x & 31;
    const unsigned hole = __ballot_sync(kFullMask, active && final_cell == kRemoved);
    const unsigned rem = __ballot_sync(kFullMask, newly_removed);
    if (lane == 0 && i < p.size) p.remove_bits[i >> 5] = hole;
    int vmax = visits;
    unsigned vsum = (unsigned)visits;
    int rsum = rechecks;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        vmax = max(vmax, __shfl_xor_sync(kFullMask, vmax, o));
        vsum += __shfl_xor_sync(kFullMask, vsum, o);
        rsum += __shfl_xor_sync(kFullMask, rsum, o);
    }
    if (lane == 0) {
        if (rem) atomicAdd(&st->remove_count, __popc(rem));
        if (vsum) atomicAdd(reinterpret_cast<unsigned long long*>(&st->total_visits), (unsigned long long)vsum);
        if (vmax) atomicMax(&st->max_visits, vmax);
        if (rsum) atomicAdd(&st->recheck_count, rsum);
    }
}

// Warp-aggregated deposit: lanes holding the same cell in a contiguous run add
// their weights with a segmented shuffle reduction; the run head issues four FP64
// atomics into node_charge[c2n[cell][k]].  key < 0 = no contribution.
__device__ __forceinline__ void warp_deposit(const MeshArgs& m, double* node_charge, int32_t key,
                                             double l0, double l1, double l2, double l3) {
    const int lane = threadIdx.x & 31;
    const int32_t prev = __shfl_up_sync(kFullMask, key, 1);
    const bool head = (lane == 0) || (prev != key);
    const unsigned heads = __ballot_sync(kFullMask, head);
    const unsigned later = (lane == 31) ? 0u : (heads & (~0u << (lane + 1)));
    const int seg_end = later ? (__ffs(later) - 2) : 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double a0 = __shfl_down_sync(kFullMask, l0, o);
        const double a1 = __shfl_down_sync(kFullMask, l1, o);
        const double a2 = __shfl_down_sync(kFullMask, l2, o);
        const double a3 = __shfl_down_sync(kFullMask, l3, o);
        if (lane + o <= seg_end) {
            l0 += a0;
            l1 += a1;
            l2 += a2;
            l3 += a3;
        }
    }
    if (head && key >= 0) {
        const int4 nodes = ldg_i4(m.conn + (int64_t)key * 8 + 4);
        const uint32_t nn = (uint32_t)m.n_nodes;
        if ((uint32_t)nodes.x < nn) atomicAdd(node_charge + nodes.x, l0);
        if ((uint32_t)nodes.y < nn) atomicAdd(node_charge + nodes.y, l1);
        if ((uint32_t)nodes.z < nn) atomicAdd(node_charge + nodes.z, l2);
        if ((uint32_t)nodes.w < nn) atomicAdd(node_charge + nodes.w, l3);
    }
}

// ------------------------------------------------------------------ FP64 move

template <bool kDeposit>
__global__ void __launch_bounds__(kMoveBlock) move_f64_kernel(MeshArgs m, PartArgs p, double* node_charge,
                                                              oppb_move_status* st, int32_t max_hops) {
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < p.size;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int status = kDone;
    int visits = 0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (active && cell != kRemoved) {
        const double x = ld_stream(p.pos + i);
        const double y = ld_stream(p.pos + p.stride + i);
        const double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        for (;;) {
            if ((uint32_t)cell >= (uint32_t)m.n_cells) {
                raise_error(st, OPPB_ERR_CELL_RANGE, (int32_t)i);
                status = kFailed;
                break;
            }
            lambda_f64(m, cell, x, y, z, l);
            visits++;
            if (inside_f64(l)) {
                status = kDone;
                break;
            }
            const int mi = argmin4(l);
            const int32_t nb = __ldg(m.conn + (int64_t)cell * 8 + mi);
            if (nb < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = nb;
            if (visits >= max_hops) {
                raise_error(st, OPPB_ERR_HOP_LIMIT, (int32_t)i);
                status = kFailed;
                break;
            }
        }
        if (visits > 0) {
            st_stream(p.lc + i, l[0]);
            st_stream(p.lc + p.stride + i, l[1]);
            st_stream(p.lc + 2 * (int64_t)p.stride + i, l[2]);
            st_stream(p.lc + 3 * (int64_t)p.stride + i, l[3]);
        }
        if (cell != cell0) st_stream(p.p2c + i, cell);
    }
    warp_account(p, st, i, active, cell, status == kNeedRemove, visits, 0);
    if (kDeposit) {
        const bool dep = active && cell0 != kRemoved && status == kDone;
        warp_deposit(m, node_charge, dep ? cell : -1, dep ? l[0] : 0.0, dep ? l[1] : 0.0, dep ? l[2] : 0.0,
                     dep ? l[3] : 0.0);
    }
}

// -------------------------------------------------------- mixed FP32 / FP64 move
//
// lambda_i(x) = c_i + g_i . (x - o) with o = f32(vertex 0), c_i, g_i in f32.  The FP32
// evaluation error is below 6 * 2^-24 * S, S = |c_i| + sum_j |g_ij| |d_j|.  A decision
// is taken in FP32 only when every threshold (-1e-10, 1+1e-10) and, outside the cell,
// every argmin tie is at least `band` away and S <= kMaxS; otherwise the visit is
// recomputed with the FP64 reference expression.  Hence every decision equals the
// FP64 one.

constexpr float kMaxS = 16.0f;

template <bool kDeposit>
__global__ void __launch_bounds__(kMoveBlock) move_mixed_kernel(MeshArgs m, PartArgs p, double* node_charge,
                                                                oppb_move_status* st, int32_t max_hops,
                                                                float band) {
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < p.size;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int status = kDone;
    int visits = 0;
    int rechecks = 0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (active && cell != kRemoved) {
        const double x = ld_stream(p.pos + i);
        const double y = ld_stream(p.pos + p.stride + i);
        const double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        for (;;) {
            if ((uint32_t)cell >= (uint32_t)m.n_cells) {
                raise_error(st, OPPB_ERR_CELL_RANGE, (int32_t)i);
                status = kFailed;
                break;
            }
            visits++;
            const float4 o = ldg_f4(m.org32 + (int64_t)cell * 4);
            const float dx = (float)(x - (double)o.x);
            const float dy = (float)(y - (double)o.y);
            const float dz = (float)(z - (double)o.z);
            float lf[4];
            float smax = 0.0f;
            const float* g = m.geo32 + (int64_t)cell * 16;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float4 r = ldg_f4(g + 4 * k);
                lf[k] = fmaf(r.w, dz, fmaf(r.z, dy, fmaf(r.y, dx, r.x)));
                const float s = fabsf(r.x) + fabsf(r.y) * fabsf(dx) + fabsf(r.z) * fabsf(dy) + fabsf(r.w) * fabsf(dz);
                smax = fmaxf(smax, s);
            }
            // Classify in FP32.
            bool clear_in = smax <= kMaxS;
            bool clear_out = false;
            bool ambiguous = !(smax <= kMaxS);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                clear_in = clear_in && (lf[k] >= band) && (lf[k] <= 1.0f - band);
                clear_out = clear_out || (lf[k] <= -band) || (lf[k] >= 1.0f + band);
            }
            int mi = 0;
            if (!clear_in && !ambiguous) {
                if (!clear_out) {
                    ambiguous = true;
                } else {
                    float mv = lf[0];
#pragma unroll
                    for (int k = 1; k < 4; k++)
                        if (lf[k] < mv) {
                            mv = lf[k];
                            mi = k;
                        }
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (k != mi && !(lf[k] - mv > 2.0f * band)) ambiguous = true;
                }
            }
            bool in;
            if (ambiguous) {
                rechecks++;
                lambda_f64(m, cell, x, y, z, l);
                in = inside_f64(l);
                if (!in) mi = argmin4(l);
            } else {
                in = clear_in;
#pragma unroll
                for (int k = 0; k < 4; k++) l[k] = (double)lf[k];
            }
            if (in) {
                status = kDone;
                break;
            }
            const int32_t nb = __ldg(m.conn + (int64_t)cell * 8 + mi);
            if (nb < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = nb;
            if (visits >= max_hops) {
                raise_error(st, OPPB_ERR_HOP_LIMIT, (int32_t)i);
                status = kFailed;
                break;
            }
        }
        if (visits > 0) {
            st_stream(p.lc + i, l[0]);
            st_stream(p.lc + p.stride + i, l[1]);
            st_stream(p.lc + 2 * (int64_t)p.stride + i, l[2]);
            st_stream(p.lc + 3 * (int64_t)p.stride + i, l[3]);
        }
        if (cell != cell0) st_stream(p.p2c + i, cell);
    }
    warp_account(p, st, i, active, cell, status == kNeedRemove, visits, rechecks);
    if (kDeposit) {
        const bool dep = active && cell0 != kRemoved && status == kDone;
        warp_deposit(m, node_charge, dep ? cell : -1, dep ? l[0] : 0.0, dep ? l[1] : 0.0, dep ? l[2] : 0.0,
                     dep ? l[3] : 0.0);
    }
}

// ------------------------------------------------------------- standalone deposit

__global__ void __launch_bounds__(kMoveBlock) deposit_f64_kernel(MeshArgs m, PartArgs p, double* node_charge) {
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < p.size;
    int32_t cell = active ? ld_stream(p.p2c + i) : -1;
    const bool ok = active && (uint32_t)cell < (uint32_t)m.n_cells;
    double l0 = 0, l1 = 0, l2 = 0, l3 = 0;
    if (ok) {
        l0 = ld_stream(p.lc + i);
        l1 = ld_stream(p.lc + p.stride + i);
        l2 = ld_stream(p.lc + 2 * (int64_t)p.stride + i);
        l3 = ld_stream(p.lc + 3 * (int64_t)p.stride + i);
    }
    warp_deposit(m, node_charge, ok ? cell : -1, l0, l1, l2, l3);
}

int check_mesh(const oppb_tet_mesh* mesh, bool mixed) {
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0) return OPPB_ERR_ARG;
    if (!mesh->det || !mesh->coef || !mesh->conn) return OPPB_ERR_ARG;
    if (!aligned(mesh->det, 16) || !aligned(mesh->conn, 16)) return OPPB_ERR_ARG;
    if (mixed && (!mesh->geo32 || !mesh->org32 || !aligned(mesh->geo32, 16) || !aligned(mesh->org32, 16)))
        return OPPB_ERR_ARG;
    return OPPB_OK;
}

int check_parts(const oppb_particles* p, bool need_bits) {
    if (!p || p->size < 0 || p->stride < p->size) return OPPB_ERR_ARG;
    if (!p->pos || !p->lc || !p->p2c) return OPPB_ERR_ARG;
    if (need_bits && !p->remove_bits) return OPPB_ERR_ARG;
    return OPPB_OK;
}

MeshArgs mesh_args(const oppb_tet_mesh* mesh) {
    return MeshArgs{mesh->n_cells, mesh->n_nodes, mesh->det, mesh->coef, mesh->conn, mesh->geo32, mesh->org32};
}
PartArgs part_args(const oppb_particles* p) {
    return PartArgs{p->size, p->stride, p->pos, p->lc, p->p2c, p->remove_bits};
}

template <int kKind>  // 0 move, 1 move+deposit, 2 mixed move+deposit
int launch_move(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                oppb_move_status* status, int32_t max_hops, double band, void* stream) {
    int rc = check_mesh(mesh, kKind == 2);
    if (rc) return rc;
    rc = check_parts(parts, true);
    if (rc) return rc;
    if (!status || max_hops <= 0) return OPPB_ERR_ARG;
    if (kKind != 0 && !node_charge) return OPPB_ERR_ARG;
    if (kKind == 2 && !(band > 0.0 && band < 0.25)) return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(status, 0, sizeof(oppb_move_status), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    if (parts->size == 0) return launch_status();
    const MeshArgs m = mesh_args(mesh);
    const PartArgs p = part_args(parts);
    const int grid = ceil_div(parts->size, kMoveBlock);
    if (kKind == 0)
        move_f64_kernel<false><<<grid, kMoveBlock, 0, s>>>(m, p, nullptr, status, max_hops);
    else if (kKind == 1)
        move_f64_kernel<true><<<grid, kMoveBlock, 0, s>>>(m, p, node_charge, status, max_hops);
    else
        move_mixed_kernel<true><<<grid, kMoveBlock, 0, s>>>(m, p, node_charge, status, max_hops, (float)band);
    count_launches(1);
    return launch_status();
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_move_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, oppb_move_status* status,
                             int32_t max_hops, void* stream) {
    return oppb::launch_move<0>(mesh, parts, nullptr, status, max_hops, 0.0, stream);
}

extern "C" int oppb_move_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                                     oppb_move_status* status, int32_t max_hops, void* stream) {
    return oppb::launch_move<1>(mesh, parts, node_charge, status, max_hops, 0.0, stream);
}

extern "C" int oppb_move_deposit_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                                       double* node_charge, oppb_move_status* status, int32_t max_hops,
                                       double band, void* stream) {
    return oppb::launch_move<2>(mesh, parts, node_charge, status, max_hops, band, stream);
}

extern "C" int oppb_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                                void* stream) {
    int rc = oppb::check_mesh(mesh, false);
    if (rc) return rc;
    if (!parts || parts->size < 0 || parts->stride < parts->size || !parts->lc || !parts->p2c || !node_charge)
        return OPPB_ERR_ARG;
    if (parts->size == 0) return OPPB_OK;
    const int grid = oppb::ceil_div(parts->size, oppb::kMoveBlock);
    oppb::deposit_f64_kernel<<<grid, oppb::kMoveBlock, 0, oppb::as_stream(stream)>>>(
        oppb::mesh_args(mesh), oppb::part_args(parts), node_charge);
    oppb::count_launches(1);
    return oppb::launch_status();
}
