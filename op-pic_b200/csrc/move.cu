// Particle move (multi-hop barycentric cell location) and node-charge deposit for
// tetrahedral meshes, FP64 and mixed FP32/FP64.
//
// One thread per particle; particles in SoA (stride = capacity).  A cell visit reads
// 32-byte-aligned records with 256-bit loads through the read-only path: FP64 = 4 loads
// of the 128-B det record + 1 of the 32-B nav record {coef, c2c}; mixed = 2 loads of the
// f32 lambda rows + 1 of {origin, c2c}.  The L1 data pipe pays one wavefront per distinct
// cell per load instruction, so fewer, wider loads per visit is what bounds this kernel.
//
// The FP64 arithmetic uses explicit round-to-nearest intrinsics so nothing is contracted
// into FMAs: each lambda_i is bit-identical to the reference expression
//   coef * (((d0 - d1*x) + d2*y) - d3*z)          (apps/app_fempic/kernels.h:110-117)
// and the inside test / argmin follow kernels.h:121-146 exactly.
//
// Deposit (kDep): lanes of a warp holding the same cell in a contiguous run are summed
// with a segmented shuffle reduction; the run heads then either issue four FP64 global
// atomics (kDepWarp) or add into a per-CTA shared-memory table of node sums (open
// addressing) that is flushed with one global atomic per distinct node (kDepTable).

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kMoveBlock = 256;
constexpr int kSlots = 256;            // shared node-sum table (power of two, one slot per thread)
constexpr int kMaxProbe = 16;          // linear-probe bound; beyond it the sum goes straight to global
constexpr double kTol = 1e-10;         // KERNEL_TOLERENCE, apps/app_fempic/kernels.h:44
constexpr int kDepNone = 0, kDepWarp = 1, kDepTable = 2;
static_assert(kSlots == kMoveBlock, "table init/flush assume one slot per thread");

enum : int { kDone = 0, kNeedMove = 1, kNeedRemove = 2, kFailed = 3 };

struct PartArgs {
    int32_t size;
    int32_t stride;
    const double* pos;
    double* lc;
    int32_t* p2c;
    uint32_t* remove_bits;
};

struct NodeTable {
    int keys[kSlots];
    double vals[kSlots];
};

// lambda_0..3 of point (x,y,z) in cell c, evaluated exactly as the FP64 reference.
// Also returns the cell's neighbours (nav record).
__device__ __forceinline__ void visit_f64(const oppb_tet_mesh& m, int32_t c, double x, double y, double z,
                                          double l[4], int nb[4]) {
    const double* d = m.det + (int64_t)c * 16;
    double r[16];
    ldg256(d, r[0], r[1], r[2], r[3]);
    ldg256(d + 4, r[4], r[5], r[6], r[7]);
    ldg256(d + 8, r[8], r[9], r[10], r[11]);
    ldg256(d + 12, r[12], r[13], r[14], r[15]);
    double coef, n01, n23, unused;
    ldg256(m.nav + (int64_t)c * 4, coef, n01, n23, unused);
    (void)unused;
    const long long a = __double_as_longlong(n01), b = __double_as_longlong(n23);
    nb[0] = (int)(a & 0xffffffffll);
    nb[1] = (int)(a >> 32);
    nb[2] = (int)(b & 0xffffffffll);
    nb[3] = (int)(b >> 32);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double t = __dsub_rn(r[4 * i], __dmul_rn(r[4 * i + 1], x));
        t = __dadd_rn(t, __dmul_rn(r[4 * i + 2], y));
        t = __dsub_rn(t, __dmul_rn(r[4 * i + 3], z));
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

__device__ __forceinline__ int pick(const int nb[4], int i) {
    return i == 0 ? nb[0] : i == 1 ? nb[1] : i == 2 ? nb[2] : nb[3];
}

// Warp-level bookkeeping shared by all move variants: removal bitmap word, remove
// count, visit statistics.  Every lane of the warp must call it.
__device__ __forceinline__ void warp_account(const PartArgs& p, oppb_move_status* st, int64_t i, bool active,
                                             int32_t final_cell, bool newly_removed, int visits, int rechecks) {
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

__device__ __forceinline__ void table_init(NodeTable& t) {
    t.keys[threadIdx.x] = -1;
    t.vals[threadIdx.x] = 0.0;
}

// Adds v to node's slot (inserting the node), or straight to global memory when the
// probe sequence is exhausted.
__device__ __forceinline__ void table_add(NodeTable& t, double* node_charge, int node, double v) {
    uint32_t h = ((uint32_t)node * 2654435761u) >> 24;  // 8 bits
#pragma unroll 1
    for (int probe = 0; probe < kMaxProbe; probe++) {
        int k = *reinterpret_cast<volatile int*>(&t.keys[h]);
        if (k == -1) k = atomicCAS(&t.keys[h], -1, node);
        if (k == -1 || k == node) {
            atomicAdd(&t.vals[h], v);
            return;
        }
        h = (h + 1) & (kSlots - 1);
    }
    atomicAdd(node_charge + node, v);
}

__device__ __forceinline__ void table_flush(const NodeTable& t, double* node_charge) {
    const int k = t.keys[threadIdx.x];
    if (k >= 0) atomicAdd(node_charge + k, t.vals[threadIdx.x]);
}

template <int kDep>
__device__ __forceinline__ void node_add(NodeTable& t, double* node_charge, int node, double v) {
    if (kDep == kDepTable)
        table_add(t, node_charge, node, v);
    else
        atomicAdd(node_charge + node, v);
}

// Segmented sum over contiguous lanes with equal key; run heads add the four weights to
// the nodes.  key < 0 = no contribution.  Every lane of the warp must call it.
template <int kDep>
__device__ __forceinline__ void warp_deposit(const oppb_tet_mesh& m, NodeTable& t, double* node_charge, int32_t key,
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
        const int4 nodes = ldg_i4(m.c2n + (int64_t)key * 4);
        const uint32_t nn = (uint32_t)m.n_nodes;
        if ((uint32_t)nodes.x < nn) node_add<kDep>(t, node_charge, nodes.x, l0);
        if ((uint32_t)nodes.y < nn) node_add<kDep>(t, node_charge, nodes.y, l1);
        if ((uint32_t)nodes.z < nn) node_add<kDep>(t, node_charge, nodes.z, l2);
        if ((uint32_t)nodes.w < nn) node_add<kDep>(t, node_charge, nodes.w, l3);
    }
}

__device__ __forceinline__ void store_result(const PartArgs& p, int64_t i, const double l[4], int visits,
                                             int32_t cell, int32_t cell0) {
    if (visits > 0) {
        st_stream(p.lc + i, l[0]);
        st_stream(p.lc + p.stride + i, l[1]);
        st_stream(p.lc + 2 * (int64_t)p.stride + i, l[2]);
        st_stream(p.lc + 3 * (int64_t)p.stride + i, l[3]);
    }
    if (cell != cell0) st_stream(p.p2c + i, cell);
}

// ------------------------------------------------------------------ FP64 move

// Deposit epilogue shared by the move kernels.  Every thread of the CTA must call it.
template <int kDep>
__device__ __forceinline__ void deposit_epilogue(const oppb_tet_mesh& m, NodeTable& table, double* node_charge,
                                                 bool dep, int32_t cell, const double l[4]) {
    if (kDep == kDepNone) return;
    if (kDep == kDepTable) __syncthreads();  // table initialised by every thread
    warp_deposit<kDep>(m, table, node_charge, dep ? cell : -1, dep ? l[0] : 0.0, dep ? l[1] : 0.0,
                       dep ? l[2] : 0.0, dep ? l[3] : 0.0);
    if (kDep == kDepTable) {
        __syncthreads();
        table_flush(table, node_charge);
    }
}

template <int kDep>
__global__ void __launch_bounds__(kMoveBlock) move_f64_kernel(oppb_tet_mesh m, PartArgs p, double* node_charge,
                                                              oppb_move_status* st, int32_t max_hops) {
    __shared__ NodeTable table;
    if (kDep == kDepTable) table_init(table);
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
            int nb[4];
            visit_f64(m, cell, x, y, z, l, nb);
            visits++;
            if (inside_f64(l)) {
                status = kDone;
                break;
            }
            const int32_t next = pick(nb, argmin4(l));
            if (next < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = next;
            if (visits >= max_hops) {
                raise_error(st, OPPB_ERR_HOP_LIMIT, (int32_t)i);
                status = kFailed;
                break;
            }
        }
        store_result(p, i, l, visits, cell, cell0);
    }
    warp_account(p, st, i, active, cell, status == kNeedRemove, visits, 0);
    deposit_epilogue<kDep>(m, table, node_charge, active && cell0 != kRemoved && status == kDone, cell, l);
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

template <int kDep>
__global__ void __launch_bounds__(kMoveBlock) move_mixed_kernel(oppb_tet_mesh m, PartArgs p, double* node_charge,
                                                                oppb_move_status* st, int32_t max_hops,
                                                                float band) {
    __shared__ NodeTable table;
    if (kDep == kDepTable) table_init(table);
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
            float nv[8], g0[8], g1[8];
            ldg256(m.nav32 + (int64_t)cell * 8, nv);
            ldg256(m.geo32 + (int64_t)cell * 16, g0);
            ldg256(m.geo32 + (int64_t)cell * 16 + 8, g1);
            const float dx = (float)(x - (double)nv[0]);
            const float dy = (float)(y - (double)nv[1]);
            const float dz = (float)(z - (double)nv[2]);
            const float rows[16] = {g0[0], g0[1], g0[2], g0[3], g0[4], g0[5], g0[6], g0[7],
                                    g1[0], g1[1], g1[2], g1[3], g1[4], g1[5], g1[6], g1[7]};
            float lf[4];
            float smax = 0.0f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float c0 = rows[4 * k], gx = rows[4 * k + 1], gy = rows[4 * k + 2], gz = rows[4 * k + 3];
                lf[k] = fmaf(gz, dz, fmaf(gy, dy, fmaf(gx, dx, c0)));
                const float s = fabsf(c0) + fabsf(gx) * fabsf(dx) + fabsf(gy) * fabsf(dy) + fabsf(gz) * fabsf(dz);
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
                int nb_unused[4];
                visit_f64(m, cell, x, y, z, l, nb_unused);
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
            const int32_t next = __float_as_int(nv[4 + mi]);
            if (next < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = next;
            if (visits >= max_hops) {
                raise_error(st, OPPB_ERR_HOP_LIMIT, (int32_t)i);
                status = kFailed;
                break;
            }
        }
        store_result(p, i, l, visits, cell, cell0);
    }
    warp_account(p, st, i, active, cell, status == kNeedRemove, visits, rechecks);
    deposit_epilogue<kDep>(m, table, node_charge, active && cell0 != kRemoved && status == kDone, cell, l);
}

// ------------------------------------------------------------- standalone deposit

template <int kDep>
__global__ void __launch_bounds__(kMoveBlock) deposit_f64_kernel(oppb_tet_mesh m, PartArgs p, double* node_charge) {
    __shared__ NodeTable table;
    if (kDep == kDepTable) table_init(table);
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < p.size;
    int32_t cell = active ? ld_stream(p.p2c + i) : -1;
    const bool ok = active && (uint32_t)cell < (uint32_t)m.n_cells;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok) {
        l[0] = ld_stream(p.lc + i);
        l[1] = ld_stream(p.lc + p.stride + i);
        l[2] = ld_stream(p.lc + 2 * (int64_t)p.stride + i);
        l[3] = ld_stream(p.lc + 3 * (int64_t)p.stride + i);
    }
    deposit_epilogue<kDep>(m, table, node_charge, ok, cell, l);
}

int check_mesh(const oppb_tet_mesh* mesh, bool mixed, bool need_c2n) {
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0) return OPPB_ERR_ARG;
    if (!mesh->det || !mesh->nav || !aligned(mesh->det, 32) || !aligned(mesh->nav, 32)) return OPPB_ERR_ARG;
    if (need_c2n && (!mesh->c2n || !aligned(mesh->c2n, 16))) return OPPB_ERR_ARG;
    if (mixed && (!mesh->geo32 || !mesh->nav32 || !aligned(mesh->geo32, 32) || !aligned(mesh->nav32, 32)))
        return OPPB_ERR_ARG;
    return OPPB_OK;
}

int check_parts(const oppb_particles* p, bool need_bits) {
    if (!p || p->size < 0 || p->stride < p->size) return OPPB_ERR_ARG;
    if (!p->pos || !p->lc || !p->p2c) return OPPB_ERR_ARG;
    if (need_bits && !p->remove_bits) return OPPB_ERR_ARG;
    return OPPB_OK;
}

PartArgs part_args(const oppb_particles* p) {
    return PartArgs{p->size, p->stride, p->pos, p->lc, p->p2c, p->remove_bits};
}

template <int kKind>  // 0 move, 1 move+deposit, 2 mixed move+deposit
int launch_move(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                oppb_move_status* status, int32_t max_hops, double band, void* stream) {
    int rc = check_mesh(mesh, kKind == 2, kKind != 0);
    if (rc) return rc;
    rc = check_parts(parts, true);
    if (rc) return rc;
    if (!status || max_hops <= 0) return OPPB_ERR_ARG;
    if (kKind != 0 && !node_charge) return OPPB_ERR_ARG;
    if (kKind == 2 && !(band > 0.0 && band < 0.25)) return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(status, 0, sizeof(oppb_move_status), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    if (parts->size == 0) return launch_status();
    const PartArgs p = part_args(parts);
    const int grid = ceil_div(parts->size, kMoveBlock);
    const bool table = tuning().deposit == OPPB_DEPOSIT_CTA_TABLE;
    if (kKind == 0)
        move_f64_kernel<kDepNone><<<grid, kMoveBlock, 0, s>>>(*mesh, p, nullptr, status, max_hops);
    else if (kKind == 1 && table)
        move_f64_kernel<kDepTable><<<grid, kMoveBlock, 0, s>>>(*mesh, p, node_charge, status, max_hops);
    else if (kKind == 1)
        move_f64_kernel<kDepWarp><<<grid, kMoveBlock, 0, s>>>(*mesh, p, node_charge, status, max_hops);
    else if (table)
        move_mixed_kernel<kDepTable><<<grid, kMoveBlock, 0, s>>>(*mesh, p, node_charge, status, max_hops,
                                                                 (float)band);
    else
        move_mixed_kernel<kDepWarp><<<grid, kMoveBlock, 0, s>>>(*mesh, p, node_charge, status, max_hops,
                                                                (float)band);
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
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0 || !mesh->c2n || !oppb::aligned(mesh->c2n, 16))
        return OPPB_ERR_ARG;
    if (!parts || parts->size < 0 || parts->stride < parts->size || !parts->lc || !parts->p2c || !node_charge)
        return OPPB_ERR_ARG;
    if (parts->size == 0) return OPPB_OK;
    const int grid = oppb::ceil_div(parts->size, oppb::kMoveBlock);
    if (oppb::tuning().deposit == OPPB_DEPOSIT_CTA_TABLE)
        oppb::deposit_f64_kernel<oppb::kDepTable><<<grid, oppb::kMoveBlock, 0, oppb::as_stream(stream)>>>(
            *mesh, oppb::part_args(parts), node_charge);
    else
        oppb::deposit_f64_kernel<oppb::kDepWarp><<<grid, oppb::kMoveBlock, 0, oppb::as_stream(stream)>>>(
            *mesh, oppb::part_args(parts), node_charge);
    oppb::count_launches(1);
    return oppb::launch_status();
}
