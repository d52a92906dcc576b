// Particle move (multi-hop barycentric cell location) and node-charge deposit for
// tetrahedral meshes, FP64 and mixed FP32/FP64.
//
// One thread per particle; particles in SoA (stride = capacity).  A cell visit is a
// dependent gather of the cell's record with 256-bit loads through the read-only path:
// FP64 = 4 loads of the 128-B det record + 1 of the 32-B nav record {coef, c2c}; mixed =
// 2 loads of the 64-B f32 record {3 lambda rows, origin}, + the 16-B c2c on a hop.  Lanes
// of a warp share cells only while the particles are still close to their sorted order,
// so a load instruction pays up to one L1 sector per lane; the L1 data pipe is what
// bounds the kernel, hence few wide loads per visit and a 32-register cap (full
// occupancy hides the dependent-gather latency).
//
// The FP64 arithmetic uses explicit round-to-nearest intrinsics so nothing is contracted
// into FMAs: each lambda_i is bit-identical to the reference expression
//   coef * (((d0 - d1*x) + d2*y) - d3*z)          (apps/app_fempic/kernels.h:110-117)
// and the inside test / argmin follow kernels.h:121-146 exactly.
//
// Deposit (kDep): lanes ending in the same cell are grouped with a warp match; the lowest
// lane of a group sums the group's weights by shuffles and issues four FP64 atomics
// (kDepWarp), or adds into a per-CTA shared-memory node table flushed once per node
// (kDepTable).  The atomics of CTA b go to node-sum copy b % R (copy 0 = node_charge,
// copies 1..R-1 in the caller's workspace) so that neighbouring CTAs, which deposit on the
// same nodes, do not serialise on one address; the copies are added afterwards.  The
// deterministic mode (kDepExact) groups lanes the same way but sums weights cut to
// multiples of 2^-52 as integers, with 64-bit integer atomics into two sums per node that a
// finishing kernel turns into FP64: the result does not depend on the order of the additions.

#include "oppb_common.cuh"
#include "oppb_dh.h"
#include "tet_f64.cuh"

namespace oppb {
namespace {

constexpr int kMoveBlock = 256;
constexpr int kMinBlocks = 8;          // 8 x 256 threads per SM: 32 registers per thread
constexpr int kThreadsPerSm = kMoveBlock * kMinBlocks;  // every block shape keeps 32 registers a thread
constexpr int kSlots = 256;            // shared node-sum table (power of two, one slot per thread)
constexpr int kMaxProbe = 16;          // linear-probe bound; beyond it the sum goes straight to global
constexpr int kDepNone = 0, kDepWarp = 1, kDepTable = 2, kDepExact = 3;
static_assert(kSlots == kMoveBlock, "table init/flush assume one slot per thread");

enum : int { kDone = 0, kNeedMove = 1, kNeedRemove = 2, kFailed = 3 };

struct PartArgs {
    int32_t size;         // the particle count; with count_dev, an upper bound of it
    int32_t stride;
    double* pos;          // written only by the fused push
    double* vel;          // fused push only
    double* lc;
    int32_t* p2c;
    uint32_t* remove_bits;
    const int32_t* count_dev;  // oppb_set_count::size (device), or nullptr
    int32_t pending;           // particles injected since *count_dev was set
};

// The particle count of a launch: the host's, or the device count plus the pending
// injections, capped by the host's bound (include/oppb_graph.h).  Written by earlier
// launches of the stream, so a plain load sees it.
__device__ __forceinline__ int32_t live_count(const PartArgs& p) {
    if (!p.count_dev) return p.size;
    const int32_t n = *p.count_dev + p.pending;
    return n < p.size ? n : p.size;
}

// Push prologue of the fused entry points: calculate_new_pos_vel_kernel
// (apps/app_fempic/kernels.h:93-103) run on the particle's registers before its walk, the
// role OPP_DO_ONCE gives a push inside a move loop (opp_lib/include/opp_seq.h:64).
struct PushArgs {
    double qm, dt;     // FP64 push
    float qmdt, dtf;   // mixed push: f32(q/m*dt), f32(dt)
};

// Node-sum target of this CTA: copy (blockIdx.x % replicas).
struct DepositArgs {
    double* node_charge;
    double* copies;     // replicas - 1 arrays of n_nodes, or nullptr
    int32_t replicas;
    unsigned long long* exact;  // OPPB_DEPOSIT_EXACT: [2][n_nodes] sums of multiples of 2^-20, of 2^-52
};

struct NodeTable {
    int keys[kSlots];
    double vals[kSlots];
};

// Direct-hop seed (include/oppb_dh.h): the structured grid, passed by value.
struct DhArgs {
    const int32_t* map;
    double min[3];
    double inv;
    unsigned long long dims[3];
};

// Cell of the grid box holding (x, y, z), or kRemoved: opp_dev_findStructuredCellIndex3D and
// opp_dev_checkForGlobalMove (opp_lib/include/device_kernels/cuda_inline_kernels.h).  Each
// index is (pos - min) * (1/h) truncated by a round-toward-zero conversion that saturates
// (negative and NaN give 0), the conversion the reference's (size_t) cast compiles to.
__device__ __forceinline__ int32_t dh_seed(const DhArgs& g, double x, double y, double z) {
    const unsigned long long ix = __double2ull_rz(__dmul_rn(__dsub_rn(x, g.min[0]), g.inv));
    const unsigned long long iy = __double2ull_rz(__dmul_rn(__dsub_rn(y, g.min[1]), g.inv));
    const unsigned long long iz = __double2ull_rz(__dmul_rn(__dsub_rn(z, g.min[2]), g.inv));
    if (ix >= g.dims[0] || iy >= g.dims[1] || iz >= g.dims[2]) return kRemoved;
    return __ldg(g.map + (int64_t)(ix + g.dims[0] * (iy + g.dims[1] * iz)));
}

__device__ __forceinline__ double* deposit_target(const DepositArgs& d, int32_t n_nodes) {
    const int r = d.replicas > 1 ? (int)(blockIdx.x % (unsigned)d.replicas) : 0;
    return r == 0 ? d.node_charge : d.copies + (int64_t)(r - 1) * n_nodes;
}

// The FP64 re-evaluation of the mixed path, kept out of line: it is rare, and inlined it
// would raise the register count of the whole kernel.
__device__ __noinline__ void recheck_f64(const oppb_tet_mesh& m, int32_t c, double x, double y, double z,
                                         double* l) {
    int nb[4];
    visit_f64(m, c, x, y, z, l, nb);
}

// Bookkeeping shared by all move variants: the warp's removal bitmap word, then the CTA's
// remove count, visit sum, visit maximum and recheck count, reduced in shared memory and
// added to the status with one atomic per counter per CTA.  Every CTA updates the same
// few status words, so per-warp atomics there serialise in L2 and cost as much as a
// large share of the move itself.  Every thread of the CTA must call it.
template <int kBlock = kMoveBlock>
__device__ __forceinline__ void cta_account(const PartArgs& p, oppb_move_status* st, int64_t i, bool active,
                                            int32_t final_cell, bool newly_removed, int visits, int rechecks) {
    constexpr int kWarps = kBlock / 32;
    static_assert(kWarps >= 1 && kWarps <= 32 && (kWarps & (kWarps - 1)) == 0, "a power-of-two warp count");
    __shared__ unsigned long long s_sum[kWarps];
    __shared__ int s_cnt[kWarps][3];  // removed, max visits, rechecks
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned hole = __ballot_sync(kFullMask, active && final_cell == kRemoved);
    const unsigned rem = __ballot_sync(kFullMask, newly_removed);
    if (lane == 0 && active) p.remove_bits[i >> 5] = hole;  // lane 0 active: the word holds live particles
    // Warp reductions in the integer reduce unit (shuffles would load the L1 data pipe the
    // visits are bound by).  The visit sum is taken in 16-bit halves so that 32 lanes
    // cannot overflow 32 bits whatever max_hops is.
    const int vmax = (int)__reduce_max_sync(kFullMask, (unsigned)visits);
    const int rsum = (int)__reduce_add_sync(kFullMask, (unsigned)rechecks);
    const unsigned long long vsum =
        ((unsigned long long)__reduce_add_sync(kFullMask, (unsigned)visits >> 16) << 16) +
        __reduce_add_sync(kFullMask, (unsigned)visits & 0xffffu);
    if (lane == 0) {
        s_sum[warp] = vsum;
        s_cnt[warp][0] = __popc(rem);
        s_cnt[warp][1] = vmax;
        s_cnt[warp][2] = rsum;
    }
    __syncthreads();
    if (warp == 0) {
        const bool mine = lane < kWarps;
        unsigned long long s = mine ? s_sum[lane] : 0ull;
        int r = mine ? s_cnt[lane][0] : 0, m = mine ? s_cnt[lane][1] : 0, c = mine ? s_cnt[lane][2] : 0;
#pragma unroll
        for (int o = kWarps / 2; o > 0; o >>= 1) {
            s += __shfl_xor_sync(kFullMask, s, o);
            r += __shfl_xor_sync(kFullMask, r, o);
            m = max(m, __shfl_xor_sync(kFullMask, m, o));
            c += __shfl_xor_sync(kFullMask, c, o);
        }
        if (lane == 0) {
            if (r) atomicAdd(&st->remove_count, r);
            if (s) atomicAdd(reinterpret_cast<unsigned long long*>(&st->total_visits), s);
            if (m) atomicMax(&st->max_visits, m);
            if (c) atomicAdd(&st->recheck_count, c);
        }
    }
}

__device__ __forceinline__ void table_init(NodeTable& t) {
    t.keys[threadIdx.x] = -1;
    t.vals[threadIdx.x] = 0.0;
}

// Adds v to node's slot (inserting the node), or straight to global memory when the
// probe sequence is exhausted.
__device__ __forceinline__ void table_add(NodeTable& t, double* target, int node, double v) {
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
    atomicAdd(target + node, v);
}

template <int kDep>
__device__ __forceinline__ void node_add(NodeTable& t, double* target, int node, double v) {
    if (kDep == kDepTable)
        table_add(t, target, node, v);
    else
        atomicAdd(target + node, v);
}

// Lanes with equal key form a group; the group's lowest lane sums the group's weights
// (shuffle loop over the group members) in FP64 and adds them to the cell's four nodes.
// T is the weights' type: FP32 weights (mixed path) take half the shuffles of FP64 ones.
// key < 0 = no contribution.  Every lane of the warp must call it.
template <int kDep, typename T>
__device__ __forceinline__ void warp_deposit(const oppb_tet_mesh& m, NodeTable& t, double* target, int32_t key,
                                             T l0, T l1, T l2, T l3) {
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(kFullMask, key);
    const bool leader = (lane == __ffs(peers) - 1) && key >= 0;
    unsigned rest = leader ? (peers & ~(1u << lane)) : 0u;
    double s0 = l0, s1 = l1, s2 = l2, s3 = l3;
    while (__any_sync(kFullMask, rest != 0)) {
        const int src = rest ? __ffs(rest) - 1 : lane;
        const T a0 = __shfl_sync(kFullMask, l0, src);
        const T a1 = __shfl_sync(kFullMask, l1, src);
        const T a2 = __shfl_sync(kFullMask, l2, src);
        const T a3 = __shfl_sync(kFullMask, l3, src);
        if (rest) {
            s0 += a0;
            s1 += a1;
            s2 += a2;
            s3 += a3;
            rest &= rest - 1;
        }
    }
    if (leader) {
        const int4 nodes = ldg_i4(m.c2n + (int64_t)key * 4);
        const uint32_t nn = (uint32_t)m.n_nodes;
        if ((uint32_t)nodes.x < nn) node_add<kDep>(t, target, nodes.x, s0);
        if ((uint32_t)nodes.y < nn) node_add<kDep>(t, target, nodes.y, s1);
        if ((uint32_t)nodes.z < nn) node_add<kDep>(t, target, nodes.z, s2);
        if ((uint32_t)nodes.w < nn) node_add<kDep>(t, target, nodes.w, s3);
    }
}

// Fixed-point parts of a weight for OPPB_DEPOSIT_EXACT: u = floor(w 2^52) (w 2^52 is exact,
// a power-of-two scaling, and so is its floor; |u| < 2^63 for |w| < 2^11) split as
// u = a 2^32 + b with a = u >> 32 (the floor of u / 2^32) and b = u mod 2^32, so that
// w = a 2^-20 + b 2^-52 + r with 0 <= r < 2^-52 for weights of either sign.
__device__ __forceinline__ void exact_parts(double w, int32_t& a, uint32_t& b) {
    const long long u = __double2ll_rz(floor(__dmul_rn(w, 4503599627370496.0)));
    a = (int32_t)(u >> 32);
    b = (uint32_t)(u & 0xffffffffll);
}

// The warp-grouped deposit of OPPB_DEPOSIT_EXACT: each lane cuts its four weights to fixed
// point, the lowest lane of a cell group adds the group's integers, and the sums go to the
// integer node sums with 64-bit atomics.  Integer sums do not depend on their order.
template <typename T>
__device__ __forceinline__ void warp_deposit_exact(const oppb_tet_mesh& m, unsigned long long* acc, int32_t key,
                                                   T l0, T l1, T l2, T l3) {
    const int lane = threadIdx.x & 31;
    int32_t a0, a1, a2, a3;
    uint32_t b0, b1, b2, b3;
    exact_parts((double)l0, a0, b0);
    exact_parts((double)l1, a1, b1);
    exact_parts((double)l2, a2, b2);
    exact_parts((double)l3, a3, b3);
    const unsigned peers = __match_any_sync(kFullMask, key);
    const bool leader = (lane == __ffs(peers) - 1) && key >= 0;
    unsigned rest = leader ? (peers & ~(1u << lane)) : 0u;
    long long h0 = a0, h1 = a1, h2 = a2, h3 = a3;
    unsigned long long g0 = b0, g1 = b1, g2 = b2, g3 = b3;
    while (__any_sync(kFullMask, rest != 0)) {
        const int src = rest ? __ffs(rest) - 1 : lane;
        const int32_t x0 = __shfl_sync(kFullMask, a0, src), x1 = __shfl_sync(kFullMask, a1, src);
        const int32_t x2 = __shfl_sync(kFullMask, a2, src), x3 = __shfl_sync(kFullMask, a3, src);
        const uint32_t y0 = __shfl_sync(kFullMask, b0, src), y1 = __shfl_sync(kFullMask, b1, src);
        const uint32_t y2 = __shfl_sync(kFullMask, b2, src), y3 = __shfl_sync(kFullMask, b3, src);
        if (rest) {
            h0 += x0, h1 += x1, h2 += x2, h3 += x3;
            g0 += y0, g1 += y1, g2 += y2, g3 += y3;
            rest &= rest - 1;
        }
    }
    if (leader) {
        const int4 nodes = ldg_i4(m.c2n + (int64_t)key * 4);
        const uint32_t nn = (uint32_t)m.n_nodes;
        unsigned long long* lo = acc + nn;
        if ((uint32_t)nodes.x < nn) atomicAdd(acc + nodes.x, (unsigned long long)h0), atomicAdd(lo + nodes.x, g0);
        if ((uint32_t)nodes.y < nn) atomicAdd(acc + nodes.y, (unsigned long long)h1), atomicAdd(lo + nodes.y, g1);
        if ((uint32_t)nodes.z < nn) atomicAdd(acc + nodes.z, (unsigned long long)h2), atomicAdd(lo + nodes.z, g2);
        if ((uint32_t)nodes.w < nn) atomicAdd(acc + nodes.w, (unsigned long long)h3), atomicAdd(lo + nodes.w, g3);
    }
}

// Deposit epilogue shared by the move kernels.  Every thread of the CTA must call it.
template <int kDep, typename T>
__device__ __forceinline__ void deposit_epilogue(const oppb_tet_mesh& m, NodeTable& table, const DepositArgs& d,
                                                 bool dep, int32_t cell, const T l[4]) {
    if (kDep == kDepNone) return;
    if (kDep == kDepExact) {
        const T zero = 0;
        warp_deposit_exact<T>(m, d.exact, dep ? cell : -1, dep ? l[0] : zero, dep ? l[1] : zero, dep ? l[2] : zero,
                              dep ? l[3] : zero);
        return;
    }
    double* target = deposit_target(d, m.n_nodes);
    if (kDep == kDepTable) __syncthreads();  // table initialised by every thread
    const T zero = 0;
    warp_deposit<kDep, T>(m, table, target, dep ? cell : -1, dep ? l[0] : zero, dep ? l[1] : zero,
                          dep ? l[2] : zero, dep ? l[3] : zero);
    if (kDep == kDepTable) {
        __syncthreads();
        const int k = table.keys[threadIdx.x];
        if (k >= 0) atomicAdd(target + k, table.vals[threadIdx.x]);
    }
}

template <typename T>
__device__ __forceinline__ void store_result(const PartArgs& p, int64_t i, const T l[4], int visits,
                                             int32_t cell, int32_t cell0) {
    if (visits > 0) {
        st_stream(p.lc + i, (double)l[0]);
        st_stream(p.lc + p.stride + i, (double)l[1]);
        st_stream(p.lc + 2 * (int64_t)p.stride + i, (double)l[2]);
        st_stream(p.lc + 3 * (int64_t)p.stride + i, (double)l[3]);
    }
    if (cell != cell0) st_stream(p.p2c + i, cell);
}

// v += (q/m) dt E[cell]; x += v dt, stored back and left in x, y, z.  The operation order
// and rounding are those of push_f64_kernel (FP64) and push_mixed_kernel (FP32 increments on
// FP64 state), so a fused step is bit-identical to push + move.
template <bool kMixed>
__device__ __forceinline__ void push_prologue(const oppb_tet_mesh& m, const PartArgs& p, const PushArgs& a,
                                              int64_t i, int32_t cell, double& x, double& y, double& z) {
    const double2 e01 = ldg_d2(m.ef + (int64_t)cell * 4);
    const double2 e2_ = ldg_d2(m.ef + (int64_t)cell * 4 + 2);
    const double e[3] = {e01.x, e01.y, e2_.x};
    double xs[3] = {x, y, z};
    const double coefficient1 = __dmul_rn(a.qm, a.dt);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double* vp = p.vel + (int64_t)d * p.stride + i;
        double v;
        if (kMixed) {
            const float dv = __fmul_rn(a.qmdt, __double2float_rn(e[d]));
            v = __dadd_rn(ld_stream(vp), (double)dv);
            xs[d] = __dadd_rn(xs[d], (double)__fmul_rn(__double2float_rn(v), a.dtf));
        } else {
            v = __dadd_rn(ld_stream(vp), __dmul_rn(coefficient1, e[d]));
            xs[d] = __dadd_rn(xs[d], __dmul_rn(v, a.dt));
        }
        st_stream(vp, v);
        st_stream(p.pos + (int64_t)d * p.stride + i, xs[d]);
    }
    x = xs[0];
    y = xs[1];
    z = xs[2];
}

// ------------------------------------------------------------------ FP64 move

// kBlock: threads per CTA (oppb_tuning.move_block; 256 for the CTA-table deposit, whose
// node table has one slot per thread), with 2048 / kBlock CTAs resident per SM.
template <int kDep, bool kPush, bool kSeed, bool kDevCount = false, int kBlock = kMoveBlock>
__global__ void __launch_bounds__(kBlock, kThreadsPerSm / kBlock)
    move_f64_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep, oppb_move_status* st, int32_t max_hops,
                    PushArgs push, DhArgs dh) {
    static_assert(kBlock == kMoveBlock || kDep != kDepTable, "the node table is sized for 256 threads");
    __shared__ NodeTable table;
    const int32_t n = kDevCount ? live_count(p) : p.size;
    if (kDevCount && (int64_t)blockIdx.x * kBlock >= n) return;  // beyond the device count (whole block)
    if (kDep == kDepTable) table_init(table);
    const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < n;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int status = kDone;
    int visits = 0;
    int err = 0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (active && cell != kRemoved) {
        double x = ld_stream(p.pos + i);
        double y = ld_stream(p.pos + p.stride + i);
        double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        if (kPush && (uint32_t)cell < (uint32_t)m.n_cells) push_prologue<false>(m, p, push, i, cell, x, y, z);
        if (kSeed) {  // the walk starts from the grid box's cell (after the push, as the reference)
            cell = dh_seed(dh, x, y, z);
            if (cell == kRemoved) status = kNeedRemove;
        }
        while (!kSeed || cell != kRemoved) {
            if ((uint32_t)cell >= (uint32_t)m.n_cells) {
                err = OPPB_ERR_CELL_RANGE;
                break;
            }
            int nb[4];
            visit_f64(m, cell, x, y, z, l, nb);
            visits++;
            if (inside_f64(l)) break;
            const int32_t next = pick(nb, argmin4(l));
            if (next < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = next;
            if (visits >= max_hops) {
                err = OPPB_ERR_HOP_LIMIT;
                break;
            }
        }
        if (err) {
            raise_error(st, err, (int32_t)i);
            status = kFailed;
        }
        store_result(p, i, l, visits, cell, cell0);
    }
    cta_account<kBlock>(p, st, i, active, cell, status == kNeedRemove, visits, 0);
    deposit_epilogue<kDep>(m, table, dep, active && cell0 != kRemoved && status == kDone, cell, l);
}

// ------------------------------------------------ FP64 move, two lanes per particle
//
// oppb_tuning.move_lanes = 2.  A cell visit of the one-lane kernel is five 256-bit loads by
// one lane, each touching its own L1 line when the warp's lanes sit in different cells, so
// the L1 data pipe serves five wavefronts per visit.  Here a lane pair walks one particle:
// lane h reads the half [8h, 8h+8) of the 128-B det record (vertices 2h and 2h+1, two
// 256-bit loads) and 16 B of the nav record (h = 0: coef and c2c[0..1]; h = 1: c2c[2..3]),
// and computes lambda_2h and lambda_2h+1 with the reference's expression; both lanes of a
// pair read the same lines, so a visit costs three wavefronts.  The pair agrees on the
// inside test with a vote, gathers the other two lambdas by shuffles for the first-index
// argmin, and takes the neighbour from the lane that holds it: the decisions and lambdas
// are bit-identical to move_f64_kernel's.
//
// The CTA works in three phases.  (1) Thread t loads (and pushes) particle t with coalesced
// accesses into shared memory.  (2) The 128 pairs take particles from a CTA counter until
// the CTA's 256 are walked, so a long walk does not hold the other lanes of its warp idle.
// (3) Thread t stores particle t's result and runs the accounting and deposit of the
// one-lane kernel.

constexpr int kInfoVisits = 0x3fffffff, kInfoRemoved = 1 << 30, kInfoFailed = 1 << 31;

// One lambda of the reference expression coef * (((d0 - d1 x) + d2 y) - d3 z).
__device__ __forceinline__ double lambda_f64(double coef, double d0, double d1, double d2, double d3, double x,
                                             double y, double z) {
    double t = __dsub_rn(d0, __dmul_rn(d1, x));
    t = __dadd_rn(t, __dmul_rn(d2, y));
    t = __dsub_rn(t, __dmul_rn(d3, z));
    return __dmul_rn(coef, t);
}

__device__ __forceinline__ bool in_band_f64(double l) { return (l > -kTol) && (__dsub_rn(l, 1.0) < kTol); }

template <int kDep, bool kPush, bool kDevCount, int kOcc>
__global__ void __launch_bounds__(kMoveBlock, kOcc)
    move_f64_pair_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep, oppb_move_status* st, int32_t max_hops,
                         PushArgs push) {
    __shared__ NodeTable table;
    __shared__ double s_x[3][kMoveBlock];
    __shared__ double s_l[4][kMoveBlock];
    __shared__ int32_t s_cell[kMoveBlock];
    __shared__ int32_t s_cell0[kMoveBlock];
    __shared__ int32_t s_info[kMoveBlock];
    __shared__ int s_next;
    const int32_t n = kDevCount ? live_count(p) : p.size;
    const int64_t base = (int64_t)blockIdx.x * kMoveBlock;
    if (kDevCount && base >= n) return;  // beyond the device count (whole block)
    if (kDep == kDepTable) table_init(table);
    const int t = threadIdx.x;
    {
    const int64_t i = base + t;
    const bool active = i < n;
    const int32_t cell0 = active ? ld_stream(p.p2c + i) : kRemoved;
    // (1) load and push
    if (active && cell0 != kRemoved) {
        double x = ld_stream(p.pos + i);
        double y = ld_stream(p.pos + p.stride + i);
        double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        if (kPush && (uint32_t)cell0 < (uint32_t)m.n_cells) push_prologue<false>(m, p, push, i, cell0, x, y, z);
        s_x[0][t] = x;
        s_x[1][t] = y;
        s_x[2][t] = z;
    }
    s_cell[t] = cell0;
    s_cell0[t] = cell0;
    s_info[t] = 0;
    if (t == 0) s_next = 0;
    }
    __syncthreads();
    // (2) pairs walk the CTA's particles
    {
        const int count = (int64_t)n - base < kMoveBlock ? (int)((int64_t)n - base) : kMoveBlock;
        const int lane = t & 31;
        const int h = lane & 1;
        const int src0 = lane & 30;
        const unsigned pm = 3u << src0;
        for (;;) {
            int slot = 0;
            if (h == 0) slot = atomicAdd(&s_next, 1);
            slot = __shfl_sync(pm, slot, src0);
            if (slot >= count) break;
            int32_t cell = s_cell[slot];
            if (cell == kRemoved) continue;
            double la = 0.0, lb = 0.0;  // lambda_2h, lambda_2h+1
            int visits = 0, err = 0;
            bool removed = false;
            for (;;) {
                if ((uint32_t)cell >= (uint32_t)m.n_cells) {
                    err = OPPB_ERR_CELL_RANGE;
                    break;
                }
                const double* d = m.det + (int64_t)cell * 16 + 8 * h;
                double a0, b0, g0, d0, a1, b1, g1, d1;
                ldg256(d, a0, b0, g0, d0);
                ldg256(d + 4, a1, b1, g1, d1);
                const double2 nv = ldg_d2(m.nav + (int64_t)cell * 4 + 2 * h);
                const double coef = __shfl_sync(pm, nv.x, src0);
                // the position from shared memory at every visit: registers are what the walk is short of
                const double x = s_x[0][slot], y = s_x[1][slot], z = s_x[2][slot];
                la = lambda_f64(coef, a0, b0, g0, d0, x, y, z);
                lb = lambda_f64(coef, a1, b1, g1, d1, x, y, z);
                visits++;
                if (__all_sync(pm, in_band_f64(la) && in_band_f64(lb))) break;
                const double oa = __shfl_xor_sync(pm, la, 1), ob = __shfl_xor_sync(pm, lb, 1);
                const double l[4] = {h ? oa : la, h ? ob : lb, h ? la : oa, h ? lb : ob};
                const int mi = argmin4(l);
                // c2c[0..1] are lane 0's nv.y, c2c[2..3] lane 1's nv.x.
                const double pair_bits = __shfl_sync(pm, h ? nv.x : nv.y, src0 + (mi >> 1));
                const long long b = __double_as_longlong(pair_bits);
                const int32_t next = (mi & 1) ? (int32_t)(b >> 32) : (int32_t)(b & 0xffffffffll);
                if (next < 0) {
                    cell = kRemoved;
                    removed = true;
                    break;
                }
                cell = next;
                if (visits >= max_hops) {
                    err = OPPB_ERR_HOP_LIMIT;
                    break;
                }
            }
            s_l[2 * h][slot] = la;
            s_l[2 * h + 1][slot] = lb;
            if (h == 0) {
                s_cell[slot] = cell;
                s_info[slot] = visits | (removed ? kInfoRemoved : 0) | (err ? kInfoFailed : 0);
                if (err) raise_error(st, err, (int32_t)(base + slot));
            }
        }
    }
    __syncthreads();
    // (3) results, accounting, deposit
    const int64_t i = base + t;
    const bool active = i < n;
    const int32_t cell0 = s_cell0[t];
    int visits = 0;
    bool newly_removed = false, failed = false;
    int32_t cell = cell0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (active && cell0 != kRemoved) {
        const int info = s_info[t];
        visits = info & kInfoVisits;
        newly_removed = (info & kInfoRemoved) != 0;
        failed = (info & kInfoFailed) != 0;
        cell = s_cell[t];
#pragma unroll
        for (int k = 0; k < 4; k++) l[k] = s_l[k][t];
        store_result(p, i, l, visits, cell, cell0);
    }
    cta_account(p, st, i, active, cell, newly_removed, visits, 0);
    deposit_epilogue<kDep>(m, table, dep, active && cell0 != kRemoved && !newly_removed && !failed, cell, l);
}

// ------------------------------------ FP64 move, cell records staged by bulk async copies
//
// oppb_tuning.move_stage = 1.  The one-lane walk, with each visit's 160-B cell record (the
// 128-B det record and the 32-B nav record) brought into the lane's slot of shared memory by
// two bulk asynchronous copies (cp.async.bulk, handled by the copy engine rather than the L1
// load pipe that bounds the 256-bit-load kernel) instead of five 256-bit loads.  A warp visits
// in lock step: lane 0 posts the expected bytes of the warp's active lanes on the warp's
// mbarrier, every active lane issues its two copies, the warp waits on the barrier's phase,
// and each lane reads its record from shared memory (a 176-B slot stride, so that eight lanes'
// 128-bit reads hit distinct banks) and evaluates it with the reference expression.  Every
// wait is bounded: a wait that runs out records OPPB_ERR_WAIT_LIMIT, waits once more (bounded)
// for the copies in flight and ends the walks.  Decisions, lambdas and counts are
// bit-identical to move_f64_kernel's.

constexpr int kStageOcc = 4;            // CTAs per SM: 45 KB of record slots each
constexpr int kStageSlot = 22;          // doubles per lane slot: 160 B of record + 16 B of padding
constexpr long kStagePolls = 1L << 20;  // bound on the barrier polls of one visit (each suspends <= 1 us)

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) { return (uint32_t)__cvta_generic_to_shared(ptr); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-B aligned) from global memory into
// this CTA's shared memory, completing `bytes` transactions on the mbarrier.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Polls the warp's barrier for `parity`, at most kStagePolls times; the result is the warp's.
__device__ __forceinline__ bool warp_wait_phase(uint64_t* bar, uint32_t parity) {
    bool done = false;
    for (long k = 0; k < kStagePolls && !done; k++) done = __all_sync(kFullMask, mbar_try_wait(bar, parity));
    return done;
}

template <int kDep, bool kPush, bool kDevCount>
__global__ void __launch_bounds__(kMoveBlock, kStageOcc)
    move_f64_stage_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep, oppb_move_status* st, int32_t max_hops,
                          PushArgs push) {
    __shared__ NodeTable table;
    __shared__ __align__(16) double s_rec[kMoveBlock * kStageSlot];
    __shared__ __align__(8) uint64_t s_bar[kMoveBlock / 32];
    const int32_t n = kDevCount ? live_count(p) : p.size;
    if (kDevCount && (int64_t)blockIdx.x * kMoveBlock >= n) return;  // beyond the device count (whole block)
    if (kDep == kDepTable) table_init(table);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t* bar = &s_bar[warp];
    if (lane == 0) mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < n;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int status = kDone, visits = 0, err = 0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    double x = 0.0, y = 0.0, z = 0.0;
    bool walking = active && cell != kRemoved;
    if (walking) {
        x = ld_stream(p.pos + i);
        y = ld_stream(p.pos + p.stride + i);
        z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        if (kPush && (uint32_t)cell < (uint32_t)m.n_cells) push_prologue<false>(m, p, push, i, cell, x, y, z);
    }
    double* slot = s_rec + threadIdx.x * kStageSlot;
    uint32_t parity = 0;
    for (;;) {
        if (walking && (uint32_t)cell >= (uint32_t)m.n_cells) {
            err = OPPB_ERR_CELL_RANGE;
            walking = false;
        }
        const unsigned wm = __ballot_sync(kFullMask, walking);
        if (!wm) break;
        if (lane == 0) mbar_arrive_expect_tx(bar, 160u * (uint32_t)__popc(wm));
        if (walking) {
            // this lane's reads of its slot (the previous visit) come before the copy's writes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_copy_g2s(slot, m.det + (int64_t)cell * 16, 128, bar);
            bulk_copy_g2s(slot + 16, m.nav + (int64_t)cell * 4, 32, bar);
        }
        if (!warp_wait_phase(bar, parity)) {
            if (lane == 0) raise_error(st, OPPB_ERR_WAIT_LIMIT, (int32_t)i);
            warp_wait_phase(bar, parity);  // the copies in flight, once more (bounded)
            if (walking) err = OPPB_ERR_WAIT_LIMIT;
            break;
        }
        parity ^= 1u;
        if (walking) {
            const double2* r = reinterpret_cast<const double2*>(slot);
            const double2 coef_n01 = r[8], n23_pad = r[9];
            const double coef = coef_n01.x;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const double2 ab = r[2 * v], gd = r[2 * v + 1];
                double t = __dsub_rn(ab.x, __dmul_rn(ab.y, x));
                t = __dadd_rn(t, __dmul_rn(gd.x, y));
                t = __dsub_rn(t, __dmul_rn(gd.y, z));
                l[v] = __dmul_rn(coef, t);
            }
            visits++;
            if (inside_f64(l)) {
                walking = false;
            } else {
                const int mi = argmin4(l);
                const long long b = __double_as_longlong(mi < 2 ? coef_n01.y : n23_pad.x);
                const int32_t next = (mi & 1) ? (int32_t)(b >> 32) : (int32_t)(b & 0xffffffffll);
                if (next < 0) {
                    cell = kRemoved;
                    status = kNeedRemove;
                    walking = false;
                } else {
                    cell = next;
                    if (visits >= max_hops) {
                        err = OPPB_ERR_HOP_LIMIT;
                        walking = false;
                    }
                }
            }
        }
    }
    if (err) {
        if (err != OPPB_ERR_WAIT_LIMIT) raise_error(st, err, (int32_t)i);
        status = kFailed;
    }
    if (active && cell0 != kRemoved) store_result(p, i, l, visits, cell, cell0);
    cta_account(p, st, i, active, cell, status == kNeedRemove, visits, 0);
    deposit_epilogue<kDep>(m, table, dep, active && cell0 != kRemoved && status == kDone, cell, l);
}

// -------------------------------------------------------- mixed FP32 / FP64 move
//
// lambda_i(x) = c_i + g_i . (x - o) for i = 0..2 with o = f32(vertex 0), c_i, g_i in f32,
// and lambda_3 = ((1 - lambda_0) - lambda_1) - lambda_2: a visit reads one 64-B record
// (two sectors).  With u = 2^-24, d = f32(x - o) and S_i = |c_i| + sum_j |g_ij| |d_j|, the
// FP32 error of lambda_0..2 is below 6u S_i (rounding of c, g, d and of the three FMAs),
// and that of lambda_3 below 6u (S_0 + S_1 + S_2) + 3u (1 + S_0 + S_1 + S_2) (the three
// subtractions), so below 9u (1 + S) with S = S_0 + S_1 + S_2.  For S <= kMaxS = 16 every
// error is below 9.2e-6 < band = 1e-5.  S is bounded per visit by 1.001 + G max_j |d_j|,
// G the cell's rounded-up sum of |g_ij| (the record's last word, +inf for a cell whose
// sum of |c_i| exceeds 1.001), evaluated with one FMA and compared with kMaxS less 2^-20 of
// it, which covers that FMA's rounding.  A decision is taken in FP32 only when every
// threshold (-1e-10, 1+1e-10) and, outside the cell, every argmin tie is at least `band`
// away and the bound is within kMaxS; otherwise the visit is recomputed with the FP64
// reference expression.  Hence every decision equals the FP64 one.

constexpr float kMaxS = 16.0f * (1.0f - 0x1p-20f);

// The band's thresholds, precomputed on the host: kernel parameters live in the constant
// bank and are used as instruction operands without occupying registers.
struct Band {
    float lo;      // band
    float neg;     // -band
    float in_hi;   // 1 - band
    float out_hi;  // 1 + band
    float tie;     // 2 * band
};

template <int kDep, bool kPush, bool kSeed, bool kDevCount = false, int kBlock = kMoveBlock>
__global__ void __launch_bounds__(kBlock, kThreadsPerSm / kBlock)
    move_mixed_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep, oppb_move_status* st, int32_t max_hops,
                      Band band, PushArgs push, DhArgs dh) {
    static_assert(kBlock == kMoveBlock || kDep != kDepTable, "the node table is sized for 256 threads");
    __shared__ NodeTable table;
    const int32_t n = kDevCount ? live_count(p) : p.size;
    if (kDevCount && (int64_t)blockIdx.x * kBlock >= n) return;  // beyond the device count (whole block)
    if (kDep == kDepTable) table_init(table);
    const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < n;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int status = kDone;
    int visits = 0;
    int rechecks = 0;
    int err = 0;
    // The last visit's lambdas in FP32 (stored as p_lc and deposited: the mixed path keeps
    // cell decisions exact, weights to FP32 precision).  lr receives the rare FP64
    // re-evaluation; it lives in local memory because the out-of-line recheck writes it,
    // so it is touched on that path only.
    float lf[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    double lr[4];
    if (active && cell != kRemoved && (uint32_t)cell >= (uint32_t)m.n_cells) err = OPPB_ERR_CELL_RANGE;
    if (active && cell != kRemoved && !err) {
        double x = ld_stream(p.pos + i);
        double y = ld_stream(p.pos + p.stride + i);
        double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        if (kPush) push_prologue<true>(m, p, push, i, cell, x, y, z);
        if (kSeed) {
            cell = dh_seed(dh, x, y, z);
            if (cell == kRemoved) status = kNeedRemove;
            else if ((uint32_t)cell >= (uint32_t)m.n_cells) err = OPPB_ERR_CELL_RANGE;
        }
        while (!kSeed || (cell != kRemoved && !err)) {
            visits++;
            float g0[8], g1[8];  // rows 0..2, then the origin
            ldg256(m.geo32 + (int64_t)cell * 16, g0);
            ldg256(m.geo32 + (int64_t)cell * 16 + 8, g1);
            const float dx = (float)(x - (double)g1[4]);
            const float dy = (float)(y - (double)g1[5]);
            const float dz = (float)(z - (double)g1[6]);
            const float ssum = fmaf(g1[7], fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))), 1.001f);
            const float rows[12] = {g0[0], g0[1], g0[2], g0[3], g0[4], g0[5], g0[6], g0[7],
                                    g1[0], g1[1], g1[2], g1[3]};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float c0 = rows[4 * k], gx = rows[4 * k + 1], gy = rows[4 * k + 2], gz = rows[4 * k + 3];
                lf[k] = fmaf(gz, dz, fmaf(gy, dy, fmaf(gx, dx, c0)));
            }
            lf[3] = ((1.0f - lf[0]) - lf[1]) - lf[2];
            // Classify in FP32.
            bool clear_in = ssum <= kMaxS;
            bool clear_out = false;
            bool ambiguous = !(ssum <= kMaxS);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                clear_in = clear_in && (lf[k] >= band.lo) && (lf[k] <= band.in_hi);
                clear_out = clear_out || (lf[k] <= band.neg) || (lf[k] >= band.out_hi);
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
                        if (k != mi && !(lf[k] - mv > band.tie)) ambiguous = true;
                }
            }
            bool in = clear_in;
            if (ambiguous) {
                rechecks++;
                recheck_f64(m, cell, x, y, z, lr);
                in = inside_f64(lr);
                if (!in) mi = argmin4(lr);
#pragma unroll
                for (int k = 0; k < 4; k++) lf[k] = (float)lr[k];
            }
            if (in) break;
            // The neighbour is read only when the particle hops on (16 B of nav32), so the
            // last visit of a particle costs two sectors.
            const int32_t next = __ldg(reinterpret_cast<const int32_t*>(m.nav32 + (int64_t)cell * 8 + 4) + mi);
            if (next < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            if ((uint32_t)next >= (uint32_t)m.n_cells) {
                err = OPPB_ERR_CELL_RANGE;
                break;
            }
            cell = next;
            if (visits >= max_hops) {
                err = OPPB_ERR_HOP_LIMIT;
                break;
            }
        }
    }
    if (err) {
        raise_error(st, err, (int32_t)i);
        status = kFailed;
    }
    if (active && cell0 != kRemoved) store_result(p, i, lf, visits, cell, cell0);
    cta_account<kBlock>(p, st, i, active, cell, status == kNeedRemove, visits, rechecks);
    deposit_epilogue<kDep>(m, table, dep, active && cell0 != kRemoved && status == kDone, cell, lf);
}

// ------------------------------------------------ FP64 move on FP32 walk decisions
//
// oppb_tuning.move_walk32 = 1 (FP64 move + deposit, on a mesh that also holds the mixed
// path's records).  The walk is move_mixed_kernel's: every inside test and argmin is decided
// from the 64-B FP32 record, or, inside the band, by the FP64 reference expression, so each
// decision is the FP64 one and the particle visits the FP64 kernel's cells.  The FP64
// lambdas are then evaluated once, with the reference expression, at the last cell visited
// (the cell the particle ends in, or the one it left the mesh from): p_lc, p2c, the deposit,
// the removals and the visit counts are move_f64_kernel's bit for bit (its recheck count stays
// 0, as the FP64 kernel's).  A visit costs two 256-bit loads instead of five; the last cell
// five more.
constexpr float kWalk32Band = 1e-5f;  // above the FP32 lambdas' proven error (9.2e-6)

// kOcc: resident CTAs per SM it is compiled for, 8 (32 registers, 24 B of spills) or 6 (39
// registers, 8 B).
template <int kDep, bool kPush, bool kSeed, bool kDevCount = false, int kOcc = kMinBlocks>
__global__ void __launch_bounds__(kMoveBlock, kOcc)
    move_walk32_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep, oppb_move_status* st, int32_t max_hops,
                       PushArgs push, DhArgs dh) {
    __shared__ NodeTable table;
    const int32_t n = kDevCount ? live_count(p) : p.size;
    if (kDevCount && (int64_t)blockIdx.x * kMoveBlock >= n) return;  // beyond the device count (whole block)
    if (kDep == kDepTable) table_init(table);
    const int64_t i = (int64_t)blockIdx.x * kMoveBlock + threadIdx.x;
    const bool active = i < n;
    int32_t cell = active ? ld_stream(p.p2c + i) : kRemoved;
    const int32_t cell0 = cell;
    int32_t last = cell;  // the cell of the last visit
    int status = kDone;
    int visits = 0;
    int err = 0;
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    double lr[4];  // the rare FP64 re-evaluation inside the band (written out of line)
    const float bl = kWalk32Band, bneg = -kWalk32Band, bin = 1.0f - kWalk32Band, bout = 1.0f + kWalk32Band,
                btie = 2.0f * kWalk32Band;
    if (active && cell != kRemoved) {
        double x = ld_stream(p.pos + i);
        double y = ld_stream(p.pos + p.stride + i);
        double z = ld_stream(p.pos + 2 * (int64_t)p.stride + i);
        if (kPush && (uint32_t)cell < (uint32_t)m.n_cells) push_prologue<false>(m, p, push, i, cell, x, y, z);
        if (kSeed) {  // the walk starts from the grid box's cell (after the push, as the reference)
            cell = dh_seed(dh, x, y, z);
            if (cell == kRemoved) status = kNeedRemove;
        }
        while (!kSeed || cell != kRemoved) {
            if ((uint32_t)cell >= (uint32_t)m.n_cells) {
                err = OPPB_ERR_CELL_RANGE;
                break;
            }
            last = cell;
            visits++;
            float g0[8], g1[8];  // rows 0..2, then the origin
            ldg256(m.geo32 + (int64_t)cell * 16, g0);
            ldg256(m.geo32 + (int64_t)cell * 16 + 8, g1);
            const float dx = (float)(x - (double)g1[4]);
            const float dy = (float)(y - (double)g1[5]);
            const float dz = (float)(z - (double)g1[6]);
            const float ssum = fmaf(g1[7], fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))), 1.001f);
            const float rows[12] = {g0[0], g0[1], g0[2], g0[3], g0[4], g0[5], g0[6], g0[7],
                                    g1[0], g1[1], g1[2], g1[3]};
            float lf[4];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float c0 = rows[4 * k], gx = rows[4 * k + 1], gy = rows[4 * k + 2], gz = rows[4 * k + 3];
                lf[k] = fmaf(gz, dz, fmaf(gy, dy, fmaf(gx, dx, c0)));
            }
            lf[3] = ((1.0f - lf[0]) - lf[1]) - lf[2];
            // The mixed kernel's classification (its comment states the error bound).
            bool clear_in = ssum <= kMaxS;
            bool clear_out = false;
            bool ambiguous = !(ssum <= kMaxS);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                clear_in = clear_in && (lf[k] >= bl) && (lf[k] <= bin);
                clear_out = clear_out || (lf[k] <= bneg) || (lf[k] >= bout);
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
                        if (k != mi && !(lf[k] - mv > btie)) ambiguous = true;
                }
            }
            bool in = clear_in;
            if (ambiguous) {
                recheck_f64(m, cell, x, y, z, lr);
                in = inside_f64(lr);
                if (!in) mi = argmin4(lr);
            }
            if (in) break;
            const int32_t next = __ldg(reinterpret_cast<const int32_t*>(m.nav32 + (int64_t)cell * 8 + 4) + mi);
            if (next < 0) {
                cell = kRemoved;
                status = kNeedRemove;
                break;
            }
            cell = next;
            if (visits >= max_hops) {
                err = OPPB_ERR_HOP_LIMIT;
                break;
            }
        }
        if (visits > 0) {  // the FP64 lambdas of the last cell visited, as move_f64_kernel leaves them
            int nb[4];
            visit_f64(m, last, x, y, z, l, nb);
        }
        if (err) {
            raise_error(st, err, (int32_t)i);
            status = kFailed;
        }
        store_result(p, i, l, visits, cell, cell0);
    }
    cta_account(p, st, i, active, cell, status == kNeedRemove, visits, 0);
    deposit_epilogue<kDep>(m, table, dep, active && cell0 != kRemoved && status == kDone, cell, l);
}

// ------------------------------------------------------------- standalone deposit

template <int kDep>
__global__ void __launch_bounds__(kMoveBlock, kMinBlocks)
    deposit_f64_kernel(oppb_tet_mesh m, PartArgs p, DepositArgs dep) {
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
    deposit_epilogue<kDep>(m, table, dep, ok, cell, l);
}

// node_charge[n] += sum over copies r of copies[r][n].
__global__ void __launch_bounds__(256) reduce_copies_kernel(double* node_charge, const double* copies, int32_t n,
                                                            int32_t n_copies) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double s = node_charge[k];
        for (int r = 0; r < n_copies; r++) s += copies[(int64_t)r * n + k];
        node_charge[k] = s;
    }
}

// OPPB_DEPOSIT_EXACT: node_charge[n] += hi[n] 2^-20 + lo[n] 2^-52.  The carry of lo above
// 2^32 moves into hi first, so both terms are exact in FP64 (|hi| < 2^53) and their sum is
// rounded once.
__global__ void __launch_bounds__(256) exact_finish_kernel(double* node_charge, const unsigned long long* acc,
                                                           int32_t n) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long lo = acc[n + k];
        const long long hi = (long long)(acc[k] + (lo >> 32));
        const double v = __dadd_rn(__dmul_rn(__ll2double_rn(hi), 0x1p-20),
                                   __dmul_rn(__ull2double_rn(lo & 0xffffffffull), 0x1p-52));
        node_charge[k] = __dadd_rn(node_charge[k], v);
    }
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

PartArgs part_args(const oppb_particles* p, const int32_t* count_dev = nullptr, int32_t pending = 0) {
    return PartArgs{p->size, p->stride, p->pos, p->vel, p->lc, p->p2c, p->remove_bits, count_dev, pending};
}

int replicas_for(size_t workspace_bytes, const void* workspace, int32_t n_nodes) {
    const int want = tuning().replicas > 0 ? tuning().replicas : 1;
    if (!workspace || want <= 1 || !aligned(workspace, 8)) return 1;
    const size_t fit = workspace_bytes / ((size_t)n_nodes * sizeof(double)) + 1;
    return (int)(fit < (size_t)want ? fit : (size_t)want);
}

// Zeroes the copies (or the exact mode's integer sums) before, and folds them into
// node_charge after, the deposit launch.
struct Replicas {
    DepositArgs args;
    int n_nodes;
    int begin(cudaStream_t s) {
        if (args.exact)
            return cudaMemsetAsync(args.exact, 0, 2 * (size_t)n_nodes * sizeof(unsigned long long), s) == cudaSuccess
                       ? OPPB_OK
                       : OPPB_ERR_LAUNCH;
        if (args.replicas > 1 &&
            cudaMemsetAsync(args.copies, 0, (size_t)(args.replicas - 1) * n_nodes * sizeof(double), s) != cudaSuccess)
            return OPPB_ERR_LAUNCH;
        return OPPB_OK;
    }
    void end(cudaStream_t s) {
        const int grid = ceil_div(n_nodes, 256) < 148 * 8 ? ceil_div(n_nodes, 256) : 148 * 8;
        if (args.exact) {
            exact_finish_kernel<<<grid, 256, 0, s>>>(args.node_charge, args.exact, n_nodes);
            count_launches(1);
            return;
        }
        if (args.replicas <= 1) return;
        reduce_copies_kernel<<<grid, 256, 0, s>>>(args.node_charge, args.copies, n_nodes, args.replicas - 1);
        count_launches(1);
    }
};

bool exact_mode() { return tuning().deposit == OPPB_DEPOSIT_EXACT; }

// The deposit's targets; *rc = OPPB_ERR_WORKSPACE when the exact mode's sums do not fit.
Replicas make_replicas(double* node_charge, void* workspace, size_t workspace_bytes, int32_t n_nodes, int* rc) {
    *rc = OPPB_OK;
    if (exact_mode()) {
        if (!workspace || !aligned(workspace, 8) || workspace_bytes < 2 * (size_t)n_nodes * sizeof(unsigned long long))
            *rc = OPPB_ERR_WORKSPACE;
        return Replicas{DepositArgs{node_charge, nullptr, 1, static_cast<unsigned long long*>(workspace)}, n_nodes};
    }
    const int r = replicas_for(workspace_bytes, workspace, n_nodes);
    return Replicas{DepositArgs{node_charge, r > 1 ? static_cast<double*>(workspace) : nullptr, r, nullptr}, n_nodes};
}

enum MoveKind { kMoveOnly, kMoveDepositF64, kMoveDepositMixed };

// The pair kernel for the tuned deposit, compiled for kOcc resident CTAs per SM.
template <bool kPush, bool kDevCount, int kOcc>
void launch_pair(int grid, cudaStream_t s, bool table, bool exact, const oppb_tet_mesh& m, const PartArgs& p,
                 const DepositArgs& d, oppb_move_status* st, int32_t max_hops, const PushArgs& push) {
    if (table)
        move_f64_pair_kernel<kDepTable, kPush, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops, push);
    else if (exact)
        move_f64_pair_kernel<kDepExact, kPush, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops, push);
    else
        move_f64_pair_kernel<kDepWarp, kPush, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops, push);
}

// The FP32-walk FP64 kernel for the tuned deposit, compiled for kOcc resident CTAs per SM.
template <bool kPush, bool kSeed, bool kDevCount, int kOcc>
void launch_walk32(int grid, cudaStream_t s, bool table, bool exact, const oppb_tet_mesh& m, const PartArgs& p,
                   const DepositArgs& d, oppb_move_status* st, int32_t max_hops, const PushArgs& push,
                   const DhArgs& dh) {
    if (table)
        move_walk32_kernel<kDepTable, kPush, kSeed, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops,
                                                                                               push, dh);
    else if (exact)
        move_walk32_kernel<kDepExact, kPush, kSeed, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops,
                                                                                               push, dh);
    else
        move_walk32_kernel<kDepWarp, kPush, kSeed, kDevCount, kOcc><<<grid, kMoveBlock, 0, s>>>(m, p, d, st, max_hops,
                                                                                              push, dh);
}

// The one-lane kernels with the warp-grouped deposit at block shape kBlock.
template <bool kMixed, bool kPush, bool kSeed, bool kDevCount, int kBlock>
void launch_warp_shape(int32_t size, cudaStream_t s, const oppb_tet_mesh& m, const PartArgs& p,
                       const DepositArgs& d, oppb_move_status* st, int32_t max_hops, const Band& bd,
                       const PushArgs& push, const DhArgs& dh) {
    const int grid = ceil_div(size, kBlock);
    if constexpr (kMixed)
        move_mixed_kernel<kDepWarp, kPush, kSeed, kDevCount, kBlock><<<grid, kBlock, 0, s>>>(m, p, d, st, max_hops,
                                                                                            bd, push, dh);
    else
        move_f64_kernel<kDepWarp, kPush, kSeed, kDevCount, kBlock><<<grid, kBlock, 0, s>>>(m, p, d, st, max_hops,
                                                                                          push, dh);
}

// ... at the tuned block shape (oppb_tuning.move_block).
template <bool kMixed, bool kPush, bool kSeed, bool kDevCount>
void launch_warp(int32_t size, cudaStream_t s, const oppb_tet_mesh& m, const PartArgs& p, const DepositArgs& d,
                 oppb_move_status* st, int32_t max_hops, const Band& bd, const PushArgs& push, const DhArgs& dh) {
    switch (tuning().move_block) {
        case 128:
            launch_warp_shape<kMixed, kPush, kSeed, kDevCount, 128>(size, s, m, p, d, st, max_hops, bd, push, dh);
            break;
        case 512:
            launch_warp_shape<kMixed, kPush, kSeed, kDevCount, 512>(size, s, m, p, d, st, max_hops, bd, push, dh);
            break;
        default:
            launch_warp_shape<kMixed, kPush, kSeed, kDevCount, kMoveBlock>(size, s, m, p, d, st, max_hops, bd, push,
                                                                           dh);
    }
}

template <int kKind, bool kPush, bool kSeed = false, bool kDevCount = false>
int launch_move(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                oppb_move_status* status, int32_t max_hops, double band, const PushArgs& push, void* workspace,
                size_t ws_bytes, void* stream, const DhArgs& dh = DhArgs{}, const int32_t* count_dev = nullptr,
                int32_t pending = 0) {
    constexpr bool kMixed = kKind == kMoveDepositMixed;
    int rc = check_mesh(mesh, kMixed, kKind != kMoveOnly);
    if (rc) return rc;
    rc = check_parts(parts, true);
    if (rc) return rc;
    if (!status || max_hops <= 0) return OPPB_ERR_ARG;
    if (kKind != kMoveOnly && !node_charge) return OPPB_ERR_ARG;
    if (kMixed && !(band > 0.0 && band < 0.25)) return OPPB_ERR_ARG;
    if (kPush && (!parts->vel || !mesh->ef || !aligned(mesh->ef, 16))) return OPPB_ERR_ARG;
    if (kSeed && !dh.map) return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(status, 0, sizeof(oppb_move_status), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    if (parts->size == 0) return launch_status();
    if (kDevCount != (count_dev != nullptr) || pending < 0) return OPPB_ERR_ARG;
    const PartArgs p = part_args(parts, count_dev, pending);
    const int grid = ceil_div(parts->size, kMoveBlock);
    Replicas rep{};
    if (kKind != kMoveOnly) {
        rep = make_replicas(node_charge, workspace, ws_bytes, mesh->n_nodes, &rc);
        if (rc) return rc;
    }
    if ((rc = rep.begin(s))) return rc;
    const bool table = tuning().deposit == OPPB_DEPOSIT_CTA_TABLE;
    const bool exact = exact_mode();
    const float bf = (float)band;
    const Band bd{bf, -bf, 1.0f - bf, 1.0f + bf, 2.0f * bf};
    if constexpr (kKind == kMoveOnly)
        move_f64_kernel<kDepNone, kPush, kSeed, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args, status, max_hops,
                                                                           push, dh);
    else if constexpr (kKind == kMoveDepositF64) {
        if (tuning().move_walk32 != 0 && mesh->geo32 && mesh->nav32 && aligned(mesh->geo32, 32) &&
            aligned(mesh->nav32, 32)) {  // walk on the FP32 records, FP64 lambdas at the last cell
            if (tuning().move_walk32 == 2)
                launch_walk32<kPush, kSeed, kDevCount, 6>(grid, s, table, exact, *mesh, p, rep.args, status,
                                                          max_hops, push, dh);
            else
                launch_walk32<kPush, kSeed, kDevCount, kMinBlocks>(grid, s, table, exact, *mesh, p, rep.args, status,
                                                                   max_hops, push, dh);
        } else if (!kSeed && tuning().move_lanes != 2 && tuning().move_stage == 1) {  // records staged by bulk copies
            if (table)
                move_f64_stage_kernel<kDepTable, kPush, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args,
                                                                                              status, max_hops, push);
            else if (exact)
                move_f64_stage_kernel<kDepExact, kPush, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args,
                                                                                              status, max_hops, push);
            else
                move_f64_stage_kernel<kDepWarp, kPush, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args,
                                                                                             status, max_hops, push);
        } else if (!kSeed && tuning().move_lanes == 2) {  // a particle per lane pair
            if (tuning().move_occupancy == 5)
                launch_pair<kPush, kDevCount, 5>(grid, s, table, exact, *mesh, p, rep.args, status, max_hops, push);
            else
                launch_pair<kPush, kDevCount, kMinBlocks>(grid, s, table, exact, *mesh, p, rep.args, status, max_hops,
                                                          push);
        } else if (table)
            move_f64_kernel<kDepTable, kPush, kSeed, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args, status,
                                                                                max_hops, push, dh);
        else if (exact)
            move_f64_kernel<kDepExact, kPush, kSeed, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args, status,
                                                                                max_hops, push, dh);
        else
            launch_warp<false, kPush, kSeed, kDevCount>(parts->size, s, *mesh, p, rep.args, status, max_hops, bd, push,
                                                        dh);
    } else if (exact)
        move_mixed_kernel<kDepExact, kPush, kSeed, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args, status,
                                                                              max_hops, bd, push, dh);
    else if (table)
        move_mixed_kernel<kDepTable, kPush, kSeed, kDevCount><<<grid, kMoveBlock, 0, s>>>(*mesh, p, rep.args, status,
                                                                              max_hops, bd, push, dh);
    else
        launch_warp<true, kPush, kSeed, kDevCount>(parts->size, s, *mesh, p, rep.args, status, max_hops, bd, push, dh);
    count_launches(1);
    rep.end(s);
    return launch_status();
}

// oppb_move_ex: the options select one instantiation of launch_move.
template <bool kSeed>
int move_ex(const oppb_tet_mesh* mesh, const oppb_particles* parts, const oppb_move_options& o,
            double* node_charge, oppb_move_status* status, int32_t max_hops, void* ws, size_t ws_bytes,
            void* stream, const DhArgs& dh) {
    const bool mixed = o.precision == OPPB_PRECISION_MIXED;
    if (o.precision != OPPB_PRECISION_F64 && !mixed) return OPPB_ERR_ARG;
    if ((o.deposit != 0 && o.deposit != 1) || (o.push != 0 && o.push != 1)) return OPPB_ERR_ARG;
    if (o.push && !o.deposit) return OPPB_ERR_ARG;   // the push prologue exists on the deposit kernels
    if (mixed && !o.deposit) return OPPB_ERR_ARG;    // the mixed move always deposits
    // The coefficients of oppb_push_f64 / oppb_push_mixed: q/m and dt, f32(q/m * dt) and f32(dt).
    const PushArgs push{o.qm, o.dt, (float)(o.qm * o.dt), (float)o.dt};
    // The device count (oppb_set_count::size is its first member), or the host's parts->size.
    const int32_t* cd = o.set_count ? reinterpret_cast<const int32_t*>(o.set_count) : nullptr;
    const int32_t pd = o.pending;
    if (cd) {  // device-counted launches: the deposit kernels, walks from the previous cell
        if (kSeed || !o.deposit) return OPPB_ERR_ARG;
        if (mixed)
            return o.push ? launch_move<kMoveDepositMixed, true, false, true>(mesh, parts, node_charge, status,
                                                                              max_hops, o.band, push, ws, ws_bytes,
                                                                              stream, dh, cd, pd)
                          : launch_move<kMoveDepositMixed, false, false, true>(mesh, parts, node_charge, status,
                                                                               max_hops, o.band, push, ws, ws_bytes,
                                                                               stream, dh, cd, pd);
        return o.push ? launch_move<kMoveDepositF64, true, false, true>(mesh, parts, node_charge, status, max_hops,
                                                                        0.0, push, ws, ws_bytes, stream, dh, cd, pd)
                      : launch_move<kMoveDepositF64, false, false, true>(mesh, parts, node_charge, status, max_hops,
                                                                         0.0, push, ws, ws_bytes, stream, dh, cd, pd);
    }
    if (!o.deposit)
        return launch_move<kMoveOnly, false, kSeed>(mesh, parts, nullptr, status, max_hops, 0.0, push, nullptr, 0,
                                                    stream, dh, cd, pd);
    if (mixed)
        return o.push ? launch_move<kMoveDepositMixed, true, kSeed>(mesh, parts, node_charge, status, max_hops,
                                                                    o.band, push, ws, ws_bytes, stream, dh, cd, pd)
                      : launch_move<kMoveDepositMixed, false, kSeed>(mesh, parts, node_charge, status, max_hops,
                                                                     o.band, push, ws, ws_bytes, stream, dh, cd, pd);
    return o.push ? launch_move<kMoveDepositF64, true, kSeed>(mesh, parts, node_charge, status, max_hops, 0.0,
                                                              push, ws, ws_bytes, stream, dh, cd, pd)
                  : launch_move<kMoveDepositF64, false, kSeed>(mesh, parts, node_charge, status, max_hops, 0.0,
                                                               push, ws, ws_bytes, stream, dh, cd, pd);
}

}  // namespace
}  // namespace oppb

extern "C" size_t oppb_deposit_workspace_bytes(int32_t n_nodes) {
    const int r = oppb::tuning().replicas;
    if (n_nodes > 0 && oppb::exact_mode()) return 2 * (size_t)n_nodes * sizeof(unsigned long long);
    if (n_nodes <= 0 || r <= 1) return 0;
    return (size_t)(r - 1) * (size_t)n_nodes * sizeof(double);
}

extern "C" int oppb_move_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, oppb_move_status* status,
                             int32_t max_hops, void* stream) {
    return oppb::launch_move<oppb::kMoveOnly, false>(mesh, parts, nullptr, status, max_hops, 0.0, oppb::PushArgs{},
                                                    nullptr, 0, stream);
}

extern "C" int oppb_move_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                                     oppb_move_status* status, int32_t max_hops, void* workspace,
                                     size_t workspace_bytes, void* stream) {
    return oppb::launch_move<oppb::kMoveDepositF64, false>(mesh, parts, node_charge, status, max_hops, 0.0,
                                                          oppb::PushArgs{}, workspace, workspace_bytes, stream);
}

extern "C" int oppb_move_deposit_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                                       double* node_charge, oppb_move_status* status, int32_t max_hops,
                                       double band, void* workspace, size_t workspace_bytes, void* stream) {
    return oppb::launch_move<oppb::kMoveDepositMixed, false>(mesh, parts, node_charge, status, max_hops, band,
                                                            oppb::PushArgs{}, workspace, workspace_bytes, stream);
}

extern "C" int oppb_push_move_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                                          double* node_charge, oppb_move_status* status, int32_t max_hops,
                                          double charge_over_mass, double dt, void* workspace,
                                          size_t workspace_bytes, void* stream) {
    const oppb::PushArgs push{charge_over_mass, dt, 0.0f, 0.0f};
    return oppb::launch_move<oppb::kMoveDepositF64, true>(mesh, parts, node_charge, status, max_hops, 0.0, push,
                                                         workspace, workspace_bytes, stream);
}

extern "C" int oppb_push_move_deposit_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                                            double* node_charge, oppb_move_status* status, int32_t max_hops,
                                            double band, double charge_over_mass, double dt, void* workspace,
                                            size_t workspace_bytes, void* stream) {
    // The same FP32 coefficients as oppb_push_mixed: f32(q/m * dt) and f32(dt).
    const oppb::PushArgs push{charge_over_mass, dt, (float)(charge_over_mass * dt), (float)dt};
    return oppb::launch_move<oppb::kMoveDepositMixed, true>(mesh, parts, node_charge, status, max_hops, band, push,
                                                           workspace, workspace_bytes, stream);
}

extern "C" int oppb_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, double* node_charge,
                                void* workspace, size_t workspace_bytes, void* stream) {
    using namespace oppb;
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0 || !mesh->c2n || !aligned(mesh->c2n, 16))
        return OPPB_ERR_ARG;
    if (!parts || parts->size < 0 || parts->stride < parts->size || !parts->lc || !parts->p2c || !node_charge)
        return OPPB_ERR_ARG;
    if (parts->size == 0) return OPPB_OK;
    cudaStream_t s = as_stream(stream);
    int rc = OPPB_OK;
    Replicas rep = make_replicas(node_charge, workspace, workspace_bytes, mesh->n_nodes, &rc);
    if (rc || (rc = rep.begin(s))) return rc;
    const int grid = ceil_div(parts->size, kMoveBlock);
    if (tuning().deposit == OPPB_DEPOSIT_CTA_TABLE)
        deposit_f64_kernel<kDepTable><<<grid, kMoveBlock, 0, s>>>(*mesh, part_args(parts), rep.args);
    else if (exact_mode())
        deposit_f64_kernel<kDepExact><<<grid, kMoveBlock, 0, s>>>(*mesh, part_args(parts), rep.args);
    else
        deposit_f64_kernel<kDepWarp><<<grid, kMoveBlock, 0, s>>>(*mesh, part_args(parts), rep.args);
    count_launches(1);
    rep.end(s);
    return launch_status();
}

extern "C" int oppb_move_ex(const oppb_tet_mesh* mesh, const oppb_particles* parts, const oppb_move_options* opt,
                            double* node_charge, oppb_move_status* status, int32_t max_hops, void* workspace,
                            size_t ws_bytes, void* stream) {
    if (!opt) return OPPB_ERR_ARG;
    if (!opt->dh)
        return oppb::move_ex<false>(mesh, parts, *opt, node_charge, status, max_hops, workspace, ws_bytes, stream,
                                    oppb::DhArgs{});
    const oppb_dh_grid& g = *opt->dh;
    if (!g.map || !(g.inv_spacing > 0.0) || g.dims[0] <= 0 || g.dims[1] <= 0 || g.dims[2] <= 0) return OPPB_ERR_ARG;
    const oppb::DhArgs dh{g.map,
                          {g.min[0], g.min[1], g.min[2]},
                          g.inv_spacing,
                          {(unsigned long long)g.dims[0], (unsigned long long)g.dims[1], (unsigned long long)g.dims[2]}};
    return oppb::move_ex<true>(mesh, parts, *opt, node_charge, status, max_hops, workspace, ws_bytes, stream, dh);
}
