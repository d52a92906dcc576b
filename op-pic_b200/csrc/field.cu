// FemPIC node-side loops and the field solve on the GPU (include/oppb_field.h).
//
// compute_node_charge_density_kernel and compute_electric_field_kernel are one thread per
// node / cell, each product and sum rounded on its own in the reference's order (this file
// is compiled with -fmad=false), so their results equal the reference's bit for bit for the
// same inputs.
//
// compute_phi is one cooperative launch: the grid runs init_f1_and_J, build_f1_vector and
// build_j_matrix (cell integrals added with FP64 atomics, as the reference's device
// kernels do), B = K D - F0 - F1, then Jacobi-preconditioned CG on J Y = B, D -= Y and the
// node potentials, separated by grid-wide barriers.  The iteration count is bounded by
// max_iter, every barrier is the cooperative grid's (all blocks are resident by
// construction of the launch), and no host synchronisation is needed, so a stream capture
// of the call is one graph node.  The dot products are reduced deterministically: each block
// writes its partial sum, and after the barrier every block sums all partials in block
// order, so all blocks hold the same scalars and a run repeats bit for bit.

#include <cooperative_groups.h>

#include <cstring>

#include "oppb_common.cuh"
#include "oppb_field.h"

namespace cg = cooperative_groups;

namespace oppb {
namespace {

constexpr int kFieldBlock = 256;
constexpr int kMaxCoopBlocks = 148 * 8;
constexpr int kWarps = kFieldBlock / 32;

struct FieldArgs {
    int32_t n_nodes, n_cells, neq;
    const int32_t* node_to_eq;
    const int32_t* c2n;
    const double* det_j;
    const double* n_bnd_pot;
    const int64_t* k_rowptr;
    const int32_t* k_col;
    const double* k_val;
    const double* f0;
    double* d;
    double* f1;
    const double* ion_den;
    double* potential;
    oppb_field_status* status;
    // work
    double *t1, *t2, *t3, *diag, *x, *r, *p, *q;
    double* partial_a;  // [kMaxCoopBlocks]
    double* partial_b;  // [kMaxCoopBlocks][2]
    // constants
    double n0, phi0, kte, qe, eps0, rtol, atol;
    int32_t max_iter;
    // K by diagonals (n_diag > 0): dia_val[j * neq + r] = K[r][r + dia_off[j]], offsets ascending.
    int32_t n_diag;
    int32_t dia_off[OPPB_FIELD_MAX_DIAG];
    const double* dia_val;
};

// Sum of v over the block, returned to every thread (fixed order: deterministic).
__device__ double block_sum(double v, double* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    __syncthreads();  // sm may still be read by a previous call
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) s += sm[w];
    return s;
}

// Sum over blocks of partial[b * stride + k], in block order, by every block.
__device__ double grid_sum(const double* partial, int stride, int k, double* sm) {
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kFieldBlock) v += partial[b * stride + k];
    return block_sum(v, sm);
}

// Shape function a at Gauss point (i, j, k) of the 2x2x2 rule (evaluate_na in the reference's
// build_f1_vector / build_j_matrix).
__device__ __forceinline__ double shape_na(int a, int i, int j, int k) {
    const double g = __dsqrt_rn(1.0 / 3.0);
    const double li = i ? g : -g, lj = j ? g : -g, lk = k ? g : -g;
    const double ni = 0.5 * (li + 1), nj = 0.5 * (lj + 1), nk = 0.5 * (lk + 1);
    return a == 0 ? ni : a == 1 ? nj : a == 2 ? nk : ((1 - ni) - nj) - nk;
}

// Row u of J v (K with its diagonal replaced by du) or, with kDiag false, of K v: four column
// indices and values are loaded before their four vector gathers, so each thread keeps several
// independent loads in flight; the terms are still added one by one in column order.  K is
// read-only for the whole launch (non-coherent loads); v is not (plain loads: the vectors are
// rewritten between grid barriers).
template <bool kDiag>
__device__ __forceinline__ double row_dot(const FieldArgs& a, int64_t u, double du, const double* v) {
    if (a.n_diag > 0) {
        // By diagonals: neighbouring rows read neighbouring values of every diagonal and of v,
        // so a warp's loads are coalesced.  Offsets ascend, so the nonzero terms are added in
        // the CSR row's column order; the zeros of a diagonal where the row has no entry add
        // +0 or -0 to a sum that starts at +0 and so is never -0, which leaves it unchanged.
        double s = 0.0;
#pragma unroll 4
        for (int j = 0; j < a.n_diag; j++) {
            const int32_t off = a.dia_off[j];
            const int64_t c = u + off;
            double kv = __ldg(a.dia_val + (int64_t)j * a.neq + u);
            if (kDiag && off == 0) kv = du;
            const double vc = (c >= 0 && c < a.neq) ? v[c] : 0.0;
            s += kv * vc;
        }
        return s;
    }
    int64_t k = __ldg(a.k_rowptr + u);
    const int64_t end = __ldg(a.k_rowptr + u + 1);
    double s = 0.0;
    for (; k + 4 <= end; k += 4) {
        const int32_t c0 = __ldg(a.k_col + k), c1 = __ldg(a.k_col + k + 1);
        const int32_t c2 = __ldg(a.k_col + k + 2), c3 = __ldg(a.k_col + k + 3);
        double v0 = __ldg(a.k_val + k), v1 = __ldg(a.k_val + k + 1);
        double v2 = __ldg(a.k_val + k + 2), v3 = __ldg(a.k_val + k + 3);
        const double p0 = v[c0], p1 = v[c1], p2 = v[c2], p3 = v[c3];
        if (kDiag) {
            v0 = c0 == u ? du : v0;
            v1 = c1 == u ? du : v1;
            v2 = c2 == u ? du : v2;
            v3 = c3 == u ? du : v3;
        }
        s += v0 * p0;
        s += v1 * p1;
        s += v2 * p2;
        s += v3 * p3;
    }
    for (; k < end; k++) {
        const int32_t c = __ldg(a.k_col + k);
        const double vk = (kDiag && c == u) ? du : __ldg(a.k_val + k);
        s += vk * v[c];
    }
    return s;
}

__global__ void __launch_bounds__(kFieldBlock) field_newton_kernel(FieldArgs a) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double sm[kWarps];
    const int64_t tid = (int64_t)blockIdx.x * kFieldBlock + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * kFieldBlock;
    const double qe_eps0 = a.qe / a.eps0;

    // init_f1_and_J (field_solver/device.cpp init_f1_kernel, init_J_kernel).
    for (int64_t n = tid; n < a.n_nodes; n += nth) {
        const int32_t e = a.node_to_eq[n];
        if (e >= 0) a.t1[e] = qe_eps0 * (a.ion_den[n] + a.n0 * exp((a.d[e] - a.phi0) / a.kte));
    }
    for (int64_t u = tid; u < a.neq; u += nth) {
        a.t2[u] = 0.0;
        a.t3[u] = -a.qe / a.eps0 * a.n0 * exp((a.d[u] - a.phi0) / a.kte) * (1 / a.kte);
    }
    grid.sync();

    // build_f1_vector and build_j_matrix: per cell and unknown vertex, the 8-point integrals
    // of tempNEQ1 and tempNEQ3 times the shape function, added into F1 and tempNEQ2.
    for (int64_t c = tid; c < a.n_cells; c += nth) {
        const double dj = a.det_j[c];
        for (int v = 0; v < 4; v++) {
            const int32_t e = a.node_to_eq[a.c2n[c * 4 + v]];
            if (e < 0) continue;
            const double s1 = a.t1[e], s3 = a.t3[e];
            double ff1 = 0.0, ff3 = 0.0;
            for (int k = 0; k < 2; k++)
                for (int j = 0; j < 2; j++)
                    for (int i = 0; i < 2; i++) {
                        const double na = shape_na(v, i, j, k);
                        ff1 += s1 * na * dj * 1.0 * 1.0 * 1.0;
                        ff3 += s3 * na * dj * 1.0 * 1.0 * 1.0;
                    }
            atomicAdd(a.f1 + e, ff1 * (1.0 / 8.0));
            atomicAdd(a.t2 + e, ff3 * (1.0 / 8.0));
        }
    }
    grid.sync();

    // B = K D - F0 - F1; J's diagonal = K's - tempNEQ2; CG start x = 0, r = B, p = r / diag.
    double bb = 0.0, rz = 0.0;
    for (int64_t u = tid; u < a.neq; u += nth) {
        double kd = 0.0, kuu = 0.0;
        for (int64_t k = a.k_rowptr[u]; k < a.k_rowptr[u + 1]; k++) {
            const int32_t col = a.k_col[k];
            kd += a.k_val[k] * a.d[col];
            if (col == u) kuu = a.k_val[k];
        }
        const double b = (kd - a.f0[u]) - a.f1[u];
        const double dg = kuu + (-a.t2[u]);
        a.diag[u] = dg;
        a.x[u] = 0.0;
        a.r[u] = b;
        const double z = b / dg;
        a.p[u] = z;
        bb += b * b;
        rz += b * z;
    }
    bb = block_sum(bb, sm);
    rz = block_sum(rz, sm);
    if (threadIdx.x == 0) {
        a.partial_b[blockIdx.x * 2] = bb;
        a.partial_b[blockIdx.x * 2 + 1] = rz;
    }
    grid.sync();
    bb = grid_sum(a.partial_b, 2, 0, sm);
    rz = grid_sum(a.partial_b, 2, 1, sm);
    const double b_norm = sqrt(bb);
    const double stop = fmax(a.rtol * b_norm, a.atol);
    double rr = bb;
    int it = 0;
    while (it < a.max_iter && sqrt(rr) > stop) {
        double pq = 0.0;
        for (int64_t u = tid; u < a.neq; u += nth) {  // q = J p
            const double s = row_dot<true>(a, u, a.diag[u], a.p);
            a.q[u] = s;
            pq += a.p[u] * s;
        }
        pq = block_sum(pq, sm);
        if (threadIdx.x == 0) a.partial_a[blockIdx.x] = pq;
        grid.sync();
        pq = grid_sum(a.partial_a, 1, 0, sm);
        const double alpha = rz / pq;
        double rz_new = 0.0, rr_new = 0.0;
        for (int64_t u = tid; u < a.neq; u += nth) {
            a.x[u] += alpha * a.p[u];
            const double ru = a.r[u] - alpha * a.q[u];
            a.r[u] = ru;
            rz_new += ru * (ru / a.diag[u]);
            rr_new += ru * ru;
        }
        rz_new = block_sum(rz_new, sm);
        rr_new = block_sum(rr_new, sm);
        if (threadIdx.x == 0) {
            a.partial_b[blockIdx.x * 2] = rz_new;
            a.partial_b[blockIdx.x * 2 + 1] = rr_new;
        }
        grid.sync();
        rz_new = grid_sum(a.partial_b, 2, 0, sm);
        rr_new = grid_sum(a.partial_b, 2, 1, sm);
        const double beta = rz_new / rz;
        rz = rz_new;
        rr = rr_new;
        for (int64_t u = tid; u < a.neq; u += nth) a.p[u] = a.r[u] / a.diag[u] + beta * a.p[u];
        grid.sync();
        it++;
    }

    // D -= Y (VecAXPY(D, -1, Y)), then compute_node_potential.
    for (int64_t u = tid; u < a.neq; u += nth) a.d[u] = a.d[u] - a.x[u];
    grid.sync();
    for (int64_t n = tid; n < a.n_nodes; n += nth) {
        const int32_t e = a.node_to_eq[n];
        a.potential[n] = a.n_bnd_pot[n] + ((e >= 0) ? a.d[e] : 0);
    }
    if (tid == 0) {
        a.status->iterations = it;
        a.status->converged = sqrt(rr) <= stop;
        a.status->resid = b_norm > 0.0 ? sqrt(rr) / b_norm : 0.0;
        a.status->b_norm = b_norm;
    }
}

__global__ void __launch_bounds__(256) node_charge_density_kernel(double* den, const double* vol, double spwt,
                                                                   int32_t n) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i < n) den[i] *= (spwt / vol[i]);
}

__global__ void __launch_bounds__(256) electric_field_kernel(const int32_t* c2n, oppb_cell_layout nl,
                                                             const double* sd, oppb_cell_layout sl,
                                                             const double* phi, double* ef, oppb_cell_layout el,
                                                             int32_t n, int32_t accumulate) {
    const int64_t c = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (c >= n) return;
    double p[4];
#pragma unroll
    for (int v = 0; v < 4; v++) p[v] = __ldg(phi + __ldg(c2n + c * nl.cell_stride + v * nl.comp_stride));
    const double* s = sd + c * sl.cell_stride;
#pragma unroll
    for (int dim = 0; dim < 3; dim++) {
        const double c1 = __ldg(s + (0 * 3 + dim) * sl.comp_stride) * p[0];
        const double c2 = __ldg(s + (1 * 3 + dim) * sl.comp_stride) * p[1];
        const double c3 = __ldg(s + (2 * 3 + dim) * sl.comp_stride) * p[2];
        const double c4 = __ldg(s + (3 * 3 + dim) * sl.comp_stride) * p[3];
        double* e = ef + c * el.cell_stride + dim * el.comp_stride;
        *e = (accumulate ? *e : 0.0) - (c1 + c2 + c3 + c4);
    }
}

// Doubles mapped to 64-bit words whose unsigned order is the doubles' order (negative values
// complemented, positive ones with the sign bit set), so atomicMax on the words is a max.
__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ unsigned long long g_max_key;

__global__ void __launch_bounds__(256) reduce_max_kernel(const double* x, int64_t n, int32_t absolute) {
    __shared__ unsigned long long sm[8];
    unsigned long long k = 0ull;  // below every key of a non-NaN double
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        const double v = absolute ? fabs(x[i]) : x[i];
        const unsigned long long kv = order_key(v);
        k = kv > k ? kv : k;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(kFullMask, k, o);
        k = other > k ? other : k;
    }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = k;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) k = sm[w] > k ? sm[w] : k;
        atomicMax(&g_max_key, k);
    }
}

int coop_grid(int* blocks) {
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, field_newton_kernel, kFieldBlock, 0) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    if (!coop || per_sm <= 0) return OPPB_ERR_LAUNCH;
    const int want = sms * (per_sm < 4 ? per_sm : 4);
    *blocks = want < kMaxCoopBlocks ? want : kMaxCoopBlocks;
    return OPPB_OK;
}

}  // namespace
}  // namespace oppb

extern "C" size_t oppb_field_work_doubles(int32_t neq) {
    if (neq < 0) return 0;
    return 8 * (size_t)(neq > 0 ? neq : 1) + 3 * (size_t)oppb::kMaxCoopBlocks;
}

extern "C" int oppb_node_charge_density(double* n_charge_den, const double* n_vol, double spwt, int32_t n_nodes,
                                        void* stream) {
    if (n_nodes < 0 || (n_nodes > 0 && (!n_charge_den || !n_vol))) return OPPB_ERR_ARG;
    if (n_nodes == 0) return OPPB_OK;
    oppb::node_charge_density_kernel<<<oppb::ceil_div(n_nodes, 256), 256, 0, oppb::as_stream(stream)>>>(
        n_charge_den, n_vol, spwt, n_nodes);
    oppb::count_launches(1);
    return oppb::launch_status();
}

extern "C" int oppb_electric_field_ex(const int32_t* c2n, oppb_cell_layout c2n_layout, const double* c_sd,
                                      oppb_cell_layout sd_layout, const double* node_potential, double* c_ef,
                                      oppb_cell_layout ef_layout, int32_t n_cells, int32_t accumulate,
                                      void* stream) {
    if (n_cells < 0 || (accumulate != 0 && accumulate != 1)) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    if (!c2n || !c_sd || !node_potential || !c_ef) return OPPB_ERR_ARG;
    oppb::electric_field_kernel<<<oppb::ceil_div(n_cells, 256), 256, 0, oppb::as_stream(stream)>>>(
        c2n, c2n_layout, c_sd, sd_layout, node_potential, c_ef, ef_layout, n_cells, accumulate);
    oppb::count_launches(1);
    return oppb::launch_status();
}

extern "C" int oppb_electric_field(const int32_t* c2n, const double* c_sd, const double* node_potential,
                                   double* c_ef, int32_t ef_stride, int32_t n_cells, void* stream) {
    if (ef_stride < 3) return OPPB_ERR_ARG;
    return oppb_electric_field_ex(c2n, oppb_cell_layout{4, 1}, c_sd, oppb_cell_layout{12, 1}, node_potential, c_ef,
                                  oppb_cell_layout{ef_stride, 1}, n_cells, 0, stream);
}

extern "C" int oppb_reduce_max(const double* x, int64_t n, int32_t absolute, double init, double* result,
                               void* stream) {
    if (!result || n < 0 || (n > 0 && !x) || (absolute != 0 && absolute != 1)) return OPPB_ERR_ARG;
    *result = init;
    if (n == 0) return OPPB_OK;
    cudaStream_t s = oppb::as_stream(stream);
    unsigned long long* key = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&key), oppb::g_max_key) != cudaSuccess ||
        cudaMemsetAsync(key, 0, sizeof(unsigned long long), s) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    const int blocks = oppb::ceil_div(n, 256) < 148 * 8 ? oppb::ceil_div(n, 256) : 148 * 8;
    oppb::reduce_max_kernel<<<blocks, 256, 0, s>>>(x, n, absolute);
    oppb::count_launches(1);
    unsigned long long k = 0;
    if (cudaMemcpyAsync(&k, key, sizeof k, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    if (k != 0ull) {  // decode the largest key (0 = no value, n > 0 makes that impossible)
        const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double v;
        memcpy(&v, &b, sizeof v);
        if (v > *result) *result = v;  // MAX(value, init) of the reference's kernels
    }
    return oppb::launch_status();
}

extern "C" int oppb_field_solve(const oppb_field_device* f, const oppb_field_consts* c, const double* ion_den,
                                double* node_potential, oppb_field_status* status, void* stream) {
    using namespace oppb;
    if (!f || !c || !ion_den || !node_potential || !status) return OPPB_ERR_ARG;
    if (f->n_nodes <= 0 || f->n_cells <= 0 || f->neq < 0 || !f->node_to_eq || !f->c2n || !f->det_j ||
        !f->n_bnd_pot || !f->k_rowptr || !f->d || !f->f1 || !f->work || !f->f0 || (f->neq > 0 && (!f->k_col ||
        !f->k_val)))
        return OPPB_ERR_ARG;
    if (c->max_iter < 0 || !(c->kte != 0.0) || !(c->eps0 != 0.0) || !(c->rtol >= 0.0) || !(c->atol >= 0.0))
        return OPPB_ERR_ARG;
    int blocks = 0;
    int rc = coop_grid(&blocks);
    if (rc) return rc;
    const size_t n = (size_t)(f->neq > 0 ? f->neq : 1);
    double* w = f->work;
    FieldArgs a{};
    a.n_nodes = f->n_nodes, a.n_cells = f->n_cells, a.neq = f->neq;
    a.node_to_eq = f->node_to_eq, a.c2n = f->c2n, a.det_j = f->det_j, a.n_bnd_pot = f->n_bnd_pot;
    a.k_rowptr = f->k_rowptr, a.k_col = f->k_col, a.k_val = f->k_val, a.f0 = f->f0;
    a.d = f->d, a.f1 = f->f1, a.ion_den = ion_den, a.potential = node_potential, a.status = status;
    a.t1 = w, a.t2 = w + n, a.t3 = w + 2 * n, a.diag = w + 3 * n, a.x = w + 4 * n, a.r = w + 5 * n;
    a.p = w + 6 * n, a.q = w + 7 * n;
    a.partial_a = w + 8 * n;
    a.partial_b = w + 8 * n + kMaxCoopBlocks;
    a.n0 = c->n0, a.phi0 = c->phi0, a.kte = c->kte, a.qe = c->qe, a.eps0 = c->eps0;
    a.rtol = c->rtol, a.atol = c->atol, a.max_iter = c->max_iter;
    if (f->n_diag < 0 || f->n_diag > OPPB_FIELD_MAX_DIAG || (f->n_diag > 0 && !f->dia_val)) return OPPB_ERR_ARG;
    a.n_diag = f->n_diag;
    for (int j = 0; j < OPPB_FIELD_MAX_DIAG; j++) a.dia_off[j] = f->dia_off[j];
    a.dia_val = f->dia_val;
    void* args[] = {&a};
    if (cudaLaunchCooperativeKernel((const void*)field_newton_kernel, dim3(blocks), dim3(kFieldBlock), args, 0,
                                    as_stream(stream)) != cudaSuccess)
        return OPPB_ERR_LAUNCH;
    count_launches(1);
    return launch_status();
}
