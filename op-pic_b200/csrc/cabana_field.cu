// CabanaPIC's mesh loops on the GPU (include/oppb_cabana.h): the field interpolation, the
// current gathered from the accumulators, the leapfrog B and E updates, the ghost-cell copies and
// folds, and the field energy.  One thread per cell, the user kernels' expressions of
// apps/app_cabanapic/kernels.h with each product and sum rounded on its own in the same order
// (this file is compiled with -fmad=false), so every cell value equals the seq backend's for the
// same inputs; the energy is a sum over cells, reduced in a fixed order that is not the seq
// backend's cell order.  Cell dats are SoA [dim][stride]; a neighbour argument is one column of
// a cell map (the map's device copy plus idx * its stride), as the generated loops index them.

#include "oppb_cabana.h"
#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kCellBlock = 256;
constexpr int kEnergyBlocks = 1024;

__device__ __forceinline__ double col(const double* d, int64_t stride, int k, int32_t c) {
    return d[(int64_t)k * stride + c];
}

struct Nb9 {
    const int32_t* e[6];
    const int32_t* b[3];
};
struct Nb6 {
    const int32_t* c[6];
};
struct Nb3 {
    const int32_t* c[3];
};

// interpolate_mesh_fields_kernel (kernels.h:21-99): the 18 interpolation coefficients of a
// non-ghost cell from E at the cell and its x, y, z, xy, yz, xz upper neighbours and B at the
// cell and its x, y, z upper neighbours.
__global__ void __launch_bounds__(kCellBlock) interpolate_kernel(int32_t n, int64_t s, const double* __restrict__ e,
                                                                 const double* __restrict__ b, Nb9 nb,
                                                                 double* __restrict__ interp,
                                                                 const int32_t* __restrict__ ghost) {
    const int32_t c = blockIdx.x * kCellBlock + threadIdx.x;
    if (c >= n || ghost[c] != 0) return;
    const double fourth = 1.0 / 4.0, half = 1.0 / 2.0;
    const int32_t cx = nb.e[0][c], cy = nb.e[1][c], cz = nb.e[2][c], cxy = nb.e[3][c], cyz = nb.e[4][c],
                  cxz = nb.e[5][c];
    const int32_t bx = nb.b[0][c], by = nb.b[1][c], bz = nb.b[2][c];
    double w0, w1, w2, w3;
    auto put4 = [&](int k) {
        interp[(int64_t)(k + 0) * s + c] = fourth * ((w3 + w0) + (w1 + w2));
        interp[(int64_t)(k + 1) * s + c] = fourth * ((w3 - w0) + (w1 - w2));
        interp[(int64_t)(k + 2) * s + c] = fourth * ((w3 - w0) - (w1 - w2));
        interp[(int64_t)(k + 3) * s + c] = fourth * ((w3 + w0) - (w1 + w2));
    };
    w0 = col(e, s, 0, c), w1 = col(e, s, 0, cy), w2 = col(e, s, 0, cz), w3 = col(e, s, 0, cyz);
    put4(0);  // ex, dexdy, dexdz, d2exdydz
    w0 = col(e, s, 1, c), w1 = col(e, s, 1, cz), w2 = col(e, s, 1, cx), w3 = col(e, s, 1, cxz);
    put4(4);  // ey, deydz, deydx, d2eydzdx
    w0 = col(e, s, 2, c), w1 = col(e, s, 2, cx), w2 = col(e, s, 2, cy), w3 = col(e, s, 2, cxy);
    put4(8);  // ez, dezdx, dezdy, d2ezdxdy
    const int32_t up[3] = {bx, by, bz};
#pragma unroll
    for (int d = 0; d < 3; d++) {  // cbx, dcbxdx; cby, dcbydy; cbz, dcbzdz
        w0 = col(b, s, d, c);
        w1 = col(b, s, d, up[d]);
        interp[(int64_t)(12 + 2 * d) * s + c] = half * (w1 + w0);
        interp[(int64_t)(13 + 2 * d) * s + c] = half * (w1 - w0);
    }
}

// accumulate_current_to_cells_kernel (kernels.h:110-135): J of a cell with iter_acc set from its
// own accumulators and those of its x, y, z, xy, yz, xz lower neighbours.
__global__ void __launch_bounds__(kCellBlock) accumulate_kernel(int32_t n, int64_t s, double* __restrict__ j,
                                                                const double* __restrict__ acc, Nb6 nb,
                                                                const int32_t* __restrict__ mask, double3 coef) {
    const int32_t c = blockIdx.x * kCellBlock + threadIdx.x;
    if (c >= n || mask[c] != 1) return;
    const int32_t xd = nb.c[0][c], yd = nb.c[1][c], zd = nb.c[2][c], xyd = nb.c[3][c], yzd = nb.c[4][c],
                  xzd = nb.c[5][c];
    // CellAcc: jfx = 0, jfy = 4, jfz = 8
    j[c] = coef.x * (((col(acc, s, 0, c) + col(acc, s, 1, yd)) + col(acc, s, 2, zd)) + col(acc, s, 3, yzd));
    j[s + c] = coef.y * (((col(acc, s, 4, c) + col(acc, s, 5, zd)) + col(acc, s, 6, xd)) + col(acc, s, 7, xzd));
    j[2 * s + c] =
        coef.z * (((col(acc, s, 8, c) + col(acc, s, 9, xd)) + col(acc, s, 10, yd)) + col(acc, s, 11, xyd));
}

// half_advance_b_kernel (kernels.h:138-158): B -= half a step of curl E at a non-ghost cell, E at
// its x, y, z upper neighbours.
__global__ void __launch_bounds__(kCellBlock) half_advance_b_kernel(int32_t n, int64_t s, Nb3 nb,
                                                                    const double* __restrict__ e,
                                                                    double* __restrict__ b,
                                                                    const int32_t* __restrict__ ghost, double3 p) {
    const int32_t c = blockIdx.x * kCellBlock + threadIdx.x;
    if (c >= n || ghost[c] != 0) return;
    const int32_t cx = nb.c[0][c], cy = nb.c[1][c], cz = nb.c[2][c];
    const double e0x = col(e, s, 0, c), e0y = col(e, s, 1, c), e0z = col(e, s, 2, c);
    b[c] = b[c] - ((0.5 * p.y) * (col(e, s, 2, cy) - e0z) - (0.5 * p.z) * (col(e, s, 1, cz) - e0y));
    b[s + c] = b[s + c] - ((0.5 * p.z) * (col(e, s, 0, cz) - e0x) - (0.5 * p.x) * (col(e, s, 2, cx) - e0z));
    b[2 * s + c] = b[2 * s + c] - ((0.5 * p.x) * (col(e, s, 1, cx) - e0y) - (0.5 * p.y) * (col(e, s, 0, cy) - e0x));
}

// advance_e_kernel (kernels.h:161-183): E += -dt/eps0 J + curl B at a cell with iter_adv_e set, B
// at its x, y, z lower neighbours.
__global__ void __launch_bounds__(kCellBlock) advance_e_kernel(int32_t n, int64_t s, Nb3 nb,
                                                               const double* __restrict__ b,
                                                               const double* __restrict__ j, double* __restrict__ e,
                                                               const int32_t* __restrict__ mask, double3 p,
                                                               double dt_eps0) {
    const int32_t c = blockIdx.x * kCellBlock + threadIdx.x;
    if (c >= n || mask[c] != 1) return;
    const int32_t cx = nb.c[0][c], cy = nb.c[1][c], cz = nb.c[2][c];
    const double b0x = col(b, s, 0, c), b0y = col(b, s, 1, c), b0z = col(b, s, 2, c);
    e[c] = e[c] + ((-dt_eps0 * j[c]) + (p.y * (b0z - col(b, s, 2, cy)) - p.z * (b0y - col(b, s, 1, cz))));
    e[s + c] = e[s + c] + ((-dt_eps0 * j[s + c]) + (p.z * (b0x - col(b, s, 0, cz)) - p.x * (b0z - col(b, s, 2, cx))));
    e[2 * s + c] =
        e[2 * s + c] + ((-dt_eps0 * j[2 * s + c]) + (p.x * (b0y - col(b, s, 1, cx)) - p.y * (b0x - col(b, s, 0, cy))));
}

// update_ghosts_B_kernel (dim < 0: the three components copied) and update_ghosts_kernel (dim >= 0:
// that component added, as an OPP_INC through the map) of kernels.h:199-224, for the cells whose
// mask[m_idx] is 1.
__global__ void __launch_bounds__(kCellBlock) ghosts_kernel(int32_t n, int64_t s, const int32_t* __restrict__ mask,
                                                            int32_t m_idx, const double* from, double* to,
                                                            const int32_t* __restrict__ to_map, int32_t dim) {
    const int32_t c = blockIdx.x * kCellBlock + threadIdx.x;
    if (c >= n || mask[(int64_t)m_idx * s + c] != 1) return;
    const int32_t t = to_map[c];
    if (dim < 0) {
#pragma unroll
        for (int d = 0; d < 3; d++) to[(int64_t)d * s + t] = from[(int64_t)d * s + c];
    } else {
        atomicAdd(to + (int64_t)dim * s + t, from[(int64_t)dim * s + c]);
    }
}

// compute_energy_kernel's terms (kernels.h:228-238): per block the sum of
// (fx fx + fy fy) + fz fz over its non-ghost cells, grid-stride, a fixed tree per block.
__global__ void __launch_bounds__(kCellBlock) energy_partial_kernel(int32_t n, int64_t s,
                                                                    const int32_t* __restrict__ ghost,
                                                                    const double* __restrict__ f,
                                                                    double* __restrict__ partial) {
    __shared__ double sm[kCellBlock];
    double v = 0.0;
    for (int32_t c = blockIdx.x * kCellBlock + threadIdx.x; c < n; c += gridDim.x * kCellBlock)
        if (ghost[c] == 0) {
            const double fx = col(f, s, 0, c), fy = col(f, s, 1, c), fz = col(f, s, 2, c);
            v = v + ((fx * fx + fy * fy) + fz * fz);
        }
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int w = kCellBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

// The block partials added in block order into *out (one thread).
__global__ void energy_final_kernel(const double* __restrict__ partial, int32_t blocks, double* out) {
    double v = 0.0;
    for (int32_t k = 0; k < blocks; k++) v = v + partial[k];
    *out = *out + v;
}

int check_cells(int32_t n, int64_t stride) { return (n < 0 || stride < n) ? OPPB_ERR_ARG : OPPB_OK; }

template <class T, int N>
bool all_set(const T* const (&p)[N]) {
    for (int k = 0; k < N; k++)
        if (!p[k]) return false;
    return true;
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_cabana_interpolate(int32_t n_cells, int64_t stride, const double* c_e, const double* c_b,
                                       const int32_t* const nb_e[6], const int32_t* const nb_b[3], double* c_interp,
                                       const int32_t* c_mask_ghost, void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || !nb_e || !nb_b) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    Nb9 nb{};
    for (int k = 0; k < 6; k++) nb.e[k] = nb_e[k];
    for (int k = 0; k < 3; k++) nb.b[k] = nb_b[k];
    if (!c_e || !c_b || !c_interp || !c_mask_ghost || !all_set(nb.e) || !all_set(nb.b)) return OPPB_ERR_ARG;
    interpolate_kernel<<<ceil_div(n_cells, kCellBlock), kCellBlock, 0, as_stream(stream)>>>(
        n_cells, stride, c_e, c_b, nb, c_interp, c_mask_ghost);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_cabana_accumulate(int32_t n_cells, int64_t stride, double* c_j, const double* c_acc,
                                      const int32_t* const nb_lower[6], const int32_t* c_mask_right,
                                      const double acc_coef[3], void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || !nb_lower || !acc_coef) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    Nb6 nb{};
    for (int k = 0; k < 6; k++) nb.c[k] = nb_lower[k];
    if (!c_j || !c_acc || !c_mask_right || !all_set(nb.c)) return OPPB_ERR_ARG;
    accumulate_kernel<<<ceil_div(n_cells, kCellBlock), kCellBlock, 0, as_stream(stream)>>>(
        n_cells, stride, c_j, c_acc, nb, c_mask_right, make_double3(acc_coef[0], acc_coef[1], acc_coef[2]));
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_cabana_half_advance_b(int32_t n_cells, int64_t stride, const int32_t* const nb_upper[3],
                                          const double* c_e, double* c_b, const int32_t* c_mask_ghost,
                                          const double p[3], void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || !nb_upper || !p) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    Nb3 nb{};
    for (int k = 0; k < 3; k++) nb.c[k] = nb_upper[k];
    if (!c_e || !c_b || !c_mask_ghost || !all_set(nb.c)) return OPPB_ERR_ARG;
    half_advance_b_kernel<<<ceil_div(n_cells, kCellBlock), kCellBlock, 0, as_stream(stream)>>>(
        n_cells, stride, nb, c_e, c_b, c_mask_ghost, make_double3(p[0], p[1], p[2]));
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_cabana_advance_e(int32_t n_cells, int64_t stride, const int32_t* const nb_lower[3],
                                     const double* c_b, const double* c_j, double* c_e, const int32_t* c_mask_right,
                                     const double p[3], double dt_eps0, void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || !nb_lower || !p) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    Nb3 nb{};
    for (int k = 0; k < 3; k++) nb.c[k] = nb_lower[k];
    if (!c_b || !c_j || !c_e || !c_mask_right || !all_set(nb.c)) return OPPB_ERR_ARG;
    advance_e_kernel<<<ceil_div(n_cells, kCellBlock), kCellBlock, 0, as_stream(stream)>>>(
        n_cells, stride, nb, c_b, c_j, c_e, c_mask_right, make_double3(p[0], p[1], p[2]), dt_eps0);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_cabana_update_ghosts(int32_t n_cells, int64_t stride, const int32_t* mask, int32_t m_idx,
                                         const double* from, double* to, const int32_t* to_map, int32_t dim,
                                         void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || m_idx < 0 || m_idx >= 6 || dim < -1 || dim > 2) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    if (!mask || !from || !to || !to_map) return OPPB_ERR_ARG;
    ghosts_kernel<<<ceil_div(n_cells, kCellBlock), kCellBlock, 0, as_stream(stream)>>>(n_cells, stride, mask, m_idx,
                                                                                       from, to, to_map, dim);
    count_launches(1);
    return launch_status();
}

extern "C" size_t oppb_cabana_energy_workspace_bytes(void) { return sizeof(double) * oppb::kEnergyBlocks; }

extern "C" int oppb_cabana_energy(int32_t n_cells, int64_t stride, const int32_t* c_mask_ghost, const double* field,
                                  double* energy, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace oppb;
    if (check_cells(n_cells, stride) || !energy) return OPPB_ERR_ARG;
    if (n_cells == 0) return OPPB_OK;
    if (!c_mask_ghost || !field || !workspace || !aligned(workspace, 8)) return OPPB_ERR_ARG;
    if (workspace_bytes < oppb_cabana_energy_workspace_bytes()) return OPPB_ERR_WORKSPACE;
    const int blocks = ceil_div(n_cells, kCellBlock) < kEnergyBlocks ? ceil_div(n_cells, kCellBlock) : kEnergyBlocks;
    cudaStream_t s = as_stream(stream);
    double* partial = static_cast<double*>(workspace);
    energy_partial_kernel<<<blocks, kCellBlock, 0, s>>>(n_cells, stride, c_mask_ghost, field, partial);
    energy_final_kernel<<<1, 1, 0, s>>>(partial, blocks, energy);
    count_launches(2);
    return launch_status();
}
