// Packing of the reference's SoA cell dats into the records the move kernels read,
// and the f32 records of the mixed-precision path.

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kPackBlock = 256;

__global__ void pack_kernel(int32_t n_cells, int32_t n_nodes, int32_t stride, const double* __restrict__ c_det,
                            const double* __restrict__ c_volume, const int32_t* __restrict__ c2c,
                            const int32_t* __restrict__ c2n, const double* __restrict__ c_ef,
                            const double* __restrict__ n_pos, int32_t n_pos_stride, double* __restrict__ det,
                            double* __restrict__ coef, int32_t* __restrict__ conn, double* __restrict__ ef,
                            float* __restrict__ geo32, float* __restrict__ org32, int32_t* invalid_out) {
    const int64_t c = (int64_t)blockIdx.x * kPackBlock + threadIdx.x;
    int bad = 0;
    if (c < n_cells) {
        double d[16];
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] = c_det[(int64_t)k * stride + c];
#pragma unroll
        for (int k = 0; k < 8; k++)
            reinterpret_cast<double2*>(det + c * 16)[k] = make_double2(d[2 * k], d[2 * k + 1]);
        // coefficient2 of apps/app_fempic/kernels.h:110, correctly rounded.
        const double cf = __ddiv_rn(1.0 / 6.0, c_volume[c]);
        coef[c] = cf;
        int4 nb, nd;
        nb.x = c2c[c];
        nb.y = c2c[(int64_t)stride + c];
        nb.z = c2c[2 * (int64_t)stride + c];
        nb.w = c2c[3 * (int64_t)stride + c];
        nd.x = c2n[c];
        nd.y = c2n[(int64_t)stride + c];
        nd.z = c2n[2 * (int64_t)stride + c];
        nd.w = c2n[3 * (int64_t)stride + c];
        const int nbv[4] = {nb.x, nb.y, nb.z, nb.w};
        const int ndv[4] = {nd.x, nd.y, nd.z, nd.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            bad += (nbv[k] < -1 || nbv[k] >= n_cells);
            bad += (ndv[k] < 0 || ndv[k] >= n_nodes);
        }
        reinterpret_cast<int4*>(conn + c * 8)[0] = nb;
        reinterpret_cast<int4*>(conn + c * 8)[1] = nd;
        if (c_ef) {
            reinterpret_cast<double2*>(ef + c * 4)[0] = make_double2(c_ef[c], c_ef[(int64_t)stride + c]);
            reinterpret_cast<double2*>(ef + c * 4)[1] = make_double2(c_ef[2 * (int64_t)stride + c], 0.0);
        }
        if (geo32 && n_pos && nd.x >= 0 && nd.x < n_nodes) {
            // Origin: vertex 0 rounded to f32; lambda_i(o) and grad(lambda_i) from the
            // FP64 coefficients, lambda_i(x) = coef*(alpha - beta*x + gamma*y - delta*z).
            const float ox = (float)n_pos[nd.x];
            const float oy = (float)n_pos[(int64_t)n_pos_stride + nd.x];
            const float oz = (float)n_pos[2 * (int64_t)n_pos_stride + nd.x];
            reinterpret_cast<float4*>(org32 + c * 4)[0] = make_float4(ox, oy, oz, 0.0f);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double a = d[4 * i], b = d[4 * i + 1], g = d[4 * i + 2], e = d[4 * i + 3];
                const double li = cf * (((a - b * (double)ox) + g * (double)oy) - e * (double)oz);
                reinterpret_cast<float4*>(geo32 + c * 16)[i] =
                    make_float4((float)li, (float)(-cf * b), (float)(cf * g), (float)(-cf * e));
            }
        }
    }
    if (invalid_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(kFullMask, bad, o);
        if ((threadIdx.x & 31) == 0 && bad) atomicAdd(invalid_out, bad);
    }
}

__global__ void set_ef_kernel(int32_t n_cells, int32_t stride, const double* __restrict__ c_ef, double* ef) {
    const int64_t c = (int64_t)blockIdx.x * kPackBlock + threadIdx.x;
    if (c < n_cells) {
        reinterpret_cast<double2*>(ef + c * 4)[0] = make_double2(c_ef[c], c_ef[(int64_t)stride + c]);
        reinterpret_cast<double2*>(ef + c * 4)[1] = make_double2(c_ef[2 * (int64_t)stride + c], 0.0);
    }
}

}  // namespace
}  // namespace oppb

extern "C" void oppb_tet_mesh_bytes(int32_t n_cells, size_t out_bytes[6]) {
    const size_t n = n_cells > 0 ? (size_t)n_cells : 0;
    out_bytes[0] = n * 16 * sizeof(double);
    out_bytes[1] = n * sizeof(double);
    out_bytes[2] = n * 8 * sizeof(int32_t);
    out_bytes[3] = n * 4 * sizeof(double);
    out_bytes[4] = n * 16 * sizeof(float);
    out_bytes[5] = n * 4 * sizeof(float);
}

extern "C" int oppb_tet_mesh_pack(oppb_tet_mesh* mesh, int32_t soa_stride, const double* c_det,
                                  const double* c_volume, const int32_t* c2c, const int32_t* c2n,
                                  const double* c_ef, const double* n_pos, int32_t n_pos_stride,
                                  int32_t* invalid_out, void* stream) {
    using namespace oppb;
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0 || soa_stride < mesh->n_cells) return OPPB_ERR_ARG;
    if (!c_det || !c_volume || !c2c || !c2n || !mesh->det || !mesh->coef || !mesh->conn) return OPPB_ERR_ARG;
    if (!aligned(mesh->det, 16) || !aligned(mesh->conn, 16)) return OPPB_ERR_ARG;
    if (c_ef && (!mesh->ef || !aligned(mesh->ef, 16))) return OPPB_ERR_ARG;
    const bool mixed = mesh->geo32 != nullptr || mesh->org32 != nullptr;
    if (mixed && (!mesh->geo32 || !mesh->org32 || !n_pos || n_pos_stride < mesh->n_nodes ||
                  !aligned(mesh->geo32, 16) || !aligned(mesh->org32, 16)))
        return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (invalid_out && cudaMemsetAsync(invalid_out, 0, sizeof(int32_t), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    const int grid = ceil_div(mesh->n_cells, kPackBlock);
    pack_kernel<<<grid, kPackBlock, 0, s>>>(mesh->n_cells, mesh->n_nodes, soa_stride, c_det, c_volume, c2c, c2n,
                                            c_ef, mixed ? n_pos : nullptr, n_pos_stride, mesh->det, mesh->coef,
                                            mesh->conn, mesh->ef, mixed ? mesh->geo32 : nullptr, mesh->org32,
                                            invalid_out);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_tet_mesh_set_ef(oppb_tet_mesh* mesh, int32_t soa_stride, const double* c_ef, void* stream) {
    using namespace oppb;
    if (!mesh || !mesh->ef || !c_ef || mesh->n_cells <= 0 || soa_stride < mesh->n_cells) return OPPB_ERR_ARG;
    if (!aligned(mesh->ef, 16)) return OPPB_ERR_ARG;
    const int grid = ceil_div(mesh->n_cells, kPackBlock);
    set_ef_kernel<<<grid, kPackBlock, 0, as_stream(stream)>>>(mesh->n_cells, soa_stride, c_ef, mesh->ef);
    count_launches(1);
    return launch_status();
}
