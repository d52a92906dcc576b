// Packing of the reference's SoA cell dats into the 32-byte-aligned records the move
// kernels read with 256-bit loads, and the f32 records of the mixed-precision path.

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kPackBlock = 256;

struct PackIn {
    int32_t n_cells, n_nodes, stride, n_pos_stride;
    const double* c_det;
    const double* c_volume;
    const int32_t* c2c;
    const int32_t* c2n;
    const double* c_ef;
    const double* n_pos;
};

__global__ void pack_kernel(PackIn in, oppb_tet_mesh m, int32_t* invalid_out) {
    const int64_t c = (int64_t)blockIdx.x * kPackBlock + threadIdx.x;
    const int64_t s = in.stride;
    int bad = 0;
    if (c < in.n_cells) {
        double d[16];
        double cf = 0.0;
        if (in.c_det) {
#pragma unroll
            for (int k = 0; k < 16; k++) d[k] = in.c_det[k * s + c];
#pragma unroll
            for (int k = 0; k < 4; k++)
                reinterpret_cast<double4*>(m.det + c * 16)[k] = make_double4(d[4 * k], d[4 * k + 1], d[4 * k + 2],
                                                                             d[4 * k + 3]);
            // coefficient2 of apps/app_fempic/kernels.h:110, correctly rounded.
            cf = __ddiv_rn(1.0 / 6.0, in.c_volume[c]);
            m.nav[c * 4] = cf;
        }
        if (in.c2c) {
            int nb[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                nb[k] = in.c2c[k * s + c];
                bad += (nb[k] < -1 || nb[k] >= in.n_cells);
            }
            // nav bytes 8..23 hold c2c[0..3]; bytes 24..31 stay zero.
            int2* q = reinterpret_cast<int2*>(m.nav + c * 4 + 1);
            q[0] = make_int2(nb[0], nb[1]);
            q[1] = make_int2(nb[2], nb[3]);
            q[2] = make_int2(0, 0);
            if (m.nav32) reinterpret_cast<int4*>(m.nav32 + c * 8)[1] = make_int4(nb[0], nb[1], nb[2], nb[3]);
        }
        int4 nd = make_int4(-1, -1, -1, -1);
        if (in.c2n) {
            nd = make_int4(in.c2n[c], in.c2n[s + c], in.c2n[2 * s + c], in.c2n[3 * s + c]);
            const int ndv[4] = {nd.x, nd.y, nd.z, nd.w};
#pragma unroll
            for (int k = 0; k < 4; k++) bad += (ndv[k] < 0 || ndv[k] >= in.n_nodes);
            reinterpret_cast<int4*>(m.c2n + c * 4)[0] = nd;
        }
        if (in.c_ef) {
            reinterpret_cast<double4*>(m.ef + c * 4)[0] =
                make_double4(in.c_ef[c], in.c_ef[s + c], in.c_ef[2 * s + c], 0.0);
        }
        if (m.geo32 && in.n_pos && in.c_det && in.c2n && nd.x >= 0 && nd.x < in.n_nodes) {
            // Origin: vertex 0 rounded to f32; lambda_i(o) and grad(lambda_i) from the
            // FP64 coefficients, lambda_i(x) = coef*(alpha - beta*x + gamma*y - delta*z),
            // for vertices 0..2 (the move derives lambda_3 from their sum), then o.
            const int64_t ps = in.n_pos_stride;
            const float ox = (float)in.n_pos[nd.x];
            const float oy = (float)in.n_pos[ps + nd.x];
            const float oz = (float)in.n_pos[2 * ps + nd.x];
            reinterpret_cast<float4*>(m.nav32 + c * 8)[0] = make_float4(ox, oy, oz, 0.0f);
            // The record's last word bounds the rows' gradients: G = sum_ij |g_ij| of the stored
            // f32 values, rounded up, so that S = sum_i (|c_i| + sum_j |g_ij| |d_j|) <= 1.001 +
            // G max_j |d_j|; a cell whose sum_i |c_i| exceeds 1.001 (c_i = lambda_i(o) with o its
            // vertex 0 is 1, 0, 0 to rounding) gets G = +inf, so all its visits are re-checked.
            double gsum = 0.0, csum = 0.0;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const double a = d[4 * i], b = d[4 * i + 1], g = d[4 * i + 2], e = d[4 * i + 3];
                const double li = cf * (((a - b * (double)ox) + g * (double)oy) - e * (double)oz);
                const float4 row = make_float4((float)li, (float)(-cf * b), (float)(cf * g), (float)(-cf * e));
                reinterpret_cast<float4*>(m.geo32 + c * 16)[i] = row;
                csum += fabs((double)row.x);
                gsum += fabs((double)row.y) + fabs((double)row.z) + fabs((double)row.w);
            }
            const float gbound = csum <= 1.001 ? __double2float_ru(gsum * (1.0 + 0x1p-20)) : __int_as_float(0x7f800000);
            reinterpret_cast<float4*>(m.geo32 + c * 16)[3] = make_float4(ox, oy, oz, gbound);
        }
    }
    if (invalid_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(kFullMask, bad, o);
        if ((threadIdx.x & 31) == 0 && bad) atomicAdd(invalid_out, bad);
    }
}

}  // namespace
}  // namespace oppb

extern "C" void oppb_tet_mesh_bytes(int32_t n_cells, size_t out_bytes[6]) {
    const size_t n = n_cells > 0 ? (size_t)n_cells : 0;
    out_bytes[0] = n * 16 * sizeof(double);  // det
    out_bytes[1] = n * 4 * sizeof(double);   // nav
    out_bytes[2] = n * 4 * sizeof(int32_t);  // c2n
    out_bytes[3] = n * 4 * sizeof(double);   // ef
    out_bytes[4] = n * 16 * sizeof(float);   // geo32
    out_bytes[5] = n * 8 * sizeof(float);    // nav32
}

extern "C" int oppb_tet_mesh_pack(oppb_tet_mesh* mesh, int32_t soa_stride, const double* c_det,
                                  const double* c_volume, const int32_t* c2c, const int32_t* c2n,
                                  const double* c_ef, const double* n_pos, int32_t n_pos_stride,
                                  int32_t* invalid_out, void* stream) {
    using namespace oppb;
    if (!mesh || mesh->n_cells <= 0 || mesh->n_nodes <= 0 || soa_stride < mesh->n_cells) return OPPB_ERR_ARG;
    if ((c_det == nullptr) != (c_volume == nullptr)) return OPPB_ERR_ARG;
    if (c_det && (!mesh->det || !mesh->nav || !aligned(mesh->det, 32) || !aligned(mesh->nav, 32))) return OPPB_ERR_ARG;
    if (c2c && (!mesh->nav || !aligned(mesh->nav, 32))) return OPPB_ERR_ARG;
    if (c2n && (!mesh->c2n || !aligned(mesh->c2n, 16))) return OPPB_ERR_ARG;
    if (c_ef && (!mesh->ef || !aligned(mesh->ef, 32))) return OPPB_ERR_ARG;
    if ((mesh->geo32 == nullptr) != (mesh->nav32 == nullptr)) return OPPB_ERR_ARG;
    if (mesh->geo32 && (!aligned(mesh->geo32, 32) || !aligned(mesh->nav32, 32))) return OPPB_ERR_ARG;
    const bool mixed = mesh->geo32 != nullptr && n_pos != nullptr;
    if (mixed && (!c_det || !c2n || n_pos_stride < mesh->n_nodes)) return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (invalid_out && cudaMemsetAsync(invalid_out, 0, sizeof(int32_t), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    const PackIn in{mesh->n_cells, mesh->n_nodes, soa_stride, n_pos_stride, c_det, c_volume, c2c, c2n, c_ef,
                    mixed ? n_pos : nullptr};
    oppb_tet_mesh m = *mesh;
    if (!mixed && !c2c) m.nav32 = nullptr;
    if (!mixed) m.geo32 = nullptr;
    pack_kernel<<<ceil_div(mesh->n_cells, kPackBlock), kPackBlock, 0, s>>>(in, m, invalid_out);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_tet_mesh_set_ef(oppb_tet_mesh* mesh, int32_t soa_stride, const double* c_ef, void* stream) {
    return oppb_tet_mesh_pack(mesh, soa_stride, nullptr, nullptr, nullptr, nullptr, c_ef, nullptr, 0, nullptr, stream);
}
