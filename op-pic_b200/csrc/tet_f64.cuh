// The FP64 barycentric cell test of the FemPIC move, shared by the move kernels and the
// direct-hop grid build (which must decide "point inside cell" exactly as the move does).
//
// The arithmetic uses explicit round-to-nearest intrinsics so nothing is contracted into
// FMAs: each lambda_i is bit-identical to the reference expression
//   coef * (((d0 - d1*x) + d2*y) - d3*z)          (apps/app_fempic/kernels.h:110-117)
// and the inside test / argmin follow kernels.h:121-146 exactly.
#pragma once

#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr double kTol = 1e-10;  // KERNEL_TOLERENCE, apps/app_fempic/kernels.h:44

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

}  // namespace
}  // namespace oppb
