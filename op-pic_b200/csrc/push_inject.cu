// Particle push (leap-frog velocity/position update) and injection from the inlet
// surface.  FP64 arithmetic uses explicit round-to-nearest intrinsics so the results
// are bit-identical to the seq backend's scalar expressions.

#include <algorithm>

#include "oppb_common.cuh"
#include "oppb_graph.h"

namespace oppb {
namespace {

constexpr int kPushBlock = 256;

// calculate_new_pos_vel_kernel, apps/app_fempic/kernels.h:93-103:
//   coefficient1 = q/m * dt;  v[i] += coefficient1 * E[i];  x[i] += v[i] * dt.
__global__ void __launch_bounds__(kPushBlock) push_f64_kernel(int32_t size, int32_t stride, int32_t n_cells,
                                                              const int32_t* __restrict__ p2c,
                                                              const double* __restrict__ ef, double* pos,
                                                              double* vel, double qm, double dt) {
    const int64_t i = (int64_t)blockIdx.x * kPushBlock + threadIdx.x;
    if (i >= size) return;
    const int32_t c = ld_stream(p2c + i);
    if ((uint32_t)c >= (uint32_t)n_cells) return;
    const double coefficient1 = __dmul_rn(qm, dt);
    const double2 e01 = ldg_d2(ef + (int64_t)c * 4);
    const double2 e2_ = ldg_d2(ef + (int64_t)c * 4 + 2);
    const double e[3] = {e01.x, e01.y, e2_.x};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double* vp = vel + (int64_t)d * stride + i;
        double* xp = pos + (int64_t)d * stride + i;
        const double v = __dadd_rn(ld_stream(vp), __dmul_rn(coefficient1, e[d]));
        st_stream(vp, v);
        st_stream(xp, __dadd_rn(ld_stream(xp), __dmul_rn(v, dt)));
    }
}

// FP32 increments on FP64 state: dv = f32(q/m*dt) * f32(E), v += dv; dx = f32(v) * f32(dt), x += dx.
__global__ void __launch_bounds__(kPushBlock) push_mixed_kernel(int32_t size, int32_t stride, int32_t n_cells,
                                                                const int32_t* __restrict__ p2c,
                                                                const double* __restrict__ ef, double* pos,
                                                                double* vel, float qmdt, float dtf) {
    const int64_t i = (int64_t)blockIdx.x * kPushBlock + threadIdx.x;
    if (i >= size) return;
    const int32_t c = ld_stream(p2c + i);
    if ((uint32_t)c >= (uint32_t)n_cells) return;
    const double2 e01 = ldg_d2(ef + (int64_t)c * 4);
    const double2 e2_ = ldg_d2(ef + (int64_t)c * 4 + 2);
    const double e[3] = {e01.x, e01.y, e2_.x};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double* vp = vel + (int64_t)d * stride + i;
        double* xp = pos + (int64_t)d * stride + i;
        const float dv = __fmul_rn(qmdt, __double2float_rn(e[d]));
        const double v = __dadd_rn(ld_stream(vp), (double)dv);
        st_stream(vp, v);
        const float dx = __fmul_rn(__double2float_rn(v), dtf);
        st_stream(xp, __dadd_rn(ld_stream(xp), (double)dx));
    }
}

// First inlet face j with k < dist[j] (the last face if none).
__device__ __forceinline__ int face_of(const int32_t* __restrict__ dist, int32_t n_faces, int64_t k) {
    int lo = 0, hi = n_faces;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (k < __ldg(dist + mid))
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo < n_faces ? lo : n_faces - 1;
}

__global__ void __launch_bounds__(kPushBlock) assign_faces_kernel(int32_t start, int32_t count, int32_t n_faces,
                                                                  const int32_t* __restrict__ dist, int32_t* p2c) {
    const int64_t k = (int64_t)blockIdx.x * kPushBlock + threadIdx.x;
    if (k < count) p2c[(int64_t)start + k] = face_of(dist, n_faces, k);
}

template <typename T>
__global__ void fill_kernel(T* dst, int64_t count, T value) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = value;
}

// Injection: face of injected particle k = first j with k < dist[j]; then
// inject_ions_kernel (apps/app_fempic/kernels.h:63-90) plus the thermal velocity.  With a
// device count (cnt), start is cnt->size; a batch that would not fit in the stride writes
// nothing and records OPPB_ERR_CAPACITY.
__global__ void __launch_bounds__(kPushBlock) inject_kernel(oppb_set_count* cnt, int32_t start_host, int32_t count,
                                                            int32_t stride,
                                                            int32_t n_faces, int32_t n_cells,
                                                            const int32_t* __restrict__ dist,
                                                            const int32_t* __restrict__ if2c,
                                                            const double* __restrict__ geom,
                                                            const double* __restrict__ ef,
                                                            const double* __restrict__ rnd, int32_t rstride,
                                                            int32_t rdim, double ion_velocity, double qm, double dt,
                                                            double* pos, double* vel, int32_t* p2c) {
    const int64_t k = (int64_t)blockIdx.x * kPushBlock + threadIdx.x;
    int32_t start = start_host;
    if (cnt) {
        start = cnt->size;
        if ((int64_t)start + count > stride || start < 0) {
            if (k == 0) atomicCAS(&cnt->error, 0, OPPB_ERR_CAPACITY);
            return;
        }
    }
    if (k >= count) return;
    // Without a distribution the face index is already in p2c (opp_inc_part_count_with_distribution).
    const int face = dist ? face_of(dist, n_faces, k) : p2c[(int64_t)start + k];
    if ((uint32_t)face >= (uint32_t)n_faces) {
        p2c[(int64_t)start + k] = kRemoved;
        return;
    }
    const int32_t cell = __ldg(if2c + face);
    if ((uint32_t)cell >= (uint32_t)n_cells) {
        p2c[(int64_t)start + k] = kRemoved;
        return;
    }
    const double* g = geom + (int64_t)face * 12;
    double a = rnd[k];
    double b = rnd[(int64_t)rstride + k];
    if (__dadd_rn(a, b) > 1) {
        a = __dsub_rn(1.0, a);
        b = __dsub_rn(1.0, b);
    }
    const double half_dt = __dmul_rn(0.5, dt);
    const int64_t p = (int64_t)start + k;
    const double2 e01 = ldg_d2(ef + (int64_t)cell * 4);
    const double2 e2_ = ldg_d2(ef + (int64_t)cell * 4 + 2);
    const double e[3] = {e01.x, e01.y, e2_.x};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double x = __dadd_rn(__dadd_rn(__dmul_rn(a, g[d]), __dmul_rn(b, g[3 + d])), g[9 + d]);
        double v = __dmul_rn(g[6 + d], ion_velocity);
        v = __dsub_rn(v, __dmul_rn(__dmul_rn(qm, e[d]), half_dt));
        if (rdim >= 5) v = __dadd_rn(v, rnd[(int64_t)(2 + d) * rstride + k]);
        pos[(int64_t)d * stride + p] = x;
        vel[(int64_t)d * stride + p] = v;
    }
    p2c[p] = cell;
}

int check_push(const oppb_tet_mesh* mesh, const oppb_particles* parts) {
    if (!mesh || !mesh->ef || mesh->n_cells <= 0 || !aligned(mesh->ef, 16)) return OPPB_ERR_ARG;
    if (!parts || parts->size < 0 || parts->stride < parts->size || !parts->pos || !parts->vel || !parts->p2c)
        return OPPB_ERR_ARG;
    return OPPB_OK;
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_push_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts, double qm, double dt,
                             void* stream) {
    using namespace oppb;
    const int rc = check_push(mesh, parts);
    if (rc) return rc;
    if (parts->size == 0) return OPPB_OK;
    push_f64_kernel<<<ceil_div(parts->size, kPushBlock), kPushBlock, 0, as_stream(stream)>>>(
        parts->size, parts->stride, mesh->n_cells, parts->p2c, mesh->ef, parts->pos, parts->vel, qm, dt);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_push_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts, double qm, double dt,
                               void* stream) {
    using namespace oppb;
    const int rc = check_push(mesh, parts);
    if (rc) return rc;
    if (parts->size == 0) return OPPB_OK;
    push_mixed_kernel<<<ceil_div(parts->size, kPushBlock), kPushBlock, 0, as_stream(stream)>>>(
        parts->size, parts->stride, mesh->n_cells, parts->p2c, mesh->ef, parts->pos, parts->vel,
        (float)(qm * dt), (float)dt);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_inject_f64(const oppb_tet_mesh* mesh, const oppb_inlet* inlet, const oppb_particles* parts,
                               int32_t start, int32_t count, const double* rnd, int32_t rnd_stride, int32_t rnd_dim,
                               double ion_velocity, double qm, double dt, void* stream) {
    using namespace oppb;
    if (!mesh || !mesh->ef || !aligned(mesh->ef, 16) || !inlet || inlet->n_faces <= 0 || !inlet->if2c ||
        !inlet->geom)
        return OPPB_ERR_ARG;
    if (!parts || !parts->pos || !parts->vel || !parts->p2c || start < 0 || count < 0) return OPPB_ERR_ARG;
    if (count > 0 && (!rnd || rnd_stride < count || (rnd_dim != 2 && rnd_dim != 5))) return OPPB_ERR_ARG;
    if ((int64_t)start + count > parts->stride) return OPPB_ERR_CAPACITY;
    if (count == 0) return OPPB_OK;
    inject_kernel<<<ceil_div(count, kPushBlock), kPushBlock, 0, as_stream(stream)>>>(
        nullptr, start, count, parts->stride, inlet->n_faces, mesh->n_cells, inlet->dist, inlet->if2c, inlet->geom,
        mesh->ef, rnd, rnd_stride, rnd_dim, ion_velocity, qm, dt, parts->pos, parts->vel, parts->p2c);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_inject_dev(const oppb_tet_mesh* mesh, const oppb_inlet* inlet, const oppb_particles* parts,
                               oppb_set_count* count, int32_t n_inject, const double* rnd, int32_t rnd_stride,
                               int32_t rnd_dim, double ion_velocity, double qm, double dt, void* stream) {
    using namespace oppb;
    if (!mesh || !mesh->ef || !aligned(mesh->ef, 16) || !inlet || inlet->n_faces <= 0 || !inlet->if2c ||
        !inlet->geom || !inlet->dist)
        return OPPB_ERR_ARG;
    if (!parts || !parts->pos || !parts->vel || !parts->p2c || !count || n_inject < 0 || parts->stride < 0)
        return OPPB_ERR_ARG;
    if (n_inject > 0 && (!rnd || rnd_stride < n_inject || (rnd_dim != 2 && rnd_dim != 5))) return OPPB_ERR_ARG;
    if (n_inject > parts->stride) return OPPB_ERR_CAPACITY;
    if (n_inject == 0) return OPPB_OK;
    inject_kernel<<<ceil_div(n_inject, kPushBlock), kPushBlock, 0, as_stream(stream)>>>(
        count, 0, n_inject, parts->stride, inlet->n_faces, mesh->n_cells, inlet->dist, inlet->if2c, inlet->geom,
        mesh->ef, rnd, rnd_stride, rnd_dim, ion_velocity, qm, dt, parts->pos, parts->vel, parts->p2c);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_assign_faces(const oppb_inlet* inlet, int32_t* p2c, int32_t start, int32_t count, void* stream) {
    using namespace oppb;
    if (!inlet || inlet->n_faces <= 0 || !inlet->dist || !p2c || start < 0 || count < 0) return OPPB_ERR_ARG;
    if (count == 0) return OPPB_OK;
    assign_faces_kernel<<<ceil_div(count, kPushBlock), kPushBlock, 0, as_stream(stream)>>>(start, count, inlet->n_faces,
                                                                                        inlet->dist, p2c);
    count_launches(1);
    return launch_status();
}

extern "C" int oppb_fill(void* dst, int64_t count, int32_t elem_bytes, uint64_t pattern, void* stream) {
    using namespace oppb;
    if (count < 0 || (count > 0 && !dst) || (elem_bytes != 4 && elem_bytes != 8)) return OPPB_ERR_ARG;
    if (!aligned(dst, (size_t)elem_bytes)) return OPPB_ERR_ARG;
    if (count == 0) return OPPB_OK;
    const int grid = (int)std::min<int64_t>(ceil_div(count, 256), 148 * 16);
    if (elem_bytes == 8)
        fill_kernel<uint64_t><<<grid, 256, 0, as_stream(stream)>>>(static_cast<uint64_t*>(dst), count, pattern);
    else
        fill_kernel<uint32_t><<<grid, 256, 0, as_stream(stream)>>>(static_cast<uint32_t*>(dst), count,
                                                                   (uint32_t)pattern);
    count_launches(1);
    return launch_status();
}
