// Shared device helpers of the oppb kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "oppb.h"

namespace oppb {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int32_t kRemoved = OPPB_REMOVED_CELL;

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// Process-wide count of kernels launched by the library (abi.cu).
void count_launches(int n);
// Process-wide launch choices (abi.cu).
const oppb_tuning& tuning();

inline int launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? OPPB_OK : OPPB_ERR_LAUNCH;
}

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// Read-only loads through the non-coherent (L1/texture) path.
__device__ __forceinline__ double2 ldg_d2(const double* p) {
    return __ldg(reinterpret_cast<const double2*>(p));
}
__device__ __forceinline__ int4 ldg_i4(const int32_t* p) { return __ldg(reinterpret_cast<const int4*>(p)); }
__device__ __forceinline__ float4 ldg_f4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// 256-bit read-only loads (sm_100): one instruction per 32-byte cell record chunk.
__device__ __forceinline__ void ldg256(const double* p, double& a, double& b, double& c, double& d) {
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void ldg256(const float* p, float (&v)[8]) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
}

// Streaming loads/stores for particle data that is touched once per step.
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(double* p, double v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(int32_t* p, int32_t v) { __stcs(p, v); }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Records the first device-side error of a launch.
__device__ __forceinline__ void raise_error(oppb_move_status* st, int32_t code, int32_t index) {
    if (atomicCAS(&st->error, 0, code) == 0) st->error_index = index;
}

}  // namespace oppb
