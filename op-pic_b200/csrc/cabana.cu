// CabanaPIC particle hot path: relativistic Boris push, streak walk across hex-cell faces and
// the charge-conserving current deposit into the 12 per-cell accumulators, one launch.
//
// One thread per particle; a particle's calls of the reference kernel (the first one with the
// push, then one per face crossing) run in a warp-wide loop so that every call's deposit goes
// through one warp reduction: lanes whose deposits target the same cell are summed in shared
// memory and each such group issues 12 FP64 atomics.  Particles are initialised cell by cell
// and move a few hundredths of a cell per step, so a warp's lanes spread over a few cells and
// the reduction turns 384 atomics per warp into a few dozen.
//
// FP64 expressions are written in the reference's order and this file is compiled with
// -fmad=false (no contraction), so positions, momenta, streaks and cells are bit-identical to
// the seq backend (apps/app_cabanapic/kernels.h:109-355).

#include "oppb_cabana.h"
#include "oppb_common.cuh"

namespace oppb {
namespace {

constexpr int kCabBlock = 256;
constexpr int kCabWarps = kCabBlock / 32;
constexpr int kSparseLanes = 4;  // at most this many depositing lanes: plain atomics, no staging
constexpr int kStageStride = 14;  // doubles per staged row: 12 used, 16-B aligned rows

struct HexArgs {
    int32_t n_cells;
    const int32_t* c2f;
    const double* interp;
    const float* interp32;  // FP32-momentum form
};

struct CabParts {
    int32_t size;
    int32_t stride;
    double* pos;
    double* vel;
    float* vel32;  // FP32-momentum form: p_vel in FP32
    double* streak;
    const double* weight;
    int32_t* p2c;
};

// CALC_J(X,Y,Z) of apps/app_cabanapic/kernels.h:11-26 into j[0..3].
__device__ __forceinline__ void calc_j(double* j, double q, double u, double dy, double dz, double v5) {
    double v0, v1, v2, v3, v4;
    v4 = q * u;
    v1 = v4 * dy;
    v0 = v4 - v1;
    v1 += v4;
    v4 = 1.0 + dz;
    v2 = v0 * v4;
    v3 = v1 * v4;
    v4 = 1.0 - dz;
    v0 *= v4;
    v1 *= v4;
    v0 += v5;
    v1 -= v5;
    v2 -= v5;
    v3 += v5;
    j[0] = v0;
    j[1] = v1;
    j[2] = v2;
    j[3] = v3;
}

// weight_current_to_accumulator_kernel (kernels.h:109-136): the 12 values one call adds.
__device__ __forceinline__ void weight_current(double* j, double q, double ux, double uy, double uz, double dx,
                                               double dy, double dz) {
    const double v5 = q * ux * uy * uz * (1.0 / 3.0);
    calc_j(j + 0, q, ux, dy, dz, v5);
    calc_j(j + 4, q, uy, dz, dx, v5);
    calc_j(j + 8, q, uz, dx, dy, v5);
}

// The OPP_DO_ONCE block of move_deposit_kernel (kernels.h:148-253): Boris push of u from the
// cell's interpolated fields at the particle's position; returns true when the particle stays
// in its cell (pos updated, j filled), else leaves the normalised displacement in s.
__device__ __forceinline__ bool push_once(const double* __restrict__ rec, double qdt_2mc, double cdx, double cdy,
                                          double cdz, double q, double pos[3], double u[3], double s[3], double* j) {
    double r[20];
    ldg256(rec, r[0], r[1], r[2], r[3]);
    ldg256(rec + 4, r[4], r[5], r[6], r[7]);
    ldg256(rec + 8, r[8], r[9], r[10], r[11]);
    ldg256(rec + 12, r[12], r[13], r[14], r[15]);
    ldg256(rec + 16, r[16], r[17], r[18], r[19]);
    const double ex = r[0], dexdy = r[1], dexdz = r[2], d2exdydz = r[3];
    const double ey = r[4], deydz = r[5], deydx = r[6], d2eydzdx = r[7];
    const double ez = r[8], dezdx = r[9], dezdy = r[10], d2ezdxdy = r[11];
    double cbx = r[12], cby = r[14], cbz = r[16];
    const double dcbxdx = r[13], dcbydy = r[15], dcbzdz = r[17];
    const double dx = pos[0], dy = pos[1], dz = pos[2];

    const double hax = qdt_2mc * ((ex + dy * dexdy) + dz * (dexdz + dy * d2exdydz));
    const double hay = qdt_2mc * ((ey + dz * deydz) + dx * (deydx + dz * d2eydzdx));
    const double haz = qdt_2mc * ((ez + dx * dezdx) + dy * (dezdy + dx * d2ezdxdy));
    cbx = cbx + dx * dcbxdx;
    cby = cby + dy * dcbydy;
    cbz = cbz + dz * dcbzdz;

    double ux = u[0], uy = u[1], uz = u[2];
    ux += hax;
    uy += hay;
    uz += haz;
    double v0 = __ddiv_rn(qdt_2mc, __dsqrt_rn(1.0 + (ux * ux + (uy * uy + uz * uz))));
    double v1 = cbx * cbx + (cby * cby + cbz * cbz);
    double v2 = (v0 * v0) * v1;
    double v3 = v0 * (1.0 + v2 * ((1.0 / 3.0) + v2 * (2.0 / 15.0)));
    double v4 = __ddiv_rn(v3, 1.0 + v1 * (v3 * v3));
    v4 += v4;
    v0 = ux + v3 * (uy * cbz - uz * cby);
    v1 = uy + v3 * (uz * cbx - ux * cbz);
    v2 = uz + v3 * (ux * cby - uy * cbx);
    ux += v4 * (v1 * cbz - v2 * cby);
    uy += v4 * (v2 * cbx - v0 * cbz);
    uz += v4 * (v0 * cby - v1 * cbx);
    ux += hax;
    uy += hay;
    uz += haz;
    u[0] = ux;
    u[1] = uy;
    u[2] = uz;

    v0 = __ddiv_rn(1.0, __dsqrt_rn(1.0 + (ux * ux + (uy * uy + uz * uz))));
    ux *= cdx;
    uy *= cdy;
    uz *= cdz;
    ux *= v0;
    uy *= v0;
    uz *= v0;
    v0 = dx + ux;
    v1 = dy + uy;
    v2 = dz + uz;
    v3 = v0 + ux;
    v4 = v1 + uy;
    const double v5 = v2 + uz;
    if (v3 <= 1.0 && v4 <= 1.0 && v5 <= 1.0 && -v3 <= 1.0 && -v4 <= 1.0 && -v5 <= 1.0) {
        pos[0] = v3;
        pos[1] = v4;
        pos[2] = v5;
        weight_current(j, q, ux, uy, uz, v0, v1, v2);
        return true;
    }
    s[0] = ux;
    s[1] = uy;
    s[2] = uz;
    return false;
}

// The same OPP_DO_ONCE push with FP32 momentum (the FP32-momentum form of the two-stream
// workload): u is stored and updated in FP32 from the cell's FP32 field record at the FP32
// rounding of the position, in the FP64 expression's order with correctly rounded divides and
// square roots; the displacement it produces returns to FP64 for the position, the face test
// and the current deposit, as in push_once.
__device__ __forceinline__ bool push_once_f32(const float* __restrict__ rec, float qdt_2mc, float cdx, float cdy,
                                              float cdz, double q, double pos[3], float u[3], double s[3],
                                              double* j) {
    float r[20];
    const float4* r4 = reinterpret_cast<const float4*>(rec);
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const float4 v = __ldg(r4 + k);
        r[4 * k] = v.x;
        r[4 * k + 1] = v.y;
        r[4 * k + 2] = v.z;
        r[4 * k + 3] = v.w;
    }
    const float ex = r[0], dexdy = r[1], dexdz = r[2], d2exdydz = r[3];
    const float ey = r[4], deydz = r[5], deydx = r[6], d2eydzdx = r[7];
    const float ez = r[8], dezdx = r[9], dezdy = r[10], d2ezdxdy = r[11];
    float cbx = r[12], cby = r[14], cbz = r[16];
    const float dcbxdx = r[13], dcbydy = r[15], dcbzdz = r[17];
    const float dx = __double2float_rn(pos[0]), dy = __double2float_rn(pos[1]), dz = __double2float_rn(pos[2]);

    const float hax = qdt_2mc * ((ex + dy * dexdy) + dz * (dexdz + dy * d2exdydz));
    const float hay = qdt_2mc * ((ey + dz * deydz) + dx * (deydx + dz * d2eydzdx));
    const float haz = qdt_2mc * ((ez + dx * dezdx) + dy * (dezdy + dx * d2ezdxdy));
    cbx = cbx + dx * dcbxdx;
    cby = cby + dy * dcbydy;
    cbz = cbz + dz * dcbzdz;

    float ux = u[0], uy = u[1], uz = u[2];
    ux += hax;
    uy += hay;
    uz += haz;
    float v0 = __fdiv_rn(qdt_2mc, __fsqrt_rn(1.0f + (ux * ux + (uy * uy + uz * uz))));
    float v1 = cbx * cbx + (cby * cby + cbz * cbz);
    float v2 = (v0 * v0) * v1;
    const float v3 = v0 * (1.0f + v2 * ((1.0f / 3.0f) + v2 * (2.0f / 15.0f)));
    float v4 = __fdiv_rn(v3, 1.0f + v1 * (v3 * v3));
    v4 += v4;
    v0 = ux + v3 * (uy * cbz - uz * cby);
    v1 = uy + v3 * (uz * cbx - ux * cbz);
    v2 = uz + v3 * (ux * cby - uy * cbx);
    ux += v4 * (v1 * cbz - v2 * cby);
    uy += v4 * (v2 * cbx - v0 * cbz);
    uz += v4 * (v0 * cby - v1 * cbx);
    ux += hax;
    uy += hay;
    uz += haz;
    u[0] = ux;
    u[1] = uy;
    u[2] = uz;

    v0 = __fdiv_rn(1.0f, __fsqrt_rn(1.0f + (ux * ux + (uy * uy + uz * uz))));
    ux *= cdx;
    uy *= cdy;
    uz *= cdz;
    ux *= v0;
    uy *= v0;
    uz *= v0;
    const double sx = ux, sy = uy, sz = uz;  // the displacement, back in FP64
    const double w0 = pos[0] + sx, w1 = pos[1] + sy, w2 = pos[2] + sz;
    const double w3 = w0 + sx, w4 = w1 + sy, w5 = w2 + sz;
    if (w3 <= 1.0 && w4 <= 1.0 && w5 <= 1.0 && -w3 <= 1.0 && -w4 <= 1.0 && -w5 <= 1.0) {
        pos[0] = w3;
        pos[1] = w4;
        pos[2] = w5;
        weight_current(j, q, sx, sy, sz, w0, w1, w2);
        return true;
    }
    s[0] = sx;
    s[1] = sy;
    s[2] = sz;
    return false;
}

// One streak segment (kernels.h:256-354): deposits into j, advances pos and s; returns the
// crossed face (0..5, Face order) or -1 when the streak ends in this cell.
__device__ __forceinline__ int streak_step(double q, double pos[3], double s[3], double* j) {
    double s_midx = pos[0], s_midy = pos[1], s_midz = pos[2];
    double s_dispx = s[0], s_dispy = s[1], s_dispz = s[2];
    const double dirx = (s_dispx > 0) ? 1.0 : -1.0;
    const double diry = (s_dispy > 0) ? 1.0 : -1.0;
    const double dirz = (s_dispz > 0) ? 1.0 : -1.0;
    const double v0 = (s_dispx == 0) ? 3.4e38 : __ddiv_rn(dirx - s_midx, s_dispx);
    const double v1 = (s_dispy == 0) ? 3.4e38 : __ddiv_rn(diry - s_midy, s_dispy);
    const double v2 = (s_dispz == 0) ? 3.4e38 : __ddiv_rn(dirz - s_midz, s_dispz);
    double v3 = 2.0;
    int axis = 3;
    if (v0 < v3) v3 = v0, axis = 0;
    if (v1 < v3) v3 = v1, axis = 1;
    if (v2 < v3) v3 = v2, axis = 2;
    v3 *= 0.5;
    s_dispx *= v3;
    s_dispy *= v3;
    s_dispz *= v3;
    s_midx += s_dispx;
    s_midy += s_dispy;
    s_midz += s_dispz;
    weight_current(j, q, s_dispx, s_dispy, s_dispz, s_midx, s_midy, s_midz);
    s[0] -= s_dispx;
    s[1] -= s_dispy;
    s[2] -= s_dispz;
    pos[0] += (s_dispx + s_dispx);
    pos[1] += (s_dispy + s_dispy);
    pos[2] += (s_dispz + s_dispz);
    if (axis == 3) return -1;
    const double d = axis == 0 ? dirx : axis == 1 ? diry : dirz;
    // The particle leaves through the face at +-1 and enters the neighbour at -+1, exactly.
    if (axis == 0)
        pos[0] = -d;
    else if (axis == 1)
        pos[1] = -d;
    else
        pos[2] = -d;
    return axis + (d > 0 ? 3 : 0);
}

// Staging of one warp's deposits: 32 rows of 12 values (rows 16-B aligned).
struct WarpStage {
    double vals[32][kStageStride];
    int32_t keys[32];
};

// Adds every lane's 12 values j to acc[k * acc_stride + key] (key < 0: nothing).  Lanes with
// the same key form a group (warp match, whatever their positions: the two counter-streaming
// species interleave lane by lane and drift apart); lanes 0..11 sum one column each over a
// group's rows in shared memory and issue one atomic per column and group.  Every lane of
// the warp must call it.
__device__ __forceinline__ void warp_deposit(WarpStage& ws, double* acc, int32_t acc_stride, int32_t key,
                                             const double* j) {
    const int lane = threadIdx.x & 31;
    // Calls after the first one (face crossings) involve a few lanes of a warp: their
    // deposits go straight to global atomics.
    if (__popc(__ballot_sync(kFullMask, key >= 0)) <= kSparseLanes) {
        if (key >= 0) {
#pragma unroll
            for (int c = 0; c < 12; c++) atomicAdd(acc + (int64_t)c * acc_stride + key, j[c]);
        }
        return;
    }
    const unsigned peers = __match_any_sync(kFullMask, key);
    unsigned leaders = __ballot_sync(kFullMask, key >= 0 && lane == __ffs(peers) - 1);
    if (leaders == 0u) return;
    __syncwarp();  // the previous call's readers are done with the stage
    double2* row = reinterpret_cast<double2*>(&ws.vals[lane][0]);
#pragma unroll
    for (int c = 0; c < 6; c++) row[c] = make_double2(j[2 * c], j[2 * c + 1]);
    ws.keys[lane] = key;
    __syncwarp();
    while (leaders) {  // warp-uniform
        const int leader = __ffs(leaders) - 1;
        leaders &= leaders - 1;
        unsigned members = __shfl_sync(kFullMask, peers, leader);
        if (lane < 12) {
            double sum = 0.0;
            while (members) {
                const int r = __ffs(members) - 1;
                members &= members - 1;
                sum += ws.vals[r][lane];
            }
            atomicAdd(acc + (int64_t)lane * acc_stride + ws.keys[leader], sum);
        }
    }
}

// FP32 copies of the constants the FP32 push reads.
struct ConstsF32 {
    float qdt_2mc, cdx, cdy, cdz;
};

// kOcc: resident CTAs per SM the kernel is compiled for (oppb_tuning.cabana_occupancy): 0 = the
// compiler's register count (FP64 form 76 registers, 3 CTAs per SM; FP32-momentum form 64, 4),
// 4 (64 registers, no spills) or 5 (48 registers, about 100 B of spills a thread).
template <bool kF32Mom, int kOcc>
__global__ void __launch_bounds__(kCabBlock, kOcc > 0 ? kOcc : 1) cabana_move_deposit_kernel(HexArgs m, CabParts p,
                                                                        oppb_cabana_consts k, ConstsF32 kf,
                                                                        double* acc, int32_t acc_stride,
                                                                        oppb_move_status* st, int32_t max_hops) {
    __shared__ __align__(16) WarpStage stage[kCabWarps];
    const int64_t i = (int64_t)blockIdx.x * kCabBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool active = i < p.size;
    int32_t cell = active ? ld_stream(p.p2c + i) : -1;
    const int32_t cell0 = cell;
    int err = 0;
    bool going = active;
    if (going && (uint32_t)cell >= (uint32_t)m.n_cells) {
        err = OPPB_ERR_CELL_RANGE;
        going = false;
    }
    double pos[3] = {0.0, 0.0, 0.0}, u[3] = {0.0, 0.0, 0.0}, s[3] = {0.0, 0.0, 0.0};
    float uf[3] = {0.0f, 0.0f, 0.0f};
    double q = 0.0;
    const int64_t sd = p.stride;
    if (going) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            pos[d] = ld_stream(p.pos + d * sd + i);
            if (kF32Mom)
                uf[d] = __ldcs(p.vel32 + d * sd + i);
            else
                u[d] = ld_stream(p.vel + d * sd + i);
        }
        q = __ldg(p.weight + i) * k.qsp;
    }
    const bool pushed = going;
    bool streaking = false;
    int calls = 0;
    while (__any_sync(kFullMask, going)) {
        double j[12];
        int32_t key = -1;
        if (going) {
            calls++;
            key = cell;
            // The first call pushes (OPP_DO_ONCE); unless the particle stays in its cell, it
            // goes on, in the same call, with the first streak segment.
            bool stay = false;
            if (calls == 1) {
                if (kF32Mom)
                    stay = push_once_f32(m.interp32 + (int64_t)cell * 20, kf.qdt_2mc, kf.cdx, kf.cdy, kf.cdz, q, pos,
                                         uf, s, j);
                else
                    stay = push_once(m.interp + (int64_t)cell * 20, k.qdt_2mc, k.cdt_d[0], k.cdt_d[1], k.cdt_d[2],
                                     q, pos, u, s, j);
                streaking = !stay;
            }
            if (stay) {
                going = false;
            } else {
                const int face = streak_step(q, pos, s, j);
                if (face < 0) {
                    going = false;
                } else {
                    const int4 f0 = ldg_i4(m.c2f + (int64_t)cell * 8);
                    const int2 f1 = __ldg(reinterpret_cast<const int2*>(m.c2f + (int64_t)cell * 8 + 4));
                    const int32_t next = face == 0 ? f0.x
                                         : face == 1 ? f0.y
                                         : face == 2 ? f0.z
                                         : face == 3 ? f0.w
                                         : face == 4 ? f1.x
                                                     : f1.y;
                    if ((uint32_t)next >= (uint32_t)m.n_cells) {
                        err = OPPB_ERR_CELL_RANGE;
                        going = false;
                    } else {
                        cell = next;
                        if (calls >= max_hops) {
                            err = OPPB_ERR_HOP_LIMIT;
                            going = false;
                        }
                    }
                }
            }
        }
        warp_deposit(stage[warp], acc, acc_stride, key, j);
    }
    if (err) raise_error(st, err, (int32_t)i);
    if (pushed) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            st_stream(p.pos + d * sd + i, pos[d]);
            if (kF32Mom)
                __stcs(p.vel32 + d * sd + i, uf[d]);
            else
                st_stream(p.vel + d * sd + i, u[d]);
            if (streaking) st_stream(p.streak + d * sd + i, s[d]);
        }
        if (cell != cell0) st_stream(p.p2c + i, cell);
    }
    // Visit statistics: warp reductions in the integer unit, one atomic per counter per warp.
    const unsigned vsum = __reduce_add_sync(kFullMask, (unsigned)calls);
    const unsigned vmax = __reduce_max_sync(kFullMask, (unsigned)calls);
    if (lane == 0) {
        if (vsum) atomicAdd(reinterpret_cast<unsigned long long*>(&st->total_visits), (unsigned long long)vsum);
        if (vmax) atomicMax(&st->max_visits, (int)vmax);
    }
}

// c2ngc SoA [6][stride] -> c2f [n][8]; c_interp SoA [18][stride] -> interp [n][20].
__global__ void __launch_bounds__(256) hex_pack_kernel(int32_t n_cells, int32_t stride, const int32_t* c2ngc,
                                                       const double* c_interp, int32_t* c2f, double* interp,
                                                       float* interp32) {
    const int64_t c = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (c >= n_cells) return;
    if (c2ngc) {
        int32_t f[8];
#pragma unroll
        for (int k = 0; k < 6; k++) f[k] = c2ngc[(int64_t)k * stride + c];
        f[6] = f[7] = 0;
        int4* o = reinterpret_cast<int4*>(c2f + c * 8);
        o[0] = make_int4(f[0], f[1], f[2], f[3]);
        o[1] = make_int4(f[4], f[5], f[6], f[7]);
    }
    if (c_interp) {
        double r[20];
#pragma unroll
        for (int k = 0; k < 18; k++) r[k] = c_interp[(int64_t)k * stride + c];
        r[18] = r[19] = 0.0;
        double2* o = reinterpret_cast<double2*>(interp + c * 20);
#pragma unroll
        for (int k = 0; k < 10; k++) o[k] = make_double2(r[2 * k], r[2 * k + 1]);
        if (interp32) {  // the FP32-momentum form's record: the same 20 values rounded to FP32
            float4* o32 = reinterpret_cast<float4*>(interp32 + c * 20);
#pragma unroll
            for (int k = 0; k < 5; k++)
                o32[k] = make_float4(__double2float_rn(r[4 * k]), __double2float_rn(r[4 * k + 1]),
                                     __double2float_rn(r[4 * k + 2]), __double2float_rn(r[4 * k + 3]));
        }
    }
}

}  // namespace
}  // namespace oppb

extern "C" int oppb_hex_mesh_pack(const oppb_hex_mesh* mesh, int32_t stride, const int32_t* c2ngc,
                                  const double* c_interp, void* stream) {
    using namespace oppb;
    if (!mesh || mesh->n_cells <= 0 || stride < mesh->n_cells) return OPPB_ERR_ARG;
    if (c2ngc && (!mesh->c2f || !aligned(mesh->c2f, 32))) return OPPB_ERR_ARG;
    if (c_interp && (!mesh->interp || !aligned(mesh->interp, 32))) return OPPB_ERR_ARG;
    if (mesh->interp32 && !aligned(mesh->interp32, 16)) return OPPB_ERR_ARG;
    if (!c2ngc && !c_interp) return OPPB_OK;
    hex_pack_kernel<<<ceil_div(mesh->n_cells, 256), 256, 0, as_stream(stream)>>>(
        mesh->n_cells, stride, c2ngc, c_interp, mesh->c2f, mesh->interp, mesh->interp32);
    count_launches(1);
    return launch_status();
}

namespace oppb {
namespace {
template <bool kF32Mom>
int launch_cabana(const oppb_hex_mesh* mesh, const oppb_cabana_particles* parts, float* vel32,
                  const oppb_cabana_consts* consts, double* acc, int32_t acc_stride, oppb_move_status* status,
                  int32_t max_hops, void* stream) {
    if (!mesh || mesh->n_cells <= 0 || !mesh->c2f || !mesh->interp || !aligned(mesh->c2f, 32) ||
        !aligned(mesh->interp, 32))
        return OPPB_ERR_ARG;
    if (kF32Mom && (!mesh->interp32 || !aligned(mesh->interp32, 16) || !vel32)) return OPPB_ERR_ARG;
    if (!parts || parts->size < 0 || parts->stride < parts->size) return OPPB_ERR_ARG;
    if (!parts->pos || (!kF32Mom && !parts->vel) || !parts->streak_mid || !parts->weight || !parts->p2c)
        return OPPB_ERR_ARG;
    if (!consts || !acc || acc_stride < mesh->n_cells || !status || max_hops <= 0) return OPPB_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(status, 0, sizeof(oppb_move_status), s) != cudaSuccess) return OPPB_ERR_LAUNCH;
    if (parts->size == 0) return launch_status();
    const HexArgs m{mesh->n_cells, mesh->c2f, mesh->interp, mesh->interp32};
    const CabParts p{parts->size, parts->stride, parts->pos, parts->vel, vel32, parts->streak_mid, parts->weight,
                     parts->p2c};
    // FP32 constants: the round-to-nearest FP32 values of the FP64 ones.
    const ConstsF32 kf{(float)consts->qdt_2mc, (float)consts->cdt_d[0], (float)consts->cdt_d[1],
                       (float)consts->cdt_d[2]};
    const int occ = tuning().cabana_occupancy;
    auto kernel = occ == 5   ? cabana_move_deposit_kernel<kF32Mom, 5>
                  : occ == 4 ? cabana_move_deposit_kernel<kF32Mom, 4>
                             : cabana_move_deposit_kernel<kF32Mom, 0>;
    kernel<<<ceil_div(parts->size, kCabBlock), kCabBlock, 0, s>>>(
        m, p, *consts, kf, acc, acc_stride, status, max_hops);
    count_launches(1);
    return launch_status();
}
}  // namespace
}  // namespace oppb

extern "C" int oppb_cabana_move_deposit(const oppb_hex_mesh* mesh, const oppb_cabana_particles* parts,
                                        const oppb_cabana_consts* consts, double* acc, int32_t acc_stride,
                                        oppb_move_status* status, int32_t max_hops, void* stream) {
    return oppb::launch_cabana<false>(mesh, parts, nullptr, consts, acc, acc_stride, status, max_hops, stream);
}

extern "C" int oppb_cabana_move_deposit_mixed(const oppb_hex_mesh* mesh, const oppb_cabana_particles* parts,
                                              float* vel32, const oppb_cabana_consts* consts, double* acc,
                                              int32_t acc_stride, oppb_move_status* status, int32_t max_hops,
                                              void* stream) {
    return oppb::launch_cabana<true>(mesh, parts, vel32, consts, acc, acc_stride, status, max_hops, stream);
}
