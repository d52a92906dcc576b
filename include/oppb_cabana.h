/* C ABI of the B200 backend for OP-PIC's CabanaPIC particle hot path: the relativistic Boris
 * push, the streak walk across hex-cell faces and the charge-conserving current deposit into
 * the 12 per-cell accumulators, all in one launch (apps/app_cabanapic/kernels.h:109-355;
 * generated CUDA body apps_codegen/app_cabanapic_cg/cuda/move_deposit_kernel_loop.hpp:305-358).
 *
 * Conventions are those of oppb.h: plain pointers, int status (OPPB_OK ...), an explicit
 * stream (cudaStream_t as void*), no allocation.  Particle dats and c_acc use the reference's
 * device layout, SoA [dim][stride]; the mesh is packed once per field update into 32-byte
 * records read with 256-bit loads.
 */
#ifndef OPPB_CABANA_H
#define OPPB_CABANA_H

#include <stddef.h>
#include <stdint.h>

#include "oppb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Hex mesh (ghost cells included, as the reference's cell set) in the packed layout:
 *   c2f    [n_cells][8]  i32 : c2ngc_map faces xd, yd, zd, xu, yu, zu (Face order,
 *                              apps/app_cabanapic/cabana_defs.h:134-141), then 2 unused words
 *   interp [n_cells][20] f64 : c_interp, the 18 CellInterp values (cabana_defs.h:95-114),
 *                              then 2 unused doubles (160-B records)
 *   interp32 [n_cells][20] f32 : the same values rounded to FP32, for the FP32-momentum form
 *                              (may be NULL; 16-byte aligned)
 * Buffers are owned by the caller, 32-byte aligned. */
typedef struct oppb_hex_mesh {
    int32_t  n_cells;
    int32_t* c2f;
    double*  interp;
    float*   interp32;
} oppb_hex_mesh;

/* Particles, SoA [dim][stride]: p_pos (cell-local coordinates in [-1,1]^3), p_vel (momentum
 * u = gamma v / c), p_streak_mid, p_weight, and the p2c map. */
typedef struct oppb_cabana_particles {
    int32_t size;
    int32_t stride;
    double* pos;
    double* vel;
    double* streak_mid;
    const double* weight;
    int32_t* p2c;
} oppb_cabana_particles;

/* The CONST_* values the kernel reads (cabana_opp.cpp:99-105): CONST_qdt_2mc, CONST_cdt_d,
 * CONST_qsp. */
typedef struct oppb_cabana_consts {
    double qdt_2mc;
    double cdt_d[3];
    double qsp;
} oppb_cabana_consts;

/* Packs the reference's device dats into `mesh`: c2ngc SoA [6][stride] into c2f, c_interp SoA
 * [18][stride] into interp.  Either source may be NULL (that record is left as it is), so the
 * per-step field update repacks interp only. */
int oppb_hex_mesh_pack(const oppb_hex_mesh* mesh, int32_t stride, const int32_t* c2ngc,
                       const double* c_interp, void* stream);

/* opp_particle_move__move_deposit_kernel (cabana_opp.cpp:158-164) for particles [0, size):
 * per particle the first call does the Boris push (OPP_DO_ONCE) and either stays in its cell
 * or starts the streak; every call deposits the current of its segment into the cell's 12
 * accumulators; a face crossing moves the particle to c2f[face] and the next call continues
 * the streak.  acc is c_acc, SoA [12][acc_stride], accumulated into (the caller zeroes it, as
 * opp_reset_dat does).  status counts calls in total_visits (hops + 1 per particle) and
 * max_visits; the hop bound sets OPPB_ERR_HOP_LIMIT, a cell index out of range
 * OPPB_ERR_CELL_RANGE.  Positions, momenta, streaks and cells are bit-identical to the seq
 * backend; accumulator sums are order-dependent (FP64 atomics).  Periodic meshes remove no
 * particle: status->remove_count stays 0. */
int oppb_cabana_move_deposit(const oppb_hex_mesh* mesh, const oppb_cabana_particles* parts,
                             const oppb_cabana_consts* consts, double* acc, int32_t acc_stride,
                             oppb_move_status* status, int32_t max_hops, void* stream);

/* The FP32-momentum form of the two-stream workload (FP64 position, FP32 momentum): as
 * oppb_cabana_move_deposit, with p_vel held in FP32 in vel32 (SoA [3][stride], parts->vel
 * unused) and the OPP_DO_ONCE Boris push computed in FP32 from mesh->interp32, in the FP64
 * expression's order with correctly rounded divides and square roots.  The push's
 * displacement returns to FP64: positions, the streak walk, cells and the 12-accumulator
 * current deposit are FP64 as in the FP64 form. */
int oppb_cabana_move_deposit_mixed(const oppb_hex_mesh* mesh, const oppb_cabana_particles* parts, float* vel32,
                                   const oppb_cabana_consts* consts, double* acc, int32_t acc_stride,
                                   oppb_move_status* status, int32_t max_hops, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_CABANA_H */
