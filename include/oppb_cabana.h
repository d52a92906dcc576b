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

/* ------------------------------------------------------------ the mesh loops of the app
 * The generated main's cell loops (apps_codegen/app_cabanapic_cg/cabana_opp.cpp:144-299; user
 * kernels apps/app_cabanapic/kernels.h), one thread per cell of [0, n_cells), each value as the
 * seq backend computes it.  Cell dats are SoA [dim][stride] (stride >= n_cells).  A neighbour
 * argument is one column of a cell map's device copy (map + idx * stride): the cell each cell
 * reads through that argument. */

/* interpolate_mesh_fields_kernel: c_interp (18 values) of every cell with c_mask_ghost 0 from
 * c_e at the cell and at nb_e = its xu_y_z, x_yu_z, x_y_zu, xu_yu_z, x_yu_zu, xu_y_zu neighbours,
 * and c_b at the cell and at nb_b = its xu_y_z, x_yu_z, x_y_zu neighbours. */
int oppb_cabana_interpolate(int32_t n_cells, int64_t stride, const double* c_e, const double* c_b,
                            const int32_t* const nb_e[6], const int32_t* const nb_b[3], double* c_interp,
                            const int32_t* c_mask_ghost, void* stream);

/* accumulate_current_to_cells_kernel: c_j of every cell with c_mask_right 1 from c_acc at the
 * cell and at nb_lower = its xd_y_z, x_yd_z, x_y_zd, xd_yd_z, x_yd_zd, xd_y_zd neighbours, times
 * acc_coef (CONST_acc_coef). */
int oppb_cabana_accumulate(int32_t n_cells, int64_t stride, double* c_j, const double* c_acc,
                           const int32_t* const nb_lower[6], const int32_t* c_mask_right, const double acc_coef[3],
                           void* stream);

/* half_advance_b_kernel: c_b of every cell with c_mask_ghost 0 less half a step of curl c_e,
 * c_e at nb_upper = its xu_y_z, x_yu_z, x_y_zu neighbours; p = CONST_p. */
int oppb_cabana_half_advance_b(int32_t n_cells, int64_t stride, const int32_t* const nb_upper[3], const double* c_e,
                               double* c_b, const int32_t* c_mask_ghost, const double p[3], void* stream);

/* advance_e_kernel: c_e of every cell with c_mask_right 1 plus -dt_eps0 c_j + curl c_b, c_b at
 * nb_lower = its xd_y_z, x_yd_z, x_y_zd neighbours; p = CONST_p, dt_eps0 = CONST_dt_eps0. */
int oppb_cabana_advance_e(int32_t n_cells, int64_t stride, const int32_t* const nb_lower[3], const double* c_b,
                          const double* c_j, double* c_e, const int32_t* c_mask_right, const double p[3],
                          double dt_eps0, void* stream);

/* update_ghosts_B_kernel (dim = -1: the three components of `from` at cell c copied to `to` at
 * to_map[c]) and update_ghosts_kernel (dim 0..2: that component added there), for the cells c
 * whose mask (a 6-component cell dat: c_mask_ugb or c_mask_ug) holds 1 at m_idx.  Cells written
 * must not be read by the same call (the app's ghost maps pair interior and ghost cells). */
int oppb_cabana_update_ghosts(int32_t n_cells, int64_t stride, const int32_t* mask, int32_t m_idx, const double* from,
                              double* to, const int32_t* to_map, int32_t dim, void* stream);

/* compute_energy_kernel: adds to *energy (device) the sum over the cells with c_mask_ghost 0 of
 * fx fx + fy fy + fz fz.  The sum is taken in a fixed order (deterministic), not the seq
 * backend's cell order, so it matches the reference's to rounding.  The workspace holds the
 * block partials (oppb_cabana_energy_workspace_bytes, 8-byte aligned). */
size_t oppb_cabana_energy_workspace_bytes(void);
int oppb_cabana_energy(int32_t n_cells, int64_t stride, const int32_t* c_mask_ghost, const double* field,
                       double* energy, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_CABANA_H */
