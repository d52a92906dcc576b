/* C ABI of the B200 backend for OP-PIC's NESO-advection particle path
 * (apps_codegen/app_neso_advection_mdir_cg): the periodic position update
 * (opp_par_loop_all__update_pos_kernel) and the axis-wise multi-hop move
 * (opp_particle_move__move_kernel), for one instance or for a batch of independent
 * instances of different mesh and particle counts advanced by one persistent launch.
 *
 * Conventions are those of oppb.h (plain pointers, int status, explicit stream, no
 * allocation).  Particle dats of all instances are concatenated in the reference's device
 * layout, SoA [2][stride]; p2c and the neighbour map hold instance-local cell indices.
 */
#ifndef OPPB_ADVEC_H
#define OPPB_ADVEC_H

#include <stddef.h>
#include <stdint.h>

#include "oppb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One instance: its particles [part_offset, part_offset + n_parts) of the concatenated dats,
 * its cells [cell_offset, cell_offset + n_cells) of the packed cell records, and its
 * CONST_dt, CONST_cell_width, CONST_extents (advec_opp.cpp).  grid_nx > 0 declares the cells
 * the periodic grid_nx x (n_cells / grid_nx) grid of the app's init_mesh (advec_misc.h:115-141:
 * cell x + nx y with c_pos_ll = (x w, y w) and the VOXEL_MAP neighbours), as
 * oppb_advec_check_grid verifies: the move then computes each cell's corner and neighbours
 * from its index instead of reading its record (the same values, bit for bit).  0 = read the
 * records. */
typedef struct oppb_advec_instance {
    int64_t part_offset;
    int32_t n_parts;
    int32_t cell_offset;
    int32_t n_cells;
    int32_t grid_nx;
    double  dt;
    double  cell_width;
    double  extents[2];
} oppb_advec_instance;

/* Direct-hop seed of one instance (the global move of the reference's move loop,
 * opp_dev_checkForGlobalMove2D_kernel with opp_dev_findStructuredCellIndex2D,
 * opp_lib/include/device_kernels/cuda_inline_kernels.h): the map of its grid (device,
 * filled by oppb_dh_build_quad), the grid's lower corner, 1/spacing and box counts.  Before a
 * particle's walk, box (x, y) = ((pos - min) * inv_spacing truncated toward zero, negative
 * giving 0); a box at or past the count on either axis, or one without a cell, removes the
 * particle (p2c = OPPB_REMOVED_CELL, counted in status->remove_count), else the walk starts
 * from the box's cell. */
typedef struct oppb_advec_dh {
    const int32_t* map;
    double  min[2];
    double  inv_spacing;
    int64_t dims[2];
} oppb_advec_dh;

/* A batch.  instances: device array [n_instances].  tile_prefix: device array
 * [n_instances + 1], the first 256-particle work item of each instance (prefix sum of
 * ceil(n_parts / 256)).  Blocks take items in order, a chunk at a time, from work_counter,
 * so the items in flight stay within one or two instances (their cell records stay in L2)
 * whatever the speed of each block.  cells: packed records [total cells][4] f64 = c_pos_ll x, y, then
 * c2c (CellMap order xd_y, xu_y, x_yd, x_yu) as four int32; 32-byte aligned. */
typedef struct oppb_advec_batch {
    int32_t n_instances;
    int32_t n_work;            /* tile_prefix[n_instances] */
    const oppb_advec_instance* instances;
    const int32_t* tile_prefix;
    const double* cells;
    int64_t stride;            /* capacity of the concatenated particle dats */
    double*  pos;              /* p_pos  [2][stride] */
    const double* vel;         /* p_vel  [2][stride] */
    int32_t* mdir;             /* p_move_dir [2][stride] */
    int32_t* p2c;              /* p2c [stride] */
    int32_t* work_counter;     /* device scratch, one int32: the launch hands out work items in
                                  order from it (the launcher zeroes it on the launch's stream) */
    const oppb_advec_dh* dh;   /* device array [n_instances], or NULL: walks start from p2c.
                                  Particles at OPPB_REMOVED_CELL are skipped either way. */
} oppb_advec_batch;

/* Packs one instance's c_pos_ll (SoA [2][ld]) and c2c_map (SoA [4][ld]) into
 * cells[cell_offset .. cell_offset + n_cells). */
int oppb_advec_pack_cells(double* cells, int32_t cell_offset, int32_t n_cells, int32_t ld,
                          const double* c_pos_ll, const int32_t* c2c, void* stream);

/* Writes to *mismatches (device int32) the number of cells of one instance whose packed record
 * (cells + 4 * cell_offset, n_cells records) differs in any bit from the periodic nx-wide grid's
 * corner (x w, y w) and neighbours; 0 means the instance may set grid_nx = nx.  No counterpart
 * in the reference (its move always reads c_pos_ll and c_c_map).  OPPB_ERR_ARG unless
 * n_cells is a multiple of nx. */
int oppb_advec_check_grid(const double* cells, int32_t cell_offset, int32_t n_cells, int32_t nx,
                          double cell_width, int32_t* mismatches, void* stream);

/* update_pos_kernel then move_kernel for every particle of every instance, fused per
 * particle (the position stays in registers), in one persistent launch.  Bit-identical to
 * the seq backend running the two loops on each instance (with opp_global_move on, when
 * batch->dh is set).  status is accumulated into, not
 * cleared (zero it before a sequence of steps, e.g. one captured CUDA graph of many steps):
 * total_visits / max_visits count move calls; the first hop-bound overrun or out-of-range
 * cell sets error / error_index (index into the concatenated dats). */
int oppb_advec_step(const oppb_advec_batch* batch, oppb_move_status* status, int32_t max_hops,
                    void* stream);

/* The two loops separately, as the generated main calls them:
 * opp_par_loop_all__update_pos_kernel (apps_codegen/app_neso_advection_mdir_cg/cuda/update_pos_kernel_loop.hpp)
 * and opp_particle_move__move_kernel (.../cuda/move_kernel_loop.hpp).  The update reads the
 * batch's pos and vel only (mdir, p2c and cells may be NULL); the move reads pos, mdir, p2c and
 * cells (vel may be NULL). */
int oppb_advec_update_pos(const oppb_advec_batch* batch, void* stream);
int oppb_advec_move(const oppb_advec_batch* batch, oppb_move_status* status, int32_t max_hops,
                    void* stream);

/* verify_kernel of one instance (apps/app_neso_advection/kernels.h:115-151; the generated loop
 * opp_par_loop_all__verify_kernel): adds to *incorrect (device int32) the number of particles
 * i < n_parts whose position pos (SoA [2][stride]) lies outside the closed box
 * [ix w, ix w + w] x [iy w, iy w + w] of their cell, (ix, iy) from the cell's global index
 * g = c_gbl_idx[p2c[i]] as g mod nx, g div nx (a negative ix or iy counts as incorrect). */
int oppb_advec_verify(const double* pos, int64_t stride, const int32_t* p2c, const int32_t* c_gbl_idx,
                      int32_t n_parts, int32_t nx, double cell_width, int32_t* incorrect, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_ADVEC_H */
