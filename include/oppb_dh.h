/* C ABI of the direct-hop (DH) seed of the FemPIC move (and, at the end, of the 2-D grids of
 * the NESO-advection move): OP-PIC's structured cell mapper
 * (opp_lib/include/opp_direct_hop_core.h CellMapper, seq build
 * opp_lib/src/seq/opp_direct_hop_seq.cpp) and the global-move pre-pass of the move loop
 * (apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:112-131, CUDA
 * opp_dev_checkForGlobalMove3D_kernel in opp_lib/include/device_kernels/cuda_inline_kernels.h).
 *
 * A uniform grid of spacing h covers the mesh's bounding box.  Every grid box holds one mesh
 * cell (or none); with the seed on, every particle's walk starts from the cell of the box its
 * position falls in instead of from its previous cell.
 *
 * Conventions are those of oppb.h (plain pointers, int status, explicit stream).  The map is
 * built on the GPU: cells are binned into the grid boxes their bounding boxes overlap, and
 * each query takes the lowest-index cell that contains the point among its box's candidates.
 * That is the reference's answer, which is the first cell, in index order, that contains the
 * point, found there by a search over all cells per point.
 */
#ifndef OPPB_DH_H
#define OPPB_DH_H

#include <stddef.h>
#include <stdint.h>

#include "oppb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The structured grid (CellMapper fields).  min/max: the global bounding box of the nodes
 * widened by `expansion` (BoundingBox(n_pos, 3, expansion), opp_direct_hop_core.h:70-120);
 * dims: boxes per axis (CellMapper::init_host, :317-380); map: device [size] mesh cell of
 * each box, x fastest (index = x + X*y + X*Y*z), OPPB_REMOVED_CELL where no cell. */
typedef struct oppb_dh_grid {
    double   min[3];
    double   max[3];
    double   spacing;       /* grid_spacing                                    */
    double   inv_spacing;   /* 1.0 / spacing (CellMapper::oneOverGridSpacing)  */
    int64_t  dims[3];
    int64_t  size;          /* dims[0] * dims[1] * dims[2]                     */
    int32_t* map;           /* device [size], filled by oppb_dh_build          */
} oppb_dh_grid;

/* Host: the bounding box of the node positions (host AoS [n_nodes][3]) widened by expansion,
 * as opp::BoundingBox(n_pos, 3, expansion) computes it (opp_direct_hop_core.h:70-120). */
int oppb_dh_bounding_box(const double* n_pos, int32_t n_nodes, const double expansion[3],
                         double min_out[3], double max_out[3]);

/* Host: the grid over a box, as CellMapper::init_host counts its boxes (:317-380, floating-point
 * loop counts included).  Leaves map untouched.  OPPB_ERR_ARG for spacing <= 0, a non-finite
 * box or a grid of more than 2^31 boxes. */
int oppb_dh_grid_from_box(const double min[3], const double max[3], double spacing, oppb_dh_grid* grid);

/* Host: oppb_dh_bounding_box then oppb_dh_grid_from_box. */
int oppb_dh_grid_init(const double* n_pos, int32_t n_nodes, double spacing, const double expansion[3],
                      oppb_dh_grid* grid);

/* Device: fills grid->map (generateStructuredMesh, opp_direct_hop_seq.cpp:134-302, steps 1 and
 * 3: box centroid, then the centroid nudged by h/100 along x, y and z in turn, then the
 * lowest-index cell holding one of the box's 8 corners).  The cells' global ids are their
 * indices (one unpartitioned mesh).  n_pos: device SoA [3][n_nodes].  Uses the mesh's FP64
 * records (det, nav) and c2n.  Workspace: when ws_bytes is too small (or workspace is NULL)
 * the call returns OPPB_ERR_WORKSPACE with *ws_needed set, after synchronising the stream
 * once to read the number of (cell, box) pairs; call again with that much. */
int oppb_dh_build(const oppb_tet_mesh* mesh, const double* n_pos, oppb_dh_grid* grid, void* workspace,
                  size_t ws_bytes, size_t* ws_needed, void* stream);

/* ------------------------------------------------------- 2-D grids (NESO advection)
 * The global move of the advection app (apps_codegen/app_neso_advection_mdir_cg/advec_opp.cpp:
 * 97-103: BoundingBox(c_pos_ll, DIM, expansion), opp_init_direct_hop_cg; CUDA pre-pass
 * opp_dev_checkForGlobalMove2D_kernel).  The grid has one box along z (min = max = 0). */

/* Host: BoundingBox(pos, 2, expansion) of host AoS [n][2] points (the cells' lower-left
 * corners c_pos_ll in the app): z stays 0, x/y widened as oppb_dh_bounding_box widens them. */
int oppb_dh_bounding_box_2d(const double* pos, int32_t n, const double expansion[3], double min_out[3],
                            double max_out[3]);

/* Host: oppb_dh_bounding_box_2d then oppb_dh_grid_from_box (dims[2] = 1). */
int oppb_dh_grid_init_2d(const double* pos, int32_t n, double spacing, const double expansion[3],
                         oppb_dh_grid* grid);

/* Device: fills grid->map for the square cells of one advection instance (generateStructuredMesh,
 * as oppb_dh_build, with the app's all-cell checker, apps_codegen/app_neso_advection_mdir_cg/
 * seq/move_kernel_loop.hpp:194-219: the lowest-index cell whose move_kernel call ends with
 * MOVE_DONE, i.e. with 0 <= p - c_pos_ll <= cell_width on both axes).  cells: the instance's
 * first packed record ({c_pos_ll, c2c}, include/oppb_advec.h), device, 32-byte aligned.
 * Workspace as oppb_dh_build.  OPPB_ERR_ARG unless grid->dims[2] == 1. */
int oppb_dh_build_quad(const double* cells, int32_t n_cells, double cell_width, oppb_dh_grid* grid,
                       void* workspace, size_t ws_bytes, size_t* ws_needed, void* stream);

/* ------------------------------------------------------------- general move entry point */

#define OPPB_PRECISION_F64   0
#define OPPB_PRECISION_MIXED 1

/* One call for every variant of the move launch.  deposit: 0 = move only (FP64 only),
 * 1 = node-charge deposit fused.  push: 1 = calculate_new_pos_vel as the kernel's prologue
 * (needs deposit).  dh: the direct-hop seed (NULL = walk from the previous cell), applied
 * after the push, as the reference's global-move pre-pass runs after the push loop: a
 * position outside the grid, or in a box with no cell, removes the particle (the CUDA
 * backend's rule), else the walk starts from the box's cell.  set_count: the particle count
 * in device memory (include/oppb_graph.h; NULL = parts->size is the count): the move then
 * processes [0, min(set_count->size + pending, parts->size)), parts->size being the upper
 * bound that sizes the grid. */
struct oppb_set_count;
typedef struct oppb_move_options {
    int32_t precision;            /* OPPB_PRECISION_*                                  */
    int32_t deposit;
    int32_t push;
    int32_t reserved;
    double  qm, dt;               /* push constants (CONST_charge/CONST_mass, CONST_dt) */
    double  band;                 /* mixed path: FP64 re-check band (e.g. 1e-5)        */
    const oppb_dh_grid* dh;       /* host struct; map on the device; may be NULL        */
    const struct oppb_set_count* set_count;  /* device; may be NULL                      */
    int32_t pending;              /* particles injected since set_count->size was set   */
    int32_t reserved2;
} oppb_move_options;

/* The move of oppb.h (oppb_move_f64 / oppb_move_deposit_* / oppb_push_move_deposit_*) with
 * options; identical results for the same options without dh.  node_charge, workspace as
 * oppb_move_deposit_f64. */
int oppb_move_ex(const oppb_tet_mesh* mesh, const oppb_particles* parts, const oppb_move_options* opt,
                 double* node_charge, oppb_move_status* status, int32_t max_hops, void* workspace,
                 size_t ws_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_DH_H */
