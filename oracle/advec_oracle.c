/* TEST INFRASTRUCTURE ONLY — CPU restatement of OP-PIC's NESO-advection particle path, the
 * checker of the CUDA kernels in op-pic_b200/csrc/advec.cu.  Nothing in the product links it.
 *
 * Follows the generated seq backend of apps_codegen/app_neso_advection_mdir_cg:
 *   update_pos_kernel  kernels.h (seq/update_pos_kernel_loop.hpp), periodic wrap with the
 *                      library's FMOD(a, b) = a - b * trunc(a / b) (opp_lib/include/opp_util.h:48)
 *   move_kernel        kernels.h (seq/move_kernel_loop.hpp:16-70): direction chosen once
 *                      (OPP_DO_ONCE), then hops in x until inside, then in y
 *   hop driver         seq/move_kernel_loop.hpp:95-117 with opp_check_part_move_status
 *                      (opp_lib/include/opp_seq.h:64-86)
 * Layouts are the seq backend's AoS: pos/vel [n][2], mdir [n][2] int, p2c [n],
 * c2c [n_cells][4] (xd_y, xu_y, x_yd, x_yu), c_pos_ll [n_cells][2].
 *
 * Compiled with -ffp-contract=off: one rounding per written operation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

/* update_pos_kernel on one particle. */
static void update_pos(const double* vel, double* pos, double dt, const double* extents) {
    for (int dm = 0; dm < 2; dm++) {
        const double offset = vel[dm] * dt;
        pos[dm] += offset;
        const int n_extent_offset_int = (int)(fabs(pos[dm]) + 2.0);
        const double temp_pos = pos[dm] + n_extent_offset_int * extents[dm];
        pos[dm] = temp_pos - extents[dm] * trunc(temp_pos / extents[dm]);
    }
}

enum { kDone = 0, kNeedMove = 1 };

/* One call of move_kernel; *c is the current cell, updated on a hop. */
static int move_once(int first, const double* pos, int32_t* mdir, const double* ll, const int32_t* c2c, int32_t* c,
                     double cell_width, const double* extents) {
    const double dx = pos[0] - ll[0];
    const double dy = pos[1] - ll[1];
    if (first) {
        const int xp = ((dx > cell_width) && (extents[0] > 2 * dx - cell_width)) ||
                       ((dx < 0) && (extents[0] < cell_width - 2 * dx));
        const int yp = ((dy > cell_width) && (extents[1] > 2 * dy - cell_width)) ||
                       ((dy < 0) && (extents[1] < cell_width - 2 * dy));
        mdir[0] = xp ? 1 : -1;
        mdir[1] = yp ? 1 : -1;
    }
    if ((dx >= 0.0) && (dx <= cell_width)) {
        mdir[0] = 0;
    } else if (mdir[0] > 0) {
        *c = c2c[1];
        return kNeedMove;
    } else if (mdir[0] < 0) {
        *c = c2c[0];
        return kNeedMove;
    }
    if ((dy >= 0.0) && (dy <= cell_width)) {
        mdir[1] = 0;
    } else if (mdir[1] > 0) {
        *c = c2c[3];
        return kNeedMove;
    } else if (mdir[1] < 0) {
        *c = c2c[2];
        return kNeedMove;
    }
    return kDone;
}

/* ------------------------------------------------------------------ direct hop (2-D)
 *
 * The structured cell mapper of the global move on the 2-D advection mesh
 * (opp_lib/include/opp_direct_hop_core.h BoundingBox / CellMapper, seq build
 * opp_lib/src/seq/opp_direct_hop_seq.cpp:134-302) with the app's all-cell checker
 * (apps_codegen/app_neso_advection_mdir_cg/seq/move_kernel_loop.hpp:166-226), and the
 * global-move pre-pass of the move loop (:121-143; the CUDA rule for a position outside the
 * grid, opp_dev_findStructuredCellIndex2D / opp_dev_checkForGlobalMove in
 * opp_lib/include/device_kernels/cuda_inline_kernels.h).  box[6] = {min x, y, z, max x, y, z},
 * z = 0; the map is x fastest (index = x + X*y). */

#define ADV_REMOVED 2147483647 /* MAX_CELL_INDEX */
#define ADV_DBL_MAX 1.7976931348623157e308
#define ADV_DBL_MIN 2.2250738585072014e-308 /* MIN_REAL = numeric_limits<double>::min() */

/* BoundingBox(c_pos_ll, 2, expansion) (opp_direct_hop_core.h:70-120: z stays 0, the x/y
 * widening reads expansion x for both minima and expansion y for both maxima) and
 * CellMapper::init_host's box counts (:317-380).  Returns 0, or 1 for a grid above 2^31 boxes. */
int oracle_advec_dh_grid_init(int32_t n_cells, const double* c_pos_ll, double spacing, const double* expansion,
                              double* box, int64_t* dims) {
    double mn[3] = {ADV_DBL_MAX, ADV_DBL_MAX, 0.0};
    double mx[3] = {ADV_DBL_MIN, ADV_DBL_MIN, 0.0};
    for (int32_t i = 0; i < n_cells; i++)
        for (int d = 0; d < 2; d++) {
            const double v = c_pos_ll[(int64_t)i * 2 + d];
            if (v < mn[d]) mn[d] = v;
            if (mx[d] < v) mx[d] = v;
        }
    mn[0] -= (expansion[0] + 1e-12); /* BOUND_OFFSET, opp_direct_hop_core.h:37 */
    mn[1] -= (expansion[0] + 1e-12);
    mx[0] += (expansion[1] - 1e-12);
    mx[1] += (expansion[1] - 1e-12);
    for (int d = 0; d < 3; d++) {
        int64_t a = 0;
        for (double v = mn[d]; v < mx[d]; v += spacing)
            if (++a > ((int64_t)1 << 31)) return 1;
        dims[d] = a + 1;
        box[d] = mn[d];
        box[3 + d] = mx[d];
    }
    return ((double)dims[0] * (double)dims[1] * (double)dims[2] > 2147483646.0) ? 1 : 0;
}

/* The all-cell checker: the first cell, in index order, for which one call of move_kernel
 * (direction chosen, as its first call) ends with MOVE_DONE at point p, i.e. whose closed
 * square [ll, ll + cell_width]^2 holds p by the kernel's own differences. */
static int32_t adv_first_cell(const double* p, int32_t n_cells, const double* c_pos_ll, double cell_width,
                              const double* extents) {
    static const int32_t dummy_c2c[4] = {0, 0, 0, 0};
    for (int32_t c = 0; c < n_cells; c++) {
        int32_t mdir[2] = {1, 1}, next = c;
        if (move_once(1, p, mdir, c_pos_ll + 2 * (int64_t)c, dummy_c2c, &next, cell_width, extents) == kDone)
            return c;
    }
    return ADV_REMOVED;
}

/* generateStructuredMesh for one box on one unpartitioned mesh (global cell id = index):
 * step 1 the box centroid (getCentroidOfBox for dim 2, the upper bound as in
 * ASSIGN_CENTROID_TO_DIM, opp_defs.h:121-127), nudged by h/100 along x, then y while no cell
 * holds it (the z nudge that follows leaves x and y, all the checker reads, as they are, so
 * it finds nothing new); step 3 the lowest cell holding one of the box's 4 corners, each
 * clamped to the upper bound (GET_VERT, opp_defs.h:115). */
static int32_t adv_dh_box(int32_t n_cells, const double* c_pos_ll, double cell_width, const double* extents,
                          const double* box, double spacing, const int64_t* dims, int64_t index) {
    const double* mn = box;
    const double* mx = box + 3;
    const int64_t ix = index % dims[0], iy = index / dims[0];
    const double corner[2] = {mn[0] + (double)ix * spacing, mn[1] + (double)iy * spacing};
    double c[2];
    for (int d = 0; d < 2; d++)
        c[d] = (corner[d] + spacing <= mx[d]) ? corner[d] + spacing * 0.5 : (corner[d] + mx[d]) * 0.5;
    int32_t cid = adv_first_cell(c, n_cells, c_pos_ll, cell_width, extents);
    for (int d = 0; d < 2 && cid == ADV_REMOVED; d++) {
        c[d] += spacing / 100.0;
        cid = adv_first_cell(c, n_cells, c_pos_ll, cell_width, extents);
    }
    if (cid == ADV_REMOVED) {
        for (int k = 0; k < 4; k++) {
            double v[2];
            for (int d = 0; d < 2; d++) {
                const double t = ((k >> d) & 1) ? corner[d] + spacing : corner[d];
                v[d] = (t > mx[d]) ? mx[d] : t;
            }
            const int32_t f = adv_first_cell(v, n_cells, c_pos_ll, cell_width, extents);
            if (f < cid) cid = f;
        }
    }
    return cid;
}

void oracle_advec_dh_build(int32_t n_cells, const double* c_pos_ll, double cell_width, const double* extents,
                           const double* box, double spacing, const int64_t* dims, int32_t* map) {
    const int64_t size = dims[0] * dims[1];
    for (int64_t index = 0; index < size; index++)
        map[index] = adv_dh_box(n_cells, c_pos_ll, cell_width, extents, box, spacing, dims, index);
}

/* Truncation of a box coordinate as the CUDA backend's (size_t) cast runs on the device
 * (round toward zero, saturating: negative and NaN give 0). */
static uint64_t adv_dh_index(double t) {
    if (!(t > 0.0)) return 0;
    if (t >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)t;
}

/* The pre-pass over [0,n): p2c = the cell of the box holding the position, or REMOVED outside
 * the grid or in a box without a cell.  Particles at REMOVED stay there.  Returns the number
 * of particles it removed. */
int32_t oracle_advec_dh_seed(int32_t n, const double* pos, int32_t* p2c, const double* box_min, double inv,
                             const int64_t* dims, const int32_t* map) {
    int32_t removed = 0;
    for (int32_t i = 0; i < n; i++) {
        if (p2c[i] == ADV_REMOVED) continue;
        const uint64_t ix = adv_dh_index((pos[2 * (int64_t)i] - box_min[0]) * inv);
        const uint64_t iy = adv_dh_index((pos[2 * (int64_t)i + 1] - box_min[1]) * inv);
        const int out = ix >= (uint64_t)dims[0] || iy >= (uint64_t)dims[1];
        const int32_t cell = out ? ADV_REMOVED : map[ix + (uint64_t)dims[0] * iy];
        p2c[i] = cell;
        if (cell == ADV_REMOVED) removed++;
    }
    return removed;
}

/* The move loop alone (opp_particle_move__move_kernel over [0,n)): the pre-pass when dh_map is
 * not NULL (dh_box_min, dh_inv, dh_dims: the grid), then every particle's walk; particles at
 * REMOVED are skipped, as the move loop skips them.  Returns 0, or -1 if a particle exceeded
 * max_hops; adds the move calls to *visits and the particles the pre-pass removed to *removed. */
int oracle_advec_move_dh(int32_t n, const double* pos, int32_t* mdir, int32_t* p2c, const int32_t* c2c,
                         const double* c_pos_ll, const double* extents, double cell_width, int32_t max_hops,
                         const int32_t* dh_map, const double* dh_box_min, double dh_inv, const int64_t* dh_dims,
                         int64_t* visits, int64_t* removed) {
    if (dh_map) *removed += oracle_advec_dh_seed(n, pos, p2c, dh_box_min, dh_inv, dh_dims, dh_map);
    for (int32_t p = 0; p < n; p++) {
        int32_t c = p2c[p];
        if (c == ADV_REMOVED) continue;
        int first = 1, calls = 0;
        for (;;) {
            const int st = move_once(first, pos + 2 * (int64_t)p, mdir + 2 * (int64_t)p, c_pos_ll + 2 * (int64_t)c,
                                     c2c + 4 * (int64_t)c, &c, cell_width, extents);
            first = 0;
            calls++;
            if (st == kDone) break;
            if (calls >= max_hops) {
                *visits += calls;
                return -1;
            }
        }
        p2c[p] = c;
        *visits += calls;
    }
    return 0;
}

/* `steps` iterations of the generated main loop (advec_opp.cpp): update_pos over all particles,
 * then the move loop (oracle_advec_move_dh).  Returns 0, or -1 if a particle exceeded
 * max_hops; *visits_out = move calls in the last step, *removed_out (may be NULL) = particles
 * the pre-pass removed over all steps. */
int oracle_advec_steps_dh(int32_t n, double* pos, const double* vel, int32_t* mdir, int32_t* p2c, const int32_t* c2c,
                          const double* c_pos_ll, double dt, const double* extents, double cell_width, int32_t steps,
                          int32_t max_hops, const int32_t* dh_map, const double* dh_box_min, double dh_inv,
                          const int64_t* dh_dims, int64_t* visits_out, int64_t* removed_out) {
    int64_t visits = 0, removed = 0;
    int rc = 0;
    for (int32_t s = 0; s < steps && rc == 0; s++) {
        for (int32_t p = 0; p < n; p++) update_pos(vel + 2 * (int64_t)p, pos + 2 * (int64_t)p, dt, extents);
        visits = 0;
        rc = oracle_advec_move_dh(n, pos, mdir, p2c, c2c, c_pos_ll, extents, cell_width, max_hops, dh_map, dh_box_min,
                                  dh_inv, dh_dims, &visits, &removed);
    }
    *visits_out = visits;
    if (removed_out) *removed_out = removed;
    return rc;
}

/* `steps` iterations of the generated main loop without the direct hop. */
int oracle_advec_steps(int32_t n, double* pos, const double* vel, int32_t* mdir, int32_t* p2c, const int32_t* c2c,
                       const double* c_pos_ll, double dt, const double* extents, double cell_width, int32_t steps,
                       int32_t max_hops, int64_t* visits_out) {
    return oracle_advec_steps_dh(n, pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, steps, max_hops,
                                 NULL, NULL, 0.0, NULL, visits_out, NULL);
}
