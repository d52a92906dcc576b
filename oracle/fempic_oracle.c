/*
 * fempic_oracle.c — TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C, single-threaded restatement of the OP-PIC seq backend for the FemPIC
 * particle hot path, in the seq backend's host layout (AoS: pos[n*3], lc[n*4],
 * c_det[c*16], c2c[c*4], c2n[c*4]).  It is what the CUDA kernels are checked
 * against; nothing in the product links or calls it.  Compiled with
 * -ffp-contract=off so each product and sum is rounded on its own, exactly as the
 * reference's scalar expressions are written.  Its agreement with the reference
 * itself is pinned by the compiled reference seq backend (oracle/ref_harness.cpp).
 *
 * Reference paths are relative to the OP-PIC source tree.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_REMOVED 2147483647 /* MAX_CELL_INDEX, opp_lib/include/opp_defs.h:150 */
#define ORACLE_TOL 1e-10          /* KERNEL_TOLERENCE, apps/app_fempic/kernels.h:44 */

enum { MOVE_DONE = 0, NEED_MOVE = 1, NEED_REMOVE = 2 }; /* opp_defs.h:197-202 */

/*
 * move_kernel of apps/app_fempic/kernels.h:106-161 (generated seq twin
 * apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:7-62) for one cell visit.
 * Writes lc[0..3]; returns the move status and, for NEED_MOVE, the next cell.
 */
static int move_visit(const double* x, double* lc, double volume, const double* det,
                      const int32_t* c2c_row, int32_t* p2c) {
    const double coefficient2 = (1.0 / 6.0) / volume;
    for (int i = 0; i < 4; i++) {
        lc[i] = coefficient2 * (det[i * 4 + 0] - det[i * 4 + 1] * x[0] + det[i * 4 + 2] * x[1] -
                                det[i * 4 + 3] * x[2]);
    }
    if ((lc[0] > (-1) * ORACLE_TOL) && ((lc[0] - 1.0) < ORACLE_TOL) &&
        (lc[1] > (-1) * ORACLE_TOL) && ((lc[1] - 1.0) < ORACLE_TOL) &&
        (lc[2] > (-1) * ORACLE_TOL) && ((lc[2] - 1.0) < ORACLE_TOL) &&
        (lc[3] > (-1) * ORACLE_TOL) && ((lc[3] - 1.0) < ORACLE_TOL)) {
        return MOVE_DONE;
    }
    int min_i = 0;
    double min_lc = lc[0];
    for (int i = 1; i < 4; i++) {
        if (lc[i] < min_lc) {
            min_lc = lc[i];
            min_i = i;
        }
    }
    if (c2c_row[min_i] >= 0) {
        *p2c = c2c_row[min_i];
        return NEED_MOVE;
    }
    *p2c = ORACLE_REMOVED;
    return NEED_REMOVE;
}

/*
 * Hop driver of opp_particle_move__move_kernel (seq loop
 * apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:88-110,141-146) with the
 * status rule of opp_check_part_move_status (opp_lib/include/opp_seq.h:68-86):
 * particles already at the removed cell are skipped; NEED_REMOVE counts a removal.
 * max_hops bounds the visits per particle (the reference loop is unbounded): on
 * hitting it the particle keeps its current cell and -1 is returned.
 * visits (may be NULL) receives the cell visits of each particle.
 * Returns the total number of cell visits.
 */
int64_t oracle_move(int32_t n, const double* pos, double* lc, int32_t* p2c, const int32_t* c2c,
                    const double* c_volume, const double* c_det, int32_t max_hops,
                    int32_t* remove_count, int32_t* visits) {
    int64_t total = 0;
    int32_t removed = 0;
    int failed = 0;
    for (int32_t i = 0; i < n; i++) {
        int32_t* cell = p2c + i;
        if (visits) visits[i] = 0;
        if (cell[0] == ORACLE_REMOVED) continue;
        int status;
        int32_t hops = 0;
        do {
            const int32_t c = cell[0];
            status = move_visit(pos + (int64_t)i * 3, lc + (int64_t)i * 4, c_volume[c],
                                c_det + (int64_t)c * 16, c2c + (int64_t)c * 4, cell);
            hops++;
            if (status == NEED_MOVE && hops >= max_hops) {
                failed = 1;
                break;
            }
        } while (status == NEED_MOVE);
        if (status == NEED_REMOVE) removed++;
        if (visits) visits[i] = hops;
        total += hops;
    }
    *remove_count = removed;
    return failed ? -1 : total;
}

/*
 * deposit_charge_on_nodes_kernel (apps/app_fempic/kernels.h:164-175) over [0,n) in
 * index order, as the seq loop does
 * (apps_codegen/app_fempic_cg/seq/deposit_charge_on_nodes_kernel_loop.hpp:40-58).
 */
void oracle_deposit(int32_t n, const double* lc, const int32_t* p2c, const int32_t* c2n,
                    double* node_charge) {
    for (int32_t i = 0; i < n; i++) {
        const int32_t* map0 = c2n + (int64_t)p2c[i] * 4;
        node_charge[map0[0]] += lc[(int64_t)i * 4 + 0];
        node_charge[map0[1]] += lc[(int64_t)i * 4 + 1];
        node_charge[map0[2]] += lc[(int64_t)i * 4 + 2];
        node_charge[map0[3]] += lc[(int64_t)i * 4 + 3];
    }
}

/* calculate_new_pos_vel_kernel (apps/app_fempic/kernels.h:93-103) over [0,n). */
void oracle_push(int32_t n, const int32_t* p2c, const double* c_ef, double* pos, double* vel,
                 double qm, double dt) {
    const double coefficient1 = qm * dt;
    for (int32_t p = 0; p < n; p++) {
        const double* ef = c_ef + (int64_t)p2c[p] * 3;
        for (int i = 0; i < 3; i++) {
            vel[(int64_t)p * 3 + i] += (coefficient1 * ef[i]);
            pos[(int64_t)p * 3 + i] += vel[(int64_t)p * 3 + i] * dt;
        }
    }
}

/* The mixed-precision push: FP32 increments on FP64 state (dv = f32(qm*dt)*f32(E),
 * v += dv; dx = f32(v)*f32(dt), x += dx). */
void oracle_push_mixed(int32_t n, const int32_t* p2c, const double* c_ef, double* pos, double* vel,
                       double qm, double dt) {
    const float coefficient1 = (float)(qm * dt);
    const float dtf = (float)dt;
    for (int32_t p = 0; p < n; p++) {
        const double* ef = c_ef + (int64_t)p2c[p] * 3;
        for (int i = 0; i < 3; i++) {
            const float dv = coefficient1 * (float)ef[i];
            const double v = vel[(int64_t)p * 3 + i] + (double)dv;
            vel[(int64_t)p * 3 + i] = v;
            const float dx = (float)v * dtf;
            pos[(int64_t)p * 3 + i] += (double)dx;
        }
    }
}

/*
 * Injection of `count` particles at slots [start, start+count):
 *  - face of the k-th injected particle by the seq rule of
 *    opp_inc_part_count_with_distribution_core
 *    (opp_lib/src/core/opp_increase_part_count_core.cpp:134-142);
 *  - inject_ions_kernel (apps/app_fempic/kernels.h:63-90) with rnd row k = (a, b, ...)
 *    as dummy_part_random, followed by the thermal velocity rnd[k][2..4].
 * rnd is AoS [count][5].
 */
void oracle_inject(int32_t start, int32_t count, const int32_t* dist, const int32_t* if2c,
                   const double* if_u, const double* if_v, const double* if_norm,
                   const double* if_n_pos, const double* c_ef, const double* rnd,
                   double ion_velocity, double qm, double dt, double* pos, double* vel,
                   int32_t* p2c) {
    int32_t j = 0;
    for (int32_t k = 0; k < count; k++) {
        if (k >= dist[j]) j++;
        p2c[start + k] = j;
    }
    for (int32_t k = 0; k < count; k++) {
        const int64_t p = (int64_t)start + k;
        const int32_t face = p2c[p];
        const int32_t cell = if2c[face];
        const double* ef = c_ef + (int64_t)cell * 3;
        double a = rnd[(int64_t)k * 5 + 0];
        double b = rnd[(int64_t)k * 5 + 1];
        if ((a + b) > 1) {
            a = (1 - a);
            b = (1 - b);
        }
        for (int i = 0; i < 3; i++) {
            pos[p * 3 + i] = a * if_u[face * 3 + i] + b * if_v[face * 3 + i] + if_n_pos[face * 9 + i];
            vel[p * 3 + i] = (if_norm[face * 3 + i] * ion_velocity);
            vel[p * 3 + i] -= qm * ef[i] * (0.5 * dt);
            vel[p * 3 + i] += rnd[(int64_t)k * 5 + 2 + i];
        }
        p2c[p] = cell;
    }
}

/*
 * particle_hole_fill_core (opp_lib/src/core/opp_particle_organize_core.cpp:124-218):
 * ascending holes j (p2c == removed) are filled from the last live particle walking
 * down, stopping when that index is at or before j or remove_count holes are filled.
 * dats[d] is an AoS array of dat_bytes[d] bytes per particle.  Returns pairs moved.
 */
int32_t oracle_hole_fill(int32_t size, int32_t remove_count, const int32_t* p2c, int32_t n_dats,
                         char** dats, const int32_t* dat_bytes, int32_t* pair_from, int32_t* pair_to) {
    int32_t removed_count = 0;
    int32_t back_index = size - 1;
    int32_t n_pairs = 0;
    for (int32_t j = 0; j < size; j++) {
        if (p2c[j] != ORACLE_REMOVED) continue;
        while (back_index >= 0 && p2c[back_index] == ORACLE_REMOVED) back_index--;
        if (back_index <= j || removed_count >= remove_count) break;
        pair_to[n_pairs] = j;
        pair_from[n_pairs] = back_index;
        n_pairs++;
        back_index--;
        removed_count++;
    }
    for (int32_t d = 0; d < n_dats; d++) {
        for (int32_t k = 0; k < n_pairs; k++) {
            memcpy(dats[d] + (int64_t)pair_to[k] * dat_bytes[d],
                   dats[d] + (int64_t)pair_from[k] * dat_bytes[d], (size_t)dat_bytes[d]);
        }
    }
    return n_pairs;
}

/* FNV-1a 64 of n bytes: the digest the reference harness records per step. */
uint64_t oracle_fnv1a(const void* p, int64_t n) {
    const unsigned char* b = (const unsigned char*)p;
    uint64_t h = 1469598103934665603ull;
    for (int64_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

/*
 * opp_particle_sort_core (opp_lib/src/core/opp_particle_organize_core.cpp:98-121):
 * permutation = sort_iota_by_key(p2c, size) (opp_lib/include/opp_util.h:211-221) taken
 * STABLE (ties keep index order), then every dat gathered.  A counting sort over
 * keys in [0, n_cells] with the removed cell mapped to n_cells is that stable order.
 * perm (may be NULL) receives the source index of each destination slot.
 */
int oracle_sort(int32_t size, int32_t n_cells, int32_t n_dats, char** dats, const int32_t* dat_bytes,
                int32_t key_dat, int32_t* perm) {
    const int32_t* p2c = (const int32_t*)dats[key_dat];
    int64_t* count = (int64_t*)calloc((size_t)n_cells + 2, sizeof(int64_t));
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)(size > 0 ? size : 1));
    if (!count || !order) {
        free(count);
        free(order);
        return 1;
    }
    for (int32_t i = 0; i < size; i++) {
        const int32_t k = (p2c[i] == ORACLE_REMOVED) ? n_cells : p2c[i];
        count[k + 1]++;
    }
    for (int32_t k = 0; k <= n_cells; k++) count[k + 1] += count[k];
    for (int32_t i = 0; i < size; i++) {
        const int32_t k = (p2c[i] == ORACLE_REMOVED) ? n_cells : p2c[i];
        order[count[k]++] = i;
    }
    for (int32_t d = 0; d < n_dats; d++) {
        const int32_t b = dat_bytes[d];
        char* tmp = (char*)malloc((size_t)b * (size_t)(size > 0 ? size : 1));
        if (!tmp) {
            free(count);
            free(order);
            return 1;
        }
        for (int32_t j = 0; j < size; j++) memcpy(tmp + (int64_t)j * b, dats[d] + (int64_t)order[j] * b, (size_t)b);
        memcpy(dats[d], tmp, (size_t)b * (size_t)size);
        free(tmp);
    }
    if (perm) memcpy(perm, order, sizeof(int32_t) * (size_t)size);
    free(count);
    free(order);
    return 0;
}

/* ------------------------------------------------------------------ direct hop
 *
 * The structured cell mapper of the global move (opp_lib/include/opp_direct_hop_core.h,
 * seq build opp_lib/src/seq/opp_direct_hop_seq.cpp) and the global-move pre-pass of the
 * move loop (apps_codegen/app_fempic_cg/seq/move_kernel_loop.hpp:112-131).  box[6] =
 * {min x, y, z, max x, y, z}; the map is x fastest (index = x + X*y + X*Y*z).
 */

#define ORACLE_DBL_MAX 1.7976931348623157e308
#define ORACLE_DBL_MIN 2.2250738585072014e-308 /* MIN_REAL = numeric_limits<double>::min() */

/* BoundingBox(n_pos, 3, expansion) (opp_direct_hop_core.h:70-120; the x/y widening
 * reads expansion x for both minima and expansion y for both maxima, as written there)
 * and CellMapper::init_host's box counts (:317-380): 1 + the number of iterations of
 * `for (v = min; v < max; v += h)`.  Returns 0, or 1 for a grid above 2^31 boxes. */
int oracle_dh_grid_init(int32_t n_nodes, const double* n_pos, double spacing, const double* expansion,
                        double* box, int64_t* dims) {
    double mn[3] = {ORACLE_DBL_MAX, ORACLE_DBL_MAX, ORACLE_DBL_MAX};
    double mx[3] = {ORACLE_DBL_MIN, ORACLE_DBL_MIN, ORACLE_DBL_MIN};
    for (int32_t i = 0; i < n_nodes; i++)
        for (int d = 0; d < 3; d++) {
            const double v = n_pos[(int64_t)i * 3 + d];
            if (v < mn[d]) mn[d] = v;
            if (mx[d] < v) mx[d] = v;
        }
    mn[0] -= (expansion[0] + 1e-12); /* BOUND_OFFSET, opp_direct_hop_core.h:37 */
    mn[1] -= (expansion[0] + 1e-12);
    mx[0] += (expansion[1] - 1e-12);
    mx[1] += (expansion[1] - 1e-12);
    mn[2] -= (expansion[2] + 1e-12);
    mx[2] += (expansion[2] - 1e-12);
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

/* The checker of opp_init_direct_hop_cg (seq move_kernel_loop.hpp:170-198): the first cell,
 * in index order, for which move_kernel ends with MOVE_DONE at point x. */
static int32_t dh_first_cell(const double* x, int32_t n_cells, const double* c_volume, const double* c_det) {
    static const int32_t dummy_c2c[4] = {0, 0, 0, 0};
    double lc[4];
    for (int32_t c = 0; c < n_cells; c++) {
        int32_t next = c;
        if (move_visit(x, lc, c_volume[c], c_det + (int64_t)c * 16, dummy_c2c, &next) == MOVE_DONE) return c;
    }
    return ORACLE_REMOVED;
}

/* CellMapper::generateStructuredMesh (opp_direct_hop_seq.cpp:134-302) on one unpartitioned
 * mesh (global cell id = index): step 1 the box centroid (getCentroidOfBox, with the box's
 * upper bound as in ASSIGN_CENTROID_TO_DIM, opp_defs.h:121-127), nudged by h/100 along x,
 * then y, then z while no cell holds it; step 3 the lowest cell holding one of the box's
 * corners, each clamped to the upper bound (GET_VERT, opp_defs.h:115).  Search over all
 * cells per query, as the reference does. */
static int32_t dh_box(int32_t n_cells, const double* c_volume, const double* c_det, const double* box,
                      double spacing, const int64_t* dims, int64_t index) {
    const double* mn = box;
    const double* mx = box + 3;
    const int64_t dx = index % dims[0], dy = (index / dims[0]) % dims[1], dz = index / (dims[0] * dims[1]);
    const double corner[3] = {mn[0] + (double)dx * spacing, mn[1] + (double)dy * spacing,
                              mn[2] + (double)dz * spacing};
    double c[3];
    for (int d = 0; d < 3; d++)
        c[d] = (corner[d] + spacing <= mx[d]) ? corner[d] + spacing * 0.5 : (corner[d] + mx[d]) * 0.5;
    int32_t cid = dh_first_cell(c, n_cells, c_volume, c_det);
    for (int d = 0; d < 3 && cid == ORACLE_REMOVED; d++) {
        c[d] += spacing / 100.0;
        cid = dh_first_cell(c, n_cells, c_volume, c_det);
    }
    if (cid == ORACLE_REMOVED) {
        for (int k = 0; k < 8; k++) {
            double v[3];
            for (int d = 0; d < 3; d++) {
                const double t = ((k >> d) & 1) ? corner[d] + spacing : corner[d];
                v[d] = (t > mx[d]) ? mx[d] : t;
            }
            const int32_t f = dh_first_cell(v, n_cells, c_volume, c_det);
            if (f < cid) cid = f;
        }
    }
    return cid;
}

void oracle_dh_build(int32_t n_cells, const double* c_volume, const double* c_det, const double* box,
                     double spacing, const int64_t* dims, int32_t* map) {
    const int64_t size = dims[0] * dims[1] * dims[2];
    for (int64_t index = 0; index < size; index++)
        map[index] = dh_box(n_cells, c_volume, c_det, box, spacing, dims, index);
}

/* The map entries of the boxes idx[0..n) only (spot checks of large grids). */
void oracle_dh_boxes(int32_t n_cells, const double* c_volume, const double* c_det, const double* box,
                     double spacing, const int64_t* dims, int32_t n, const int64_t* idx, int32_t* out) {
    for (int32_t k = 0; k < n; k++) out[k] = dh_box(n_cells, c_volume, c_det, box, spacing, dims, idx[k]);
}

/* Truncation of the box index as the CUDA backend's (size_t) cast of a double runs on the
 * device (round toward zero, saturating: negative and NaN give 0). */
static uint64_t dh_index(double t) {
    if (!(t > 0.0)) return 0;
    if (t >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)t;
}

/* Global-move pre-pass over [0,n) (seq move_kernel_loop.hpp:112-131 with
 * findStructuredCellIndex3D, opp_direct_hop_core.h:410-429, and the CUDA rule for a
 * position outside the grid, opp_dev_findStructuredCellIndex3D / opp_dev_checkForGlobalMove
 * in opp_lib/include/device_kernels/cuda_inline_kernels.h): p2c = the box's cell, or
 * REMOVED outside the grid or in a box without a cell.  Particles at REMOVED stay there.
 * Returns the number of particles it removed. */
int32_t oracle_dh_seed(int32_t n, const double* pos, int32_t* p2c, const double* box_min, double inv,
                       const int64_t* dims, const int32_t* map) {
    int32_t removed = 0;
    for (int32_t i = 0; i < n; i++) {
        if (p2c[i] == ORACLE_REMOVED) continue;
        const double* x = pos + (int64_t)i * 3;
        uint64_t ix[3];
        int out = 0;
        for (int d = 0; d < 3; d++) {
            ix[d] = dh_index((x[d] - box_min[d]) * inv);
            if (ix[d] >= (uint64_t)dims[d]) out = 1;
        }
        const int32_t cell = out ? ORACLE_REMOVED
                                 : map[ix[0] + (uint64_t)dims[0] * (ix[1] + (uint64_t)dims[1] * ix[2])];
        p2c[i] = cell;
        if (cell == ORACLE_REMOVED) removed++;
    }
    return removed;
}
