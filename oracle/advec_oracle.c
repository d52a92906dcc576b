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

/* `steps` iterations of the generated main loop (advec_opp.cpp): update_pos over all particles,
 * then the move over all particles.  Returns 0, or -1 if a particle exceeded max_hops;
 * *visits_out = move calls in the last step. */
int oracle_advec_steps(int32_t n, double* pos, const double* vel, int32_t* mdir, int32_t* p2c, const int32_t* c2c,
                       const double* c_pos_ll, double dt, const double* extents, double cell_width, int32_t steps,
                       int32_t max_hops, int64_t* visits_out) {
    int64_t visits = 0;
    for (int32_t s = 0; s < steps; s++) {
        for (int32_t p = 0; p < n; p++) update_pos(vel + 2 * (int64_t)p, pos + 2 * (int64_t)p, dt, extents);
        visits = 0;
        for (int32_t p = 0; p < n; p++) {
            int32_t c = p2c[p];
            int first = 1, calls = 0;
            for (;;) {
                const int st = move_once(first, pos + 2 * (int64_t)p, mdir + 2 * (int64_t)p,
                                         c_pos_ll + 2 * (int64_t)c, c2c + 4 * (int64_t)c, &c, cell_width, extents);
                first = 0;
                calls++;
                if (st == kDone) break;
                if (calls >= max_hops) {
                    *visits_out = visits + calls;
                    return -1;
                }
            }
            p2c[p] = c;
            visits += calls;
        }
    }
    *visits_out = visits;
    return 0;
}
