/* TEST INFRASTRUCTURE ONLY — CPU restatement of OP-PIC's CabanaPIC particle hot path, the
 * checker of the CUDA kernel in op-pic_b200/csrc/cabana.cu.  Nothing in the product links it.
 *
 * Follows the generated seq backend of the electromagnetic PIC app:
 *   move_deposit_kernel                 apps/app_cabanapic/kernels.h:139-355
 *   weight_current_to_accumulator_kernel apps/app_cabanapic/kernels.h:109-136 (CALC_J :11-26)
 *   hop driver                          apps_codegen/app_cabanapic_cg/seq/move_deposit_kernel_loop.hpp
 *                                       (do/while with opp_check_part_move_status,
 *                                       opp_lib/include/opp_seq.h:64-86: OPP_DO_ONCE is true on
 *                                       the first call of a particle only)
 * Layouts are the seq backend's AoS: pos/vel/streak [n][3], weight [n], p2c [n],
 * c2ngc [n_cells][6] (faces xd, yd, zd, xu, yu, zu), interp [n_cells][18] (CellInterp order),
 * acc [n_cells][12] (jfx 0..3, jfy 0..3, jfz 0..3).
 *
 * Compiled with -ffp-contract=off: every expression is evaluated in the written order with
 * one rounding per operation, as the pinned reference build is.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

/* CALC_J(X,Y,Z) of kernels.h:11-26, then the four adds into acc[base..base+3]. */
static void calc_j(double* acc, double q, double u, double dy, double dz, double v5) {
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
    acc[0] += v0;
    acc[1] += v1;
    acc[2] += v2;
    acc[3] += v3;
}

/* weight_current_to_accumulator_kernel, kernels.h:109-136. */
static void weight_current(double* cell_acc, double q, double ux, double uy, double uz, double dx, double dy,
                           double dz) {
    const double v5 = q * ux * uy * uz * (1.0 / 3.0);
    calc_j(cell_acc + 0, q, ux, dy, dz, v5);  /* CALC_J(x,y,z) -> jfx */
    calc_j(cell_acc + 4, q, uy, dz, dx, v5);  /* CALC_J(y,z,x) -> jfy */
    calc_j(cell_acc + 8, q, uz, dx, dy, v5);  /* CALC_J(z,x,y) -> jfz */
}

enum { kDone = 0, kNeedMove = 1 };

/* The OPP_DO_ONCE push of move_deposit_kernel (apps/app_cabanapic/kernels.h:148-253) up to the
 * normalised displacement u * cdt_d / gamma, FP64; vel is updated. */
static void push_f64(const double* pos, double* vel, const double* interp, double qdt_2mc, const double* cdt_d,
                     double disp[3]) {
    const double ex = interp[0], dexdy = interp[1], dexdz = interp[2], d2exdydz = interp[3];
    const double ey = interp[4], deydz = interp[5], deydx = interp[6], d2eydzdx = interp[7];
    const double ez = interp[8], dezdx = interp[9], dezdy = interp[10], d2ezdxdy = interp[11];
    double cbx = interp[12];
    const double dcbxdx = interp[13];
    double cby = interp[14];
    const double dcbydy = interp[15];
    double cbz = interp[16];
    const double dcbzdz = interp[17];
    const double dx = pos[0], dy = pos[1], dz = pos[2];

    const double hax = qdt_2mc * ((ex + dy * dexdy) + dz * (dexdz + dy * d2exdydz));
    const double hay = qdt_2mc * ((ey + dz * deydz) + dx * (deydx + dz * d2eydzdx));
    const double haz = qdt_2mc * ((ez + dx * dezdx) + dy * (dezdy + dx * d2ezdxdy));
    cbx = cbx + dx * dcbxdx;
    cby = cby + dy * dcbydy;
    cbz = cbz + dz * dcbzdz;

    double ux = vel[0], uy = vel[1], uz = vel[2];
    ux += hax;
    uy += hay;
    uz += haz;
    double v0 = qdt_2mc / sqrt(1.0 + (ux * ux + (uy * uy + uz * uz)));
    double v1 = cbx * cbx + (cby * cby + cbz * cbz);
    double v2 = (v0 * v0) * v1;
    double v3 = v0 * (1.0 + v2 * ((1.0 / 3.0) + v2 * (2.0 / 15.0)));
    double v4 = v3 / (1.0 + v1 * (v3 * v3));
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
    vel[0] = ux;
    vel[1] = uy;
    vel[2] = uz;

    v0 = 1.0 / sqrt(1.0 + (ux * ux + (uy * uy + uz * uz)));
    ux *= cdt_d[0];
    uy *= cdt_d[1];
    uz *= cdt_d[2];
    ux *= v0;
    uy *= v0;
    uz *= v0;
    disp[0] = ux;
    disp[1] = uy;
    disp[2] = uz;
}

/* The same push with FP32 momentum (the FP32-momentum form the library also offers, not a
 * reference loop): the fields and the position rounded to FP32, the FP64 expression's
 * operations in FP32 (IEEE division and square root), FP32 momentum; the displacement is
 * returned in FP64. */
static void push_f32(const double* pos, float* vel, const double* interp, double qdt_2mc, const double* cdt_d,
                     double disp[3]) {
    float r[18];
    for (int k = 0; k < 18; k++) r[k] = (float)interp[k];
    const float ex = r[0], dexdy = r[1], dexdz = r[2], d2exdydz = r[3];
    const float ey = r[4], deydz = r[5], deydx = r[6], d2eydzdx = r[7];
    const float ez = r[8], dezdx = r[9], dezdy = r[10], d2ezdxdy = r[11];
    float cbx = r[12];
    const float dcbxdx = r[13];
    float cby = r[14];
    const float dcbydy = r[15];
    float cbz = r[16];
    const float dcbzdz = r[17];
    const float dx = (float)pos[0], dy = (float)pos[1], dz = (float)pos[2];
    const float q2 = (float)qdt_2mc;

    const float hax = q2 * ((ex + dy * dexdy) + dz * (dexdz + dy * d2exdydz));
    const float hay = q2 * ((ey + dz * deydz) + dx * (deydx + dz * d2eydzdx));
    const float haz = q2 * ((ez + dx * dezdx) + dy * (dezdy + dx * d2ezdxdy));
    cbx = cbx + dx * dcbxdx;
    cby = cby + dy * dcbydy;
    cbz = cbz + dz * dcbzdz;

    float ux = vel[0], uy = vel[1], uz = vel[2];
    ux += hax;
    uy += hay;
    uz += haz;
    float v0 = q2 / sqrtf(1.0f + (ux * ux + (uy * uy + uz * uz)));
    float v1 = cbx * cbx + (cby * cby + cbz * cbz);
    float v2 = (v0 * v0) * v1;
    const float v3 = v0 * (1.0f + v2 * ((1.0f / 3.0f) + v2 * (2.0f / 15.0f)));
    float v4 = v3 / (1.0f + v1 * (v3 * v3));
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
    vel[0] = ux;
    vel[1] = uy;
    vel[2] = uz;

    v0 = 1.0f / sqrtf(1.0f + (ux * ux + (uy * uy + uz * uz)));
    ux *= (float)cdt_d[0];
    uy *= (float)cdt_d[1];
    uz *= (float)cdt_d[2];
    ux *= v0;
    uy *= v0;
    uz *= v0;
    disp[0] = ux;
    disp[1] = uy;
    disp[2] = uz;
}

/* One call of move_deposit_kernel for particle p in cell c; returns kDone or kNeedMove
 * (then *c is the next cell).  disp: the push's displacement on the first call (OPP_DO_ONCE),
 * NULL on the later calls. */
static int move_deposit_once(const double* disp, double* pos, double* streak, double weight, double* cell_acc,
                             const int32_t* c2f, int32_t* c, double qsp) {
    if (disp) {
        const double ux = disp[0], uy = disp[1], uz = disp[2];
        const double dx = pos[0], dy = pos[1], dz = pos[2];
        const double v0 = dx + ux;
        const double v1 = dy + uy;
        const double v2 = dz + uz;
        const double v3 = v0 + ux;
        const double v4 = v1 + uy;
        const double v5 = v2 + uz;
        if (v3 <= 1.0 && v4 <= 1.0 && v5 <= 1.0 && -v3 <= 1.0 && -v4 <= 1.0 && -v5 <= 1.0) {
            pos[0] = v3;
            pos[1] = v4;
            pos[2] = v5;
            weight_current(cell_acc, weight * qsp, ux, uy, uz, v0, v1, v2);
            return kDone;
        }
        streak[0] = ux;
        streak[1] = uy;
        streak[2] = uz;
    }
    double s_midx = pos[0], s_midy = pos[1], s_midz = pos[2];
    double s_dispx = streak[0], s_dispy = streak[1], s_dispz = streak[2];
    const double s_dir[3] = {(s_dispx > 0) ? 1.0 : -1.0, (s_dispy > 0) ? 1.0 : -1.0, (s_dispz > 0) ? 1.0 : -1.0};
    const double v0 = (s_dispx == 0) ? 3.4e38 : (s_dir[0] - s_midx) / s_dispx;
    const double v1 = (s_dispy == 0) ? 3.4e38 : (s_dir[1] - s_midy) / s_dispy;
    const double v2 = (s_dispz == 0) ? 3.4e38 : (s_dir[2] - s_midz) / s_dispz;
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
    weight_current(cell_acc, weight * qsp, s_dispx, s_dispy, s_dispz, s_midx, s_midy, s_midz);
    streak[0] -= s_dispx;
    streak[1] -= s_dispy;
    streak[2] -= s_dispz;
    pos[0] += (s_dispx + s_dispx);
    pos[1] += (s_dispy + s_dispy);
    pos[2] += (s_dispz + s_dispz);
    if (axis != 3) {
        const double d = s_dir[axis];
        pos[axis] = d;
        const int face = axis + (d > 0 ? 3 : 0);
        *c = c2f[face];
        pos[axis] = -d;
        return kNeedMove;
    }
    return kDone;
}

/* The generated seq move loop over particles [0, n): returns the total number of kernel
 * calls (hops + 1 per particle) in *visits_out; -1 if a particle exceeded max_hops.
 * vel32 = NULL: FP64 momentum in vel (the reference's form); else FP32 momentum in vel32. */
static int move_deposit_all(int32_t n, double* pos, double* vel, float* vel32, double* streak, const double* weight,
                            int32_t* p2c, const int32_t* c2ngc, const double* interp, double* acc, double qdt_2mc,
                            const double* cdt_d, double qsp, int32_t max_hops, int64_t* visits_out) {
    int64_t visits = 0;
    for (int32_t p = 0; p < n; p++) {
        int32_t c = p2c[p];
        int calls = 0;
        double disp[3];
        double* pp = pos + 3 * (int64_t)p;
        if (vel32)
            push_f32(pp, vel32 + 3 * (int64_t)p, interp + 18 * (int64_t)c, qdt_2mc, cdt_d, disp);
        else
            push_f64(pp, vel + 3 * (int64_t)p, interp + 18 * (int64_t)c, qdt_2mc, cdt_d, disp);
        for (;;) {
            const int st = move_deposit_once(calls == 0 ? disp : NULL, pp, streak + 3 * (int64_t)p, weight[p],
                                             acc + 12 * (int64_t)c, c2ngc + 6 * (int64_t)c, &c, qsp);
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
    *visits_out = visits;
    return 0;
}

int oracle_cabana_move_deposit(int32_t n, double* pos, double* vel, double* streak, const double* weight,
                               int32_t* p2c, const int32_t* c2ngc, const double* interp, double* acc,
                               double qdt_2mc, const double* cdt_d, double qsp, int32_t max_hops,
                               int64_t* visits_out) {
    return move_deposit_all(n, pos, vel, NULL, streak, weight, p2c, c2ngc, interp, acc, qdt_2mc, cdt_d, qsp,
                            max_hops, visits_out);
}

/* The FP32-momentum form: vel32 [n][3] FP32. */
int oracle_cabana_move_deposit_mixed(int32_t n, double* pos, float* vel32, double* streak, const double* weight,
                                     int32_t* p2c, const int32_t* c2ngc, const double* interp, double* acc,
                                     double qdt_2mc, const double* cdt_d, double qsp, int32_t max_hops,
                                     int64_t* visits_out) {
    return move_deposit_all(n, pos, NULL, vel32, streak, weight, p2c, c2ngc, interp, acc, qdt_2mc, cdt_d, qsp,
                            max_hops, visits_out);
}
