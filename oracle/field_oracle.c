/*
 * field_oracle.c — TEST INFRASTRUCTURE ONLY (the parity oracle of the FemPIC field phase).
 *
 * Plain-C, single-threaded restatement of FemPIC's node-side loops and field solve:
 *   - compute_node_charge_density_kernel, compute_electric_field_kernel
 *     (apps/app_fempic/kernels.h:178-202): pinned to the reference's generated seq loops
 *     by oracle/field_ref_harness.cpp;
 *   - FESolver's set-up and compute_phi
 *     (apps_codegen/app_fempic_cg/field_solver/{field_solver,host}.cpp): the reference
 *     solves J Y = B with PETSc's KSPCG, which is absent here, so the solve is parity
 *     unpinned; this restatement uses Jacobi-preconditioned CG with the same stopping
 *     rule as the library, and its set-up (equation map, detJ, shape derivatives, K, F0)
 *     follows the reference's loops in their operation order.
 * Compiled with -ffp-contract=off.  Reference paths are relative to the OP-PIC tree.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FO_NODE_NORMAL 0
#define FO_NODE_OPEN 1
#define FO_SCALING 100.0 /* SCALLING, field_solver.cpp:21 */

/* compute_node_charge_density_kernel (kernels.h:178-183) over [0, n). */
void oracle_node_charge_density(int32_t n, double* den, const double* vol, double spwt) {
    for (int32_t i = 0; i < n; i++) den[i] *= (spwt / vol[i]);
}

/* opp_reset_dat(c_ef) then compute_electric_field_kernel (kernels.h:186-202) over the cells;
 * c_sd [nc][4][3], c2n [nc][4], ef [nc][3]. */
void oracle_electric_field(int32_t nc, const int32_t* c2n, const double* c_sd, const double* phi, double* ef) {
    for (int32_t c = 0; c < nc; c++) {
        const int32_t* n = c2n + (int64_t)c * 4;
        const double* sd = c_sd + (int64_t)c * 12;
        for (int dim = 0; dim < 3; dim++) {
            const double c1 = (sd[0 * 3 + dim] * phi[n[0]]);
            const double c2 = (sd[1 * 3 + dim] * phi[n[1]]);
            const double c3 = (sd[2 * 3 + dim] * phi[n[2]]);
            const double c4 = (sd[3 * 3 + dim] * phi[n[3]]);
            double e = 0.0;
            e -= (c1 + c2 + c3 + c4);
            ef[(int64_t)c * 3 + dim] = e;
        }
    }
}

static double fo_det3(double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

static void fo_inverse(double m[3][3], double v[3][3]) {
    const double a = m[0][0], b = m[0][1], c = m[0][2], d = m[1][0], e = m[1][1], f = m[1][2];
    const double g = m[2][0], h = m[2][1], i = m[2][2];
    v[0][0] = (e * i - f * h);
    v[1][0] = -(d * i - f * g);
    v[2][0] = (d * h - e * g);
    v[0][1] = -(b * i - c * h);
    v[1][1] = (a * i - c * g);
    v[2][1] = -(a * h - b * g);
    v[0][2] = (b * f - c * e);
    v[1][2] = -(a * f - c * d);
    v[2][2] = (a * e - b * d);
    const double det = a * v[0][0] + b * v[1][0] + c * v[2][0];
    double vmax = 0;
    for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) vmax = fabs(v[r][s]) > vmax ? fabs(v[r][s]) : vmax;
    double idet = 0;
    if (!(fabs(vmax) / fabs(det) > 1e12)) idet = 1 / det;
    for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) v[r][s] *= idet;
}

static int cmp_col(const void* x, const void* y) {
    const int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    return (a > b) - (a < b);
}

/* FESolver's set-up: calculate_neq / init_node_to_eq_map (field_solver.cpp:178-210),
 * compute_nx (:553-594), pre_assembly with add_ke / add_fe (:330-391, :501-551) and
 * enrich_cell_shape_deriv (:474-499).  node_to_eq [nn] (-1 for Dirichlet), det_j [nc],
 * c_sd [nc*12], f0 [nn] (first neq used); K as CSR (rowptr [nn+1], col/val with room for
 * 16*nc entries).  Returns neq, or -1 on a bad node index. */
int32_t oracle_field_setup(int32_t nn, int32_t nc, const double* n_pos, const int32_t* n_type,
                           const double* n_bnd_pot, const int32_t* c2n, int32_t* node_to_eq, double* det_j,
                           double* c_sd, double* f0, int64_t* rowptr, int32_t* col, double* val,
                           int64_t* nnz_out) {
    int32_t neq = 0;
    for (int32_t n = 0; n < nn; n++)
        node_to_eq[n] = (n_type[n] == FO_NODE_NORMAL || n_type[n] == FO_NODE_OPEN) ? neq++ : -1;
    /* Per-row lists in arrival order: at most 16 entries per cell over all rows. */
    int32_t* cnt = calloc((size_t)neq + 1, sizeof(int32_t));
    for (int64_t e = 0; e < nc; e++)
        for (int a = 0; a < 4; a++) {
            const int32_t nd = c2n[e * 4 + a];
            if (nd < 0 || nd >= nn) {
                free(cnt);
                return -1;
            }
            if (node_to_eq[nd] >= 0) cnt[node_to_eq[nd]] += 4;
        }
    int64_t* start = calloc((size_t)neq + 1, sizeof(int64_t));
    for (int32_t r = 0; r < neq; r++) start[r + 1] = start[r] + cnt[r];
    int32_t* rc = malloc(sizeof(int32_t) * (size_t)(start[neq] ? start[neq] : 1));
    double* rv = malloc(sizeof(double) * (size_t)(start[neq] ? start[neq] : 1));
    int32_t* len = calloc((size_t)neq + 1, sizeof(int32_t));
    for (int32_t r = 0; r < neq; r++) f0[r] = 0.0;
    static const double na_xi[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    for (int64_t e = 0; e < nc; e++) {
        const int32_t* con = c2n + e * 4;
        double x_xi[3][3], xi_x[3][3], nx[4][3], ke[4][4];
        for (int dim = 0; dim < 3; dim++)
            for (int j = 0; j < 3; j++) {
                x_xi[dim][j] = 0;
                for (int a = 0; a < 4; a++) x_xi[dim][j] += (na_xi[a][j] * n_pos[(int64_t)con[a] * 3 + dim]);
            }
        det_j[e] = fo_det3(x_xi);
        fo_inverse(x_xi, xi_x);
        for (int a = 0; a < 4; a++)
            for (int d = 0; d < 3; d++) {
                nx[a][d] = 0.0;
                for (int k = 0; k < 3; k++) nx[a][d] += (na_xi[a][k] * xi_x[k][d] * FO_SCALING);
                c_sd[e * 12 + a * 3 + d] = (nx[a][d] / FO_SCALING);
            }
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                ke[a][b] = 0.0;
                for (int k = 0; k < 2; k++)
                    for (int j = 0; j < 2; j++)
                        for (int i = 0; i < 2; i++) {
                            double dot = 0.0;
                            for (int d = 0; d < 3; d++) dot += (nx[a][d] * nx[b][d]);
                            ke[a][b] += (dot * det_j[e] * 1.0 * 1.0 * 1.0);
                        }
            }
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                const int32_t p = node_to_eq[con[a]];
                if (p < 0) continue;
                const int32_t q = node_to_eq[con[b]];
                if (q < 0) continue;
                int32_t k = 0;
                while (k < len[p] && rc[start[p] + k] != q) k++;
                if (k == len[p]) {
                    rc[start[p] + k] = q;
                    rv[start[p] + k] = ke[a][b];
                    len[p]++;
                } else {
                    rv[start[p] + k] += ke[a][b];
                }
            }
        for (int a = 0; a < 4; a++) {
            double fh = 0, fg = 0;
            for (int b = 0; b < 4; b++) fg -= (ke[a][b] * n_bnd_pot[con[b]]);
            const int32_t p = node_to_eq[con[a]];
            if (p >= 0) f0[p] += (fh + fg);
        }
    }
    const double scalar2 = 1.0 / (FO_SCALING * FO_SCALING);
    int64_t at = 0;
    for (int32_t r = 0; r < neq; r++) {
        /* sort (col, val) pairs of the row by column: sort an index permutation */
        int32_t n = len[r];
        int32_t* key = malloc(sizeof(int32_t) * 2 * (size_t)(n ? n : 1));
        for (int32_t k = 0; k < n; k++) {
            key[2 * k] = rc[start[r] + k];
            key[2 * k + 1] = k;
        }
        qsort(key, (size_t)n, 2 * sizeof(int32_t), cmp_col);
        rowptr[r] = at;
        for (int32_t k = 0; k < n; k++) {
            col[at] = key[2 * k];
            val[at] = rv[start[r] + key[2 * k + 1]] * scalar2;
            at++;
        }
        free(key);
    }
    rowptr[neq] = at;
    for (int32_t r = 0; r < neq; r++) f0[r] *= scalar2;
    *nnz_out = at;
    free(cnt);
    free(start);
    free(rc);
    free(rv);
    free(len);
    return neq;
}

/* Shape function a at Gauss point (i, j, k) (host.cpp evaluate_na with l = -+sqrt(1/3)). */
static double fo_na(int a, int i, int j, int k) {
    const double l[2] = {-sqrt(1.0 / 3.0), sqrt(1.0 / 3.0)};
    switch (a) {
        case 0: return 0.5 * (l[i] + 1);
        case 1: return 0.5 * (l[j] + 1);
        case 2: return 0.5 * (l[k] + 1);
        default: return 1 - 0.5 * (l[i] + 1) - 0.5 * (l[j] + 1) - 0.5 * (l[k] + 1);
    }
}

/* FESolver::compute_phi (field_solver.cpp:115-176 with host.cpp's init_f1_and_J,
 * build_f1_vector, build_j_matrix, compute_node_potential): d [neq] and f1 [neq] are the
 * Newton state and the accumulated F1 (updated in place), potential [nn] the result.  The
 * linear step is Jacobi-preconditioned CG from Y = 0, stopped when ||r|| <= max(rtol ||B||,
 * atol) or after max_iter iterations.  Returns the iterations; *resid = ||r|| / ||B||. */
int32_t oracle_field_solve(int32_t nn, int32_t nc, int32_t neq, const int32_t* node_to_eq, const int32_t* c2n,
                           const double* det_j, const double* n_bnd_pot, const int64_t* rowptr,
                           const int32_t* col, const double* val, const double* f0, double* d, double* f1,
                           const double* ion_den, double n0, double phi0, double kte, double qe, double eps0,
                           double rtol, double atol, int32_t max_iter, double* potential, double* resid) {
    const size_t m = (size_t)(neq > 0 ? neq : 1);
    double* t1 = calloc(m, sizeof(double));
    double* t2 = calloc(m, sizeof(double));
    double* t3 = calloc(m, sizeof(double));
    double* b = calloc(m, sizeof(double));
    double* dg = calloc(m, sizeof(double));
    double* x = calloc(m, sizeof(double));
    double* r = calloc(m, sizeof(double));
    double* p = calloc(m, sizeof(double));
    double* q = calloc(m, sizeof(double));
    for (int32_t n = 0; n < nn; n++) {
        const int32_t e = node_to_eq[n];
        if (e >= 0) t1[e] = (qe / eps0) * ((ion_den[n]) + n0 * exp((d[e] - phi0) / kte));
    }
    for (int32_t u = 0; u < neq; u++) {
        t2[u] = 0;
        t3[u] = -qe / eps0 * n0 * exp((d[u] - phi0) / kte) * (1 / kte);
    }
    for (int64_t c = 0; c < nc; c++)
        for (int a = 0; a < 4; a++) {
            const int32_t e = node_to_eq[c2n[c * 4 + a]];
            if (e < 0) continue;
            double ff1 = 0.0, ff3 = 0.0;
            for (int k = 0; k < 2; k++)
                for (int j = 0; j < 2; j++)
                    for (int i = 0; i < 2; i++) {
                        const double na = fo_na(a, i, j, k);
                        ff1 += (t1[e] * na * det_j[c] * 1.0 * 1.0 * 1.0);
                        ff3 += (t3[e] * na * det_j[c] * 1.0 * 1.0 * 1.0);
                    }
            ff1 *= (1.0 / 8.0);
            ff3 *= (1.0 / 8.0);
            f1[e] += ff1;
            t2[e] += ff3;
        }
    double bb = 0.0, rz = 0.0;
    for (int32_t u = 0; u < neq; u++) {
        double kd = 0.0, kuu = 0.0;
        for (int64_t k = rowptr[u]; k < rowptr[u + 1]; k++) {
            kd += val[k] * d[col[k]];
            if (col[k] == u) kuu = val[k];
        }
        b[u] = (kd - f0[u]) - f1[u];
        dg[u] = kuu + (-t2[u]);
        r[u] = b[u];
        p[u] = b[u] / dg[u];
        bb += b[u] * b[u];
        rz += b[u] * p[u];
    }
    const double bn = sqrt(bb);
    const double stop = fmax(rtol * bn, atol);
    double rr = bb;
    int32_t it = 0;
    while (it < max_iter && sqrt(rr) > stop) {
        double pq = 0.0;
        for (int32_t u = 0; u < neq; u++) {
            double s = 0.0;
            for (int64_t k = rowptr[u]; k < rowptr[u + 1]; k++) s += (col[k] == u ? dg[u] : val[k]) * p[col[k]];
            q[u] = s;
            pq += p[u] * s;
        }
        const double alpha = rz / pq;
        double rz2 = 0.0, rr2 = 0.0;
        for (int32_t u = 0; u < neq; u++) {
            x[u] += alpha * p[u];
            r[u] -= alpha * q[u];
            rz2 += r[u] * (r[u] / dg[u]);
            rr2 += r[u] * r[u];
        }
        const double beta = rz2 / rz;
        rz = rz2;
        rr = rr2;
        for (int32_t u = 0; u < neq; u++) p[u] = r[u] / dg[u] + beta * p[u];
        it++;
    }
    for (int32_t u = 0; u < neq; u++) d[u] = d[u] - x[u];
    for (int32_t n = 0; n < nn; n++) {
        potential[n] = n_bnd_pot[n];
        if (node_to_eq[n] >= 0) potential[n] += d[node_to_eq[n]];
    }
    *resid = bn > 0 ? sqrt(rr) / bn : 0.0;
    free(t1);
    free(t2);
    free(t3);
    free(b);
    free(dg);
    free(x);
    free(r);
    free(p);
    free(q);
    return it;
}
