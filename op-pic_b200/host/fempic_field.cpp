// Host set-up of the FemPIC field solve (include/oppb_field.h): FESolver's constructor
// (apps_codegen/app_fempic_cg/field_solver/field_solver.cpp:46-99) without PETSc.  Every
// quantity is formed with the reference's operation order, so the stiffness matrix, F0 and
// the shape-function derivatives equal the reference's bit for bit; compiled with
// -ffp-contract=off.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include "oppb_field.h"

namespace {

constexpr double kScaling = 100.0;  // SCALLING, field_solver.cpp:21

template <typename T>
T* alloc(size_t n) {
    return static_cast<T*>(std::calloc(n ? n : 1, sizeof(T)));
}

// Determinant by cofactors of the first row (minifempic_funcs.h det3).
double det3(const double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// Inverse by the adjugate; a matrix whose largest adjugate entry exceeds 1e12 |det| gives the
// zero matrix, as the reference's `inverse` (minifempic_funcs.h) does.
void inverse3(const double m[3][3], double v[3][3]) {
    const double a = m[0][0], b = m[0][1], c = m[0][2];
    const double d = m[1][0], e = m[1][1], f = m[1][2];
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
        for (int s = 0; s < 3; s++) vmax = std::fabs(v[r][s]) > vmax ? std::fabs(v[r][s]) : vmax;
    const double idet = (std::fabs(vmax) / std::fabs(det) > 1e12) ? 0.0 : 1 / det;
    for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) v[r][s] *= idet;
}

}  // namespace

extern "C" int oppb_field_setup(const oppb_fempic_mesh* mp, oppb_field_system* out) {
    if (!mp || !out || !mp->n_pos || !mp->n_type || !mp->n_bnd_pot || !mp->c2n || mp->n_nodes <= 0 ||
        mp->n_cells <= 0)
        return OPPB_ERR_ARG;
    const oppb_fempic_mesh& m = *mp;
    const int64_t nn = m.n_nodes, nc = m.n_cells;
    for (int64_t k = 0; k < 4 * nc; k++)
        if (m.c2n[k] < 0 || m.c2n[k] >= nn) return OPPB_ERR_ARG;
    oppb_field_system s{};
    s.n_nodes = m.n_nodes;
    s.n_cells = m.n_cells;
    // Equation numbering (calculate_neq / init_node_to_eq_map, :178-210).
    s.node_to_eq = alloc<int32_t>((size_t)nn);
    int32_t neq = 0;
    for (int64_t n = 0; n < nn; n++)
        s.node_to_eq[n] = (m.n_type[n] == OPPB_NODE_NORMAL || m.n_type[n] == OPPB_NODE_OPEN) ? neq++ : -1;
    s.neq = neq;
    s.c2n = alloc<int32_t>((size_t)(4 * nc));
    std::memcpy(s.c2n, m.c2n, sizeof(int32_t) * 4 * (size_t)nc);
    s.n_bnd_pot = alloc<double>((size_t)nn);
    std::memcpy(s.n_bnd_pot, m.n_bnd_pot, sizeof(double) * (size_t)nn);
    s.det_j = alloc<double>((size_t)nc);
    s.c_sd = alloc<double>((size_t)(12 * nc));
    s.f0 = alloc<double>((size_t)(neq ? neq : 1));
    // Rows of K in the order contributions arrive (element order), as the reference's
    // std::map rows sum them; columns sorted afterwards.
    std::vector<std::vector<std::pair<int32_t, double>>> rows((size_t)neq);
    static const double na_xi[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    for (int64_t e = 0; e < nc; e++) {
        const int32_t* con = m.c2n + 4 * e;
        // compute_nx (:553-594): x_xi = d x / d xi, detJ, NX = na_xi * xi_x * SCALLING.
        double x_xi[3][3], xi_x[3][3], nx[4][3];
        for (int dim = 0; dim < 3; dim++)
            for (int j = 0; j < 3; j++) {
                x_xi[dim][j] = 0;
                for (int a = 0; a < 4; a++) x_xi[dim][j] += (na_xi[a][j] * m.n_pos[(int64_t)con[a] * 3 + dim]);
            }
        const double det_j = det3(x_xi);
        inverse3(x_xi, xi_x);
        for (int a = 0; a < 4; a++)
            for (int d = 0; d < 3; d++) {
                nx[a][d] = 0.0;
                for (int k = 0; k < 3; k++) nx[a][d] += (na_xi[a][k] * xi_x[k][d] * kScaling);
                s.c_sd[e * 12 + a * 3 + d] = (nx[a][d] / kScaling);  // enrich_cell_shape_deriv
            }
        s.det_j[e] = det_j;
        // pre_assembly (:330-391): ke over the 2x2x2 Gauss points (weights 1), fe = -ke g.
        double ke[4][4];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                ke[a][b] = 0.0;
                for (int q = 0; q < 8; q++) {
                    double dot = 0.0;
                    for (int d = 0; d < 3; d++) dot += (nx[a][d] * nx[b][d]);
                    ke[a][b] += (dot * det_j * 1.0 * 1.0 * 1.0);
                }
            }
        for (int a = 0; a < 4; a++) {  // add_ke (:501-536)
            const int32_t p = s.node_to_eq[con[a]];
            if (p < 0) continue;
            for (int b = 0; b < 4; b++) {
                const int32_t q = s.node_to_eq[con[b]];
                if (q < 0) continue;
                auto& row = rows[(size_t)p];
                bool found = false;
                for (auto& cv : row)
                    if (cv.first == q) {
                        cv.second += ke[a][b];
                        found = true;
                        break;
                    }
                if (!found) row.emplace_back(q, ke[a][b]);
            }
        }
        for (int a = 0; a < 4; a++) {  // fe and add_fe (:538-551)
            double fh = 0, fg = 0;
            for (int b = 0; b < 4; b++) fg -= (ke[a][b] * m.n_bnd_pot[con[b]]);
            const int32_t p = s.node_to_eq[con[a]];
            if (p >= 0) s.f0[p] += (fh + fg);
        }
    }
    // Downscaling by 1/SCALLING^2 (MatScale / VecScale, :387-388).
    const double scalar2 = 1.0 / (kScaling * kScaling);
    s.k_rowptr = alloc<int64_t>((size_t)neq + 1);
    int64_t nnz = 0;
    for (int32_t r = 0; r < neq; r++) nnz += (int64_t)rows[(size_t)r].size();
    s.k_col = alloc<int32_t>((size_t)nnz);
    s.k_val = alloc<double>((size_t)nnz);
    int64_t at = 0;
    for (int32_t r = 0; r < neq; r++) {
        auto& row = rows[(size_t)r];
        std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        s.k_rowptr[r] = at;
        for (const auto& cv : row) {
            s.k_col[at] = cv.first;
            s.k_val[at] = cv.second * scalar2;
            at++;
        }
        std::vector<std::pair<int32_t, double>>().swap(row);
    }
    s.k_rowptr[neq] = at;
    s.nnz = nnz;
    for (int32_t r = 0; r < neq; r++) s.f0[r] *= scalar2;
    // The diagonal form, when K's entries lie on few diagonals.
    std::vector<int32_t> offs;
    bool banded = true;
    for (int32_t r = 0; r < neq && banded; r++)
        for (int64_t k = s.k_rowptr[r]; k < s.k_rowptr[r + 1]; k++) {
            const int32_t o = s.k_col[k] - r;
            if (std::find(offs.begin(), offs.end(), o) == offs.end()) {
                if ((int)offs.size() == OPPB_FIELD_MAX_DIAG) {
                    banded = false;
                    break;
                }
                offs.push_back(o);
            }
        }
    if (banded && !offs.empty() && (double)offs.size() * neq <= 1.5 * (double)nnz) {
        std::sort(offs.begin(), offs.end());
        s.n_diag = (int32_t)offs.size();
        for (int j = 0; j < s.n_diag; j++) s.dia_off[j] = offs[(size_t)j];
        s.dia_val = alloc<double>((size_t)s.n_diag * neq);
        for (int64_t q = 0; q < (int64_t)s.n_diag * neq; q++) s.dia_val[q] = 0.0;
        for (int32_t r = 0; r < neq; r++)
            for (int64_t k = s.k_rowptr[r]; k < s.k_rowptr[r + 1]; k++) {
                const int j = (int)(std::lower_bound(offs.begin(), offs.end(), s.k_col[k] - r) - offs.begin());
                s.dia_val[(int64_t)j * neq + r] = s.k_val[k];
            }
    }
    *out = s;
    return OPPB_OK;
}

extern "C" void oppb_field_system_free(oppb_field_system* s) {
    if (!s) return;
    std::free(s->node_to_eq);
    std::free(s->c2n);
    std::free(s->det_j);
    std::free(s->c_sd);
    std::free(s->n_bnd_pot);
    std::free(s->k_rowptr);
    std::free(s->k_col);
    std::free(s->k_val);
    std::free(s->f0);
    std::free(s->dia_val);
    *s = oppb_field_system{};
}
