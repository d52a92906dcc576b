// Host set-up of the FemPIC application: box tetrahedral mesh, reference cell
// geometry, inlet surface, injection distribution and the static FEM field.
// Compiled with -ffp-contract=off so every product below is rounded on its own,
// as the reference's scalar C++ evaluates it.

#include "oppb_fempic.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

// 3x3 determinant, cofactor expansion along the first row
// (apps/app_fempic/minifempic_funcs.h:69-73).
double det3(const double M[3][3]) {
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

// 4x4 determinant along the first row (minifempic_funcs.h:75-103).
double det4(const double M[4][4]) {
    double S[4][3][3];
    static const int cols[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    for (int s = 0; s < 4; s++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) S[s][i][j] = M[i + 1][cols[s][j]];
    return M[0][0] * det3(S[0]) - M[0][1] * det3(S[1]) + M[0][2] * det3(S[2]) -
           M[0][3] * det3(S[3]);
}

template <typename T>
T* alloc(size_t n) {
    T* p = static_cast<T*>(std::calloc(n ? n : 1, sizeof(T)));
    return p;
}

// Vertices (opposite-face rule, minifempic_funcs.h:386-437) of the face opposite vertex v.
const int kFace[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
// Vertex triples of the alpha..delta cofactors of vertex v (minifempic_funcs.h:323-330).
const int kCof[4][3] = {{1, 2, 3}, {3, 2, 0}, {3, 0, 1}, {1, 0, 2}};

uint64_t face_key(int a, int b, int c) {
    int t[3] = {a, b, c};
    std::sort(t, t + 3);
    return (uint64_t(uint32_t(t[0])) << 42) | (uint64_t(uint32_t(t[1])) << 21) | uint64_t(uint32_t(t[2]));
}

}  // namespace

extern "C" void oppb_fempic_mesh_free(oppb_fempic_mesh* m) {
    if (!m) return;
    void* ptrs[] = {m->n_pos, m->n_vol, m->n_type, m->n_bnd_pot, m->c2n, m->c2c,
                    m->c_det, m->c_vol, m->c_sd, m->c_ef, m->c_centroid, m->if2c,
                    m->if2n, m->if_u, m->if_v, m->if_norm, m->if_area, m->if_n_pos};
    for (void* p : ptrs) std::free(p);
    std::memset(m, 0, sizeof(*m));
}

extern "C" int oppb_fempic_box_mesh(int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                                    double lz, oppb_fempic_mesh* out) {
    if (!out || nx <= 0 || ny <= 0 || nz <= 0 || !(lx > 0) || !(ly > 0) || !(lz > 0)) return 1;
    std::memset(out, 0, sizeof(*out));
    const int64_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
    const int64_t n_nodes = NX * NY * NZ;
    const int64_t n_hex = int64_t(nx) * ny * nz;
    const int64_t n_cells = 6 * n_hex;
    if (n_cells > INT32_MAX / 4 || n_nodes >= (int64_t(1) << 21)) return 1;
    oppb_fempic_mesh& m = *out;
    m.n_nodes = int32_t(n_nodes);
    m.n_cells = int32_t(n_cells);
    m.n_ifaces = 2 * nx * ny;

    m.n_pos = alloc<double>(3 * n_nodes);
    m.n_vol = alloc<double>(n_nodes);
    m.n_type = alloc<int32_t>(n_nodes);
    m.n_bnd_pot = alloc<double>(n_nodes);
    m.c2n = alloc<int32_t>(4 * n_cells);
    m.c2c = alloc<int32_t>(4 * n_cells);
    m.c_det = alloc<double>(16 * n_cells);
    m.c_vol = alloc<double>(n_cells);
    m.c_sd = alloc<double>(12 * n_cells);
    m.c_ef = alloc<double>(3 * n_cells);
    m.c_centroid = alloc<double>(3 * n_cells);
    m.if2c = alloc<int32_t>(m.n_ifaces);
    m.if2n = alloc<int32_t>(3 * m.n_ifaces);
    m.if_u = alloc<double>(3 * m.n_ifaces);
    m.if_v = alloc<double>(3 * m.n_ifaces);
    m.if_norm = alloc<double>(3 * m.n_ifaces);
    m.if_area = alloc<double>(m.n_ifaces);
    m.if_n_pos = alloc<double>(9 * m.n_ifaces);

    const double hx = lx / nx, hy = ly / ny, hz = lz / nz;
    auto nid = [&](int64_t i, int64_t j, int64_t k) { return int32_t(i + NX * (j + NY * k)); };
    for (int64_t k = 0; k < NZ; k++)
        for (int64_t j = 0; j < NY; j++)
            for (int64_t i = 0; i < NX; i++) {
                double* p = m.n_pos + 3 * nid(i, j, k);
                p[0] = (i == nx) ? lx : double(i) * hx;
                p[1] = (j == ny) ? ly : double(j) * hy;
                p[2] = (k == nz) ? lz : double(k) * hz;
            }

    // Kuhn split: tet t walks 000 -> e_a -> e_a+e_b -> 111 for the t-th axis permutation.
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int64_t k = 0; k < nz; k++)
        for (int64_t j = 0; j < ny; j++)
            for (int64_t i = 0; i < nx; i++) {
                const int64_t h = i + nx * (j + ny * k);
                for (int t = 0; t < 6; t++) {
                    int b[3] = {0, 0, 0};
                    int32_t* con = m.c2n + 4 * (6 * h + t);
                    con[0] = nid(i, j, k);
                    b[perm[t][0]] = 1;
                    con[1] = nid(i + b[0], j + b[1], k + b[2]);
                    b[perm[t][1]] = 1;
                    con[2] = nid(i + b[0], j + b[1], k + b[2]);
                    con[3] = nid(i + 1, j + 1, k + 1);
                }
            }

    // Volumes with the ABCD -> ADBC flip, then the alpha..delta cofactors.
    for (int64_t c = 0; c < n_cells; c++) {
        int32_t* con = m.c2n + 4 * c;
        double M[4][4];
        for (int v = 0; v < 4; v++) {
            M[v][0] = 1;
            for (int d = 0; d < 3; d++) M[v][d + 1] = m.n_pos[3 * con[v] + d];
        }
        double vol = (1.0 / 6.0) * det4(M);
        if (vol < 0) {
            std::swap(con[1], con[3]);
            vol = -vol;
        }
        m.c_vol[c] = vol;
        for (int v = 0; v < 4; v++) {
            const double* p2 = m.n_pos + 3 * con[kCof[v][0]];
            const double* p3 = m.n_pos + 3 * con[kCof[v][1]];
            const double* p4 = m.n_pos + 3 * con[kCof[v][2]];
            const double A[3][3] = {{p2[0], p2[1], p2[2]}, {p3[0], p3[1], p3[2]}, {p4[0], p4[1], p4[2]}};
            const double B[3][3] = {{1, p2[1], p2[2]}, {1, p3[1], p3[2]}, {1, p4[1], p4[2]}};
            const double G[3][3] = {{1, p2[0], p2[2]}, {1, p3[0], p3[2]}, {1, p4[0], p4[2]}};
            const double D[3][3] = {{1, p2[0], p2[1]}, {1, p3[0], p3[1]}, {1, p4[0], p4[1]}};
            double* det = m.c_det + 16 * c + 4 * v;
            det[0] = det3(A);
            det[1] = det3(B);
            det[2] = det3(G);
            det[3] = det3(D);
        }
        for (int d = 0; d < 3; d++) {
            double s = 0;
            for (int v = 0; v < 4; v++) s += 0.25 * m.n_pos[3 * con[v] + d];
            m.c_centroid[3 * c + d] = s;
        }
        // grad(lambda_i) = (-beta_i, gamma_i, -delta_i) / (6 V)
        for (int v = 0; v < 4; v++) {
            const double* det = m.c_det + 16 * c + 4 * v;
            const double s6 = 6.0 * vol;
            m.c_sd[12 * c + 3 * v + 0] = -det[1] / s6;
            m.c_sd[12 * c + 3 * v + 1] = det[2] / s6;
            m.c_sd[12 * c + 3 * v + 2] = -det[3] / s6;
        }
    }

    // Face neighbours: the face opposite vertex v of cell c is shared by at most one
    // other cell; match sorted node triples.
    {
        std::vector<std::pair<uint64_t, int64_t>> faces(static_cast<size_t>(4 * n_cells));
        for (int64_t c = 0; c < n_cells; c++) {
            const int32_t* con = m.c2n + 4 * c;
            for (int v = 0; v < 4; v++) {
                faces[size_t(4 * c + v)] = {face_key(con[kFace[v][0]], con[kFace[v][1]], con[kFace[v][2]]),
                                            4 * c + v};
                m.c2c[4 * c + v] = -1;
            }
        }
        std::sort(faces.begin(), faces.end());
        for (size_t f = 0; f + 1 < faces.size(); f++) {
            if (faces[f].first == faces[f + 1].first) {
                const int64_t a = faces[f].second, b = faces[f + 1].second;
                m.c2c[a] = int32_t(b / 4);
                m.c2c[b] = int32_t(a / 4);
                f++;
            }
        }
    }

    // Node volumes: scatter lc(centroid) * volume (XtoLtet form, minifempic_funcs.h:199-211,446-461),
    // and node types: nodes of faces without a neighbour are OPEN.
    for (int64_t c = 0; c < n_cells; c++) {
        const int32_t* con = m.c2n + 4 * c;
        const double* det = m.c_det + 16 * c;
        const double* x = m.c_centroid + 3 * c;
        const double vol = m.c_vol[c];
        for (int v = 0; v < 4; v++) {
            const double lc = (1.0 / 6.0) * (det[4 * v + 0] - x[0] * det[4 * v + 1] + x[1] * det[4 * v + 2] -
                                             x[2] * det[4 * v + 3]) / vol;
            m.n_vol[con[v]] += lc * vol;
        }
        for (int v = 0; v < 4; v++)
            if (m.c2c[4 * c + v] < 0)
                for (int i = 0; i < 4; i++)
                    if (i != v && m.n_type[con[i]] == OPPB_NODE_NORMAL) m.n_type[con[i]] = OPPB_NODE_OPEN;
    }
    for (int64_t j = 0; j < NY; j++)
        for (int64_t i = 0; i < NX; i++) {
            m.n_type[nid(i, j, 0)] = OPPB_NODE_INLET;
            m.n_type[nid(i, j, nz)] = OPPB_NODE_FIXED;
        }

    // Inlet: two triangles per z=0 hex face, ordered so that the reference's normal
    // formula (minifempic_funcs.h:551-575, no inversion) points along +z.
    {
        std::vector<std::pair<uint64_t, int64_t>> bfaces;
        bfaces.reserve(size_t(2 * nx * ny));
        for (int64_t h = 0; h < int64_t(nx) * ny; h++)  // bottom hex layer k = 0
            for (int t = 0; t < 6; t++) {
                const int64_t c = 6 * h + t;
                const int32_t* con = m.c2n + 4 * c;
                for (int v = 0; v < 4; v++) {
                    if (m.c2c[4 * c + v] >= 0) continue;
                    const int32_t a = con[kFace[v][0]], b = con[kFace[v][1]], d = con[kFace[v][2]];
                    if (m.n_pos[3 * a + 2] == 0.0 && m.n_pos[3 * b + 2] == 0.0 && m.n_pos[3 * d + 2] == 0.0)
                        bfaces.push_back({face_key(a, b, d), c});
                }
            }
        std::sort(bfaces.begin(), bfaces.end());
        int32_t f = 0;
        for (int64_t j = 0; j < ny; j++)
            for (int64_t i = 0; i < nx; i++) {
                const int32_t n000 = nid(i, j, 0), n100 = nid(i + 1, j, 0);
                const int32_t n010 = nid(i, j + 1, 0), n110 = nid(i + 1, j + 1, 0);
                const int32_t tri[2][3] = {{n000, n110, n100}, {n000, n010, n110}};
                for (int s = 0; s < 2; s++, f++) {
                    const uint64_t key = face_key(tri[s][0], tri[s][1], tri[s][2]);
                    auto it = std::lower_bound(bfaces.begin(), bfaces.end(), std::make_pair(key, int64_t(-1)));
                    if (it == bfaces.end() || it->first != key) return 2;
                    m.if2c[f] = int32_t(it->second);
                    const double* p1 = m.n_pos + 3 * tri[s][0];
                    const double* p2 = m.n_pos + 3 * tri[s][1];
                    const double* p3 = m.n_pos + 3 * tri[s][2];
                    double u[3], v[3];
                    for (int d = 0; d < 3; d++) {
                        m.if2n[3 * f + d] = tri[s][d];
                        u[d] = p2[d] - p1[d];
                        v[d] = p3[d] - p1[d];
                        m.if_n_pos[9 * f + d] = p1[d];
                        m.if_n_pos[9 * f + 3 + d] = p2[d];
                        m.if_n_pos[9 * f + 6 + d] = p3[d];
                        m.if_u[3 * f + d] = u[d];
                        m.if_v[3 * f + d] = v[d];
                    }
                    const double nrm[3] = {u[2] * v[1] - u[1] * v[2], u[0] * v[2] - u[2] * v[0],
                                           u[1] * v[0] - u[0] * v[1]};
                    const double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
                    for (int d = 0; d < 3; d++) m.if_norm[3 * f + d] = nrm[d] / len;
                    m.if_area[f] = len / 2;
                }
            }
    }
    return 0;
}

extern "C" int oppb_fempic_inject_distribution(const oppb_fempic_mesh* m, int32_t total, int32_t* dist_out) {
    if (!m || !dist_out || total < 0 || m->n_ifaces <= 0) return 1;
    double area = 0;
    for (int32_t f = 0; f < m->n_ifaces; f++) area += m->if_area[f];
    // Cumulative counts from the rounded cumulative area share: the last face closes at `total`.
    double acc = 0;
    for (int32_t f = 0; f < m->n_ifaces; f++) {
        acc += m->if_area[f];
        int64_t cum = (f == m->n_ifaces - 1) ? total : int64_t(std::llround(double(total) * (acc / area)));
        if (cum > total) cum = total;
        dist_out[f] = int32_t(cum);
    }
    for (int32_t f = 1; f < m->n_ifaces; f++)
        if (dist_out[f] < dist_out[f - 1]) dist_out[f] = dist_out[f - 1];
    return 0;
}

extern "C" int oppb_fempic_solve_field(oppb_fempic_mesh* mp, double phi_inlet, double phi_fixed, double rtol,
                                       int32_t max_iter, double* n_pot_out, int32_t* iters_out,
                                       double* resid_out) {
    if (!mp) return 1;
    oppb_fempic_mesh& m = *mp;
    const int64_t nn = m.n_nodes, nc = m.n_cells;
    // Dirichlet values and an initial guess that interpolates them linearly in z.
    double zmin = m.n_pos[2], zmax = m.n_pos[2];
    for (int64_t n = 0; n < nn; n++) {
        zmin = std::min(zmin, m.n_pos[3 * n + 2]);
        zmax = std::max(zmax, m.n_pos[3 * n + 2]);
    }
    const size_t NN = static_cast<size_t>(nn);
    std::vector<double> phi(NN);
    std::vector<char> fixed(NN, 0);
    for (int64_t n = 0; n < nn; n++) {
        const double s = (m.n_pos[3 * n + 2] - zmin) / (zmax - zmin);
        phi[size_t(n)] = phi_inlet + (phi_fixed - phi_inlet) * s;
        if (m.n_type[n] == OPPB_NODE_INLET) {
            phi[size_t(n)] = phi_inlet;
            fixed[size_t(n)] = 1;
        } else if (m.n_type[n] == OPPB_NODE_FIXED) {
            phi[size_t(n)] = phi_fixed;
            fixed[size_t(n)] = 1;
        }
        m.n_bnd_pot[n] = fixed[size_t(n)] ? phi[size_t(n)] : 0.0;
    }
    // Assemble K_ij = sum_e V_e grad(l_i).grad(l_j) as CSR over all nodes.
    std::vector<std::vector<std::pair<int32_t, double>>> rows(NN);
    for (int64_t c = 0; c < nc; c++) {
        const int32_t* con = m.c2n + 4 * c;
        const double* g = m.c_sd + 12 * c;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                const double k = m.c_vol[c] * (g[3 * a] * g[3 * b] + g[3 * a + 1] * g[3 * b + 1] +
                                               g[3 * a + 2] * g[3 * b + 2]);
                rows[size_t(con[a])].push_back({con[b], k});
            }
    }
    std::vector<int64_t> rp(NN + 1, 0);
    std::vector<int32_t> ci;
    std::vector<double> cv;
    for (int64_t n = 0; n < nn; n++) {
        auto& r = rows[size_t(n)];
        std::sort(r.begin(), r.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t e = 0; e < r.size(); e++) {
            if (!ci.empty() && int64_t(ci.size()) > rp[size_t(n)] && ci.back() == r[e].first)
                cv.back() += r[e].second;
            else {
                ci.push_back(r[e].first);
                cv.push_back(r[e].second);
            }
        }
        rp[size_t(n + 1)] = int64_t(ci.size());
        std::vector<std::pair<int32_t, double>>().swap(r);
    }
    // CG on the free nodes: K_ff phi_f = -K_fd phi_d  <=>  residual r = -(K phi) on free rows.
    auto apply = [&](const std::vector<double>& x, std::vector<double>& y) {
        for (int64_t n = 0; n < nn; n++) {
            if (fixed[size_t(n)]) { y[size_t(n)] = 0; continue; }
            double s = 0;
            for (int64_t e = rp[size_t(n)]; e < rp[size_t(n + 1)]; e++) s += cv[size_t(e)] * x[size_t(ci[size_t(e)])];
            y[size_t(n)] = s;
        }
    };
    std::vector<double> r(NN), p(NN), q(NN), bvec(NN), zero(NN);
    // b = -K_fd phi_d: apply K to the Dirichlet part only.
    for (int64_t n = 0; n < nn; n++) zero[size_t(n)] = fixed[size_t(n)] ? phi[size_t(n)] : 0.0;
    apply(zero, bvec);
    double bnorm = 0;
    for (int64_t n = 0; n < nn; n++) {
        bvec[size_t(n)] = -bvec[size_t(n)];
        bnorm += bvec[size_t(n)] * bvec[size_t(n)];
    }
    bnorm = std::sqrt(bnorm);
    apply(phi, q);  // K phi on free rows (full phi) = K_ff phi_f + K_fd phi_d
    double rr = 0;
    for (int64_t n = 0; n < nn; n++) {
        r[size_t(n)] = fixed[size_t(n)] ? 0.0 : -q[size_t(n)];
        p[size_t(n)] = r[size_t(n)];
        rr += r[size_t(n)] * r[size_t(n)];
    }
    const double stop = rtol * (bnorm > 0 ? bnorm : 1.0);
    int32_t it = 0;
    while (std::sqrt(rr) > stop && it < max_iter) {
        apply(p, q);
        double pq = 0;
        for (int64_t n = 0; n < nn; n++) pq += p[size_t(n)] * q[size_t(n)];
        const double alpha = rr / pq;
        double rr2 = 0;
        for (int64_t n = 0; n < nn; n++) {
            if (fixed[size_t(n)]) continue;
            phi[size_t(n)] += alpha * p[size_t(n)];
            r[size_t(n)] -= alpha * q[size_t(n)];
            rr2 += r[size_t(n)] * r[size_t(n)];
        }
        const double beta = rr2 / rr;
        rr = rr2;
        for (int64_t n = 0; n < nn; n++) p[size_t(n)] = fixed[size_t(n)] ? 0.0 : r[size_t(n)] + beta * p[size_t(n)];
        it++;
    }
    if (iters_out) *iters_out = it;
    if (resid_out) *resid_out = std::sqrt(rr) / (bnorm > 0 ? bnorm : 1.0);
    // c_ef = 0 - (c1 + c2 + c3 + c4), c_k = sd[k][dim] * phi_k (kernels.h:186-202).
    for (int64_t c = 0; c < nc; c++) {
        const int32_t* con = m.c2n + 4 * c;
        const double* sd = m.c_sd + 12 * c;
        for (int d = 0; d < 3; d++) {
            const double c1 = sd[0 * 3 + d] * phi[size_t(con[0])];
            const double c2 = sd[1 * 3 + d] * phi[size_t(con[1])];
            const double c3 = sd[2 * 3 + d] * phi[size_t(con[2])];
            const double c4 = sd[3 * 3 + d] * phi[size_t(con[3])];
            double e = 0.0;
            e -= (c1 + c2 + c3 + c4);
            m.c_ef[3 * c + d] = e;
        }
    }
    if (n_pot_out)
        for (int64_t n = 0; n < nn; n++) n_pot_out[n] = phi[size_t(n)];
    return (std::sqrt(rr) <= stop) ? 0 : 3;
}
