// TEST INFRASTRUCTURE ONLY — driver of the compiled OP-PIC reference (seq / omp backend
// and the generated FemPIC loops of apps_codegen/app_fempic_cg/{seq,omp}) on a case file.
//
// It declares the FemPIC sets, maps and dats through the reference's own API and runs the
// particle part of the generated main loop (apps_codegen/app_fempic_cg/fempic_opp.cpp:160-215):
//   opp_inc_part_count_with_distribution -> inject_ions (+ thermal velocity from the case)
//   -> reset n_charge_den -> calculate_new_pos_vel -> move (with its finalize) -> deposit.
// The field is the static cell field of the case (no field solve).  A direct-hop case
// turns on the global move (opp_init_direct_hop_cg builds the structured map by the
// reference's own search) and the output ends with the reference's grid and map.  Per step it records
// sizes and wall times and, unless the case is a timing case (record_state 0), FNV-1a
// hashes of the particle dats and of the node charges.
//
//   ref_harness <opp params file> <case file> <out file>
//
// Built by oracle/Makefile into oracle/_ref/ only; it is the checker of the C oracle and
// the CPU baseline, never part of the product.

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "opp_lib.h"

void opp_par_loop_injected__inject_ions_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg,
                                               opp_arg, opp_arg, opp_arg, opp_arg);
void opp_par_loop_all__calculate_new_pos_vel_kernel(opp_set, opp_arg, opp_arg, opp_arg);
void opp_particle_move__move_kernel(opp_set, opp_map, opp_map, opp_arg, opp_arg, opp_arg, opp_arg);
void opp_par_loop_all__deposit_charge_on_nodes_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg);
void opp_init_direct_hop_cg(double, const opp_dat, const opp::BoundingBox&, opp_map, opp_map, opp_arg, opp_arg,
                            opp_arg, opp_arg);

namespace {

struct Header {
    char magic[8];
    int32_t n_nodes, n_cells, n_ifaces, inject, steps, n_tables, record_state, direct_hop;
    double dt, qm, ion_velocity, sigma;
};

template <typename T>
std::vector<T> read_vec(FILE* f, size_t n) {
    std::vector<T> v(n ? n : 1);
    if (n && fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "ref_harness: short read\n");
        exit(2);
    }
    return v;
}

uint64_t fnv1a(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

// Tables beyond the case's: splitmix64 uniforms and Box-Muller normals (timing runs only).
uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double unif(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

struct StepRecord {
    int32_t step, size_before_move, removed, size;
    uint64_t h_p2c, h_pos, h_vel, h_lc, h_charge;
    double t_inject, t_push, t_move, t_deposit;
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <params> <case> <out>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[2], "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", argv[2]);
        return 2;
    }
    Header h;
    if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, "OPPBCAS1", 8) != 0) {
        fprintf(stderr, "bad case file\n");
        return 2;
    }
    const size_t nc = h.n_cells, nf = h.n_ifaces, nn = h.n_nodes;
    auto c2n = read_vec<int>(f, nc * 4);
    auto c2c = read_vec<int>(f, nc * 4);
    auto c_det = read_vec<double>(f, nc * 16);
    auto c_vol = read_vec<double>(f, nc);
    auto c_ef = read_vec<double>(f, nc * 3);
    auto if2c = read_vec<int>(f, nf);
    auto if_u = read_vec<double>(f, nf * 3);
    auto if_v = read_vec<double>(f, nf * 3);
    auto if_norm = read_vec<double>(f, nf * 3);
    auto if_n_pos = read_vec<double>(f, nf * 9);
    auto if_dist = read_vec<int>(f, nf);
    auto tables = read_vec<double>(f, (size_t)h.n_tables * h.inject * 5);
    // Direct-hop cases: grid spacing, expansion[3] and the node positions follow the tables.
    std::vector<double> dh_par(4, 0.0), n_pos;
    if (h.direct_hop) {
        dh_par = read_vec<double>(f, 4);
        n_pos = read_vec<double>(f, nn * 3);
    }
    fclose(f);
    std::vector<double> n_charge(nn, 0.0);

    char* args[2] = {argv[0], argv[1]};
    opp_init(2, args);
    {
        opp_set node_set = opp_decl_set(h.n_nodes, "mesh_nodes");
        opp_set cell_set = opp_decl_set(h.n_cells, "mesh_cells");
        opp_set iface_set = opp_decl_set(h.n_ifaces, "inlet_faces_cells");
        opp_set particle_set = opp_decl_particle_set("particles", cell_set);
        opp_set dummy_part_set = opp_decl_particle_set("dummy particles", cell_set);

        opp_map c2n_map = opp_decl_map(cell_set, node_set, 4, c2n.data(), "c_v_n_map");
        opp_map c2c_map = opp_decl_map(cell_set, cell_set, 4, c2c.data(), "c_v_c_map");
        opp_map if2c_map = opp_decl_map(iface_set, cell_set, 1, if2c.data(), "if_v_c_map");

        opp_dat c_det_d = opp_decl_dat(cell_set, 16, DT_REAL, c_det.data(), "c_det");
        opp_dat c_volume = opp_decl_dat(cell_set, 1, DT_REAL, c_vol.data(), "c_volume");
        opp_dat c_ef_d = opp_decl_dat(cell_set, 3, DT_REAL, c_ef.data(), "c_ef");
        opp_dat n_charge_den = opp_decl_dat(node_set, 1, DT_REAL, n_charge.data(), "n_charge_den");
        opp_dat if_v_norm = opp_decl_dat(iface_set, 3, DT_REAL, if_v.data(), "iface_v_norm");
        opp_dat if_u_norm = opp_decl_dat(iface_set, 3, DT_REAL, if_u.data(), "iface_u_norm");
        opp_dat if_norm_d = opp_decl_dat(iface_set, 3, DT_REAL, if_norm.data(), "iface_norm");
        opp_dat if_distrib = opp_decl_dat(iface_set, 1, DT_INT, if_dist.data(), "iface_dist");
        opp_dat if_n_pos_d = opp_decl_dat(iface_set, 9, DT_REAL, if_n_pos.data(), "iface_n_pos");

        opp_dat p_pos = opp_decl_dat(particle_set, 3, DT_REAL, nullptr, "p_position");
        opp_dat p_vel = opp_decl_dat(particle_set, 3, DT_REAL, nullptr, "p_velocity");
        opp_dat p_lc = opp_decl_dat(particle_set, 4, DT_REAL, nullptr, "p_lc");
        opp_map p2c_map = opp_decl_map(particle_set, cell_set, 1, nullptr, "p2c_map");
        opp_dat dp_rand = opp_decl_dat(dummy_part_set, 2, DT_REAL, nullptr, "dummy_part_rand");

        // Global move (the params file sets opp_global_move and opp_dh_data_generate): the
        // app's set-up of fempic_opp.cpp:69-76,95,147-153 with the case's spacing/expansion.
        if (h.direct_hop) {
            std::vector<int> c_id(nc);
            for (size_t c = 0; c < nc; c++) c_id[c] = (int)c;
            opp_dat n_pos_d = opp_decl_dat(node_set, 3, DT_REAL, n_pos.data(), "n_pos");
            opp_dat c_gbl_id = opp_decl_dat(cell_set, 1, DT_INT, c_id.data(), "c_gbl_id");
            opp::BoundingBox bounding_box(n_pos_d, 3, opp_point(dh_par[1], dh_par[2], dh_par[3]));
            opp_init_direct_hop_cg(dh_par[0], c_gbl_id, bounding_box, c2c_map, p2c_map,
                                   opp_arg_dat(p_pos, OPP_READ), opp_arg_dat(p_lc, OPP_WRITE),
                                   opp_arg_dat(c_volume, p2c_map, OPP_READ),
                                   opp_arg_dat(c_det_d, p2c_map, OPP_READ));
        }

        double one = 1.0, dt = h.dt, vion = h.ion_velocity, zero = 0.0;
        opp_decl_const<OPP_REAL>(1, &zero, "CONST_spwt");
        opp_decl_const<OPP_REAL>(1, &vion, "CONST_ion_velocity");
        opp_decl_const<OPP_REAL>(1, &dt, "CONST_dt");
        opp_decl_const<OPP_REAL>(1, &zero, "CONST_plasma_den");
        opp_decl_const<OPP_REAL>(1, &one, "CONST_mass");
        opp_decl_const<OPP_REAL>(1, &h.qm, "CONST_charge");
        opp_decl_const<OPP_REAL>(1, &zero, "CONST_wall_potential");

        opp_increase_particle_count(dummy_part_set, h.inject);
        std::vector<double> thermal((size_t)h.inject * 3);
        std::vector<StepRecord> recs;
        uint64_t rng = 0x5eedull;
        using clk = std::chrono::steady_clock;
        auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };

        for (OPP_main_loop_iter = 0; OPP_main_loop_iter < h.steps; OPP_main_loop_iter++) {
            const int s = OPP_main_loop_iter;
            // Per-step random table: (a, b) into dp_rand, thermal velocity kept aside.
            double* dr = (double*)dp_rand->data;
            for (int k = 0; k < h.inject; k++) {
                if (s < h.n_tables) {
                    const double* t = tables.data() + ((size_t)s * h.inject + k) * 5;
                    dr[2 * k] = t[0];
                    dr[2 * k + 1] = t[1];
                    for (int d = 0; d < 3; d++) thermal[3 * k + d] = t[2 + d];
                } else {
                    dr[2 * k] = unif(rng);
                    dr[2 * k + 1] = unif(rng);
                    for (int d = 0; d < 3; d++) {
                        const double u1 = unif(rng) + 1e-300, u2 = unif(rng);
                        thermal[3 * k + d] = h.sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                    }
                }
            }
            StepRecord r{};
            r.step = s;
            auto t0 = clk::now();
            opp_inc_part_count_with_distribution(particle_set, h.inject, if_distrib, false);
            opp_par_loop_injected__inject_ions_kernel(
                particle_set, opp_arg_dat(p_pos, OPP_WRITE), opp_arg_dat(p_vel, OPP_WRITE),
                opp_arg_dat(p2c_map, OPP_RW), opp_arg_dat(if2c_map, p2c_map, OPP_READ),
                opp_arg_dat(c_ef_d, 0, if2c_map, p2c_map, OPP_READ), opp_arg_dat(if_u_norm, p2c_map, OPP_READ),
                opp_arg_dat(if_v_norm, p2c_map, OPP_READ), opp_arg_dat(if_norm_d, p2c_map, OPP_READ),
                opp_arg_dat(if_n_pos_d, p2c_map, OPP_READ), opp_arg_dat(dp_rand, OPP_READ, false));
            {
                double* vel = (double*)p_vel->data;
                const int start = particle_set->size - particle_set->diff;
                for (int k = 0; k < particle_set->diff; k++)
                    for (int d = 0; d < 3; d++) vel[(size_t)(start + k) * 3 + d] += thermal[3 * k + d];
            }
            opp_reset_dat(n_charge_den, opp_zero_double16);
            auto t1 = clk::now();
            opp_par_loop_all__calculate_new_pos_vel_kernel(particle_set, opp_arg_dat(c_ef_d, p2c_map, OPP_READ),
                                                           opp_arg_dat(p_pos, OPP_WRITE),
                                                           opp_arg_dat(p_vel, OPP_WRITE));
            auto t2 = clk::now();
            r.size_before_move = particle_set->size;
            opp_particle_move__move_kernel(particle_set, c2c_map, p2c_map, opp_arg_dat(p_pos, OPP_READ),
                                           opp_arg_dat(p_lc, OPP_WRITE), opp_arg_dat(c_volume, p2c_map, OPP_READ),
                                           opp_arg_dat(c_det_d, p2c_map, OPP_READ));
            auto t3 = clk::now();
            opp_par_loop_all__deposit_charge_on_nodes_kernel(
                particle_set, opp_arg_dat(p_lc, OPP_READ), opp_arg_dat(n_charge_den, 0, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 1, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 2, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 3, c2n_map, p2c_map, OPP_INC));
            auto t4 = clk::now();
            r.size = particle_set->size;
            r.removed = r.size_before_move - r.size;
            r.t_inject = secs(t0, t1);
            r.t_push = secs(t1, t2);
            r.t_move = secs(t2, t3);
            r.t_deposit = secs(t3, t4);
            if (h.record_state) {  // timing cases (record_state 0) skip the per-step digests
                const size_t n = (size_t)r.size;
                r.h_p2c = fnv1a(p2c_map->p2c_dat->data, n * sizeof(int));
                r.h_pos = fnv1a(p_pos->data, n * 3 * sizeof(double));
                r.h_vel = fnv1a(p_vel->data, n * 3 * sizeof(double));
                r.h_lc = fnv1a(p_lc->data, n * 4 * sizeof(double));
                r.h_charge = fnv1a(n_charge_den->data, nn * sizeof(double));
            }
            recs.push_back(r);
        }

        FILE* o = fopen(argv[3], "wb");
        if (!o) return 2;
        const int32_t nrec = (int32_t)recs.size();
        const int32_t fin = particle_set->size;
        fwrite(&nrec, sizeof nrec, 1, o);
        fwrite(recs.data(), sizeof(StepRecord), recs.size(), o);
        fwrite(&fin, sizeof fin, 1, o);
        if (h.record_state) {
            fwrite(p2c_map->p2c_dat->data, sizeof(int), (size_t)fin, o);
            fwrite(p_pos->data, sizeof(double), (size_t)fin * 3, o);
            fwrite(p_vel->data, sizeof(double), (size_t)fin * 3, o);
            fwrite(p_lc->data, sizeof(double), (size_t)fin * 4, o);
            fwrite(n_charge_den->data, sizeof(double), nn, o);
        }
        if (h.direct_hop) {  // the reference's grid: box counts, bounds and the map
            const int64_t dims[3] = {(int64_t)cellMapper->globalGridDimsX, (int64_t)cellMapper->globalGridDimsY,
                                     (int64_t)cellMapper->globalGridDimsZ};
            const opp_point& mn = boundingBox->getGlobalMin();
            const opp_point& mx = boundingBox->getGlobalMax();
            const double box[6] = {mn.x, mn.y, mn.z, mx.x, mx.y, mx.z};
            fwrite(dims, sizeof(int64_t), 3, o);
            fwrite(box, sizeof(double), 6, o);
            fwrite(cellMapper->structMeshToCellMapping, sizeof(int), cellMapper->globalGridSize, o);
        }
        fclose(o);
    }
    opp_exit();
    return 0;
}
