// FemPIC particle loop written against the opp_* API only, linked with libopp_b200.
//
// The structure is the generated main's (apps_codegen/app_fempic_cg/fempic_opp.cpp:80-215):
// declare sets, maps, dats and constants, then per step
//   opp_inc_part_count_with_distribution -> inject_ions -> reset n_charge_den
//   -> calculate_new_pos_vel -> opp_particle_move(move_kernel) -> deposit_charge_on_nodes.
// The field is static (the case's cell field); there is no field solve.  The mesh either
// comes from a case file (mesh arrays + per-step injection tables, the format written by
// the test drivers) or is built as a box from the parameter file (box_nx ... box_lz).
//
//   fempic_b200 <params> [case file] [out file]
//
// The out file holds per-step records (sizes, removals, FNV-1a digests of the particle
// dats, times) and the final particle state and node charges.

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "opp_fempic_solver.h"
#include "opp_lib.h"
#include "oppb_fempic.h"

void opp_par_loop_injected__inject_ions_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg,
                                               opp_arg, opp_arg, opp_arg, opp_arg);
void opp_par_loop_all__calculate_new_pos_vel_kernel(opp_set, opp_arg, opp_arg, opp_arg);
void opp_particle_move__move_kernel(opp_set, opp_map, opp_map, opp_arg, opp_arg, opp_arg, opp_arg);
void opp_par_loop_all__deposit_charge_on_nodes_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg);
void opp_init_direct_hop_cg(double, const opp_dat, const opp::BoundingBox&, opp_map, opp_map, opp_arg, opp_arg,
                            opp_arg, opp_arg);
void opp_par_loop_all__init_boundary_pot_kernel(opp_set, opp_arg, opp_arg);
void opp_par_loop_all__compute_node_charge_density_kernel(opp_set, opp_arg, opp_arg);
void opp_par_loop_all__compute_electric_field_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg);
void opp_par_loop_all__get_max_cef_kernel(opp_set, opp_arg, opp_arg);
void opp_par_loop_all__get_final_max_values_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg);

namespace {

struct CaseHeader {
    char magic[8];
    int32_t n_nodes, n_cells, n_ifaces, inject, steps, n_tables, record_state, direct_hop;
    double dt, qm, ion_velocity, sigma;
};

struct Mesh {
    int n_nodes = 0, n_cells = 0, n_ifaces = 0;
    std::vector<int> c2n, c2c, if2c, if_dist;
    std::vector<double> c_det, c_vol, c_ef, if_u, if_v, if_norm, if_n_pos;
};

template <typename T>
void read_into(std::FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n ? n : 1);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) opp_abort("case file: short read");
}

uint64_t fnv1a(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

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
    opp_init(argc, argv);
    {
        Mesh m;
        CaseHeader h{};
        std::vector<double> tables, dh_par, n_pos;
        // Field phase (an optional block tagged OPPBFLD1 at the end of the case file): node types,
        // positions and volumes, CONST_wall_potential and CONST_spwt; plasma_den and
        // electron_temperature come from the parameter file, as the reference's FESolver takes them.
        bool field = false;
        std::vector<int> f_type;
        std::vector<double> f_pos, f_vol, f_par;
        if (argc >= 3) {
            std::FILE* f = std::fopen(argv[2], "rb");
            if (!f || std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, "OPPBCAS1", 8) != 0)
                opp_abort("bad case file");
            m.n_nodes = h.n_nodes, m.n_cells = h.n_cells, m.n_ifaces = h.n_ifaces;
            const size_t nc = m.n_cells, nf = m.n_ifaces;
            read_into(f, m.c2n, nc * 4);
            read_into(f, m.c2c, nc * 4);
            read_into(f, m.c_det, nc * 16);
            read_into(f, m.c_vol, nc);
            read_into(f, m.c_ef, nc * 3);
            read_into(f, m.if2c, nf);
            read_into(f, m.if_u, nf * 3);
            read_into(f, m.if_v, nf * 3);
            read_into(f, m.if_norm, nf * 3);
            read_into(f, m.if_n_pos, nf * 9);
            read_into(f, m.if_dist, nf);
            read_into(f, tables, (size_t)h.n_tables * h.inject * 5);
            if (h.direct_hop) {  // grid spacing, expansion[3], node positions [n_nodes][3]
                read_into(f, dh_par, 4);
                read_into(f, n_pos, (size_t)m.n_nodes * 3);
            }
            char tag[8];
            if (std::fread(tag, 1, 8, f) == 8 && std::memcmp(tag, "OPPBFLD1", 8) == 0) {
                field = true;
                read_into(f, f_type, (size_t)m.n_nodes);
                read_into(f, f_pos, (size_t)m.n_nodes * 3);
                read_into(f, f_vol, (size_t)m.n_nodes);
                read_into(f, f_par, 2);  // wall_potential, spwt
            }
            std::fclose(f);
        } else {
            // Box mesh and static field from the parameter file.
            oppb_fempic_mesh bm{};
            const int nx = opp_params->get<OPP_INT>("box_nx"), ny = opp_params->get<OPP_INT>("box_ny"),
                      nz = opp_params->get<OPP_INT>("box_nz");
            if (oppb_fempic_box_mesh(nx, ny, nz, opp_params->get<OPP_REAL>("box_lx"), opp_params->get<OPP_REAL>("box_ly"),
                                     opp_params->get<OPP_REAL>("box_lz"), &bm) != 0)
                opp_abort("box mesh");
            if (oppb_fempic_solve_field(&bm, 1.0, 0.0, 1e-12, 100000, nullptr, nullptr, nullptr) != 0)
                opp_abort("field solve");
            m.n_nodes = bm.n_nodes, m.n_cells = bm.n_cells, m.n_ifaces = bm.n_ifaces;
            m.c2n.assign(bm.c2n, bm.c2n + 4 * (size_t)bm.n_cells);
            m.c2c.assign(bm.c2c, bm.c2c + 4 * (size_t)bm.n_cells);
            m.c_det.assign(bm.c_det, bm.c_det + 16 * (size_t)bm.n_cells);
            m.c_vol.assign(bm.c_vol, bm.c_vol + (size_t)bm.n_cells);
            m.c_ef.assign(bm.c_ef, bm.c_ef + 3 * (size_t)bm.n_cells);
            m.if2c.assign(bm.if2c, bm.if2c + bm.n_ifaces);
            m.if_u.assign(bm.if_u, bm.if_u + 3 * (size_t)bm.n_ifaces);
            m.if_v.assign(bm.if_v, bm.if_v + 3 * (size_t)bm.n_ifaces);
            m.if_norm.assign(bm.if_norm, bm.if_norm + 3 * (size_t)bm.n_ifaces);
            m.if_n_pos.assign(bm.if_n_pos, bm.if_n_pos + 9 * (size_t)bm.n_ifaces);
            h.inject = opp_params->get<OPP_INT>("inject_per_step");
            h.steps = opp_params->get<OPP_INT>("num_steps");
            h.dt = opp_params->get<OPP_REAL>("dt");
            h.qm = 1.0;
            h.ion_velocity = opp_params->get<OPP_REAL>("ion_velocity");
            h.sigma = opp_params->get<OPP_REAL>("thermal_sigma");
            m.if_dist.resize(bm.n_ifaces);
            oppb_fempic_inject_distribution(&bm, h.inject, m.if_dist.data());
            oppb_fempic_mesh_free(&bm);
        }

        opp_set node_set = opp_decl_set(m.n_nodes, "mesh_nodes");
        opp_set cell_set = opp_decl_set(m.n_cells, "mesh_cells");
        opp_set iface_set = opp_decl_set(m.n_ifaces, "inlet_faces_cells");
        opp_set particle_set = opp_decl_particle_set("particles", cell_set);
        opp_set dummy_part_set = opp_decl_particle_set("dummy particles", cell_set);

        opp_map c2n_map = opp_decl_map(cell_set, node_set, 4, m.c2n.data(), "c_v_n_map");
        opp_map c2c_map = opp_decl_map(cell_set, cell_set, 4, m.c2c.data(), "c_v_c_map");
        opp_map if2c_map = opp_decl_map(iface_set, cell_set, 1, m.if2c.data(), "if_v_c_map");

        opp_dat c_det = opp_decl_dat(cell_set, 16, DT_REAL, m.c_det.data(), "c_det");
        opp_dat c_volume = opp_decl_dat(cell_set, 1, DT_REAL, m.c_vol.data(), "c_volume");
        opp_dat c_ef = opp_decl_dat(cell_set, 3, DT_REAL, m.c_ef.data(), "c_ef");
        std::vector<double> zeros((size_t)m.n_nodes, 0.0);
        opp_dat n_charge_den = opp_decl_dat(node_set, 1, DT_REAL, zeros.data(), "n_charge_den");
        opp_dat if_v_norm = opp_decl_dat(iface_set, 3, DT_REAL, m.if_v.data(), "iface_v_norm");
        opp_dat if_u_norm = opp_decl_dat(iface_set, 3, DT_REAL, m.if_u.data(), "iface_u_norm");
        opp_dat if_norm = opp_decl_dat(iface_set, 3, DT_REAL, m.if_norm.data(), "iface_norm");
        opp_dat if_distrib = opp_decl_dat(iface_set, 1, DT_INT, m.if_dist.data(), "iface_dist");
        opp_dat if_n_pos = opp_decl_dat(iface_set, 9, DT_REAL, m.if_n_pos.data(), "iface_n_pos");

        opp_dat p_pos = opp_decl_dat(particle_set, 3, DT_REAL, nullptr, "p_position");
        opp_dat p_vel = opp_decl_dat(particle_set, 3, DT_REAL, nullptr, "p_velocity");
        opp_dat p_lc = opp_decl_dat(particle_set, 4, DT_REAL, nullptr, "p_lc");
        opp_map p2c_map = opp_decl_map(particle_set, cell_set, 1, nullptr, "p2c_map");
        // Injection table: (a, b, thermal vx, vy, vz) per injected particle, refreshed each step.
        opp_dat dp_rand = opp_decl_dat(dummy_part_set, 5, DT_REAL, nullptr, "dummy_part_rand");

        // Global move (opp_global_move in the parameter file): the app's direct-hop set-up
        // (fempic_opp.cpp:69-76,95,147-153) with the case's grid spacing and expansion.
        if (h.direct_hop) {
            std::vector<int> c_id((size_t)m.n_cells);
            for (int c = 0; c < m.n_cells; c++) c_id[(size_t)c] = c;
            opp_dat n_pos_d = opp_decl_dat(node_set, 3, DT_REAL, n_pos.data(), "n_pos");
            opp_dat c_gbl_id = opp_decl_dat(cell_set, 1, DT_INT, c_id.data(), "c_gbl_id");
            opp::BoundingBox bounding_box(n_pos_d, 3, opp_point(dh_par[1], dh_par[2], dh_par[3]));
            opp_init_direct_hop_cg(dh_par[0], c_gbl_id, bounding_box, c2c_map, p2c_map, opp_arg_dat(p_pos, OPP_READ),
                                   opp_arg_dat(p_lc, OPP_WRITE), opp_arg_dat(c_volume, p2c_map, OPP_READ),
                                   opp_arg_dat(c_det, p2c_map, OPP_READ));
        }


        double one = 1.0, zero = 0.0;
        double spwt = field ? f_par[1] : 0.0, wall = field ? f_par[0] : 0.0;
        opp_decl_const<OPP_REAL>(1, &spwt, "CONST_spwt");
        opp_decl_const<OPP_REAL>(1, &wall, "CONST_wall_potential");
        opp_decl_const<OPP_REAL>(1, &h.ion_velocity, "CONST_ion_velocity");
        opp_decl_const<OPP_REAL>(1, &h.dt, "CONST_dt");
        opp_decl_const<OPP_REAL>(1, &one, "CONST_mass");
        opp_decl_const<OPP_REAL>(1, &h.qm, "CONST_charge");

        // The reference main's field set-up (fempic_opp.cpp:101-110,139-141,155-156).
        opp_dat n_type_d = nullptr, n_pos_f = nullptr, n_volume = nullptr, n_bnd_pot = nullptr, n_potential = nullptr;
        opp_dat c_sd = nullptr;
        std::unique_ptr<FESolver> field_solver;
        std::vector<double> zeros_n((size_t)m.n_nodes, 0.0), zeros_sd((size_t)m.n_cells * 12, 0.0);
        if (field) {
            n_type_d = opp_decl_dat(node_set, 1, DT_INT, f_type.data(), "n_type");
            n_pos_f = opp_decl_dat(node_set, 3, DT_REAL, f_pos.data(), "n_pos_field");
            n_volume = opp_decl_dat(node_set, 1, DT_REAL, f_vol.data(), "n_vol");
            n_bnd_pot = opp_decl_dat(node_set, 1, DT_REAL, zeros_n.data(), "n_bnd_pot");
            n_potential = opp_decl_dat(node_set, 1, DT_REAL, zeros_n.data(), "n_potential");
            c_sd = opp_decl_dat(cell_set, 12, DT_REAL, zeros_sd.data(), "c_shape_deri");
            opp_par_loop_all__init_boundary_pot_kernel(node_set, opp_arg_dat(n_type_d, OPP_READ),
                                                       opp_arg_dat(n_bnd_pot, OPP_WRITE));
            field_solver = std::make_unique<FESolver>(c2n_map, n_type_d, n_pos_f, n_bnd_pot);
            field_solver->enrich_cell_shape_deriv(c_sd);
        }

        opp_increase_particle_count(dummy_part_set, h.inject);
        std::vector<StepRecord> recs;
        uint64_t rng = 0x5eedull;
        using clk = std::chrono::steady_clock;
        auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };

        for (OPP_main_loop_iter = 0; OPP_main_loop_iter < h.steps; OPP_main_loop_iter++) {
            const int s = OPP_main_loop_iter;
            double* dr = reinterpret_cast<double*>(dp_rand->data);
            for (int k = 0; k < h.inject; k++) {
                if (s < h.n_tables) {
                    std::memcpy(dr + 5 * (size_t)k, tables.data() + ((size_t)s * h.inject + k) * 5, 5 * sizeof(double));
                } else {
                    dr[5 * k] = unif(rng);
                    dr[5 * k + 1] = unif(rng);
                    for (int d = 0; d < 3; d++) {
                        const double u1 = unif(rng) + 1e-300, u2 = unif(rng);
                        dr[5 * k + 2 + d] = h.sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                    }
                }
            }
            dp_rand->dirty_hd = Device;  // host copy is the newer one: upload before device use

            StepRecord r{};
            r.step = s;
            auto t0 = clk::now();
            opp_inc_part_count_with_distribution(particle_set, h.inject, if_distrib, false);
            opp_par_loop_injected__inject_ions_kernel(
                particle_set, opp_arg_dat(p_pos, OPP_WRITE), opp_arg_dat(p_vel, OPP_WRITE),
                opp_arg_dat(p2c_map, OPP_RW), opp_arg_dat(if2c_map, p2c_map, OPP_READ),
                opp_arg_dat(c_ef, 0, if2c_map, p2c_map, OPP_READ), opp_arg_dat(if_u_norm, p2c_map, OPP_READ),
                opp_arg_dat(if_v_norm, p2c_map, OPP_READ), opp_arg_dat(if_norm, p2c_map, OPP_READ),
                opp_arg_dat(if_n_pos, p2c_map, OPP_READ), opp_arg_dat(dp_rand, OPP_READ, false));
            opp_reset_dat(n_charge_den, opp_zero_double16);
            auto t1 = clk::now();
            opp_par_loop_all__calculate_new_pos_vel_kernel(particle_set, opp_arg_dat(c_ef, p2c_map, OPP_READ),
                                                           opp_arg_dat(p_pos, OPP_WRITE), opp_arg_dat(p_vel, OPP_WRITE));
            auto t2 = clk::now();
            r.size_before_move = particle_set->size;
            opp_particle_move__move_kernel(particle_set, c2c_map, p2c_map, opp_arg_dat(p_pos, OPP_READ),
                                           opp_arg_dat(p_lc, OPP_WRITE), opp_arg_dat(c_volume, p2c_map, OPP_READ),
                                           opp_arg_dat(c_det, p2c_map, OPP_READ));
            auto t3 = clk::now();
            opp_par_loop_all__deposit_charge_on_nodes_kernel(
                particle_set, opp_arg_dat(p_lc, OPP_READ), opp_arg_dat(n_charge_den, 0, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 1, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 2, c2n_map, p2c_map, OPP_INC),
                opp_arg_dat(n_charge_den, 3, c2n_map, p2c_map, OPP_INC));
            if (field) {  // fempic_opp.cpp:195-231
                opp_par_loop_all__compute_node_charge_density_kernel(node_set, opp_arg_dat(n_charge_den, OPP_RW),
                                                                     opp_arg_dat(n_volume, OPP_READ));
                field_solver->compute_phi(opp_arg_dat(n_potential, OPP_WRITE), opp_arg_dat(n_charge_den, OPP_READ),
                                          opp_arg_dat(n_bnd_pot, OPP_READ));
                opp_reset_dat(c_ef, opp_zero_double16);
                opp_par_loop_all__compute_electric_field_kernel(
                    cell_set, opp_arg_dat(c_ef, OPP_INC), opp_arg_dat(c_sd, OPP_READ),
                    opp_arg_dat(n_potential, 0, c2n_map, OPP_READ), opp_arg_dat(n_potential, 1, c2n_map, OPP_READ),
                    opp_arg_dat(n_potential, 2, c2n_map, OPP_READ), opp_arg_dat(n_potential, 3, c2n_map, OPP_READ));
                if (opp_params->get<OPP_BOOL>("print_final")) {
                    double max_cef = 0.0, max_den = 0.0, max_pot = 0.0;
                    opp_par_loop_all__get_max_cef_kernel(cell_set, opp_arg_dat(c_ef, OPP_READ),
                                                         opp_arg_gbl(&max_cef, 1, "double", OPP_MAX));
                    opp_par_loop_all__get_final_max_values_kernel(
                        node_set, opp_arg_dat(n_charge_den, OPP_READ), opp_arg_gbl(&max_den, 1, "double", OPP_MAX),
                        opp_arg_dat(n_potential, OPP_READ), opp_arg_gbl(&max_pot, 1, "double", OPP_MAX));
                    opp_printf("Main", "ts: %d max_c_ef %2.15lE max_n_pot %2.15lE max_n_chg_den %2.15lE cg %d", s,
                               max_cef, max_pot, max_den, field_solver->last_iterations());
                }
            }
            auto t4 = clk::now();
            r.size = particle_set->size;
            r.removed = r.size_before_move - r.size;
            r.t_inject = secs(t0, t1), r.t_push = secs(t1, t2), r.t_move = secs(t2, t3), r.t_deposit = secs(t3, t4);
            if (h.record_state) {
                const size_t n = (size_t)r.size;
                r.h_p2c = fnv1a(opp_get_data<int>(p2c_map->p2c_dat), n * sizeof(int));
                r.h_pos = fnv1a(opp_get_data<double>(p_pos), n * 3 * sizeof(double));
                r.h_vel = fnv1a(opp_get_data<double>(p_vel), n * 3 * sizeof(double));
                r.h_lc = fnv1a(opp_get_data<double>(p_lc), n * 4 * sizeof(double));
                r.h_charge = 0;  // FP64 atomics: order-dependent bits, compared with a tolerance instead
            }
            recs.push_back(r);
            OPP_RUN_ON_ROOT(&& h.record_state == 0)
            opp_printf("Main", "ts: %d np %d removed %d", s, r.size, r.removed);
        }

        if (argc >= 4) {
            std::FILE* o = std::fopen(argv[3], "wb");
            if (!o) opp_abort("cannot write output");
            const int32_t nrec = (int32_t)recs.size(), fin = particle_set->size;
            std::fwrite(&nrec, sizeof nrec, 1, o);
            std::fwrite(recs.data(), sizeof(StepRecord), recs.size(), o);
            std::fwrite(&fin, sizeof fin, 1, o);
            if (h.record_state) {
                std::fwrite(opp_get_data<int>(p2c_map->p2c_dat), sizeof(int), (size_t)fin, o);
                std::fwrite(opp_get_data<double>(p_pos), sizeof(double), (size_t)fin * 3, o);
                std::fwrite(opp_get_data<double>(p_vel), sizeof(double), (size_t)fin * 3, o);
                std::fwrite(opp_get_data<double>(p_lc), sizeof(double), (size_t)fin * 4, o);
                std::fwrite(opp_get_data<double>(n_charge_den), sizeof(double), (size_t)m.n_nodes, o);
            }
            std::fclose(o);
        }
    }
    opp_exit();
    return 0;
}
