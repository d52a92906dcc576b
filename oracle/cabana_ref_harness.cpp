// TEST INFRASTRUCTURE ONLY — driver of the compiled OP-PIC reference (seq / omp backend and the
// generated CabanaPIC loops of apps_codegen/app_cabanapic_cg/{seq,omp}) on a move+deposit case.
//
// It declares the particle part of the CabanaPIC main (apps_codegen/app_cabanapic_cg/cabana_opp.cpp:
// c_set, p_set, c2ngc_map, c_interp, c_acc, p_pos, p_vel, p_streak_mid, p_weight, p2c_map and the
// CONST_* values) through the reference's own API and calls
//   opp_reset_dat(c_acc) -> opp_particle_move__move_deposit_kernel
// `calls` times with the case's fixed c_interp, as the main loop does between field updates
// (cabana_opp.cpp:158-169).  It writes the wall time of each call, the final particle dats and
// the last call's c_acc.
//
//   cabana_ref_harness <opp params file> <case file> <out file>
//
// Built by oracle/Makefile into oracle/_ref/ only; the checker of the C oracle and the CPU
// baseline, never part of the product.

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "opp_lib.h"

void opp_particle_move__move_deposit_kernel(opp_set, opp_map, opp_map, opp_arg, opp_arg, opp_arg, opp_arg,
                                            opp_arg, opp_arg);

namespace {

struct Header {
    char magic[8];
    int32_t n_cells, n_parts, calls, pad;
    double qdt_2mc, cdt_d[3], qsp, dt;
};

template <typename T>
std::vector<T> read_vec(FILE* f, size_t n) {
    std::vector<T> v(n ? n : 1);
    if (n && fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "cabana_ref_harness: short read\n");
        exit(2);
    }
    return v;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <params> <case> <out>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 2;
    Header h;
    if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, "OPPBCAB1", 8) != 0) {
        fprintf(stderr, "bad case file\n");
        return 2;
    }
    const size_t nc = h.n_cells, np = h.n_parts;
    auto c2ngc = read_vec<int>(f, nc * 6);
    auto interp = read_vec<double>(f, nc * 18);
    auto pos = read_vec<double>(f, np * 3);
    auto vel = read_vec<double>(f, np * 3);
    auto streak = read_vec<double>(f, np * 3);
    auto weight = read_vec<double>(f, np);
    auto p2c = read_vec<int>(f, np);
    fclose(f);
    std::vector<double> acc0(nc * 12, 0.0);

    char* args[2] = {argv[0], argv[1]};
    opp_init(2, args);
    std::vector<double> times;
    {
        opp_set c_set = opp_decl_set(h.n_cells, "mesh_cells");
        opp_set p_set = opp_decl_particle_set("particles", c_set);
        opp_map c2ngc_map = opp_decl_map(c_set, c_set, 6, c2ngc.data(), "c2c_non_ghost_map");
        opp_dat c_acc = opp_decl_dat(c_set, 12, DT_REAL, acc0.data(), "c_acc");
        opp_dat c_interp = opp_decl_dat(c_set, 18, DT_REAL, interp.data(), "c_interp");
        opp_dat p_pos = opp_decl_dat(p_set, 3, DT_REAL, nullptr, "p_pos");
        opp_dat p_vel = opp_decl_dat(p_set, 3, DT_REAL, nullptr, "p_vel");
        opp_dat p_streak_mid = opp_decl_dat(p_set, 3, DT_REAL, nullptr, "p_streak_mid");
        opp_dat p_weight = opp_decl_dat(p_set, 1, DT_REAL, nullptr, "p_weight");
        opp_map p2c_map = opp_decl_map(p_set, c_set, 1, nullptr, "p2c_map");

        double zero3[3] = {0.0, 0.0, 0.0}, zero = 0.0;
        opp_decl_const<OPP_REAL>(1, &h.dt, "CONST_dt");
        opp_decl_const<OPP_REAL>(1, &h.qsp, "CONST_qsp");
        opp_decl_const<OPP_REAL>(3, h.cdt_d, "CONST_cdt_d");
        opp_decl_const<OPP_REAL>(3, zero3, "CONST_p");
        opp_decl_const<OPP_REAL>(1, &h.qdt_2mc, "CONST_qdt_2mc");
        opp_decl_const<OPP_REAL>(1, &zero, "CONST_dt_eps0");
        opp_decl_const<OPP_REAL>(3, zero3, "CONST_acc_coef");

        opp_increase_particle_count(p_set, h.n_parts);
        memcpy(p_pos->data, pos.data(), np * 3 * sizeof(double));
        memcpy(p_vel->data, vel.data(), np * 3 * sizeof(double));
        memcpy(p_streak_mid->data, streak.data(), np * 3 * sizeof(double));
        memcpy(p_weight->data, weight.data(), np * sizeof(double));
        memcpy(p2c_map->p2c_dat->data, p2c.data(), np * sizeof(int));

        using clk = std::chrono::steady_clock;
        for (int k = 0; k < h.calls; k++) {
            opp_reset_dat(c_acc, opp_zero_double16);
            const auto t0 = clk::now();
            opp_particle_move__move_deposit_kernel(p_set, c2ngc_map, p2c_map, opp_arg_dat(p_vel, OPP_RW),
                                                   opp_arg_dat(p_pos, OPP_RW), opp_arg_dat(p_streak_mid, OPP_RW),
                                                   opp_arg_dat(p_weight, OPP_READ),
                                                   opp_arg_dat(c_interp, p2c_map, OPP_READ),
                                                   opp_arg_dat(c_acc, p2c_map, OPP_INC));
            times.push_back(std::chrono::duration<double>(clk::now() - t0).count());
        }

        FILE* o = fopen(argv[3], "wb");
        if (!o) return 2;
        const int32_t ncalls = h.calls, size = p_set->size;
        fwrite(&ncalls, sizeof ncalls, 1, o);
        fwrite(times.data(), sizeof(double), times.size(), o);
        fwrite(&size, sizeof size, 1, o);
        fwrite(p_pos->data, sizeof(double), (size_t)size * 3, o);
        fwrite(p_vel->data, sizeof(double), (size_t)size * 3, o);
        fwrite(p_streak_mid->data, sizeof(double), (size_t)size * 3, o);
        fwrite(p2c_map->p2c_dat->data, sizeof(int), (size_t)size, o);
        fwrite(c_acc->data, sizeof(double), nc * 12, o);
        fclose(o);
    }
    opp_exit();
    return 0;
}
