// TEST INFRASTRUCTURE ONLY — driver of the reference's generated FemPIC seq loops
// compute_node_charge_density_kernel and compute_electric_field_kernel
// (apps_codegen/app_fempic_cg/seq/, user kernels apps/app_fempic/kernels.h:178-202) on
// given inputs, through the reference's own API, as the generated main calls them
// (fempic_opp.cpp:195-215: the density loop, then opp_reset_dat(c_ef) and the field loop).
// It is the checker of the C oracle's node-side loops, never part of the product.
//
//   field_ref_harness <opp params file> <in file> <out file>
//   in:  int32 n_nodes, n_cells; f64 spwt; f64 n_charge_den[n_nodes], n_vol[n_nodes];
//        int32 c2n[n_cells*4]; f64 c_sd[n_cells*12], n_potential[n_nodes]
//   out: f64 n_charge_den[n_nodes] (after the density loop), c_ef[n_cells*3]

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "opp_lib.h"

void opp_par_loop_all__compute_node_charge_density_kernel(opp_set, opp_arg, opp_arg);
void opp_par_loop_all__compute_electric_field_kernel(opp_set, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg, opp_arg);

namespace {
template <typename T>
std::vector<T> read_vec(FILE* f, size_t n) {
    std::vector<T> v(n ? n : 1);
    if (n && fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "field_ref_harness: short read\n");
        exit(2);
    }
    return v;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <params> <in> <out>\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 2;
    int32_t hdr[2];
    double spwt = 0;
    if (fread(hdr, sizeof hdr, 1, f) != 1 || fread(&spwt, sizeof spwt, 1, f) != 1) return 2;
    const size_t nn = (size_t)hdr[0], nc = (size_t)hdr[1];
    auto den = read_vec<double>(f, nn);
    auto vol = read_vec<double>(f, nn);
    auto c2n = read_vec<int>(f, nc * 4);
    auto c_sd = read_vec<double>(f, nc * 12);
    auto pot = read_vec<double>(f, nn);
    fclose(f);
    std::vector<double> c_ef(nc * 3, 0.0);

    char* args[2] = {argv[0], argv[1]};
    opp_init(2, args);
    {
        opp_set node_set = opp_decl_set((int)nn, "mesh_nodes");
        opp_set cell_set = opp_decl_set((int)nc, "mesh_cells");
        opp_map c2n_map = opp_decl_map(cell_set, node_set, 4, c2n.data(), "c_v_n_map");
        opp_dat n_charge_den = opp_decl_dat(node_set, 1, DT_REAL, den.data(), "n_charge_den");
        opp_dat n_volume = opp_decl_dat(node_set, 1, DT_REAL, vol.data(), "n_vol");
        opp_dat n_potential = opp_decl_dat(node_set, 1, DT_REAL, pot.data(), "n_potential");
        opp_dat c_ef_d = opp_decl_dat(cell_set, 3, DT_REAL, c_ef.data(), "c_ef");
        opp_dat c_sd_d = opp_decl_dat(cell_set, 12, DT_REAL, c_sd.data(), "c_shape_deri");
        opp_decl_const<OPP_REAL>(1, &spwt, "CONST_spwt");

        opp_par_loop_all__compute_node_charge_density_kernel(node_set, opp_arg_dat(n_charge_den, OPP_RW),
                                                             opp_arg_dat(n_volume, OPP_READ));
        opp_reset_dat(c_ef_d, opp_zero_double16);
        opp_par_loop_all__compute_electric_field_kernel(
            cell_set, opp_arg_dat(c_ef_d, OPP_INC), opp_arg_dat(c_sd_d, OPP_READ),
            opp_arg_dat(n_potential, 0, c2n_map, OPP_READ), opp_arg_dat(n_potential, 1, c2n_map, OPP_READ),
            opp_arg_dat(n_potential, 2, c2n_map, OPP_READ), opp_arg_dat(n_potential, 3, c2n_map, OPP_READ));

        FILE* o = fopen(argv[3], "wb");
        if (!o) return 2;
        fwrite(n_charge_den->data, sizeof(double), nn, o);
        fwrite(c_ef_d->data, sizeof(double), nc * 3, o);
        fclose(o);
    }
    opp_exit();
    return 0;
}
