// Text I/O of the opp_* API, one source built twice by oracle/Makefile: against the reference's
// seq backend (_ref/io_check_seq) and against this repository's include/ and libopp_b200.so
// (_ref/io_check_dropin).  Test infrastructure: tests/test_gpu_dropin_io.py runs both in the same
// directory and compares what they write.
//
//   io_check <params file> <input dir> [mode] [OPP_...=value ...]
//
// The input directory holds the text files of the decl_*_txt calls (written by the test).  The
// run writes files/io_<backend>_*.dat through opp_print_dat_to_txtfile /
// opp_print_map_to_txtfile, and opp_dump_dat's output on stdout between marker lines.
// mode "dump_int" dumps an int dat instead (the reference ends the program there).  A
// "globals" line prints the run-time globals both libraries set the same way (from the
// parameter file and the OPP_...= arguments).
#include <cstdio>
#include <string>

#include "opp_lib.h"

int main(int argc, char** argv) {
    opp_init(argc, argv);
    const std::string dir = argc > 2 ? argv[2] : ".";
    const std::string mode = argc > 3 ? argv[3] : "";
    auto in = [&](const char* f) { return dir + "/" + f; };

    opp_set nodes = opp_decl_set(9, "nodes");
    opp_set cells = opp_decl_set(7, "cells");
    opp_dat c_v1 = opp_decl_dat_txt(cells, 1, DT_REAL, in("c_v1.txt").c_str(), "c_v1");
    opp_dat c_v3 = opp_decl_dat_txt(cells, 3, DT_REAL, in("c_v3.txt").c_str(), "c_v3");
    opp_dat c_v16 = opp_decl_dat_txt(cells, 16, DT_REAL, in("c_v16.txt").c_str(), "c_v16");
    opp_dat c_i2 = opp_decl_dat_txt(cells, 2, DT_INT, in("c_i2.txt").c_str(), "c_i2");
    opp_map c2n = opp_decl_map_txt(cells, nodes, 4, in("c2n.txt").c_str(), "c2n");
    OPP_maps_base_index = 1;  // c2n1.txt holds c2n's entries plus 1
    opp_map c2n1 = opp_decl_map_txt(cells, nodes, 4, in("c2n1.txt").c_str(), "c2n1");
    OPP_maps_base_index = 0;

    opp_set parts = opp_decl_particle_set(5, "parts", cells);
    int p2c_init[5] = {3, 0, 6, 6, 1};
    opp_map p2c = opp_decl_map(parts, cells, 1, p2c_init, "p2c");
    double pv_init[10] = {1.5, -0.0, 0.0, -2.25e-300, 1e300, 3.0, -7.0, 0.1, 1.0 / 3.0, -1.0 / 3.0};
    opp_dat p_v = opp_decl_dat(parts, 2, DT_REAL, pv_init, "p_v");

    opp_print_dat_to_txtfile(c_v1, "io", "c_v1.dat");
    opp_print_dat_to_txtfile(c_v3, "io", "c_v3.dat");
    opp_print_dat_to_txtfile(c_v16, "io", "c_v16.dat");
    opp_print_dat_to_txtfile(c_i2, "io", "c_i2.dat");
    opp_print_dat_to_txtfile(p_v, "io", "p_v.dat");
    opp_print_map_to_txtfile(c2n, "io", "c2n.dat");
    opp_print_map_to_txtfile(c2n1, "io", "c2n1.dat");
    opp_print_map_to_txtfile(p2c, "io", "p2c.dat");

#ifdef IO_CHECK_FETCH  // the seq backend declares opp_fetch_data but defines it only for devices
    opp_dat f = opp_fetch_data(c_v3);
    std::printf("fetch %d %d %.17g\n", f == c_v3 ? 1 : 0, f->set->size, opp_get_data<double>(f)[4]);
#endif
    std::printf("globals %d %d %.17g %d %d\n", OPP_fill_period, OPP_move_moreX_hops, OPP_part_alloc_mult,
                OPP_mpi_part_alloc_mult, OPP_dh_data_dump ? 1 : 0);
    opp_arg hargs[2] = {opp_arg_dat(c_v3, OPP_READ), opp_arg_dat(p_v, OPP_RW)};
    std::printf("halo %d %d\n", opp_mpi_halo_exchanges_grouped(cells, 1, hargs, Device_CPU),
                opp_mpi_halo_exchanges_grouped(parts, 2, hargs, Device_GPU));
    std::printf("dump begin\n");
    std::fflush(stdout);
    opp_dump_dat(mode == "dump_int" ? c_i2 : p_v);
    std::printf("dump end\n");
    std::fflush(stdout);
    opp_exit();
    return 0;
}
