// TEST INFRASTRUCTURE ONLY — driver of the compiled OP-PIC reference (seq / omp backend and the
// generated NESO-advection loops of apps_codegen/app_neso_advection_mdir_cg/{seq,omp}).
//
// It declares the sets, maps, dats and constants of advec_opp.cpp through the reference's own
// API (cell_set, c2c_map, c_pos_ll, part_set, p2c_map, p_pos, p_vel, p_mdir; CONST_extents,
// CONST_dt, CONST_cell_width, CONST_ndimcells) and runs the main loop's particle part
//   opp_par_loop_all__update_pos_kernel -> opp_particle_move__move_kernel
// `steps` times, timing each step, then writes the times and the final particle dats.  A case
// of format 2 may turn on the global move: the app's set-up of advec_opp.cpp:97-103 (cell ids,
// BoundingBox(c_pos_ll, DIM, expansion (2 cell widths, 2 cell widths, 0)),
// opp_init_direct_hop_cg with the case's grid spacing; the params file sets opp_global_move
// and opp_dh_data_generate), after which the harness also writes the reference's grid (box
// counts, bounds) and its structured map.
//
//   advec_ref_harness <opp params file> <case file> <out file>
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

void opp_par_loop_all__update_pos_kernel(opp_set, opp_arg, opp_arg);
void opp_particle_move__move_kernel(opp_set, opp_map, opp_map, opp_arg, opp_arg, opp_arg);
void opp_init_direct_hop_cg(double, const opp_dat, const opp::BoundingBox&, opp_map, opp_map, opp_arg, opp_arg,
                            opp_arg);

namespace {

struct Header {
    char magic[8];
    int32_t nx, ny, n_parts, steps;
    double dt, cell_width;
};

template <typename T>
std::vector<T> read_vec(FILE* f, size_t n) {
    std::vector<T> v(n ? n : 1);
    if (n && fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "advec_ref_harness: short read\n");
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
    if (fread(&h, sizeof h, 1, f) != 1 ||
        (memcmp(h.magic, "OPPBADV1", 8) != 0 && memcmp(h.magic, "OPPBADV2", 8) != 0)) {
        fprintf(stderr, "bad case file\n");
        return 2;
    }
    // Format 2: {int32 direct_hop, int32 unused, double grid_spacing} after the header.
    int32_t dh_flags[2] = {0, 0};
    double grid_spacing = 0.0;
    if (memcmp(h.magic, "OPPBADV2", 8) == 0 &&
        (fread(dh_flags, sizeof dh_flags, 1, f) != 1 || fread(&grid_spacing, sizeof grid_spacing, 1, f) != 1)) {
        fprintf(stderr, "bad case file\n");
        return 2;
    }
    const bool direct_hop = dh_flags[0] != 0;
    const size_t nc = (size_t)h.nx * h.ny, np = h.n_parts;
    auto c2c = read_vec<int>(f, nc * 4);
    auto c_pos_ll = read_vec<double>(f, nc * 2);
    auto pos = read_vec<double>(f, np * 2);
    auto vel = read_vec<double>(f, np * 2);
    auto mdir = read_vec<int>(f, np * 2);
    auto p2c = read_vec<int>(f, np);
    fclose(f);

    char* args[2] = {argv[0], argv[1]};
    opp_init(2, args);
    std::vector<double> times;
    {
        opp_set cell_set = opp_decl_set((int)nc, "mesh_cells");
        opp_map c2c_map = opp_decl_map(cell_set, cell_set, 4, c2c.data(), "c_c_map");
        opp_dat c_pos_ll_d = opp_decl_dat(cell_set, 2, DT_REAL, c_pos_ll.data(), "c_pos_ll");
        opp_set part_set = opp_decl_particle_set("particles", cell_set);
        opp_map p2c_map = opp_decl_map(part_set, cell_set, 1, nullptr, "p_mesh_rel");
        opp_dat p_pos = opp_decl_dat(part_set, 2, DT_REAL, nullptr, "p_pos");
        opp_dat p_vel = opp_decl_dat(part_set, 2, DT_REAL, nullptr, "p_vel");
        opp_dat p_mdir = opp_decl_dat(part_set, 2, DT_INT, nullptr, "p_move_dir");

        double extents[2] = {h.nx * h.cell_width, h.ny * h.cell_width};
        int ndimcells[2] = {h.nx, h.ny};
        opp_decl_const<OPP_REAL>(2, extents, "CONST_extents");
        opp_decl_const<OPP_REAL>(1, &h.dt, "CONST_dt");
        opp_decl_const<OPP_REAL>(1, &h.cell_width, "CONST_cell_width");
        opp_decl_const<OPP_INT>(2, ndimcells, "CONST_ndimcells");

        opp_increase_particle_count(part_set, h.n_parts);
        memcpy(p_pos->data, pos.data(), np * 2 * sizeof(double));
        memcpy(p_vel->data, vel.data(), np * 2 * sizeof(double));
        memcpy(p_mdir->data, mdir.data(), np * 2 * sizeof(int));
        memcpy(p2c_map->p2c_dat->data, p2c.data(), np * sizeof(int));

        std::vector<int> c_id(nc);
        for (size_t c = 0; c < nc; c++) c_id[c] = (int)c;  // c_index of advec_misc.h's mesh
        if (direct_hop) {
            opp_dat c_idx = opp_decl_dat(cell_set, 1, DT_INT, c_id.data(), "c_index");
            const opp_point expansion(h.cell_width * 2, h.cell_width * 2, 0.0);
            const opp::BoundingBox bounding_box(c_pos_ll_d, 2, expansion);
            opp_init_direct_hop_cg(grid_spacing, c_idx, bounding_box, c2c_map, p2c_map, opp_arg_dat(p_pos, OPP_READ),
                                   opp_arg_dat(p_mdir, OPP_RW), opp_arg_dat(c_pos_ll_d, p2c_map, OPP_READ));
        }

        using clk = std::chrono::steady_clock;
        for (int s = 0; s < h.steps; s++) {
            const auto t0 = clk::now();
            opp_par_loop_all__update_pos_kernel(part_set, opp_arg_dat(p_vel, OPP_READ), opp_arg_dat(p_pos, OPP_RW));
            opp_particle_move__move_kernel(part_set, c2c_map, p2c_map, opp_arg_dat(p_pos, OPP_READ),
                                           opp_arg_dat(p_mdir, OPP_RW), opp_arg_dat(c_pos_ll_d, p2c_map, OPP_READ));
            times.push_back(std::chrono::duration<double>(clk::now() - t0).count());
        }

        FILE* o = fopen(argv[3], "wb");
        if (!o) return 2;
        const int32_t steps = h.steps, size = part_set->size;
        fwrite(&steps, sizeof steps, 1, o);
        fwrite(times.data(), sizeof(double), times.size(), o);
        fwrite(&size, sizeof size, 1, o);
        fwrite(p_pos->data, sizeof(double), (size_t)size * 2, o);
        fwrite(p_mdir->data, sizeof(int), (size_t)size * 2, o);
        fwrite(p2c_map->p2c_dat->data, sizeof(int), (size_t)size, o);
        if (direct_hop) {  // the reference's grid: box counts, bounds and the map
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
