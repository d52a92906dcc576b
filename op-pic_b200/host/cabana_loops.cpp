// CabanaPIC's generated-loop entry points on the library's kernels (include/oppb_cabana.h), for
// one unpartitioned mesh: the functions the generated main
// apps_codegen/app_cabanapic_cg/cabana_opp.cpp:40-48 declares.  They replace the bodies of
// apps_codegen/app_cabanapic_cg/cuda/*_loop.hpp: the particle move + current deposit
// (oppb_cabana_move_deposit) and the cell loops of the field update.  An indirect argument
// (dat, idx, map) reads the dat at the map's idx-th entry of each cell: its column of the map's
// device copy is passed to the kernel.  The constants come from the main's opp_decl_const calls
// (CONST_qdt_2mc, CONST_cdt_d, CONST_qsp, CONST_p, CONST_dt_eps0, CONST_acc_coef).
#include <algorithm>
#include <initializer_list>
#include <string>
#include <utility>

#include "opp_lib.h"
#include "oppb_cabana.h"
#include "oppb_field.h"

namespace {

void check(int rc, const char* what) {
    if (rc != OPPB_OK) opp_abort(std::string(what) + ": " + oppb_status_string(rc));
}
void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) opp_abort(std::string(what) + ": " + cudaGetErrorString(e));
}

double cst(const char* name, int k = 0) { return opp_get_const(name, k); }

int64_t cell_stride(opp_set s) { return std::max(s->size, 1); }

double* ddat(const opp_arg& a) { return reinterpret_cast<double*>(a.dat->data_d); }
const int32_t* idat(const opp_arg& a) { return reinterpret_cast<const int32_t*>(a.dat->data_d); }

// The column of an indirect argument's map: the cell each cell reads through it.
const int32_t* column(const opp_arg& a) {
    if (!a.map || a.idx < 0 || a.idx >= a.map->dim) opp_abort("cabana loops: an argument needs a map entry");
    return a.map->map_d + (int64_t)a.idx * a.map->from->size;
}

// Device copies current for the arguments that are read; the written ones marked.
void prepare(std::initializer_list<const opp_arg*> args) {
    for (const opp_arg* a : args)
        if (a->argtype == OPP_ARG_DAT && a->dat) oppb_rt::sync_host_to_device(a->dat);
}
void written(std::initializer_list<const opp_arg*> args) {
    for (const opp_arg* a : args) oppb_rt::mark_device_written(a->dat);
}
void finish(const char* name) {
    check_cuda(cudaStreamSynchronize(oppb_rt::stream()), name);
    opp_profiler->end(name);
}

struct HexMesh {
    opp_map c2ngc = nullptr;  // the map packed into c2f, in the runtime generation `generation`
    int generation = -1;
    int32_t n_cells = 0;
    int32_t* c2f = nullptr;
    double* interp = nullptr;
    double* scalar = nullptr;   // the energy sum
    void* partial = nullptr;    // the energy's block partials
};
HexMesh& hex() {
    static HexMesh h;
    return h;
}

}  // namespace

// interpolate_mesh_fields_kernel (cuda/interpolate_mesh_fields_kernel_loop.hpp).
void opp_par_loop_all__interpolate_mesh_fields_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                                                      opp_arg arg3, opp_arg arg4, opp_arg arg5, opp_arg arg6,
                                                      opp_arg arg7, opp_arg arg8, opp_arg arg9, opp_arg arg10,
                                                      opp_arg arg11, opp_arg arg12) {
    opp_profiler->start("interpolate_mesh_fields_kernel");
    prepare({&arg0, &arg1, &arg11, &arg12});
    const int32_t* nb_e[6] = {column(arg2), column(arg3), column(arg4), column(arg5), column(arg6), column(arg7)};
    const int32_t* nb_b[3] = {column(arg8), column(arg9), column(arg10)};
    check(oppb_cabana_interpolate(set->size, cell_stride(set), ddat(arg0), ddat(arg1), nb_e, nb_b, ddat(arg11),
                                  idat(arg12), oppb_rt::stream()),
          "oppb_cabana_interpolate");
    written({&arg11});
    finish("interpolate_mesh_fields_kernel");
}

// move_deposit_kernel (cuda/move_deposit_kernel_loop.hpp:305-358): the Boris push, the streak
// walk through c2ngc_map and the current deposit into c_acc, then the finalize.
void opp_particle_move__move_deposit_kernel(opp_set set, opp_map c2c_map, opp_map p2c_map, opp_arg arg0,
                                            opp_arg arg1, opp_arg arg2, opp_arg arg3, opp_arg arg4, opp_arg arg5) {
    opp_profiler->start("move_deposit_kernel");
    opp_set cells = c2c_map->from;
    if (c2c_map->dim != 6 || p2c_map->p2c_dat != set->mesh_relation_dat || arg4.dat->dim != 18 ||
        arg5.dat->dim != 12 || arg4.dat->set != cells || arg5.dat->set != cells)
        opp_abort("opp_particle_move__move_deposit_kernel: unexpected arguments");
    opp_init_particle_move(set, 0, nullptr);
    prepare({&arg0, &arg1, &arg2, &arg3, &arg4, &arg5});
    oppb_rt::sync_host_to_device(set->mesh_relation_dat);
    HexMesh& h = hex();
    cudaStream_t s = oppb_rt::stream();
    const int32_t n = cells->size;
    if (h.n_cells != n) {
        cudaFree(h.c2f);
        cudaFree(h.interp);
        const size_t cells_alloc = (size_t)std::max(n, 1);
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&h.c2f), sizeof(int32_t) * 8 * cells_alloc), "cudaMalloc c2f");
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&h.interp), sizeof(double) * 20 * cells_alloc),
                   "cudaMalloc interp");
        h.n_cells = n;
        h.c2ngc = nullptr;
    }
    oppb_hex_mesh mesh{n, h.c2f, h.interp, nullptr};
    const bool packed = h.c2ngc == c2c_map && h.generation == oppb_rt::generation();
    check(oppb_hex_mesh_pack(&mesh, n, packed ? nullptr : c2c_map->map_d, ddat(arg4), s), "oppb_hex_mesh_pack");
    h.c2ngc = c2c_map;
    h.generation = oppb_rt::generation();
    oppb_cabana_particles p{set->size,
                            std::max(set->set_capacity, 1),
                            ddat(arg1),
                            ddat(arg0),
                            ddat(arg2),
                            ddat(arg3),
                            reinterpret_cast<int32_t*>(set->mesh_relation_dat->data_d)};
    oppb_cabana_consts c{cst("CONST_qdt_2mc"), {cst("CONST_cdt_d", 0), cst("CONST_cdt_d", 1), cst("CONST_cdt_d", 2)},
                         cst("CONST_qsp")};
    oppb_move_status* st = oppb_rt::move_status();
    check_cuda(cudaMemsetAsync(st, 0, sizeof(oppb_move_status), s), "status reset");
    check(oppb_cabana_move_deposit(&mesh, &p, &c, ddat(arg5), n, st, oppb_rt::max_hops(), s),
          "oppb_cabana_move_deposit");
    written({&arg0, &arg1, &arg2, &arg5});
    oppb_rt::mark_device_written(set->mesh_relation_dat);
    while (opp_finalize_particle_move(set)) {
    }
    opp_profiler->end("move_deposit_kernel");
}

// accumulate_current_to_cells_kernel (cuda/accumulate_current_to_cells_kernel_loop.hpp).
void opp_par_loop_all__accumulate_current_to_cells_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                                                          opp_arg arg3, opp_arg arg4, opp_arg arg5, opp_arg arg6,
                                                          opp_arg arg7, opp_arg arg8) {
    opp_profiler->start("accumulate_current_to_cells_kernel");
    prepare({&arg0, &arg1, &arg8});
    const int32_t* nb[6] = {column(arg2), column(arg3), column(arg4), column(arg5), column(arg6), column(arg7)};
    const double coef[3] = {cst("CONST_acc_coef", 0), cst("CONST_acc_coef", 1), cst("CONST_acc_coef", 2)};
    check(oppb_cabana_accumulate(set->size, cell_stride(set), ddat(arg0), ddat(arg1), nb, idat(arg8), coef,
                                 oppb_rt::stream()),
          "oppb_cabana_accumulate");
    written({&arg0});
    finish("accumulate_current_to_cells_kernel");
}

// half_advance_b_kernel (cuda/half_advance_b_kernel_loop.hpp).
void opp_par_loop_all__half_advance_b_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3,
                                             opp_arg arg4, opp_arg arg5) {
    opp_profiler->start("half_advance_b_kernel");
    prepare({&arg3, &arg4, &arg5});
    const int32_t* nb[3] = {column(arg0), column(arg1), column(arg2)};
    const double p[3] = {cst("CONST_p", 0), cst("CONST_p", 1), cst("CONST_p", 2)};
    check(oppb_cabana_half_advance_b(set->size, cell_stride(set), nb, ddat(arg3), ddat(arg4), idat(arg5), p,
                                     oppb_rt::stream()),
          "oppb_cabana_half_advance_b");
    written({&arg4});
    finish("half_advance_b_kernel");
}

// update_ghosts_B_kernel (cuda/update_ghosts_B_kernel_loop.hpp): the dat copied to the ghost
// cells of the map, for the cells whose c_mask_ugb holds 1 at the index global.
void opp_par_loop_all__update_ghosts_B_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3) {
    opp_profiler->start("update_ghosts_B_kernel");
    prepare({&arg0, &arg1, &arg2});
    check(oppb_cabana_update_ghosts(set->size, cell_stride(set), idat(arg0), *reinterpret_cast<int*>(arg3.data),
                                    ddat(arg1), ddat(arg2), column(arg2), -1, oppb_rt::stream()),
          "oppb_cabana_update_ghosts");
    written({&arg2});
    finish("update_ghosts_B_kernel");
}

// update_ghosts_kernel (cuda/update_ghosts_kernel_loop.hpp): one component added to the cells of
// the map, for the cells whose c_mask_ug holds 1 at the index global.
void opp_par_loop_all__update_ghosts_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3,
                                            opp_arg arg4) {
    opp_profiler->start("update_ghosts_kernel");
    prepare({&arg0, &arg1, &arg2});
    check(oppb_cabana_update_ghosts(set->size, cell_stride(set), idat(arg0), *reinterpret_cast<int*>(arg3.data),
                                    ddat(arg1), ddat(arg2), column(arg2), *reinterpret_cast<int*>(arg4.data),
                                    oppb_rt::stream()),
          "oppb_cabana_update_ghosts");
    written({&arg2});
    finish("update_ghosts_kernel");
}

// advance_e_kernel (cuda/advance_e_kernel_loop.hpp).
void opp_par_loop_all__advance_e_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3,
                                        opp_arg arg4, opp_arg arg5, opp_arg arg6) {
    opp_profiler->start("advance_e_kernel");
    prepare({&arg3, &arg4, &arg5, &arg6});
    const int32_t* nb[3] = {column(arg0), column(arg1), column(arg2)};
    const double p[3] = {cst("CONST_p", 0), cst("CONST_p", 1), cst("CONST_p", 2)};
    check(oppb_cabana_advance_e(set->size, cell_stride(set), nb, ddat(arg3), ddat(arg4), ddat(arg5), idat(arg6), p,
                                cst("CONST_dt_eps0"), oppb_rt::stream()),
          "oppb_cabana_advance_e");
    written({&arg5});
    finish("advance_e_kernel");
}

// compute_energy_kernel (cuda/compute_energy_kernel_loop.hpp): the OPP_INC double global
// receives the sum over the non-ghost cells.
void opp_par_loop_all__compute_energy_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2) {
    opp_profiler->start("compute_energy_kernel");
    prepare({&arg0, &arg1});
    HexMesh& h = hex();
    cudaStream_t s = oppb_rt::stream();
    if (!h.scalar) {
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&h.scalar), sizeof(double)), "cudaMalloc energy");
        check_cuda(cudaMalloc(&h.partial, oppb_cabana_energy_workspace_bytes()), "cudaMalloc energy partials");
    }
    check_cuda(cudaMemsetAsync(h.scalar, 0, sizeof(double), s), "energy reset");
    check(oppb_cabana_energy(set->size, cell_stride(set), idat(arg0), ddat(arg1), h.scalar, h.partial,
                             oppb_cabana_energy_workspace_bytes(), s),
          "oppb_cabana_energy");
    double sum = 0.0;
    check_cuda(cudaMemcpyAsync(&sum, h.scalar, sizeof sum, cudaMemcpyDeviceToHost, s), "energy read");
    finish("compute_energy_kernel");
    *reinterpret_cast<double*>(arg2.data) += sum;
}

// get_max_x_values_kernel (cuda/get_max_x_values_kernel_loop.hpp): each OPP_MAX global becomes the
// larger of itself and the largest x component of its dat over the cells.
void opp_par_loop_all__get_max_x_values_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3,
                                               opp_arg arg4, opp_arg arg5) {
    opp_profiler->start("get_max_x_values_kernel");
    prepare({&arg0, &arg2, &arg4});
    for (auto [dat, gbl] : {std::pair<opp_arg*, opp_arg*>{&arg0, &arg1}, {&arg2, &arg3}, {&arg4, &arg5}}) {
        double* out = reinterpret_cast<double*>(gbl->data);
        check(oppb_reduce_max(ddat(*dat), set->size, 0, *out, out, oppb_rt::stream()), "oppb_reduce_max");
    }
    opp_profiler->end("get_max_x_values_kernel");
}
