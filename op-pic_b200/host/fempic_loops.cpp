// The FemPIC generated-loop entry points (apps_codegen/app_fempic_cg/fempic_opp.cpp:40-49
// declares them with C++ linkage) on the B200 backend.  Each one replaces the body of the
// reference's generated CUDA loop with the launchers of oppb.h; argument order and access
// modes are the generated code's.

#include <cuda_runtime.h>

#include <algorithm>

#include "opp_lib.h"
#include "oppb_dh.h"
#include "oppb_fempic.h"
#include "oppb_field.h"

namespace {

void check(int rc, const char* what) {
    if (rc != OPPB_OK) opp_abort(std::string(what) + ": " + oppb_status_string(rc));
}

oppb_particles particles(opp_set set, opp_dat pos, opp_dat vel, opp_dat lc) {
    oppb_particles p{};
    p.size = set->size;
    p.stride = set->set_capacity > 0 ? set->set_capacity : 1;
    p.pos = pos ? reinterpret_cast<double*>(pos->data_d) : nullptr;
    p.vel = vel ? reinterpret_cast<double*>(vel->data_d) : nullptr;
    p.lc = lc ? reinterpret_cast<double*>(lc->data_d) : nullptr;
    p.p2c = reinterpret_cast<int32_t*>(set->mesh_relation_dat->data_d);
    p.remove_bits = oppb_rt::remove_bits(set);
    return p;
}

double charge_over_mass() { return opp_get_const("CONST_charge") / opp_get_const("CONST_mass"); }

// The global move's structured grid, set up by opp_init_direct_hop_cg when opp_global_move is on,
// for the run (the runtime generation) it was built in.
struct DirectHop {
    bool on = false;
    int generation = -1;
    oppb_dh_grid grid{};
} g_dh;

// Inlet geometry record [n_faces][12] = u, v, normal, node0, packed from the iface dats.
struct InletCache {
    opp_dat u = nullptr, v = nullptr, n = nullptr, np = nullptr;
    uint64_t ver = 0;
    double* geom = nullptr;
    int n_faces = 0;
} g_inlet;

const double* inlet_geom(opp_dat u, opp_dat v, opp_dat nrm, opp_dat npos) {
    const uint64_t ver = u->version + v->version + nrm->version + npos->version;
    if (g_inlet.geom && g_inlet.u == u && g_inlet.v == v && g_inlet.n == nrm && g_inlet.np == npos &&
        g_inlet.ver == ver)
        return g_inlet.geom;
    opp_download_dat(u);
    opp_download_dat(v);
    opp_download_dat(nrm);
    opp_download_dat(npos);
    const int nf = u->set->size;
    std::vector<double> h((size_t)nf * 12);
    for (int f = 0; f < nf; f++)
        for (int d = 0; d < 3; d++) {
            h[(size_t)f * 12 + d] = reinterpret_cast<double*>(u->data)[f * 3 + d];
            h[(size_t)f * 12 + 3 + d] = reinterpret_cast<double*>(v->data)[f * 3 + d];
            h[(size_t)f * 12 + 6 + d] = reinterpret_cast<double*>(nrm->data)[f * 3 + d];
            h[(size_t)f * 12 + 9 + d] = reinterpret_cast<double*>(npos->data)[f * 9 + d];
        }
    if (g_inlet.geom && g_inlet.n_faces < nf) {
        cudaFree(g_inlet.geom);
        g_inlet.geom = nullptr;
    }
    if (!g_inlet.geom && cudaMalloc(&g_inlet.geom, h.size() * sizeof(double)) != cudaSuccess)
        opp_abort("cudaMalloc inlet");
    if (cudaMemcpy(g_inlet.geom, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        opp_abort("inlet upload");
    g_inlet = InletCache{u, v, nrm, npos, ver, g_inlet.geom, nf};
    return g_inlet.geom;
}

}  // namespace

// inject_ions_kernel over the injected particles [size - diff, size).
void opp_par_loop_injected__inject_ions_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2, opp_arg arg3,
                                               opp_arg arg4, opp_arg arg5, opp_arg arg6, opp_arg arg7, opp_arg arg8,
                                               opp_arg arg9) {
    opp_profiler->start("inject_ions_kernel");
    (void)arg2;
    opp_dat c_ef = arg4.dat, rnd = arg9.dat;
    oppb_rt::sync_host_to_device(rnd);
    const oppb_tet_mesh& mesh = oppb_rt::tet_mesh(nullptr, nullptr, nullptr, nullptr, c_ef);
    // arg3 is the if2c map read through p2c: the face index the distribution left in p2c.
    const oppb_inlet inlet{arg5.dat->set->size, nullptr, arg3.map_data_d ? arg3.map_data_d : nullptr,
                           inlet_geom(arg5.dat, arg6.dat, arg7.dat, arg8.dat)};
    if (!inlet.if2c) opp_abort("inject_ions_kernel: if2c map has no device copy");
    oppb_particles p = particles(set, arg0.dat, arg1.dat, nullptr);
    const int rstride = rnd->set->is_particle ? rnd->set->set_capacity : rnd->set->size;
    check(oppb_inject_f64(&mesh, &inlet, &p, set->size - set->diff, set->diff,
                          reinterpret_cast<const double*>(rnd->data_d), rstride, rnd->dim,
                          opp_get_const("CONST_ion_velocity"), charge_over_mass(), opp_get_const("CONST_dt"),
                          oppb_rt::stream()),
          "oppb_inject_f64");
    oppb_rt::mark_device_written(arg0.dat);
    oppb_rt::mark_device_written(arg1.dat);
    oppb_rt::mark_device_written(set->mesh_relation_dat);
    opp_profiler->end("inject_ions_kernel");
}

// calculate_new_pos_vel_kernel over [0, size).
void opp_par_loop_all__calculate_new_pos_vel_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2) {
    opp_profiler->start("calculate_new_pos_vel_kernel");
    const oppb_tet_mesh& mesh = oppb_rt::tet_mesh(nullptr, nullptr, nullptr, nullptr, arg0.dat);
    oppb_particles p = particles(set, arg1.dat, arg2.dat, nullptr);
    check(oppb_push_f64(&mesh, &p, charge_over_mass(), opp_get_const("CONST_dt"), oppb_rt::stream()), "oppb_push_f64");
    oppb_rt::mark_device_written(arg1.dat);
    oppb_rt::mark_device_written(arg2.dat);
    opp_profiler->end("calculate_new_pos_vel_kernel");
}

// move_kernel with multi-hop, then the finalize (hole fill / sort).
void opp_particle_move__move_kernel(opp_set set, opp_map c2c_map, opp_map p2c_map, opp_arg arg0, opp_arg arg1,
                                    opp_arg arg2, opp_arg arg3) {
    opp_profiler->start("move_kernel");
    (void)p2c_map;
    opp_init_particle_move(set, 0, nullptr);
    const oppb_tet_mesh& mesh = oppb_rt::tet_mesh(arg3.dat, arg2.dat, c2c_map, nullptr, nullptr);
    oppb_particles p = particles(set, arg0.dat, nullptr, arg1.dat);
    opp_profiler->start("move_kernel_only");
    if (g_dh.on && g_dh.generation == oppb_rt::generation()) {  // global move: the walks start from the grid's cells
        oppb_move_options o{};
        o.precision = OPPB_PRECISION_F64;
        o.dh = &g_dh.grid;
        check(oppb_move_ex(&mesh, &p, &o, nullptr, oppb_rt::move_status(), oppb_rt::max_hops(), nullptr, 0,
                           oppb_rt::stream()),
              "oppb_move_ex");
    } else {
        check(oppb_move_f64(&mesh, &p, oppb_rt::move_status(), oppb_rt::max_hops(), oppb_rt::stream()),
              "oppb_move_f64");
    }
    oppb_rt::mark_device_written(arg1.dat);
    oppb_rt::mark_device_written(set->mesh_relation_dat);
    opp_profiler->end("move_kernel_only");
    while (opp_finalize_particle_move(set)) {
    }
    opp_profiler->end("move_kernel");
}

// deposit_charge_on_nodes_kernel: n_charge_den[c2n[p2c][i]] += p_lc[i].
void opp_par_loop_all__deposit_charge_on_nodes_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                                                      opp_arg arg3, opp_arg arg4) {
    opp_profiler->start("deposit_charge_on_nodes_kernel");
    (void)arg2, (void)arg3, (void)arg4;
    oppb_rt::sync_host_to_device(arg1.dat);
    const oppb_tet_mesh& mesh = oppb_rt::tet_mesh(nullptr, nullptr, nullptr, arg1.map, nullptr);
    oppb_particles p = particles(set, nullptr, nullptr, arg0.dat);
    const size_t ws_bytes = oppb_deposit_workspace_bytes(mesh.n_nodes);
    check(oppb_deposit_f64(&mesh, &p, reinterpret_cast<double*>(arg1.dat->data_d),
                           ws_bytes ? oppb_rt::workspace(ws_bytes) : nullptr, ws_bytes, oppb_rt::stream()),
          "oppb_deposit_f64");
    oppb_rt::mark_device_written(arg1.dat);
    if (cudaStreamSynchronize(oppb_rt::stream()) != cudaSuccess) opp_abort("deposit");
    opp_profiler->end("deposit_charge_on_nodes_kernel");
}

// opp_init_direct_hop_cg (apps_codegen/app_fempic_cg/cuda/move_kernel_loop.hpp:403-475): with
// opp_global_move set, builds the structured grid of spacing grid_spacing over b_box on the
// GPU (the reference searches all cells per grid box on the host, or reads a file made that
// way); every later move starts each walk from its grid box's cell.  One unpartitioned mesh:
// the cells' global ids must be their indices.
void opp_init_direct_hop_cg(double grid_spacing, const opp_dat c_gbl_id, const opp::BoundingBox& b_box,
                            opp_map c2c_map, opp_map p2c_map, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                            opp_arg arg3) {
    (void)p2c_map, (void)arg0, (void)arg1;
    useGlobalMove = opp_params->get<OPP_BOOL>("opp_global_move");
    if (!useGlobalMove) return;
    opp_profiler->start("Setup_Mover");
    opp_set cells = c2c_map->from;
    if (c_gbl_id) {
        opp_download_dat(c_gbl_id);
        const int* id = reinterpret_cast<const int*>(c_gbl_id->data);
        for (int c = 0; c < cells->size; c++)
            if (id[c] != c) opp_abort("opp_init_direct_hop_cg: c_gbl_id must be the cell index on one GPU");
    }
    if (b_box.getDim() != 3) opp_abort("opp_init_direct_hop_cg: the FemPIC grid is 3-D");
    opp_dat npos = b_box.nodePositions();
    if (!npos) opp_abort("opp_init_direct_hop_cg: the bounding box must come from the node positions");
    opp_map c2n = nullptr;  // the cell -> node map the binning reads
    for (opp_map m : opp_maps)
        if (m && m->from == cells && m->to == npos->set && m->dim == 4) c2n = m;
    if (!c2n) opp_abort("opp_init_direct_hop_cg: no cell -> node map of dimension 4 is declared");
    const opp_point& mn = b_box.getGlobalMin();
    const opp_point& mx = b_box.getGlobalMax();
    const double lo[3] = {mn.x, mn.y, mn.z}, hi[3] = {mx.x, mx.y, mx.z};
    if (g_dh.grid.map) cudaFree(g_dh.grid.map);
    g_dh = DirectHop{};
    check(oppb_dh_grid_from_box(lo, hi, grid_spacing, &g_dh.grid), "oppb_dh_grid_from_box");
    if (cudaMalloc(&g_dh.grid.map, sizeof(int32_t) * (size_t)g_dh.grid.size) != cudaSuccess)
        opp_abort("cudaMalloc direct-hop map");
    oppb_rt::sync_host_to_device(npos);
    const oppb_tet_mesh& mesh = oppb_rt::tet_mesh(arg3.dat, arg2.dat, c2c_map, c2n, nullptr);
    const double* npos_d = reinterpret_cast<const double*>(npos->data_d);
    size_t need = 0;
    int rc = oppb_dh_build(&mesh, npos_d, &g_dh.grid, nullptr, 0, &need, oppb_rt::stream());
    if (rc == OPPB_ERR_WORKSPACE)
        rc = oppb_dh_build(&mesh, npos_d, &g_dh.grid, oppb_rt::workspace(need), need, &need, oppb_rt::stream());
    check(rc, "oppb_dh_build");
    if (cudaStreamSynchronize(oppb_rt::stream()) != cudaSuccess) opp_abort("direct-hop grid build");
    g_dh.on = true;
    g_dh.generation = oppb_rt::generation();
    opp_profiler->end("Setup_Mover");
}

// ------------------------------------------------------------ node and cell loops
// The generated node- and cell-set loops of the FemPIC main (fempic_opp.cpp:40-48) around the
// field solve.  Mesh dats and maps live on the device as SoA with stride = the set size.

namespace {
oppb_cell_layout soa(opp_set set) { return oppb_cell_layout{1, (int64_t)std::max(set->size, 1)}; }
}  // namespace

// init_boundary_pot_kernel (apps/app_fempic/kernels.h:48-60): FIXED nodes get
// -CONST_wall_potential, every other node 0.  Runs on the host at set-up.
void opp_par_loop_all__init_boundary_pot_kernel(opp_set set, opp_arg arg0, opp_arg arg1) {
    opp_profiler->start("init_boundary_pot_kernel");
    opp_download_dat(arg0.dat);
    const int* type = reinterpret_cast<const int*>(arg0.dat->data);
    double* pot = reinterpret_cast<double*>(arg1.dat->data);
    const double wall = opp_get_const("CONST_wall_potential");
    for (int n = 0; n < set->size; n++) pot[n] = (type[n] == OPPB_NODE_FIXED) ? -1 * wall : 0;
    arg1.dat->dirty_hd = Device;  // the host copy is the newer one
    arg1.dat->version++;
    opp_profiler->end("init_boundary_pot_kernel");
}

// compute_node_charge_density_kernel: n_charge_den *= CONST_spwt / n_volume.
void opp_par_loop_all__compute_node_charge_density_kernel(opp_set set, opp_arg arg0, opp_arg arg1) {
    opp_profiler->start("compute_node_charge_density_kernel");
    oppb_rt::sync_host_to_device(arg0.dat);
    oppb_rt::sync_host_to_device(arg1.dat);
    check(oppb_node_charge_density(reinterpret_cast<double*>(arg0.dat->data_d),
                                   reinterpret_cast<const double*>(arg1.dat->data_d), opp_get_const("CONST_spwt"),
                                   set->size, oppb_rt::stream()),
          "oppb_node_charge_density");
    oppb_rt::mark_device_written(arg0.dat);
    opp_profiler->end("compute_node_charge_density_kernel");
}

// compute_electric_field_kernel: c_ef (OPP_INC) -= sum_i c_sd[i] * n_potential[c2n[i]].
void opp_par_loop_all__compute_electric_field_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                                                     opp_arg arg3, opp_arg arg4, opp_arg arg5) {
    opp_profiler->start("compute_electric_field_kernel");
    (void)arg3, (void)arg4, (void)arg5;
    opp_dat c_ef = arg0.dat, c_sd = arg1.dat, pot = arg2.dat;
    if (!arg2.map || !arg2.map->map_d) opp_abort("compute_electric_field_kernel: c2n map has no device copy");
    oppb_rt::sync_host_to_device(c_ef);
    oppb_rt::sync_host_to_device(c_sd);
    oppb_rt::sync_host_to_device(pot);
    check(oppb_electric_field_ex(arg2.map->map_d, soa(set), reinterpret_cast<const double*>(c_sd->data_d), soa(set),
                                 reinterpret_cast<const double*>(pot->data_d), reinterpret_cast<double*>(c_ef->data_d),
                                 soa(set), set->size, 1, oppb_rt::stream()),
          "oppb_electric_field_ex");
    oppb_rt::mark_device_written(c_ef);
    opp_profiler->end("compute_electric_field_kernel");
}

// get_max_cef_kernel: the OPP_MAX global of every component of c_ef.
void opp_par_loop_all__get_max_cef_kernel(opp_set set, opp_arg arg0, opp_arg arg1) {
    opp_dat c_ef = arg0.dat;
    oppb_rt::sync_host_to_device(c_ef);
    double* out = reinterpret_cast<double*>(arg1.data);
    const int64_t stride = std::max(set->size, 1);
    for (int d = 0; d < c_ef->dim; d++)
        check(oppb_reduce_max(reinterpret_cast<const double*>(c_ef->data_d) + d * stride, set->size, 0, *out, out,
                              oppb_rt::stream()),
              "oppb_reduce_max");
}

// get_final_max_values_kernel: OPP_MAX of |n_charge_den| and of |n_potential|.
void opp_par_loop_all__get_final_max_values_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2,
                                                   opp_arg arg3) {
    oppb_rt::sync_host_to_device(arg0.dat);
    oppb_rt::sync_host_to_device(arg2.dat);
    double* m0 = reinterpret_cast<double*>(arg1.data);
    double* m1 = reinterpret_cast<double*>(arg3.data);
    check(oppb_reduce_max(reinterpret_cast<const double*>(arg0.dat->data_d), set->size, 1, *m0, m0, oppb_rt::stream()),
          "oppb_reduce_max");
    check(oppb_reduce_max(reinterpret_cast<const double*>(arg2.dat->data_d), set->size, 1, *m1, m1, oppb_rt::stream()),
          "oppb_reduce_max");
}
