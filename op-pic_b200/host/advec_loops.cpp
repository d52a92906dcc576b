// NESO advection's generated-loop entry points on the library's advection kernels
// (include/oppb_advec.h), for one unpartitioned mesh: the functions the generated main
// apps_codegen/app_neso_advection_mdir_cg/advec_opp.cpp:40-43 declares.  They replace the bodies
// of apps_codegen/app_neso_advection_mdir_cg/cuda/{update_pos_kernel_loop,move_kernel_loop,
// verify_kernel_loop}.hpp.  The mesh is the app's periodic nx x ny grid of square cells; the
// constants come from the main's opp_decl_const calls (CONST_dt, CONST_extents, CONST_cell_width,
// CONST_ndimcells).  The instance's cells are packed once from c_pos_ll and c_c_map (again when
// c_pos_ll is rewritten) and checked against the grid the app's init_mesh builds, so that the
// move computes corners and neighbours (oppb_advec_check_grid).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "opp_lib.h"
#include "oppb_advec.h"
#include "oppb_dh.h"

namespace {

constexpr int kWorkItem = 256;  // particles per work item of the persistent launch

void check(int rc, const char* what) {
    if (rc != OPPB_OK) opp_abort(std::string(what) + ": " + oppb_status_string(rc));
}
void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) opp_abort(std::string(what) + ": " + cudaGetErrorString(e));
}
template <class T>
T* dev_alloc(size_t n) {
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    return static_cast<T*>(p);
}

struct Advec {
    opp_dat c_pos_ll = nullptr;  // the packed cells' source, its version and the runtime's generation
    int c_pos_ll_version = -1;
    int generation = -1;
    opp_map c2c = nullptr;
    int32_t n_cells = 0;
    int32_t grid_nx = 0;
    double* cells = nullptr;       // packed records [n_cells][4]
    oppb_advec_instance* inst = nullptr;
    int32_t* prefix = nullptr;
    int32_t* counter = nullptr;
    int32_t* scratch = nullptr;    // grid-check mismatches, verify count
    oppb_advec_dh* dh = nullptr;   // the global move's grid (device, one entry) or nullptr
    int32_t* dh_map = nullptr;
    oppb_advec_dh* dh_table = nullptr;  // device storage of `dh`
    int dh_generation = -1;
};

Advec& adv() {
    static Advec a;
    return a;
}

double const_at(const char* name, int k) { return opp_get_const(name, k); }

void ensure_buffers() {
    Advec& a = adv();
    if (a.inst) return;
    a.inst = dev_alloc<oppb_advec_instance>(1);
    a.prefix = dev_alloc<int32_t>(2);
    a.counter = dev_alloc<int32_t>(1);
    a.scratch = dev_alloc<int32_t>(1);
}

// The instance of `set` (all its particles) and its work items, uploaded for this launch.
void upload_instance(opp_set set) {
    Advec& a = adv();
    ensure_buffers();
    oppb_advec_instance in{};
    in.part_offset = 0;
    in.n_parts = set->size;
    in.cell_offset = 0;
    in.n_cells = a.n_cells;
    in.grid_nx = a.grid_nx;
    in.dt = const_at("CONST_dt", 0);
    in.cell_width = const_at("CONST_cell_width", 0);
    in.extents[0] = const_at("CONST_extents", 0);
    in.extents[1] = const_at("CONST_extents", 1);
    const int32_t prefix[2] = {0, (set->size + kWorkItem - 1) / kWorkItem};
    cudaStream_t s = oppb_rt::stream();
    check_cuda(cudaMemcpyAsync(a.inst, &in, sizeof in, cudaMemcpyHostToDevice, s), "instance upload");
    check_cuda(cudaMemcpyAsync(a.prefix, prefix, sizeof prefix, cudaMemcpyHostToDevice, s), "prefix upload");
}

// Packs c_pos_ll and c_c_map when they are new or c_pos_ll was rewritten, and checks the cells
// against the periodic grid (one host read of the mismatch count).
void pack_cells(opp_dat c_pos_ll, opp_map c2c) {
    Advec& a = adv();
    if (a.c_pos_ll == c_pos_ll && a.c2c == c2c && a.c_pos_ll_version == c_pos_ll->version &&
        a.generation == oppb_rt::generation())
        return;
    if (c_pos_ll->dim != 2 || c2c->dim != 4 || c2c->from != c_pos_ll->set)
        opp_abort("advection loops: c_pos_ll must be a 2-component cell dat and c_c_map a 4-entry cell map");
    oppb_rt::sync_host_to_device(c_pos_ll);
    const int32_t n = c_pos_ll->set->size;
    if (a.cells && a.n_cells != n) {
        cudaFree(a.cells);
        a.cells = nullptr;
    }
    if (!a.cells) a.cells = dev_alloc<double>((size_t)n * 4);
    a.n_cells = n;
    ensure_buffers();
    cudaStream_t s = oppb_rt::stream();
    check(oppb_advec_pack_cells(a.cells, 0, n, n, reinterpret_cast<const double*>(c_pos_ll->data_d), c2c->map_d, s),
          "oppb_advec_pack_cells");
    const int nx = (int)const_at("CONST_ndimcells", 0);
    a.grid_nx = 0;
    if (nx > 0 && n % nx == 0) {
        check(oppb_advec_check_grid(a.cells, 0, n, nx, const_at("CONST_cell_width", 0), a.scratch, s),
              "oppb_advec_check_grid");
        int32_t bad = -1;
        check_cuda(cudaMemcpyAsync(&bad, a.scratch, sizeof bad, cudaMemcpyDeviceToHost, s), "grid check");
        check_cuda(cudaStreamSynchronize(s), "grid check sync");
        if (bad == 0) a.grid_nx = nx;
    }
    a.c_pos_ll = c_pos_ll;
    a.c2c = c2c;
    a.c_pos_ll_version = c_pos_ll->version;
    a.generation = oppb_rt::generation();
}

oppb_advec_batch batch_of(opp_set set, opp_dat pos, opp_dat vel, opp_dat mdir) {
    Advec& a = adv();
    if (a.dh && a.dh_generation != oppb_rt::generation()) a.dh = nullptr;  // a grid of an earlier run
    oppb_advec_batch b{};
    b.n_instances = 1;
    b.n_work = (set->size + kWorkItem - 1) / kWorkItem;
    b.instances = a.inst;
    b.tile_prefix = a.prefix;
    b.cells = a.cells;
    b.stride = std::max(set->set_capacity, 1);
    b.pos = reinterpret_cast<double*>(pos->data_d);
    b.vel = vel ? reinterpret_cast<const double*>(vel->data_d) : nullptr;
    b.mdir = mdir ? reinterpret_cast<int32_t*>(mdir->data_d) : nullptr;
    b.p2c = reinterpret_cast<int32_t*>(set->mesh_relation_dat->data_d);
    b.work_counter = a.counter;
    b.dh = a.dh;
    return b;
}

}  // namespace

// update_pos_kernel over every particle (cuda/update_pos_kernel_loop.hpp): the periodic
// position update of apps/app_neso_advection/kernels.h:41-57.
void opp_par_loop_all__update_pos_kernel(opp_set set, opp_arg arg0, opp_arg arg1) {
    opp_profiler->start("update_pos_kernel");
    opp_dat vel = arg0.dat, pos = arg1.dat;
    if (!vel || !pos || vel->dim != 2 || pos->dim != 2 || vel->set != set || pos->set != set)
        opp_abort("opp_par_loop_all__update_pos_kernel: p_vel and p_pos must be 2-component dats of the set");
    oppb_rt::sync_host_to_device(vel);
    oppb_rt::sync_host_to_device(pos);
    upload_instance(set);
    const oppb_advec_batch b = batch_of(set, pos, vel, nullptr);
    check(oppb_advec_update_pos(&b, oppb_rt::stream()), "oppb_advec_update_pos");
    oppb_rt::mark_device_written(pos);
    check_cuda(cudaStreamSynchronize(oppb_rt::stream()), "update_pos sync");
    opp_profiler->end("update_pos_kernel");
}

// move_kernel (cuda/move_kernel_loop.hpp): the axis-wise walk of
// apps/app_neso_advection/kernels.h:60-112 from each particle's cell, or, with the global move
// on (opp_init_direct_hop_cg), from its direct-hop grid box's cell; then the finalize.
void opp_particle_move__move_kernel(opp_set set, opp_map c2c_map, opp_map p2c_map, opp_arg arg0, opp_arg arg1,
                                    opp_arg arg2) {
    opp_profiler->start("move_kernel");
    opp_dat pos = arg0.dat, mdir = arg1.dat, c_pos_ll = arg2.dat;
    if (!pos || !mdir || !c_pos_ll || pos->set != set || mdir->set != set || mdir->dim != 2 ||
        p2c_map->p2c_dat != set->mesh_relation_dat)
        opp_abort("opp_particle_move__move_kernel: unexpected arguments for the advection move");
    opp_init_particle_move(set, 0, nullptr);
    for (opp_dat d : {pos, mdir, set->mesh_relation_dat}) oppb_rt::sync_host_to_device(d);
    pack_cells(c_pos_ll, c2c_map);
    upload_instance(set);
    cudaStream_t s = oppb_rt::stream();
    oppb_move_status* st = oppb_rt::move_status();
    check_cuda(cudaMemsetAsync(st, 0, sizeof(oppb_move_status), s), "status reset");
    const oppb_advec_batch b = batch_of(set, pos, nullptr, mdir);
    check(oppb_advec_move(&b, st, oppb_rt::max_hops(), s), "oppb_advec_move");
    if (b.dh)  // only the global move's pre-pass removes particles
        check(oppb_removal_bits(b.p2c, set->size, oppb_rt::remove_bits(set), s), "oppb_removal_bits");
    oppb_rt::mark_device_written(mdir);
    oppb_rt::mark_device_written(set->mesh_relation_dat);
    while (opp_finalize_particle_move(set)) {
    }
    opp_profiler->end("move_kernel");
}

// verify_kernel (cuda/verify_kernel_loop.hpp): counts the particles outside their cell's box
// into the OPP_INC int global.
void opp_par_loop_all__verify_kernel(opp_set set, opp_arg arg0, opp_arg arg1, opp_arg arg2) {
    opp_profiler->start("verify_kernel");
    opp_dat pos = arg0.dat, c_idx = arg1.dat;
    if (!pos || !c_idx || pos->set != set || c_idx->set != set->cells_set || c_idx->dim != 1 ||
        arg2.argtype != OPP_ARG_GBL || !arg2.data)
        opp_abort("opp_par_loop_all__verify_kernel: unexpected arguments");
    oppb_rt::sync_host_to_device(pos);
    oppb_rt::sync_host_to_device(c_idx);
    oppb_rt::sync_host_to_device(set->mesh_relation_dat);
    Advec& a = adv();
    ensure_buffers();
    cudaStream_t s = oppb_rt::stream();
    check_cuda(cudaMemsetAsync(a.scratch, 0, sizeof(int32_t), s), "verify reset");
    check(oppb_advec_verify(reinterpret_cast<const double*>(pos->data_d), std::max(set->set_capacity, 1),
                            reinterpret_cast<const int32_t*>(set->mesh_relation_dat->data_d),
                            reinterpret_cast<const int32_t*>(c_idx->data_d), set->size,
                            (int)const_at("CONST_ndimcells", 0), const_at("CONST_cell_width", 0), a.scratch, s),
          "oppb_advec_verify");
    int32_t bad = 0;
    check_cuda(cudaMemcpyAsync(&bad, a.scratch, sizeof bad, cudaMemcpyDeviceToHost, s), "verify count");
    check_cuda(cudaStreamSynchronize(s), "verify sync");
    *reinterpret_cast<int*>(arg2.data) += bad;
    opp_profiler->end("verify_kernel");
}

// opp_init_direct_hop_cg of the advection app (cuda/move_kernel_loop.hpp:417-490): with
// opp_global_move set, the 2-D structured grid of spacing grid_spacing over b_box, its map
// built on the GPU from the packed cells (oppb_dh_build_quad: the lowest-index cell whose move
// from the box's corner ends in that cell, the reference's all-cell search); every later move
// seeds its walks from it.  One unpartitioned mesh: the cells' global ids must be their indices.
void opp_init_direct_hop_cg(double grid_spacing, const opp_dat c_gbl_id, const opp::BoundingBox& b_box,
                            opp_map c2c_map, opp_map p2c_map, opp_arg arg0, opp_arg arg1, opp_arg arg2) {
    (void)p2c_map, (void)arg0, (void)arg1;
    opp_profiler->start("Setup_Mover");
    useGlobalMove = opp_params->get<OPP_BOOL>("opp_global_move");
    if (useGlobalMove) {
        if (b_box.getDim() != 2) opp_abort("opp_init_direct_hop_cg: the advection grid is 2-D");
        if (c_gbl_id) {
            opp_download_dat(c_gbl_id);
            const int* id = reinterpret_cast<const int*>(c_gbl_id->data);
            for (int c = 0; c < c_gbl_id->set->size; c++)
                if (id[c] != c) opp_abort("opp_init_direct_hop_cg: c_gbl_id must be the cell index on one GPU");
        }
        pack_cells(arg2.dat, c2c_map);
        Advec& a = adv();
        const opp_point& mn = b_box.getGlobalMin();
        const opp_point& mx = b_box.getGlobalMax();
        const double lo[3] = {mn.x, mn.y, 0.0}, hi[3] = {mx.x, mx.y, 0.0};
        oppb_dh_grid g{};
        check(oppb_dh_grid_from_box(lo, hi, grid_spacing, &g), "oppb_dh_grid_from_box");
        if (a.dh_map) cudaFree(a.dh_map);
        a.dh_map = dev_alloc<int32_t>((size_t)g.size);
        g.map = a.dh_map;
        cudaStream_t s = oppb_rt::stream();
        size_t need = 0;
        int rc = oppb_dh_build_quad(a.cells, a.n_cells, const_at("CONST_cell_width", 0), &g, nullptr, 0, &need, s);
        if (rc == OPPB_ERR_WORKSPACE) {
            void* ws = oppb_rt::workspace(need);
            rc = oppb_dh_build_quad(a.cells, a.n_cells, const_at("CONST_cell_width", 0), &g, ws, need, &need, s);
        }
        check(rc, "oppb_dh_build_quad");
        oppb_advec_dh d{};
        d.map = a.dh_map;
        d.min[0] = g.min[0];
        d.min[1] = g.min[1];
        d.inv_spacing = g.inv_spacing;
        d.dims[0] = g.dims[0];
        d.dims[1] = g.dims[1];
        if (!a.dh_table) a.dh_table = dev_alloc<oppb_advec_dh>(1);
        a.dh = a.dh_table;
        a.dh_generation = oppb_rt::generation();
        check_cuda(cudaMemcpyAsync(a.dh, &d, sizeof d, cudaMemcpyHostToDevice, s), "dh upload");
        check_cuda(cudaStreamSynchronize(s), "dh sync");
    }
    opp_profiler->end("Setup_Mover");
}
