// FESolver of the opp_* drop-in runtime (include/opp_fempic_solver.h) on the B200 field
// kernels (include/oppb_field.h).

#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "opp_fempic_solver.h"
#include "oppb_field.h"

namespace {

// fempic_defs.h:60-63
constexpr double kEps0 = 8.8541878e-12;
constexpr double kQe = 1.602e-19;
constexpr double kBoltzmann = 8.617333262e-5;

void check(int rc, const char* what) {
    if (rc != OPPB_OK) opp_abort(std::string(what) + ": " + oppb_status_string(rc));
}

template <typename T>
T* upload(const T* h, size_t n) {
    T* d = nullptr;
    if (cudaMalloc(&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) opp_abort("FESolver: cudaMalloc");
    if (n && cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess) opp_abort("FESolver: upload");
    return d;
}

}  // namespace

struct FESolver::Impl {
    oppb_field_device dev{};
    oppb_field_consts consts{};
    oppb_field_status* status = nullptr;  // device
    std::vector<double> c_sd;             // [n_cells][12], host
    std::vector<void*> owned;
    int iterations = 0;
    bool converged = true;
    ~Impl() {
        for (void* p : owned) cudaFree(p);
    }
    template <typename T>
    T* keep(T* p) {
        owned.push_back(p);
        return p;
    }
};

FESolver::FESolver(const opp_map c2n_map, const opp_dat n_type, const opp_dat n_pos, const opp_dat n_bnd_pot)
    : impl_(new Impl) {
    opp_profiler->start("FSolve_setup");
    opp_download_dat(n_type);
    opp_download_dat(n_pos);
    opp_download_dat(n_bnd_pot);
    if (n_pos->dim != 3 || c2n_map->dim != 4) opp_abort("FESolver: 3-D tetrahedral meshes only");
    oppb_fempic_mesh m{};
    m.n_nodes = n_type->set->size;
    m.n_cells = c2n_map->from->size;
    m.n_pos = reinterpret_cast<double*>(n_pos->data);
    m.n_type = reinterpret_cast<int32_t*>(n_type->data);
    m.n_bnd_pot = reinterpret_cast<double*>(n_bnd_pot->data);
    m.c2n = c2n_map->map;
    oppb_field_system s{};
    check(oppb_field_setup(&m, &s), "oppb_field_setup");
    Impl& I = *impl_;
    const size_t nn = (size_t)s.n_nodes, nc = (size_t)s.n_cells, neq = (size_t)s.neq, nnz = (size_t)s.nnz;
    I.c_sd.assign(s.c_sd, s.c_sd + 12 * nc);
    oppb_field_device& d = I.dev;
    d.n_nodes = s.n_nodes;
    d.n_cells = s.n_cells;
    d.neq = s.neq;
    d.node_to_eq = I.keep(upload(s.node_to_eq, nn));
    d.c2n = I.keep(upload(s.c2n, 4 * nc));
    d.det_j = I.keep(upload(s.det_j, nc));
    d.n_bnd_pot = I.keep(upload(s.n_bnd_pot, nn));
    d.k_rowptr = I.keep(upload(s.k_rowptr, neq + 1));
    d.k_col = I.keep(upload(s.k_col, nnz));
    d.k_val = I.keep(upload(s.k_val, nnz));
    d.f0 = I.keep(upload(s.f0, neq));
    d.n_diag = s.n_diag;
    for (int j = 0; j < OPPB_FIELD_MAX_DIAG; j++) d.dia_off[j] = s.dia_off[j];
    d.dia_val = s.n_diag > 0 ? I.keep(upload(s.dia_val, (size_t)s.n_diag * neq)) : nullptr;
    oppb_field_system_free(&s);  // s is zeroed: sizes below come from the copies taken above
    const std::vector<double> zeros(neq ? neq : 1, 0.0);
    d.d = I.keep(upload(zeros.data(), zeros.size()));   // D (dLocal) starts at 0
    d.f1 = I.keep(upload(zeros.data(), zeros.size()));  // f1Local starts at 0
    const std::vector<double> work(oppb_field_work_doubles((int32_t)neq), 0.0);
    d.work = I.keep(upload(work.data(), work.size()));
    const oppb_field_status st0{};
    I.status = I.keep(upload(&st0, 1));
    oppb_field_consts& c = I.consts;
    c.n0 = opp_params->get<OPP_REAL>("plasma_den");
    c.kte = kBoltzmann * opp_params->get<OPP_REAL>("electron_temperature");
    c.phi0 = 0.0;
    c.qe = kQe;
    c.eps0 = kEps0;
    c.rtol = 1e-10;
    c.atol = 1e-10;
    c.max_iter = 10000;  // PETSc's default iteration bound
    opp_profiler->end("FSolve_setup");
}

FESolver::~FESolver() = default;

void FESolver::enrich_cell_shape_deriv(opp_dat cell_shape_deriv) {
    if (cell_shape_deriv->dim != 12 || cell_shape_deriv->set->size != impl_->dev.n_cells)
        opp_abort("enrich_cell_shape_deriv: c_sd must be a 12-component cell dat");
    std::memcpy(cell_shape_deriv->data, impl_->c_sd.data(), impl_->c_sd.size() * sizeof(double));
    cell_shape_deriv->dirty_hd = Device;  // the host copy is the newer one: upload before device use
    cell_shape_deriv->version++;
}

void FESolver::compute_phi(opp_arg arg0, opp_arg arg1, opp_arg arg2) {
    (void)arg2;  // the Dirichlet values were taken at set-up, as the reference's F0
    opp_profiler->start("compute_phi");
    Impl& I = *impl_;
    oppb_rt::sync_host_to_device(arg1.dat);
    check(oppb_field_solve(&I.dev, &I.consts, reinterpret_cast<const double*>(arg1.dat->data_d),
                           reinterpret_cast<double*>(arg0.dat->data_d), I.status, oppb_rt::stream()),
          "oppb_field_solve");
    oppb_rt::mark_device_written(arg0.dat);
    oppb_field_status st{};
    if (cudaMemcpyAsync(&st, I.status, sizeof st, cudaMemcpyDeviceToHost, oppb_rt::stream()) != cudaSuccess ||
        cudaStreamSynchronize(oppb_rt::stream()) != cudaSuccess)
        opp_abort("compute_phi: status read");
    I.iterations = st.iterations;
    I.converged = st.converged != 0;
    if (!I.converged)  // the reference prints the KSP reason and carries on
        opp_printf("FESolver", "linear solve did not converge: %d iterations, relative residual %g", st.iterations,
                   st.resid);
    opp_profiler->end("compute_phi");
}

int FESolver::last_iterations() const { return impl_->iterations; }
bool FESolver::last_converged() const { return impl_->converged; }
