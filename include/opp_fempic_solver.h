// FemPIC's field solver for the opp_* drop-in runtime: the public interface of the reference
// app's FESolver (apps_codegen/app_fempic_cg/field_solver.h:41-49) on the B200 backend
// (include/oppb_field.h), without PETSc.  An app that includes "field_solver.h" includes this
// header instead and drops field_solver/*.cpp from its link.
//
// Constants as the reference's constructor takes them: CONST_n0 = plasma_den and
// CONST_kTe = Kb * electron_temperature from opp_params, QE and EPS0 (fempic_defs.h), phi0 = 0;
// the linear solve stops at the KSP tolerances 1e-10 (field_solver.cpp:270).
#ifndef OPP_FEMPIC_SOLVER_H
#define OPP_FEMPIC_SOLVER_H

#include <memory>

#include "opp_lib.h"

class FESolver {
   public:
    FESolver(const opp_map c2n_map, const opp_dat n_type, const opp_dat n_pos, const opp_dat n_bnd_pot);
    ~FESolver();

    // compute_phi(n_potential OPP_WRITE, n_charge_den OPP_READ, n_bnd_pot OPP_READ): one Newton
    // step of the Poisson-Boltzmann potential (field_solver.cpp:115-176).
    void compute_phi(opp_arg arg0, opp_arg arg1, opp_arg arg2);
    // The shape-function derivatives (NX / SCALLING) into c_sd [n_cells][4][3].
    void enrich_cell_shape_deriv(opp_dat cell_shape_deriv);

    // CG iterations and convergence of the last compute_phi.
    int last_iterations() const;
    bool last_converged() const;

   private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

#endif  // OPP_FEMPIC_SOLVER_H
