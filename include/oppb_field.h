/* C ABI of the FemPIC node-side loops and field solve on the B200 backend: the node charge
 * density (compute_node_charge_density_kernel, apps/app_fempic/kernels.h:178-183), the
 * electric field (compute_electric_field_kernel, :186-202) and the electrostatic potential
 * of FESolver::compute_phi (apps_codegen/app_fempic_cg/field_solver/field_solver.cpp:115-176):
 * one Newton step per call on the Poisson-Boltzmann system K D - F0 - F1(D) = 0 with
 * J = K - diag(dF1/dD), the linear step J Y = B solved by FP64 conjugate gradients.
 *
 * The set-up (shape-function derivatives, equation numbering, K, F0) runs on the host once,
 * as FESolver's constructor does; every per-step part runs on the device with no host
 * synchronisation, so a stream capture of oppb_field_solve makes it one CUDA graph.
 */
#ifndef OPPB_FIELD_H
#define OPPB_FIELD_H

#include <stddef.h>
#include <stdint.h>

#include "oppb.h"
#include "oppb_fempic.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host set-up of FESolver (field_solver.cpp:46-99): compute_nx (:553-594, the derivatives
 * NX of the linear shape functions scaled by SCALLING = 100, and detJ), the equation map
 * (:178-210: NORMAL and OPEN nodes are unknowns, numbered in node order; INLET and FIXED
 * nodes are Dirichlet), pre_assembly (:330-391: K and F0 from 2x2x2 Gauss points, both
 * scaled by 1/SCALLING^2) and enrich_cell_shape_deriv (:474-499: c_sd = NX / SCALLING).
 * K is CSR over the unknowns with columns ascending in each row.  Arrays are malloc-owned.
 * When K's entries lie on at most OPPB_FIELD_MAX_DIAG diagonals (column - row offsets) that
 * hold no more than 1.5 nnz values in all, K is also given by diagonals: dia_val[j * neq + r] =
 * K[r][r + dia_off[j]] (0 where K has no entry), offsets ascending; else n_diag = 0.  A box
 * mesh in node order has 15 diagonals. */
#define OPPB_FIELD_MAX_DIAG 16
typedef struct oppb_field_system {
    int32_t  n_nodes, n_cells, neq;
    int32_t* node_to_eq;   /* [n_nodes] equation of a node, -1 for a Dirichlet node        */
    int32_t* c2n;          /* [n_cells][4] copied from the mesh                             */
    double*  det_j;        /* [n_cells] detJ of compute_nx                                  */
    double*  c_sd;         /* [n_cells][4][3] NX / SCALLING (compute_electric_field's c_sd) */
    double*  n_bnd_pot;    /* [n_nodes] Dirichlet values (0 on unknowns)                    */
    int64_t* k_rowptr;     /* [neq + 1]                                                     */
    int32_t* k_col;        /* [nnz]                                                         */
    double*  k_val;        /* [nnz]                                                         */
    double*  f0;           /* [neq]                                                         */
    int64_t  nnz;
    int32_t  n_diag;                        /* 0 = no diagonal form                      */
    int32_t  dia_off[OPPB_FIELD_MAX_DIAG];
    double*  dia_val;                       /* [n_diag][neq], or NULL                    */
} oppb_field_system;

int oppb_field_setup(const oppb_fempic_mesh* mesh, oppb_field_system* out);
void oppb_field_system_free(oppb_field_system* s);

/* The electron model and solver constants (FESolver members: CONST_n0 = plasma_den,
 * CONST_kTe = Kb * electron_temperature, CONST_phi0 = 0, CONST_QE, CONST_EPS0; the KSP
 * tolerances 1e-10, field_solver.cpp:270). */
typedef struct oppb_field_consts {
    double n0, phi0, kte, qe, eps0;
    double rtol, atol;    /* stop when ||r|| <= max(rtol * ||B||, atol)                   */
    int32_t max_iter;     /* CG iteration bound                                          */
    int32_t reserved;
} oppb_field_consts;

/* Device copy of the system plus the Newton state and CG scratch.  All pointers device. */
typedef struct oppb_field_device {
    int32_t n_nodes, n_cells, neq, reserved;
    const int32_t* node_to_eq;
    const int32_t* c2n;       /* [n_cells][4] */
    const double*  det_j;
    const double*  n_bnd_pot;
    const int64_t* k_rowptr;
    const int32_t* k_col;
    const double*  k_val;
    const double*  f0;
    double* d;                /* [neq] Newton iterate D (dLocal), zero at start            */
    double* f1;               /* [neq] F1, accumulated over calls as the reference's f1Local */
    double* work;             /* oppb_field_work_doubles(neq) doubles                       */
    int32_t n_diag;           /* K by diagonals (oppb_field_system), 0 = CSR only: the CG's */
    int32_t dia_off[OPPB_FIELD_MAX_DIAG]; /* products then read the diagonals, coalesced   */
    const double* dia_val;    /* [n_diag][neq]; the same sums, term by term in column order */
} oppb_field_device;

/* Doubles of work space a device system needs. */
size_t oppb_field_work_doubles(int32_t neq);

/* Result of a solve (device).  iterations / converged of the last call; resid = ||r|| / ||B||. */
typedef struct oppb_field_status {
    int32_t iterations;
    int32_t converged;
    double  resid;
    double  b_norm;
} oppb_field_status;

/* compute_node_charge_density_kernel over the nodes: n_charge_den *= spwt / n_vol. */
int oppb_node_charge_density(double* n_charge_den, const double* n_vol, double spwt, int32_t n_nodes,
                             void* stream);

/* FESolver::compute_phi: tempNEQ1/2/3 from D and ion_den (init_f1_and_J), F1 += the cell
 * integrals of tempNEQ1 (build_f1_vector; F1 is never reset, as in the reference), the
 * diagonal of J = K - diag(integrals of tempNEQ3) (build_j_matrix), B = K D - F0 - F1, CG on
 * J Y = B (Jacobi preconditioner, one cooperative launch), D -= Y, then node_potential =
 * n_bnd_pot + D on unknowns (compute_node_potential).  ion_den, node_potential: device
 * [n_nodes].  status: device, written at the end. */
int oppb_field_solve(const oppb_field_device* f, const oppb_field_consts* c, const double* ion_den,
                     double* node_potential, oppb_field_status* status, void* stream);

/* compute_electric_field_kernel over the cells after opp_reset_dat(c_ef):
 * c_ef[d] = 0 - (((sd0 phi0 + sd1 phi1) + sd2 phi2) + sd3 phi3) per dimension.  c_sd
 * [n_cells][4][3] and c2n [n_cells][4] in the host (AoS) layout; cell c's field goes to
 * c_ef[c * ef_stride + d] (3 for the reference's AoS c_ef, 4 for the move's packed
 * oppb_tet_mesh::ef record, whose fourth word is left alone). */
int oppb_electric_field(const int32_t* c2n, const double* c_sd, const double* node_potential, double* c_ef,
                        int32_t ef_stride, int32_t n_cells, void* stream);

/* Element (c, k) of a per-cell array at base[c * cell_stride + k * comp_stride]: AoS arrays
 * have (dim, 1), the opp_* runtime's device dats and maps (SoA) have (1, n_cells). */
typedef struct oppb_cell_layout {
    int64_t cell_stride;
    int64_t comp_stride;
} oppb_cell_layout;

/* compute_electric_field_kernel with explicit layouts: c2n components = the 4 vertices,
 * c_sd components = vertex * 3 + dimension, c_ef components = dimension.  accumulate = 1
 * subtracts from c_ef as the generated loop's OPP_INC does (the caller resets c_ef first,
 * as the generated main does); accumulate = 0 writes 0 - sum. */
int oppb_electric_field_ex(const int32_t* c2n, oppb_cell_layout c2n_layout, const double* c_sd,
                           oppb_cell_layout sd_layout, const double* node_potential, double* c_ef,
                           oppb_cell_layout ef_layout, int32_t n_cells, int32_t accumulate, void* stream);

/* Largest of init and the n values x[i] (|x[i]| when absolute = 1): the OPP_MAX global
 * reduction of get_max_cef_kernel and get_final_max_values_kernel (apps/app_fempic/kernels.h:
 * 205-223).  Synchronous: *result (host) holds the value on return.  The reduction word is
 * fixed device scratch, so calls on one device must not overlap. */
int oppb_reduce_max(const double* x, int64_t n, int32_t absolute, double init, double* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_FIELD_H */
