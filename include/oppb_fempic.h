/*
 * oppb_fempic.h — host-side (CPU) set-up utilities of the FemPIC application
 * around the particle hot path: the box tetrahedral mesh with the reference's
 * per-cell geometry, the inlet surface, the injection distribution and the
 * static electric field (linear FEM Laplace potential, FP64 conjugate gradient).
 * None of this runs per particle; it prepares the inputs of the kernels in oppb.h.
 */
#ifndef OPPB_FEMPIC_H
#define OPPB_FEMPIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Node types (apps/app_fempic/minifempic_funcs.h NodeType). */
#define OPPB_NODE_NORMAL 0
#define OPPB_NODE_OPEN   1
#define OPPB_NODE_INLET  2
#define OPPB_NODE_FIXED  3

/* Host AoS arrays (the reference's host layout), malloc-owned by the struct. */
typedef struct oppb_fempic_mesh {
    int32_t  n_nodes, n_cells, n_ifaces;
    double*  n_pos;      /* [n_nodes][3]                                     */
    double*  n_vol;      /* [n_nodes]    node volumes (minifempic_funcs.h:446-461) */
    int32_t* n_type;     /* [n_nodes]    OPPB_NODE_*                         */
    double*  n_bnd_pot;  /* [n_nodes]    Dirichlet value of INLET/FIXED nodes */
    int32_t* c2n;        /* [n_cells][4]                                     */
    int32_t* c2c;        /* [n_cells][4] face opposite vertex i, -1 = boundary */
    double*  c_det;      /* [n_cells][16] alpha,beta,gamma,delta per vertex  */
    double*  c_vol;      /* [n_cells]                                        */
    double*  c_sd;       /* [n_cells][4][3] gradient of barycentric weight i */
    double*  c_ef;       /* [n_cells][3] cell electric field                 */
    double*  c_centroid; /* [n_cells][3]                                     */
    int32_t* if2c;       /* [n_ifaces]                                       */
    int32_t* if2n;       /* [n_ifaces][3]                                    */
    double*  if_u;       /* [n_ifaces][3] node1 - node0                      */
    double*  if_v;       /* [n_ifaces][3] node2 - node0                      */
    double*  if_norm;    /* [n_ifaces][3] unit normal into the domain        */
    double*  if_area;    /* [n_ifaces]                                       */
    double*  if_n_pos;   /* [n_ifaces][9] positions of the three face nodes  */
} oppb_fempic_mesh;

/* Box [0,lx]x[0,ly]x[0,lz] of nx*ny*nz hexahedra, each cut into 6 tetrahedra that
 * share the hexahedron's main diagonal (conforming between hexahedra).  Cell c of hex
 * h = i + nx*(j + ny*k) is 6*h + t.  Geometry follows apps/app_fempic/minifempic_funcs.h:
 * volume = det4/6 with the ABCD->ADBC flip (:284-313), alpha..delta cofactors
 * (:316-382), face neighbours (:386-437), node volumes (:440-474).  The inlet is the
 * z=0 face (two triangles per hex face, normal +z); inlet nodes are INLET, z=lz nodes
 * FIXED, other boundary nodes OPEN.  Returns 0 on success. */
int oppb_fempic_box_mesh(int32_t nx, int32_t ny, int32_t nz,
                         double lx, double ly, double lz, oppb_fempic_mesh* out);

/* Linear-FEM potential with Dirichlet phi = phi_inlet on INLET nodes and phi_fixed on
 * FIXED nodes (natural boundary elsewhere), solved by FP64 CG to relative residual
 * rtol, then c_ef = -sum_i phi_i grad(lambda_i) accumulated as in
 * compute_electric_field_kernel (apps/app_fempic/kernels.h:186-202).
 * n_pot_out [n_nodes] may be NULL.  Returns 0 on convergence. */
int oppb_fempic_solve_field(oppb_fempic_mesh* m, double phi_inlet, double phi_fixed,
                            double rtol, int32_t max_iter, double* n_pot_out,
                            int32_t* iters_out, double* resid_out);

/* Cumulative injection counts per inlet face for `total` particles per step,
 * proportional to face area with no face empty when total >= n_ifaces
 * (role of init_inject_distributions, apps/app_fempic/fempic_misc.h:42-80). */
int oppb_fempic_inject_distribution(const oppb_fempic_mesh* m, int32_t total, int32_t* dist_out);

void oppb_fempic_mesh_free(oppb_fempic_mesh* m);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_FEMPIC_H */
