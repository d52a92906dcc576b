/*
 * oppb.h — C ABI of the B200 particle hot path (move, deposit, push, inject,
 * hole fill, cell sort) for unstructured tetrahedral meshes.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (OPPB_OK = 0).  Pointers named "device" must point to
 * CUDA device memory of the current device; all launches are asynchronous on
 * `stream` (a cudaStream_t passed as void*, NULL = the legacy default stream).
 * Nothing here allocates device memory: scratch space is passed in by the
 * caller (see the *_workspace_bytes queries).
 *
 * Each entry point names the reference interface whose body it replaces.
 * Reference paths are relative to the OP-PIC source tree.
 */
#ifndef OPPB_H
#define OPPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define OPPB_OK              0
#define OPPB_ERR_ARG         1  /* null pointer, negative size, bad alignment      */
#define OPPB_ERR_LAUNCH      2  /* CUDA reported an error at launch                */
#define OPPB_ERR_WORKSPACE   3  /* workspace smaller than *_workspace_bytes()      */
#define OPPB_ERR_HOP_LIMIT   4  /* device: a particle exceeded max_hops cell visits */
#define OPPB_ERR_CELL_RANGE  5  /* device: p2c / c2c / c2n index out of range       */
#define OPPB_ERR_CAPACITY    6  /* injection would exceed the set capacity          */
#define OPPB_ERR_NO_DEVICE   7  /* no CUDA device visible                           */
#define OPPB_ERR_SCRATCH_LIMIT 8 /* request larger than a fixed in-library scratch  */
#define OPPB_ERR_WAIT_LIMIT  9  /* device: a bounded wait for an asynchronous copy ran out */

/* Cell index of a removed particle: MAX_CELL_INDEX in opp_lib/include/opp_defs.h:150. */
#define OPPB_REMOVED_CELL 2147483647

/* ------------------------------------------------------------------ types */

/* Device-resident tetrahedral mesh in the packed layout the kernels read: one cell
 * visit of the FP64 move is four 256-bit loads of `det` and one of `nav`; of the mixed
 * move two of `geo32` (64 B), plus one 16-B read of the nav32 neighbours when the
 * particle hops on.  Filled by oppb_tet_mesh_pack(); buffers are
 * owned by the caller and 32-byte aligned (oppb_tet_mesh_bytes gives the sizes).
 *   det   [n_cells][16] f64 : {alpha,beta,gamma,delta} of vertex 0..3
 *                             (minifempic_funcs.h:316-382 ordering), 128-B record
 *   nav   [n_cells][4] 64-bit: coef = (1.0/6.0)/c_volume (kernels.h:110), then
 *                             c2c[0..3] as four int32 (face opposite vertex i, -1 =
 *                             boundary), then 8 unused bytes; 32-B record
 *   c2n   [n_cells][4]  i32 : cell -> node map (deposit)
 *   ef    [n_cells][4]  f64 : cell electric field x,y,z + pad
 *   geo32 [n_cells][16] f32 : mixed path, for vertices 0..2 {lambda_i(o), dlambda_i/dx,
 *                             dlambda_i/dy, dlambda_i/dz} about origin o, then o = vertex 0
 *                             rounded to f32 (3 floats) and G, the rounded-up sum of the nine
 *                             |dlambda_i/dx_j| (the FP32 error bound's factor; +inf when the
 *                             rows' |lambda_i(o)| sum above 1.001); lambda_3 is
 *                             1 - lambda_0 - lambda_1 - lambda_2 (may be NULL)
 *   nav32 [n_cells][8] 32-bit: mixed path origin o (3 floats), one unused word,
 *                             c2c[0..3] as int32 (may be NULL) */
typedef struct oppb_tet_mesh {
    int32_t  n_cells;
    int32_t  n_nodes;
    double*  det;
    double*  nav;
    int32_t* c2n;
    double*  ef;
    float*   geo32;
    float*   nav32;
} oppb_tet_mesh;

/* Particle set in the reference's device layout: SoA [dim][stride]
 * (opp_lib/src/cuda/opp_cuda_utils.cu:128-143), stride = set capacity. */
typedef struct oppb_particles {
    int32_t   size;        /* particles [0,size) are live / processed          */
    int32_t   stride;      /* SoA stride of every particle dat (capacity)      */
    double*   pos;         /* [3][stride] p_position                           */
    double*   vel;         /* [3][stride] p_velocity                           */
    double*   lc;          /* [4][stride] p_lc (barycentric weights)           */
    int32_t*  p2c;         /* [stride]    particle -> cell (mesh relation)     */
    uint32_t* remove_bits; /* [ceil(stride/32)] bit i = (p2c[i]==REMOVED) after a move */
} oppb_particles;

/* Device-side result of one move.  The move launchers zero it first. */
typedef struct oppb_move_status {
    int32_t  remove_count;   /* particles removed by this move (opp_set::particle_remove_count) */
    int32_t  error;          /* first device error (OPPB_ERR_HOP_LIMIT / _CELL_RANGE), 0 = none */
    int32_t  error_index;    /* particle index that raised `error`                              */
    int32_t  max_visits;     /* largest number of cells one particle visited                    */
    uint64_t total_visits;   /* sum over particles of cells visited                             */
    int32_t  recheck_count;  /* mixed path: particles whose decision was re-evaluated in FP64   */
    int32_t  reserved;
} oppb_move_status;

/* One particle dat for compaction / sort: SoA [dim][stride] of elem_bytes. */
typedef struct oppb_dat {
    void*   data;        /* device, current contents                         */
    void*   swap;        /* device, same shape; sort gathers into it (may be NULL for hole fill) */
    int32_t dim;
    int32_t elem_bytes;  /* 4 or 8 */
} oppb_dat;

/* Inlet faces for injection (FemPIC inlet surface, minifempic_funcs.h:508-583).
 *   dist [n_faces] i32 : cumulative particle count per face (fempic_misc.h:42-80)
 *   if2c [n_faces] i32 : cell attached to the face
 *   geom [n_faces][12] f64 : u[3], v[3], normal[3], node0 position[3]          */
typedef struct oppb_inlet {
    int32_t        n_faces;
    const int32_t* dist;
    const int32_t* if2c;
    const double*  geom;
} oppb_inlet;

/* ------------------------------------------------------------------ setup */

const char* oppb_version(void);
const char* oppb_status_string(int status);

/* Number of CUDA kernels this library has launched in the process so far (every
 * launcher adds its launches; memsets are not counted). */
uint64_t oppb_kernel_launches(void);

/* Launch choices of the move kernels (process-wide; the autotuner's output). */
#define OPPB_DEPOSIT_WARP_ATOMIC 0  /* lanes grouped by final cell (warp match), FP64 atomics per group */
#define OPPB_DEPOSIT_CTA_TABLE   1  /* per-CTA shared-memory node-sum table, one global atomic per node */
/* Deterministic mode: every weight w is cut to the fixed-point value floor(w 2^52) 2^-52 (held
 * as an int32 multiple of 2^-20 plus a uint32 multiple of 2^-52) and the node sums are integer sums,
 * so node_charge gains exactly sum_i trunc(w_i) whatever the particle order, warp grouping or
 * launch shape, bit for bit from run to run (one rounding when the integer sum is turned into
 * FP64).  Each term is within 2^-52 of its weight.  Needs 16 B per node of workspace
 * (oppb_deposit_workspace_bytes) and weights in (-2^11, 2^11). */
#define OPPB_DEPOSIT_EXACT       2
typedef struct oppb_tuning {
    int32_t deposit;     /* OPPB_DEPOSIT_* */
    int32_t replicas;    /* node-sum copies the deposit spreads its atomics over (1..64, default 8) */
    int32_t advec_items; /* NESO-advection step: 256-particle work items per block pass, i.e.
                            particles per thread in flight (1, 2 or 4; default 2) */
    int32_t sort_gather_cols; /* cell sort: particle-dat columns gathered per launch (1..16, default 16) */
    int32_t move_lanes;  /* lanes per particle of the FP64 move: 1 (0 reads as 1) = a particle per thread,
                            32 per warp; 2 = a particle per lane pair, 16 per warp, each lane reading one
                            64-B half of the cell record and computing two of the four lambdas */
    int32_t move_occupancy; /* lane-pair FP64 move: CTAs per SM it is compiled for, 8 (0 reads as 8;
                               32 registers a thread) or 5 (48 registers, no spills) */
    int32_t sort_scatter;   /* cell sort / shuffle: 0 = gather every dat by destination (scattered
                               reads, coalesced writes), 1 = scatter by source (coalesced reads,
                               scattered writes); the same result */
    int32_t move_stage;     /* FP64 move, one lane per particle: 0 = each visit's cell record read by
                               the lane's own 256-bit loads; 1 = staged into shared memory by bulk
                               asynchronous copies (cp.async.bulk, one per record half, completed on
                               a warp's mbarrier) and read from there; the same results */
    int32_t move_block;     /* threads per CTA of the one-lane FP64 and mixed moves with the warp-grouped
                               deposit: 128, 256 (0 reads as 256) or 512, with 2048 / move_block CTAs
                               resident per SM (32 registers a thread); the other deposits, the lane-pair
                               and the staged kernels use 256.  The same results */
    int32_t cabana_occupancy; /* CabanaPIC move + deposit: resident CTAs per SM it is compiled for:
                                 0 = the compiler's register count, 4 (default; 64 registers a
                                 thread) or 5 (48 registers, small spills).  The same results */
    int32_t move_walk32;      /* FP64 move + deposit: 1 = walk on the mixed path's FP32 records (each
                                 inside test and argmin decided in FP32 or, near a threshold, by the
                                 FP64 expression, so equal to the FP64 decision) and evaluate the FP64
                                 lambdas once at the last cell), compiled for 8 CTAs per SM; 2 = the
                                 same compiled for 6; used when the mesh holds geo32 and nav32
                                 (else the plain FP64 kernel runs).  0 (default) = the FP64 walk.
                                 The same results either way, bit for bit */
} oppb_tuning;

/* Set / read the tuning used by subsequent launches (OPPB_ERR_ARG on unknown values). */
int oppb_set_tuning(const oppb_tuning* tuning);
void oppb_get_tuning(oppb_tuning* out);

/* Bytes of each packed mesh buffer for n_cells cells (det, nav, c2n, ef, geo32, nav32). */
void oppb_tet_mesh_bytes(int32_t n_cells, size_t out_bytes[6]);

/* Pack the reference's device-layout cell dats (SoA [dim][soa_stride], as uploaded by
 * opp_upload_dat, opp_lib/src/cuda/opp_cuda_utils.cu:119-152) into the records of *mesh,
 * and, when mesh->geo32/nav32 are non-NULL, the mixed-precision records (needs n_pos,
 * SoA [3][n_pos_stride]).  Each input may be NULL, leaving its part of the records
 * untouched: c_det and c_volume (det, nav coef), c2c (nav and nav32 neighbours), c2n (c2n),
 * c_ef (ef); geo32 and the nav32 origin need c_det, c_volume, c2n and n_pos.  invalid_out (device
 * int32, may be NULL) receives the number of c2c entries outside {-1}u[0,n_cells) and
 * c2n entries outside [0,n_nodes); kernels never dereference such entries.
 * Replaces the per-loop SoA gathers of the generated move loop
 * (apps_codegen/app_fempic_cg/cuda/move_kernel_loop.hpp:287-301). */
int oppb_tet_mesh_pack(oppb_tet_mesh* mesh, int32_t soa_stride,
                       const double* c_det, const double* c_volume,
                       const int32_t* c2c, const int32_t* c2n, const double* c_ef,
                       const double* n_pos, int32_t n_pos_stride,
                       int32_t* invalid_out, void* stream);

/* Upload a cell electric field (SoA [3][soa_stride]) into mesh->ef. */
int oppb_tet_mesh_set_ef(oppb_tet_mesh* mesh, int32_t soa_stride, const double* c_ef, void* stream);

/* ------------------------------------------------------------------- move */

/* FP64 multi-hop move.  Body of opp_particle_move__move_kernel
 * (apps_codegen/app_fempic_cg/cuda/move_kernel_loop.hpp:189-401, user kernel
 * apps/app_fempic/kernels.h:106-161, status rule opp_lib/include/opp_seq.h:68-86):
 * writes p_lc and p2c, sets p2c = OPPB_REMOVED_CELL for particles leaving the mesh,
 * fills remove_bits and *status (device).  Cell decisions are bit-identical to the
 * FP64 seq backend.  max_hops bounds the cell visits per particle (the reference
 * loop is unbounded); hitting it sets status->error = OPPB_ERR_HOP_LIMIT. */
int oppb_move_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                  oppb_move_status* status, int32_t max_hops, void* stream);

/* Scratch bytes a deposit (fused or standalone) can use for n_nodes nodes: the node-sum
 * copies beyond the first for the tuned replica count (with less, or NULL, the deposit adds
 * straight into node_charge); with OPPB_DEPOSIT_EXACT the two integer sums per node, which
 * the deposit requires (OPPB_ERR_WORKSPACE when they do not fit). */
size_t oppb_deposit_workspace_bytes(int32_t n_nodes);

/* FP64 move with the node-charge deposit of the final cell fused in:
 * node_charge[c2n[p2c][i]] += p_lc[i] for every particle that stays
 * (apps/app_fempic/kernels.h:164-175).  Lanes of a warp ending in the same cell are
 * summed first; the sums go to FP64 atomics spread over replica copies of the node array
 * (in `workspace`, zeroed here) that are added into node_charge at the end, as the
 * reference spreads its atomics over thread-level copies (opp_lib/include/opp_cuda.h:526-588). */
int oppb_move_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                          double* node_charge, oppb_move_status* status, int32_t max_hops,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Mixed-precision move + deposit: barycentric tests in FP32 about a per-cell origin;
 * any particle whose decision lies within `band` of a threshold or tie is re-evaluated
 * with the FP64 reference formula, so cell assignment, hop counts and removals stay
 * bit-identical to oppb_move_deposit_f64.  p_lc carries FP32 accuracy (within 1e-5 of
 * FP64); node totals accumulate in FP64.  Needs mesh->geo32/nav32. */
int oppb_move_deposit_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                            double* node_charge, oppb_move_status* status, int32_t max_hops,
                            double band, void* workspace, size_t workspace_bytes, void* stream);

/* Push fused into the move as its once-per-particle prologue (the OPP_DO_ONCE pattern,
 * opp_lib/include/opp_seq.h:64): calculate_new_pos_vel_kernel (apps/app_fempic/kernels.h:93-103,
 * replacing opp_par_loop_all__calculate_new_pos_vel_kernel) on every particle with a valid
 * cell, then the move + deposit of the entry points above on the pushed position held in
 * registers.  p_pos and p_vel are written; results are bit-identical to oppb_push_f64 +
 * oppb_move_deposit_f64 (oppb_push_mixed + oppb_move_deposit_mixed for the mixed form).
 * Needs parts->vel and mesh->ef. */
int oppb_push_move_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                               double* node_charge, oppb_move_status* status, int32_t max_hops,
                               double charge_over_mass, double dt,
                               void* workspace, size_t workspace_bytes, void* stream);
int oppb_push_move_deposit_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                                 double* node_charge, oppb_move_status* status, int32_t max_hops,
                                 double band, double charge_over_mass, double dt,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- deposit */

/* Standalone deposit over [0,size): body of opp_par_loop_all__deposit_charge_on_nodes_kernel
 * (apps_codegen/app_fempic_cg/cuda/deposit_charge_on_nodes_kernel_loop.hpp:92-165). */
int oppb_deposit_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                     double* node_charge, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------- push */

/* v += (qm*dt)*E[p2c]; x += v*dt  (apps/app_fempic/kernels.h:93-103), FP64, bit-identical
 * to the seq backend.  Body of opp_par_loop_all__calculate_new_pos_vel_kernel. */
int oppb_push_f64(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                  double qm, double dt, void* stream);

/* Same update with FP32 increments on FP64 state: dv = f32(qm*dt)*f32(E),
 * v += dv; dx = f32(v)*f32(dt), x += dx. */
int oppb_push_mixed(const oppb_tet_mesh* mesh, const oppb_particles* parts,
                    double qm, double dt, void* stream);

/* ----------------------------------------------------------------- inject */

/* Inject `count` particles into slots [start, start+count): face of particle k is the
 * first face j with k < dist[j] (opp_lib/src/cuda/opp_increase_part_count.cu:86-105,
 * found by binary search), then inject_ions_kernel (apps/app_fempic/kernels.h:63-90):
 *   pos = a*u + b*v + node0  ((a,b) folded into the triangle),
 *   vel = normal*ion_velocity - qm*E*(0.5*dt) + thermal,  p2c = if2c[face].
 * When inlet->dist is NULL the face index is taken from p2c[start+k] instead, as left
 * there by oppb_assign_faces (the reference's split into the two calls).
 * rnd is SoA [rnd_dim][rnd_stride] indexed by k: a, b and, when rnd_dim == 5, the
 * thermal velocity vx, vy, vz (rnd_dim == 2 is the reference's dummy_part_random).
 * start+count must not exceed parts->stride (else OPPB_ERR_CAPACITY). */
int oppb_inject_f64(const oppb_tet_mesh* mesh, const oppb_inlet* inlet,
                    const oppb_particles* parts, int32_t start, int32_t count,
                    const double* rnd, int32_t rnd_stride, int32_t rnd_dim,
                    double ion_velocity, double qm, double dt, void* stream);

/* Face assignment of opp_inc_part_count_with_distribution: p2c[start+k] = first face j
 * with k < dist[j], k in [0,count) (opp_lib/src/cuda/opp_increase_part_count.cu:86-105;
 * the seq backend's rule, opp_increase_part_count_core.cpp:134-142, agrees whenever no face
 * is empty). */
int oppb_assign_faces(const oppb_inlet* inlet, int32_t* p2c, int32_t start, int32_t count, void* stream);

/* Fill count elements of elem_bytes (4 or 8) at dst with the low bytes of `pattern`
 * (opp_reset_dat of one component; the removed-cell fill of new particle slots). */
int oppb_fill(void* dst, int64_t count, int32_t elem_bytes, uint64_t pattern, void* stream);

/* ------------------------------------------------------------- compaction */

/* Scratch bytes oppb_hole_fill needs for `size` particles of which `remove_count` were removed. */
size_t oppb_hole_fill_workspace_bytes(int32_t size, int32_t remove_count);

/* Hole fill after a move: the k-th removed slot (ascending) receives the k-th live
 * particle counted from the back, while that particle lies behind the slot
 * (opp_lib/src/core/opp_particle_organize_core.cpp:124-218; CUDA
 * opp_lib/src/cuda/opp_particle_sorter.cu:264-363).  Holes are the set bits of
 * remove_bits over [0,size); at most remove_count pairs move.  Every dat moves
 * together.  The caller then sets size -= remove_count. */
int oppb_hole_fill(int32_t size, int32_t remove_count, const uint32_t* remove_bits,
                   int32_t stride, int32_t n_dats, const oppb_dat* dats,
                   void* workspace, size_t workspace_bytes, void* stream);

/* remove_bits for oppb_hole_fill from the cells a move left: bit i of word i / 32 set where
 * p2c[i] == OPPB_REMOVED_CELL, for i in [0, size) (ceil(size / 32) words written).  For moves
 * that mark removed particles in p2c only (the advection move's global-move pre-pass). */
int oppb_removal_bits(const int32_t* p2c, int32_t size, uint32_t* remove_bits, void* stream);

/* Largest remove_count that oppb_hole_fill_static accepts. */
#define OPPB_HOLE_FILL_STATIC_MAX_REMOVES 1048576

/* oppb_hole_fill without a workspace argument and without allocating anything: no
 * counterpart in the reference.  It is for callers that cannot call cudaMalloc at the
 * point of the move: a plugin that holds only the particle dats' device pointers while
 * another runtime owns all device memory through its own pool, or a step loop that must
 * not pay cudaMalloc/cudaFree's implicit device-wide synchronisation.  Same arguments and
 * same result as oppb_hole_fill, bit for bit.
 *
 * Its scratch is a fixed array inside the library, about 8.5 MiB on every GPU that loads
 * the library, held until the process exits; remove_count above
 * OPPB_HOLE_FILL_STATIC_MAX_REMOVES returns OPPB_ERR_SCRATCH_LIMIT and changes nothing.
 * The first call on each device looks the array's device address up with that device
 * current; make that first call before any stream capture begins.  Calls outside a capture
 * look the address up again, so the entry point stays valid after cudaDeviceReset once a
 * call outside a capture has been made on the reset device.  All calls on a device
 * share the one array, so calls that may overlap on the GPU (other streams, other host
 * threads) race and must be ordered by the caller. */
int oppb_hole_fill_static(int32_t size, int32_t remove_count, const uint32_t* remove_bits,
                          int32_t stride, int32_t n_dats, const oppb_dat* dats, void* stream);

/* Scratch bytes oppb_sort_by_cell needs. */
size_t oppb_sort_workspace_bytes(int32_t size, int32_t n_cells);

/* Stable sort of particles [0,size) by cell (removed particles, p2c = REMOVED, last),
 * then gather every dat into its `swap` buffer (opp_particle_sort_core,
 * opp_lib/src/core/opp_particle_organize_core.cpp:98-121; CUDA particle_sort_device,
 * opp_lib/src/cuda/opp_particle_sorter.cu:167-246).  dats[key_dat] must be the p2c dat.
 * perm_out (device, may be NULL) receives the source index of every destination slot.
 * Hand-written LSD radix sort (8-bit digits), no library sort. */
int oppb_sort_by_cell(int32_t size, int32_t n_cells, int32_t stride,
                      int32_t n_dats, const oppb_dat* dats, int32_t key_dat,
                      int32_t* perm_out, void* workspace, size_t workspace_bytes,
                      void* stream);

/* Shuffle of particles [0,size) for opp_fill = Shuffle_All / Shuffle_Periodic: the particles
 * with a valid cell in a random order, removed particles (p2c outside [0,n_cells)) last, then
 * every dat, the p2c dat included, gathered into its `swap` buffer (the CUDA backend's
 * particle_sort_device with shuffle = true, opp_lib/src/cuda/opp_particle_sorter.cu:167-246,
 * which sorts by random keys from a RandomFunctor seeded 123, :40-54).  Here the keys are 30
 * bits of a splitmix64 hash of (seed, index), seed != 0, sorted stably by the same radix sort:
 * deterministic for a seed, but not the reference's draws (its engine is Thrust's), so the
 * order within the live particles is not the reference's.  The seq backend's shuffle sorts by
 * cell (opp_particle_sort_core ignores the flag, opp_particle_organize_core.cpp:98-121).
 * Workspace as oppb_sort_by_cell. */
int oppb_shuffle(int32_t size, int32_t n_cells, int32_t stride, int32_t n_dats, const oppb_dat* dats,
                 int32_t key_dat, uint64_t seed, int32_t* perm_out, void* workspace, size_t workspace_bytes,
                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_H */
