/*
 * oppb_graph.h — the FemPIC particle step with its particle count kept in device memory, so
 * that whole steps (inject -> push + move + deposit -> hole fill or cell sort) can be
 * captured as one CUDA graph and replayed with no host synchronisation between them.
 *
 * The reference sizes its compaction on the host: opp_finalize_particle_move reads the
 * remove count back after every move (opp_lib/src/cuda/opp_particle_comm.cu:115-226) and the
 * next injection starts at the host's set size.  Here the count lives in an oppb_set_count
 * on the device; every kernel of a step reads it there, and oppb_step_end_dev subtracts the
 * step's removals and records the step.  Grids are sized from a host upper bound of the
 * particle count (`size_bound`: the count before the steps plus everything they can inject),
 * and blocks beyond the device count return at once.  The host reads the count and the step
 * records once per replay.
 *
 * Results are bit-identical to the host-sized entry points of oppb.h on the same inputs: the
 * same kernels run on the same particles.  One difference of form: a cell sort that finds no
 * removed particle (the reference does nothing then, opp_particle_organize_core.cpp:61-80)
 * copies every dat into its swap buffer unchanged, because the graph's later launches read
 * the swapped buffers; the contents are the same.
 *
 * Reference paths are relative to the OP-PIC source tree.
 */
#ifndef OPPB_GRAPH_H
#define OPPB_GRAPH_H

#include <stddef.h>
#include <stdint.h>

#include "oppb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device-resident count of a particle set (16 B, device memory). */
typedef struct oppb_set_count {
    int32_t size;        /* particles [0,size) are live between steps (opp_set::size)        */
    int32_t error;       /* first error of a device-sized step since the host cleared it     */
    int32_t error_step;  /* value of `steps` when that error was raised                      */
    int32_t steps;       /* steps closed by oppb_step_end_dev                                 */
} oppb_set_count;

/* What oppb_step_end_dev records of one step (32 B, device memory). */
typedef struct oppb_step_record {
    int32_t  size_before_move;  /* particles moved: the count after injection          */
    int32_t  removed;           /* particles the move removed                         */
    int32_t  size;              /* the count after the compaction                     */
    int32_t  max_visits;        /* the move status's largest cell-visit count         */
    uint64_t total_visits;
    int32_t  recheck_count;
    int32_t  error;             /* the move's error word (0 = none)                   */
} oppb_step_record;

/* oppb_inject_f64 with start = count->size read on the device: particles go to slots
 * [size, size + n_inject).  When they would not fit in parts->stride the kernel writes
 * nothing and records OPPB_ERR_CAPACITY in count->error.  parts->size is not read.  The
 * count itself is not changed here: the step's later launches take `pending` = n_inject. */
int oppb_inject_dev(const oppb_tet_mesh* mesh, const oppb_inlet* inlet, const oppb_particles* parts,
                    oppb_set_count* count, int32_t n_inject, const double* rnd, int32_t rnd_stride,
                    int32_t rnd_dim, double ion_velocity, double qm, double dt, void* stream);

/* The move entry points take the device count through oppb_move_options (oppb_dh.h):
 * set_count and pending.  Then parts->size is the upper bound that sizes the grid and the
 * move processes [0, min(set_count->size + pending, parts->size)). */

/* Scratch bytes of oppb_hole_fill_dev for counts up to size_bound. */
size_t oppb_hole_fill_dev_workspace_bytes(int32_t size_bound);

/* oppb_hole_fill over [0, count->size + pending) with remove_count = status->remove_count,
 * both read on the device (the same pairs, bit for bit).  size_bound bounds the count. */
int oppb_hole_fill_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                       const oppb_move_status* status, const uint32_t* remove_bits, int32_t stride,
                       int32_t n_dats, const oppb_dat* dats, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Scratch bytes of oppb_sort_by_cell_dev for counts up to size_bound. */
size_t oppb_sort_dev_workspace_bytes(int32_t size_bound);

/* oppb_sort_by_cell over [0, count->size + pending) read on the device: every dat is gathered
 * into its swap buffer in cell order.  When status->remove_count is 0 the dats are copied into
 * their swap buffers unchanged instead (see above); either way the caller swaps the buffers. */
int oppb_sort_by_cell_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                          const oppb_move_status* status, int32_t n_cells, int32_t stride, int32_t n_dats,
                          const oppb_dat* dats, int32_t key_dat, void* workspace, size_t workspace_bytes,
                          void* stream);

/* oppb_shuffle over [0, count->size + pending) read on the device; with status->remove_count
 * 0 a copy into the swap buffers, as oppb_sort_by_cell_dev. */
int oppb_shuffle_dev(int32_t size_bound, const oppb_set_count* count, int32_t pending,
                     const oppb_move_status* status, int32_t n_cells, int32_t stride, int32_t n_dats,
                     const oppb_dat* dats, int32_t key_dat, uint64_t seed, void* workspace, size_t workspace_bytes,
                     void* stream);

/* Closes a step (one thread): records {count->size + pending, status} into
 * records[count->steps % n_records], copies a move error into count->error (first one
 * kept), sets count->size = count->size + pending - status->remove_count and advances
 * count->steps.  The role of `set->size -= particle_remove_count` in
 * opp_finalize_particle_move (opp_lib/src/cuda/opp_particle_comm.cu:115-226). */
int oppb_step_end_dev(oppb_set_count* count, int32_t pending, const oppb_move_status* status,
                      oppb_step_record* records, int32_t n_records, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPPB_GRAPH_H */
