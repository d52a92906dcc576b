"""ctypes binding of the C ABI in include/oppb*.h.

The shared library is built in-tree (op-pic_b200/lib/liboppb.so).  Loading fails loudly
when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent.parent / "lib" / "liboppb.so"

OPPB_OK = 0
OPPB_ERR_ARG = 1
OPPB_ERR_LAUNCH = 2
OPPB_ERR_WORKSPACE = 3
OPPB_ERR_HOP_LIMIT = 4
OPPB_ERR_CELL_RANGE = 5
OPPB_ERR_CAPACITY = 6
OPPB_ERR_NO_DEVICE = 7
OPPB_ERR_SCRATCH_LIMIT = 8
OPPB_ERR_WAIT_LIMIT = 9
HOLE_FILL_STATIC_MAX_REMOVES = 1048576
REMOVED_CELL = 2147483647

c_i32, c_u32, c_i64, c_u64 = C.c_int32, C.c_uint32, C.c_int64, C.c_uint64
c_dp, c_fp, c_ip, c_vp = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int32), C.c_void_p


class TetMesh(C.Structure):
    _fields_ = [("n_cells", c_i32), ("n_nodes", c_i32), ("det", c_vp), ("nav", c_vp), ("c2n", c_vp),
                ("ef", c_vp), ("geo32", c_vp), ("nav32", c_vp)]


class Particles(C.Structure):
    _fields_ = [("size", c_i32), ("stride", c_i32), ("pos", c_vp), ("vel", c_vp), ("lc", c_vp), ("p2c", c_vp),
                ("remove_bits", c_vp)]


class MoveStatus(C.Structure):
    _fields_ = [("remove_count", c_i32), ("error", c_i32), ("error_index", c_i32), ("max_visits", c_i32),
                ("total_visits", c_u64), ("recheck_count", c_i32), ("reserved", c_i32)]


class SetCount(C.Structure):
    _fields_ = [("size", c_i32), ("error", c_i32), ("error_step", c_i32), ("steps", c_i32)]


class StepRecord(C.Structure):
    _fields_ = [("size_before_move", c_i32), ("removed", c_i32), ("size", c_i32), ("max_visits", c_i32),
                ("total_visits", c_u64), ("recheck_count", c_i32), ("error", c_i32)]


class Dat(C.Structure):
    _fields_ = [("data", c_vp), ("swap", c_vp), ("dim", c_i32), ("elem_bytes", c_i32)]


class Tuning(C.Structure):
    _fields_ = [("deposit", c_i32), ("replicas", c_i32), ("advec_items", c_i32), ("sort_gather_cols", c_i32),
                ("move_lanes", c_i32), ("move_occupancy", c_i32), ("sort_scatter", c_i32), ("move_stage", c_i32),
                ("move_block", c_i32), ("cabana_occupancy", c_i32), ("move_walk32", c_i32)]


DEPOSIT_WARP_ATOMIC = 0
DEPOSIT_CTA_TABLE = 1
DEPOSIT_EXACT = 2  # OPPB_DEPOSIT_EXACT: integer fixed-point node sums, order-independent


class Inlet(C.Structure):
    _fields_ = [("n_faces", c_i32), ("dist", c_vp), ("if2c", c_vp), ("geom", c_vp)]


class HexMesh(C.Structure):
    _fields_ = [("n_cells", c_i32), ("c2f", c_vp), ("interp", c_vp), ("interp32", c_vp)]


class CabanaParticles(C.Structure):
    _fields_ = [("size", c_i32), ("stride", c_i32), ("pos", c_vp), ("vel", c_vp), ("streak_mid", c_vp),
                ("weight", c_vp), ("p2c", c_vp)]


class CabanaConsts(C.Structure):
    _fields_ = [("qdt_2mc", C.c_double), ("cdt_d", C.c_double * 3), ("qsp", C.c_double)]


class AdvecInstance(C.Structure):
    _fields_ = [("part_offset", c_i64), ("n_parts", c_i32), ("cell_offset", c_i32), ("n_cells", c_i32),
                ("grid_nx", c_i32), ("dt", C.c_double), ("cell_width", C.c_double), ("extents", C.c_double * 2)]


class AdvecBatch(C.Structure):
    _fields_ = [("n_instances", c_i32), ("n_work", c_i32), ("instances", c_vp), ("tile_prefix", c_vp),
                ("cells", c_vp), ("stride", c_i64), ("pos", c_vp), ("vel", c_vp), ("mdir", c_vp), ("p2c", c_vp),
                ("work_counter", c_vp), ("dh", c_vp)]


class AdvecDh(C.Structure):
    _fields_ = [("map", c_vp), ("min", C.c_double * 2), ("inv_spacing", C.c_double), ("dims", c_i64 * 2)]


class DhGrid(C.Structure):
    _fields_ = [("min", C.c_double * 3), ("max", C.c_double * 3), ("spacing", C.c_double),
                ("inv_spacing", C.c_double), ("dims", c_i64 * 3), ("size", c_i64), ("map", c_vp)]


PRECISION_F64 = 0
PRECISION_MIXED = 1


class MoveOptions(C.Structure):
    _fields_ = [("precision", c_i32), ("deposit", c_i32), ("push", c_i32), ("reserved", c_i32),
                ("qm", C.c_double), ("dt", C.c_double), ("band", C.c_double), ("dh", C.POINTER(DhGrid)),
                ("set_count", c_vp), ("pending", c_i32), ("reserved2", c_i32)]


class FieldSystem(C.Structure):
    _fields_ = [("n_nodes", c_i32), ("n_cells", c_i32), ("neq", c_i32), ("node_to_eq", c_ip), ("c2n", c_ip),
                ("det_j", c_dp), ("c_sd", c_dp), ("n_bnd_pot", c_dp), ("k_rowptr", C.POINTER(c_i64)),
                ("k_col", c_ip), ("k_val", c_dp), ("f0", c_dp), ("nnz", c_i64), ("n_diag", c_i32),
                ("dia_off", c_i32 * 16), ("dia_val", c_dp)]


class FieldConsts(C.Structure):
    _fields_ = [("n0", C.c_double), ("phi0", C.c_double), ("kte", C.c_double), ("qe", C.c_double),
                ("eps0", C.c_double), ("rtol", C.c_double), ("atol", C.c_double), ("max_iter", c_i32),
                ("reserved", c_i32)]


class FieldDevice(C.Structure):
    _fields_ = [("n_nodes", c_i32), ("n_cells", c_i32), ("neq", c_i32), ("reserved", c_i32),
                ("node_to_eq", c_vp), ("c2n", c_vp), ("det_j", c_vp), ("n_bnd_pot", c_vp), ("k_rowptr", c_vp),
                ("k_col", c_vp), ("k_val", c_vp), ("f0", c_vp), ("d", c_vp), ("f1", c_vp), ("work", c_vp),
                ("n_diag", c_i32), ("dia_off", c_i32 * 16), ("dia_val", c_vp)]


class FieldStatus(C.Structure):
    _fields_ = [("iterations", c_i32), ("converged", c_i32), ("resid", C.c_double), ("b_norm", C.c_double)]


class FemPICMesh(C.Structure):
    _fields_ = [("n_nodes", c_i32), ("n_cells", c_i32), ("n_ifaces", c_i32),
                ("n_pos", c_dp), ("n_vol", c_dp), ("n_type", c_ip), ("n_bnd_pot", c_dp),
                ("c2n", c_ip), ("c2c", c_ip), ("c_det", c_dp), ("c_vol", c_dp), ("c_sd", c_dp),
                ("c_ef", c_dp), ("c_centroid", c_dp), ("if2c", c_ip), ("if2n", c_ip),
                ("if_u", c_dp), ("if_v", c_dp), ("if_norm", c_dp), ("if_area", c_dp), ("if_n_pos", c_dp)]


P = C.POINTER
_SIGS = {
    "oppb_version": (C.c_char_p, []),
    "oppb_status_string": (C.c_char_p, [C.c_int]),
    "oppb_kernel_launches": (C.c_uint64, []),
    "oppb_set_tuning": (C.c_int, [P(Tuning)]),
    "oppb_get_tuning": (None, [P(Tuning)]),
    "oppb_tet_mesh_bytes": (None, [c_i32, P(C.c_size_t)]),
    "oppb_tet_mesh_pack": (C.c_int, [P(TetMesh), c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp]),
    "oppb_tet_mesh_set_ef": (C.c_int, [P(TetMesh), c_i32, c_vp, c_vp]),
    "oppb_move_f64": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_i32, c_vp]),
    "oppb_deposit_workspace_bytes": (C.c_size_t, [c_i32]),
    "oppb_move_deposit_f64": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_vp, c_i32, c_vp, C.c_size_t, c_vp]),
    "oppb_move_deposit_mixed": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_vp, c_i32, C.c_double, c_vp,
                                          C.c_size_t, c_vp]),
    "oppb_push_move_deposit_f64": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_vp, c_i32, C.c_double, C.c_double,
                                             c_vp, C.c_size_t, c_vp]),
    "oppb_push_move_deposit_mixed": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_vp, c_i32, C.c_double, C.c_double,
                                               C.c_double, c_vp, C.c_size_t, c_vp]),
    "oppb_deposit_f64": (C.c_int, [P(TetMesh), P(Particles), c_vp, c_vp, C.c_size_t, c_vp]),
    "oppb_push_f64": (C.c_int, [P(TetMesh), P(Particles), C.c_double, C.c_double, c_vp]),
    "oppb_push_mixed": (C.c_int, [P(TetMesh), P(Particles), C.c_double, C.c_double, c_vp]),
    "oppb_inject_f64": (C.c_int, [P(TetMesh), P(Inlet), P(Particles), c_i32, c_i32, c_vp, c_i32, c_i32,
                                  C.c_double, C.c_double, C.c_double, c_vp]),
    "oppb_assign_faces": (C.c_int, [P(Inlet), c_vp, c_i32, c_i32, c_vp]),
    "oppb_fill": (C.c_int, [c_vp, c_i64, c_i32, c_u64, c_vp]),
    "oppb_hole_fill_workspace_bytes": (C.c_size_t, [c_i32, c_i32]),
    "oppb_hole_fill": (C.c_int, [c_i32, c_i32, c_vp, c_i32, c_i32, P(Dat), c_vp, C.c_size_t, c_vp]),
    "oppb_hole_fill_static": (C.c_int, [c_i32, c_i32, c_vp, c_i32, c_i32, P(Dat), c_vp]),
    "oppb_sort_workspace_bytes": (C.c_size_t, [c_i32, c_i32]),
    "oppb_sort_by_cell": (C.c_int, [c_i32, c_i32, c_i32, c_i32, P(Dat), c_i32, c_vp, c_vp, C.c_size_t, c_vp]),
    "oppb_shuffle": (C.c_int, [c_i32, c_i32, c_i32, c_i32, P(Dat), c_i32, c_u64, c_vp, c_vp, C.c_size_t, c_vp]),
    "oppb_inject_dev": (C.c_int, [P(TetMesh), P(Inlet), P(Particles), c_vp, c_i32, c_vp, c_i32, c_i32,
                                  C.c_double, C.c_double, C.c_double, c_vp]),
    "oppb_hole_fill_dev_workspace_bytes": (C.c_size_t, [c_i32]),
    "oppb_hole_fill_dev": (C.c_int, [c_i32, c_vp, c_i32, c_vp, c_vp, c_i32, c_i32, P(Dat), c_vp, C.c_size_t,
                                     c_vp]),
    "oppb_sort_dev_workspace_bytes": (C.c_size_t, [c_i32]),
    "oppb_sort_by_cell_dev": (C.c_int, [c_i32, c_vp, c_i32, c_vp, c_i32, c_i32, c_i32, P(Dat), c_i32, c_vp,
                                        C.c_size_t, c_vp]),
    "oppb_shuffle_dev": (C.c_int, [c_i32, c_vp, c_i32, c_vp, c_i32, c_i32, c_i32, P(Dat), c_i32, c_u64, c_vp,
                                   C.c_size_t, c_vp]),
    "oppb_step_end_dev": (C.c_int, [c_vp, c_i32, c_vp, c_vp, c_i32, c_vp]),
    "oppb_hex_mesh_pack": (C.c_int, [P(HexMesh), c_i32, c_vp, c_vp, c_vp]),
    "oppb_cabana_move_deposit": (C.c_int, [P(HexMesh), P(CabanaParticles), P(CabanaConsts), c_vp, c_i32, c_vp,
                                           c_i32, c_vp]),
    "oppb_cabana_move_deposit_mixed": (C.c_int, [P(HexMesh), P(CabanaParticles), c_vp, P(CabanaConsts), c_vp, c_i32,
                                                 c_vp, c_i32, c_vp]),
    "oppb_advec_pack_cells": (C.c_int, [c_vp, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp]),
    "oppb_advec_step": (C.c_int, [P(AdvecBatch), c_vp, c_i32, c_vp]),
    "oppb_advec_check_grid": (C.c_int, [c_vp, c_i32, c_i32, c_i32, C.c_double, c_vp, c_vp]),
    "oppb_advec_update_pos": (C.c_int, [P(AdvecBatch), c_vp]),
    "oppb_advec_move": (C.c_int, [P(AdvecBatch), c_vp, c_i32, c_vp]),
    "oppb_advec_verify": (C.c_int, [c_vp, c_i64, c_vp, c_vp, c_i32, c_i32, C.c_double, c_vp, c_vp]),
    "oppb_cabana_interpolate": (C.c_int, [c_i32, c_i64, c_vp, c_vp, P(c_vp), P(c_vp), c_vp, c_vp, c_vp]),
    "oppb_cabana_accumulate": (C.c_int, [c_i32, c_i64, c_vp, c_vp, P(c_vp), c_vp, P(C.c_double), c_vp]),
    "oppb_cabana_half_advance_b": (C.c_int, [c_i32, c_i64, P(c_vp), c_vp, c_vp, c_vp, P(C.c_double), c_vp]),
    "oppb_cabana_advance_e": (C.c_int, [c_i32, c_i64, P(c_vp), c_vp, c_vp, c_vp, c_vp, P(C.c_double), C.c_double,
                                        c_vp]),
    "oppb_cabana_update_ghosts": (C.c_int, [c_i32, c_i64, c_vp, c_i32, c_vp, c_vp, c_vp, c_i32, c_vp]),
    "oppb_cabana_energy_workspace_bytes": (C.c_size_t, []),
    "oppb_cabana_energy": (C.c_int, [c_i32, c_i64, c_vp, c_vp, c_vp, c_vp, C.c_size_t, c_vp]),
    "oppb_removal_bits": (C.c_int, [c_vp, c_i32, c_vp, c_vp]),
    "oppb_dh_grid_init": (C.c_int, [c_vp, c_i32, C.c_double, c_vp, P(DhGrid)]),
    "oppb_dh_build": (C.c_int, [P(TetMesh), c_vp, P(DhGrid), c_vp, C.c_size_t, P(C.c_size_t), c_vp]),
    "oppb_dh_bounding_box_2d": (C.c_int, [c_vp, c_i32, c_vp, c_vp, c_vp]),
    "oppb_dh_grid_init_2d": (C.c_int, [c_vp, c_i32, C.c_double, c_vp, P(DhGrid)]),
    "oppb_dh_build_quad": (C.c_int, [c_vp, c_i32, C.c_double, P(DhGrid), c_vp, C.c_size_t, P(C.c_size_t), c_vp]),
    "oppb_move_ex": (C.c_int, [P(TetMesh), P(Particles), P(MoveOptions), c_vp, c_vp, c_i32, c_vp, C.c_size_t,
                               c_vp]),
    "oppb_field_setup": (C.c_int, [P(FemPICMesh), P(FieldSystem)]),
    "oppb_field_system_free": (None, [P(FieldSystem)]),
    "oppb_field_work_doubles": (C.c_size_t, [c_i32]),
    "oppb_node_charge_density": (C.c_int, [c_vp, c_vp, C.c_double, c_i32, c_vp]),
    "oppb_field_solve": (C.c_int, [P(FieldDevice), P(FieldConsts), c_vp, c_vp, c_vp, c_vp]),
    "oppb_electric_field": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32, c_vp]),
    "oppb_fempic_box_mesh": (C.c_int, [c_i32, c_i32, c_i32, C.c_double, C.c_double, C.c_double, P(FemPICMesh)]),
    "oppb_fempic_solve_field": (C.c_int, [P(FemPICMesh), C.c_double, C.c_double, C.c_double, c_i32, c_dp,
                                          P(c_i32), P(C.c_double)]),
    "oppb_fempic_inject_distribution": (C.c_int, [P(FemPICMesh), c_i32, c_ip]),
    "oppb_fempic_mesh_free": (None, [P(FemPICMesh)]),
}

_lib = None


def load() -> C.CDLL:
    """Load liboppb.so (built by op-pic_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run op-pic_b200/build.py (no fallback implementation)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class OppbError(RuntimeError):
    def __init__(self, fn: str, status: int):
        msg = load().oppb_status_string(status).decode()
        super().__init__(f"{fn} failed: status {status} ({msg})")
        self.status = status


def check(fn: str, status: int) -> None:
    if status != OPPB_OK:
        raise OppbError(fn, status)


def set_tuning(deposit: int | None = None, replicas: int | None = None, advec_items: int | None = None,
               sort_gather_cols: int | None = None, move_lanes: int | None = None,
               move_occupancy: int | None = None, sort_scatter: int | None = None,
               move_stage: int | None = None, move_block: int | None = None,
               cabana_occupancy: int | None = None, move_walk32: int | None = None) -> None:
    t = Tuning()
    load().oppb_get_tuning(C.byref(t))
    if deposit is not None:
        t.deposit = deposit
    if replicas is not None:
        t.replicas = replicas
    if advec_items is not None:
        t.advec_items = advec_items
    if sort_gather_cols is not None:
        t.sort_gather_cols = sort_gather_cols
    if move_lanes is not None:
        t.move_lanes = move_lanes
    if move_occupancy is not None:
        t.move_occupancy = move_occupancy
    if sort_scatter is not None:
        t.sort_scatter = sort_scatter
    if move_stage is not None:
        t.move_stage = move_stage
    if move_block is not None:
        t.move_block = move_block
    if cabana_occupancy is not None:
        t.cabana_occupancy = cabana_occupancy
    if move_walk32 is not None:
        t.move_walk32 = move_walk32
    check("oppb_set_tuning", load().oppb_set_tuning(C.byref(t)))


def set_deposit_strategy(strategy: int) -> None:
    set_tuning(deposit=strategy)
