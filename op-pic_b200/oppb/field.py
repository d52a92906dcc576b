"""FemPIC's node-side loops and field solve on the B200 backend (include/oppb_field.h).

FieldDevice holds FESolver's system on the GPU (built once on the host by
oppb_field_setup: equation map, detJ, shape derivatives, stiffness matrix K, F0) with the
Newton state D and the accumulated F1, and runs per step:
  node_charge_density   compute_node_charge_density_kernel (n_charge_den *= spwt / n_vol)
  solve                 FESolver::compute_phi, one cooperative launch, no host sync
  electric_field        compute_electric_field_kernel into any [cell][stride] field array
The three calls capture into one CUDA graph (capture()).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from oppb import _lib as L

NODE_INLET, NODE_FIXED = 2, 3


def boundary_potential(n_type: np.ndarray, phi_inlet: float, phi_fixed: float) -> np.ndarray:
    """Dirichlet values: phi_inlet on INLET nodes, phi_fixed on FIXED nodes, 0 elsewhere."""
    out = np.zeros(len(n_type))
    out[n_type == NODE_INLET] = phi_inlet
    out[n_type == NODE_FIXED] = phi_fixed
    return out


@dataclass
class FieldConstants:
    """FESolver's electron model (CONST_n0, CONST_phi0, CONST_kTe, CONST_QE, CONST_EPS0) and
    the CG stopping rule (||r|| <= max(rtol ||B||, atol), at most max_iter iterations)."""
    n0: float
    phi0: float
    kte: float
    qe: float
    eps0: float
    rtol: float = 1e-10
    atol: float = 1e-10
    max_iter: int = 4000

    def c_struct(self) -> L.FieldConsts:
        return L.FieldConsts(self.n0, self.phi0, self.kte, self.qe, self.eps0, self.rtol, self.atol, self.max_iter, 0)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def host_system(hm, n_bnd_pot: np.ndarray) -> dict:
    """FESolver's set-up on the host (oppb_field_setup): node_to_eq, det_j, c_sd [nc][4][3],
    K as CSR (k_rowptr, k_col, k_val), K by diagonals when banded (dia_off [n_diag],
    dia_val [n_diag][neq]; n_diag = 0 otherwise) and f0, as numpy arrays."""
    lib = L.load()
    n_pos = np.ascontiguousarray(hm.n_pos, np.float64)
    n_type = np.ascontiguousarray(hm.n_type, np.int32)
    bnd = np.ascontiguousarray(n_bnd_pot, np.float64)
    c2n = np.ascontiguousarray(hm.c2n, np.int32)
    fm = L.FemPICMesh()
    fm.n_nodes, fm.n_cells = hm.n_nodes, hm.n_cells
    fm.n_pos = n_pos.ctypes.data_as(L.c_dp)
    fm.n_type = n_type.ctypes.data_as(L.c_ip)
    fm.n_bnd_pot = bnd.ctypes.data_as(L.c_dp)
    fm.c2n = c2n.ctypes.data_as(L.c_ip)
    sys_ = L.FieldSystem()
    L.check("oppb_field_setup", lib.oppb_field_setup(C.byref(fm), C.byref(sys_)))
    try:
        nn, nc, neq, nnz = sys_.n_nodes, sys_.n_cells, sys_.neq, int(sys_.nnz)

        def take(ptr, n, dt):
            return np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].astype(dt, copy=True)

        return {"n_nodes": nn, "n_cells": nc, "neq": neq, "nnz": nnz, "c2n": c2n, "n_bnd_pot": bnd,
                "node_to_eq": take(sys_.node_to_eq, nn, np.int32), "det_j": take(sys_.det_j, nc, np.float64),
                "c_sd": take(sys_.c_sd, nc * 12, np.float64).reshape(nc, 4, 3),
                "k_rowptr": take(sys_.k_rowptr, neq + 1, np.int64), "k_col": take(sys_.k_col, nnz, np.int32),
                "k_val": take(sys_.k_val, nnz, np.float64), "f0": take(sys_.f0, neq, np.float64),
                "dia_off": np.array(list(sys_.dia_off)[:sys_.n_diag], np.int32),
                "dia_val": take(sys_.dia_val, sys_.n_diag * neq, np.float64).reshape(sys_.n_diag, neq)
                if sys_.n_diag else np.zeros((0, neq))}
    finally:
        lib.oppb_field_system_free(C.byref(sys_))


class FieldDevice:
    def __init__(self, hm, device, n_bnd_pot: np.ndarray):
        lib = L.load()
        self.lib = lib
        self.device = torch.device(device)
        h = host_system(hm, n_bnd_pot)
        nn, nc, neq, nnz = h["n_nodes"], h["n_cells"], h["neq"], h["nnz"]
        self.node_to_eq, self.det_j, self.c_sd = h["node_to_eq"], h["det_j"], h["c_sd"]
        self.k_rowptr, self.k_col, self.k_val, self.f0 = h["k_rowptr"], h["k_col"], h["k_val"], h["f0"]
        c2n, bnd = h["c2n"], h["n_bnd_pot"]
        self.n_nodes, self.n_cells, self.neq, self.nnz = nn, nc, neq, nnz
        dev = self.device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.d_node_to_eq, self.d_c2n, self.d_det_j = t(self.node_to_eq), t(c2n), t(self.det_j)
        self.d_bnd = t(bnd)
        self.d_rowptr, self.d_col, self.d_val = t(self.k_rowptr), t(self.k_col), t(self.k_val)
        self.d_f0 = t(self.f0) if neq else torch.zeros(1, dtype=torch.float64, device=dev)
        self.d_c_sd = t(self.c_sd.reshape(nc, 12))
        self.d = torch.zeros(max(neq, 1), dtype=torch.float64, device=dev)   # Newton iterate D
        self.f1 = torch.zeros(max(neq, 1), dtype=torch.float64, device=dev)  # accumulated F1
        self.work = torch.zeros(int(lib.oppb_field_work_doubles(neq)), dtype=torch.float64, device=dev)
        self.status = torch.zeros(3, dtype=torch.float64, device=dev)        # oppb_field_status (24 B)
        self.potential = torch.zeros(nn, dtype=torch.float64, device=dev)
        self.dia_off = h["dia_off"]
        self.d_dia = t(h["dia_val"]) if len(self.dia_off) else None
        self.s = L.FieldDevice(nn, nc, neq, 0, _ptr(self.d_node_to_eq), _ptr(self.d_c2n), _ptr(self.d_det_j),
                               _ptr(self.d_bnd), _ptr(self.d_rowptr), _ptr(self.d_col), _ptr(self.d_val),
                               _ptr(self.d_f0), _ptr(self.d), _ptr(self.f1), _ptr(self.work))
        self.set_diagonal_form(True)

    def set_diagonal_form(self, on: bool) -> None:
        """Whether the CG's products read K by diagonals (when K has that form) or as CSR."""
        n = len(self.dia_off) if on and self.d_dia is not None else 0
        self.s.n_diag = n
        for j in range(16):
            self.s.dia_off[j] = int(self.dia_off[j]) if j < n else 0
        self.s.dia_val = _ptr(self.d_dia) if n else None

    @staticmethod
    def _stream(stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        return s.cuda_stream or None

    def node_charge_density(self, den: torch.Tensor, n_vol: torch.Tensor, spwt: float, stream=None) -> None:
        L.check("oppb_node_charge_density", self.lib.oppb_node_charge_density(
            den.data_ptr(), n_vol.data_ptr(), float(spwt), den.numel(), self._stream(stream)))

    def solve(self, ion_den: torch.Tensor, consts: FieldConstants, stream=None) -> torch.Tensor:
        """compute_phi on ion_den (device [n_nodes]); returns the node potential tensor."""
        c = consts.c_struct()
        L.check("oppb_field_solve", self.lib.oppb_field_solve(C.byref(self.s), C.byref(c), ion_den.data_ptr(),
                                                               self.potential.data_ptr(), self.status.data_ptr(),
                                                               self._stream(stream)))
        return self.potential

    def electric_field(self, ef: torch.Tensor, stride: int, stream=None) -> None:
        L.check("oppb_electric_field", self.lib.oppb_electric_field(
            self.d_c2n.data_ptr(), self.d_c_sd.data_ptr(), self.potential.data_ptr(), ef.data_ptr(), stride,
            self.n_cells, self._stream(stream)))

    def status_host(self) -> L.FieldStatus:
        return L.FieldStatus.from_buffer_copy(self.status.cpu().numpy().tobytes())

    def warm(self, den: torch.Tensor, n_vol: torch.Tensor, spwt: float, consts: FieldConstants,
             ef: torch.Tensor, stride: int) -> None:
        """First launches load the kernels: run each once outside any capture, on scratch
        outputs (a solve with no CG iteration leaves D as it is; F1 is put back)."""
        self.node_charge_density(den[:1].clone(), n_vol[:1], spwt)
        f1 = self.f1.clone()
        warm = FieldConstants(**{**consts.__dict__, "max_iter": 0})
        self.solve(torch.zeros_like(den), warm)
        self.f1.copy_(f1)
        self.electric_field(torch.empty_like(ef), stride)
        torch.cuda.synchronize(self.device)

    def launch(self, den: torch.Tensor, n_vol: torch.Tensor, spwt: float, consts: FieldConstants,
               ef: torch.Tensor, stride: int) -> None:
        """The field phase's launches on the current stream: density, potential, field."""
        self.node_charge_density(den, n_vol, spwt)
        self.solve(den, consts)
        self.electric_field(ef, stride)

    def capture(self, den: torch.Tensor, n_vol: torch.Tensor, spwt: float, consts: FieldConstants,
                ef: torch.Tensor, stride: int) -> torch.cuda.CUDAGraph:
        """The field phase of a step (density, potential, field) as one CUDA graph."""
        self.warm(den, n_vol, spwt, consts, ef, stride)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch(den, n_vol, spwt, consts, ef, stride)
        torch.cuda.current_stream().wait_stream(s)
        return g
