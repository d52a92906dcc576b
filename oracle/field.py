"""TEST INFRASTRUCTURE ONLY — Python driver of the C oracle of the FemPIC field phase
(oracle/field_oracle.c) and of the reference's generated node-side loops
(oracle/_ref/field_ref_seq, built by oracle/Makefile from the reference sources).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from oracle.oracle import _p, load
from oracle.ref_runner import REF_DIR, params_text

NODE_INLET, NODE_FIXED = 2, 3


def _sigs(lib):
    if getattr(lib, "_field_sigs", False):
        return lib
    vp, i32, d = C.c_void_p, C.c_int32, C.c_double
    lib.oracle_node_charge_density.restype = None
    lib.oracle_node_charge_density.argtypes = [i32, vp, vp, d]
    lib.oracle_electric_field.restype = None
    lib.oracle_electric_field.argtypes = [i32, vp, vp, vp, vp]
    lib.oracle_field_setup.restype = i32
    lib.oracle_field_setup.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.oracle_field_solve.restype = i32
    lib.oracle_field_solve.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                       d, d, d, d, d, d, d, i32, vp, vp]
    lib._field_sigs = True
    return lib


def node_charge_density(den: np.ndarray, vol: np.ndarray, spwt: float) -> np.ndarray:
    out = np.ascontiguousarray(den, np.float64).copy()
    _sigs(load()).oracle_node_charge_density(len(out), _p(out), _p(np.ascontiguousarray(vol, np.float64)), spwt)
    return out


def electric_field(c2n: np.ndarray, c_sd: np.ndarray, phi: np.ndarray) -> np.ndarray:
    c2n = np.ascontiguousarray(c2n, np.int32)
    ef = np.zeros((len(c2n), 3))
    _sigs(load()).oracle_electric_field(len(c2n), _p(c2n), _p(np.ascontiguousarray(c_sd, np.float64)),
                                        _p(np.ascontiguousarray(phi, np.float64)), _p(ef))
    return ef


def boundary_potential(n_type: np.ndarray, phi_inlet: float, phi_fixed: float) -> np.ndarray:
    """Dirichlet values: phi_inlet on INLET nodes, phi_fixed on FIXED nodes, 0 elsewhere."""
    out = np.zeros(len(n_type))
    out[n_type == NODE_INLET] = phi_inlet
    out[n_type == NODE_FIXED] = phi_fixed
    return out


@dataclass
class FieldConsts:
    n0: float
    phi0: float
    kte: float
    qe: float
    eps0: float
    rtol: float = 1e-10
    atol: float = 1e-10
    max_iter: int = 4000


class FieldSystem:
    """FESolver's set-up and Newton state on host arrays (oracle_field_setup / _solve)."""

    def __init__(self, n_pos, n_type, n_bnd_pot, c2n):
        lib = _sigs(load())
        n_pos = np.ascontiguousarray(n_pos, np.float64)
        self.n_type = np.ascontiguousarray(n_type, np.int32)
        self.n_bnd_pot = np.ascontiguousarray(n_bnd_pot, np.float64)
        self.c2n = np.ascontiguousarray(c2n, np.int32)
        nn, nc = len(n_pos), len(self.c2n)
        self.n_nodes, self.n_cells = nn, nc
        self.node_to_eq = np.zeros(nn, np.int32)
        self.det_j = np.zeros(nc)
        self.c_sd = np.zeros((nc, 4, 3))
        f0 = np.zeros(max(nn, 1))
        rowptr = np.zeros(nn + 1, np.int64)
        col = np.zeros(16 * nc, np.int32)
        val = np.zeros(16 * nc)
        nnz = np.zeros(1, np.int64)
        neq = lib.oracle_field_setup(nn, nc, _p(n_pos), _p(self.n_type), _p(self.n_bnd_pot), _p(self.c2n),
                                     _p(self.node_to_eq), _p(self.det_j), _p(self.c_sd), _p(f0), _p(rowptr),
                                     _p(col), _p(val), _p(nnz))
        if neq < 0:
            raise ValueError("bad cell -> node map")
        self.neq = int(neq)
        self.f0 = f0[:neq].copy()
        self.k_rowptr = rowptr[:neq + 1].copy()
        self.k_col = col[:int(nnz[0])].copy()
        self.k_val = val[:int(nnz[0])].copy()
        self.d = np.zeros(max(neq, 1))
        self.f1 = np.zeros(max(neq, 1))

    def solve(self, ion_den: np.ndarray, c: FieldConsts) -> tuple[np.ndarray, int, float]:
        """One compute_phi: returns (node potential, CG iterations, relative residual)."""
        lib = _sigs(load())
        pot = np.zeros(self.n_nodes)
        resid = np.zeros(1)
        it = lib.oracle_field_solve(self.n_nodes, self.n_cells, self.neq, _p(self.node_to_eq), _p(self.c2n),
                                    _p(self.det_j), _p(self.n_bnd_pot), _p(self.k_rowptr), _p(self.k_col),
                                    _p(self.k_val), _p(self.f0), _p(self.d), _p(self.f1),
                                    _p(np.ascontiguousarray(ion_den, np.float64)), c.n0, c.phi0, c.kte, c.qe,
                                    c.eps0, c.rtol, c.atol, c.max_iter, _p(pot), _p(resid))
        return pot, int(it), float(resid[0])


def run_reference(den, vol, spwt: float, c2n, c_sd, phi) -> tuple[np.ndarray, np.ndarray]:
    """The reference's generated seq loops: (n_charge_den after compute_node_charge_density,
    c_ef after opp_reset_dat + compute_electric_field)."""
    exe = REF_DIR / "field_ref_seq"
    if not exe.exists():
        raise FileNotFoundError(exe)
    den = np.ascontiguousarray(den, np.float64)
    c2n = np.ascontiguousarray(c2n, np.int32)
    nn, nc = len(den), len(c2n)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        with open(d / "in.bin", "wb") as f:
            f.write(np.array([nn, nc], "<i4").tobytes())
            f.write(np.array([spwt], "<f8").tobytes())
            for a, t in ((den, "<f8"), (vol, "<f8"), (c2n, "<i4"), (c_sd, "<f8"), (phi, "<f8")):
                f.write(np.ascontiguousarray(a, t).tobytes())
        (d / "params.txt").write_text(params_text("HoleFill_All", 10, 2.0))
        r = subprocess.run([str(exe), str(d / "params.txt"), str(d / "in.bin"), str(d / "out.bin")],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"field_ref_seq failed ({r.returncode}): {r.stderr[-1000:]}")
        out = np.fromfile(d / "out.bin", "<f8")
    return out[:nn].copy(), out[nn:].reshape(nc, 3).copy()
