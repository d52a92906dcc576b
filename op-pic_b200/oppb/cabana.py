"""CabanaPIC particle path on the B200 backend (include/oppb_cabana.h).

Host-side set-up mirrors the reference app where the particle path needs it:
  Deck          the constants of apps/app_cabanapic/cabana_defs.h:331-372 (dt from the Courant
                length :320-326, cdt_d, qdt_2mc, we)
  HexMesh       init_mesh's cell set with one ghost layer and the periodic non-ghost face map
                c2ngc (apps/app_cabanapic/cabana_misc_mesh_loader.h:63-150)
  two_stream    seeded particles of the two-stream workload: uniform positions in every
                non-ghost cell, counter-streaming momenta along z with a thermal spread
  CabanaDevice  device buffers (particle dats SoA [dim][capacity], packed mesh, c_acc SoA
                [12][n_cells]) and the move_deposit launch
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from oppb import _lib as L

NG = 1  # ghost layers, cabana_defs.h:41


@dataclass
class Deck:
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    nppc: int
    c: float = 1.0
    qsp: float = -1.0
    me: float = 1.0
    courant_frac: float = 0.99
    n0: float = 2.0

    def __post_init__(self):
        w1 = 0.0
        for n, length in ((self.nx, self.lx), (self.ny, self.ly), (self.nz, self.lz)):
            if n > 1:
                w0 = n / length
                w1 += w0 * w0
        courant = math.sqrt(1.0 / w1)
        self.dx, self.dy, self.dz = self.lx / self.nx, self.ly / self.ny, self.lz / self.nz
        self.dt = self.courant_frac * courant / self.c
        self.cdt_d = (self.c * self.dt / self.dx, self.c * self.dt / self.dy, self.c * self.dt / self.dz)
        self.qdt_2mc = self.qsp * self.dt / (2 * self.me * self.c)
        self.we = self.n0 * self.lx * self.ly * self.lz / (self.nx * self.ny * self.nz * self.nppc)

    def consts(self) -> L.CabanaConsts:
        return L.CabanaConsts(self.qdt_2mc, (C.c_double * 3)(*self.cdt_d), self.qsp)


class HexMesh:
    """Cells (nx+2)(ny+2)(nz+2) with index x + (nx+2)(y + (ny+2) z) (VOXEL, cabana_defs.h:49);
    c2ngc [n_cells, 6] in Face order xd, yd, zd, xu, yu, zu: periodic neighbours for non-ghost
    cells (VOXEL_MAP_NON_GHOST_PERIODIC, :59-70), the cell itself for ghost cells."""

    def __init__(self, nx: int, ny: int, nz: int):
        self.nx, self.ny, self.nz = nx, ny, nz
        gx, gy, gz = nx + 2 * NG, ny + 2 * NG, nz + 2 * NG
        self.n_cells = gx * gy * gz
        z, y, x = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
        x, y, z = x.ravel(), y.ravel(), z.ravel()
        idx = x + gx * (y + gy * z)
        order = np.argsort(idx)
        x, y, z = x[order], y[order], z[order]
        self.ghost = ((x < 1) | (y < 1) | (z < 1) | (x >= nx + 1) | (y >= ny + 1) | (z >= nz + 1)).astype(np.int32)

        def wrap(a, n):
            a = np.where(a == 0, n, a)
            return np.where(a == n + 1, 1, a)

        def voxel(a, b, c):
            return (wrap(a, nx) + gx * (wrap(b, ny) + gy * wrap(c, nz))).astype(np.int32)

        self_idx = np.arange(self.n_cells, dtype=np.int32)
        faces = [voxel(x - 1, y, z), voxel(x, y - 1, z), voxel(x, y, z - 1),
                 voxel(x + 1, y, z), voxel(x, y + 1, z), voxel(x, y, z + 1)]
        self.c2ngc = np.stack([np.where(self.ghost == 1, self_idx, f) for f in faces], axis=1).astype(np.int32)
        self.interior = np.flatnonzero(self.ghost == 0).astype(np.int32)


def synthetic_interp(mesh: HexMesh, seed: int, e_scale: float = 1e-2, b_scale: float = 1e-2) -> np.ndarray:
    """Seeded c_interp [n_cells, 18] (CellInterp order): E and B values and their first
    derivatives ~ N(0, scale^2); ghost cells zero, as interpolate_mesh_fields leaves them."""
    rng = np.random.default_rng(seed)
    interp = np.zeros((mesh.n_cells, 18))
    e_cols = list(range(12))
    b_cols = list(range(12, 18))
    n = len(mesh.interior)
    interp[np.ix_(mesh.interior, e_cols)] = rng.normal(0.0, e_scale, (n, 12))
    interp[np.ix_(mesh.interior, b_cols)] = rng.normal(0.0, b_scale, (n, 6))
    return interp


def two_stream(mesh: HexMesh, deck: Deck, v0: float, sigma: float, seed: int, cells=None):
    """Particles cell by cell (the order of the reference's enrichment): nppc per non-ghost
    cell, positions uniform in [-1,1]^3, u = (N(0,s^2), N(0,s^2), +-v0 gamma + N(0,s^2)) with
    alternating sign, zero streak, weight deck.we.  Returns AoS pos, vel, streak, weight, p2c."""
    rng = np.random.default_rng(seed)
    cells = mesh.interior if cells is None else np.asarray(cells, np.int32)
    n = len(cells) * deck.nppc
    p2c = np.repeat(cells, deck.nppc).astype(np.int32)
    pos = rng.uniform(-1.0, 1.0, (n, 3))
    gam = 1.0 / math.sqrt(1.0 - v0 * v0)
    sign = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    vel = rng.normal(0.0, sigma, (n, 3))
    vel[:, 2] += sign * v0 * gam
    return pos, vel, np.zeros((n, 3)), np.full(n, deck.we), p2c


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


class CabanaDevice:
    """Device state of the particle path: packed mesh, particle dats SoA [dim][capacity],
    c_acc SoA [12][n_cells], move status.  There is no CPU fallback.

    precision 'f64' is the reference's form (bit-identical to the seq backend); 'mixed' holds
    the momentum in FP32 (vel32) and pushes it in FP32 (oppb_cabana_move_deposit_mixed), with
    FP64 positions, cells and current deposit."""

    def __init__(self, mesh: HexMesh, device, capacity: int, precision: str = "f64"):
        if precision not in ("f64", "mixed"):
            raise ValueError(precision)
        self.precision = precision
        if not torch.cuda.is_available():
            raise RuntimeError("CabanaDevice needs a CUDA device (there is no CPU fallback)")
        self.device = torch.device(device)
        self.lib = L.load()
        nc = mesh.n_cells
        self.n_cells = nc
        self.c2f = torch.zeros(nc * 8, dtype=torch.int32, device=self.device)
        self.interp = torch.zeros(nc * 20, dtype=torch.float64, device=self.device)
        self.interp32 = torch.zeros(nc * 20, dtype=torch.float32, device=self.device) if precision == "mixed" else None
        self.mesh = L.HexMesh(nc, _ptr(self.c2f), _ptr(self.interp), _ptr(self.interp32))
        self.acc = torch.zeros((12, nc), dtype=torch.float64, device=self.device)
        self.capacity = max(capacity, 1)
        cap = self.capacity
        self.pos = torch.zeros((3, cap), dtype=torch.float64, device=self.device)
        # p_vel: FP64 in the reference's form; FP32 in the mixed form (vel32; vel unused there)
        self.vel = torch.zeros((3, cap if precision == "f64" else 1), dtype=torch.float64, device=self.device)
        self.vel32 = torch.zeros((3, cap), dtype=torch.float32, device=self.device) if precision == "mixed" else None
        self.streak = torch.zeros((3, cap), dtype=torch.float64, device=self.device)
        self.weight = torch.zeros(cap, dtype=torch.float64, device=self.device)
        self.p2c = torch.zeros(cap, dtype=torch.int32, device=self.device)
        self.status = torch.zeros(8, dtype=torch.int32, device=self.device)
        self.size = 0
        c2ngc = torch.from_numpy(np.ascontiguousarray(mesh.c2ngc.T)).to(self.device)
        L.check("oppb_hex_mesh_pack", self.lib.oppb_hex_mesh_pack(C.byref(self.mesh), nc, _ptr(c2ngc), None, None))

    def set_interp(self, interp: np.ndarray) -> None:
        """Upload c_interp [n_cells, 18] (host AoS) and repack it."""
        soa = torch.from_numpy(np.ascontiguousarray(interp.T)).to(self.device)
        L.check("oppb_hex_mesh_pack",
                self.lib.oppb_hex_mesh_pack(C.byref(self.mesh), self.n_cells, None, _ptr(soa), None))

    def set_particles(self, pos, vel, streak, weight, p2c) -> None:
        n = len(p2c)
        if n > self.capacity:
            raise ValueError("capacity exceeded")
        self.size = n
        vel_name = "vel" if self.precision == "f64" else "vel32"
        for name, a in (("pos", pos), (vel_name, vel), ("streak", streak)):
            t = getattr(self, name)
            t[:, :n] = torch.from_numpy(np.ascontiguousarray(a.T)).to(device=self.device, dtype=t.dtype)
        self.weight[:n] = torch.from_numpy(np.ascontiguousarray(weight)).to(self.device)
        self.p2c[:n] = torch.from_numpy(np.ascontiguousarray(p2c, dtype=np.int32)).to(self.device)

    def fill_two_stream(self, mesh: HexMesh, deck: Deck, v0: float, sigma: float, seed: int) -> None:
        """The two_stream construction drawn on the device (torch generator): nppc particles per
        non-ghost cell in cell order, positions uniform in [-1,1]^3, u = N(0, sigma^2) per axis
        plus +-v0 gamma along z alternating per particle, zero streak, weight deck.we."""
        n = len(mesh.interior) * deck.nppc
        if n > self.capacity or deck.nppc % 2:
            raise ValueError("capacity exceeded or odd nppc")
        self.size = n
        g = torch.Generator(device=self.device)
        g.manual_seed(seed)
        self.pos[:, :n].uniform_(-1.0, 1.0, generator=g)
        u = torch.empty((3, n), dtype=torch.float64, device=self.device)
        u.normal_(0.0, sigma, generator=g)
        drift = v0 / math.sqrt(1.0 - v0 * v0)
        pairs = u[2].view(-1, 2)
        pairs[:, 0] += drift
        pairs[:, 1] -= drift
        if self.precision == "f64":
            self.vel[:, :n] = u
        else:
            self.vel32[:, :n] = u.to(torch.float32)  # the same draw, rounded to FP32
        self.streak[:, :n].zero_()
        self.weight[:n] = deck.we
        cells = torch.from_numpy(mesh.interior).to(self.device)
        self.p2c[:n] = cells.repeat_interleave(deck.nppc)

    def view(self) -> L.CabanaParticles:
        return L.CabanaParticles(self.size, self.capacity, _ptr(self.pos), _ptr(self.vel), _ptr(self.streak),
                                 _ptr(self.weight), _ptr(self.p2c))

    def move_deposit(self, deck: Deck, max_hops: int = 4096, stream=None, zero_acc: bool = True) -> None:
        """opp_reset_dat(c_acc) + opp_particle_move__move_deposit_kernel."""
        if zero_acc:  # with the library's fill kernel, so that the call launches only library kernels
            L.check("oppb_fill", L.load().oppb_fill(_ptr(self.acc), self.acc.numel(), 8, 0,
                                                    None if stream is None else stream.cuda_stream))
        v = self.view()
        k = deck.consts()
        sp = None if stream is None else stream.cuda_stream
        if self.precision == "mixed":
            L.check("oppb_cabana_move_deposit_mixed",
                    self.lib.oppb_cabana_move_deposit_mixed(C.byref(self.mesh), C.byref(v), _ptr(self.vel32),
                                                            C.byref(k), _ptr(self.acc), self.n_cells,
                                                            _ptr(self.status), max_hops, sp))
            return
        L.check("oppb_cabana_move_deposit",
                self.lib.oppb_cabana_move_deposit(C.byref(self.mesh), C.byref(v), C.byref(k), _ptr(self.acc),
                                                  self.n_cells, _ptr(self.status), max_hops, sp))

    def status_host(self) -> L.MoveStatus:
        return L.MoveStatus.from_buffer_copy(self.status.cpu().numpy().tobytes())

    def host(self) -> dict:
        n = self.size
        vel = self.vel if self.precision == "f64" else self.vel32
        return {"pos": self.pos[:, :n].T.contiguous().cpu().numpy(), "vel": vel[:, :n].T.contiguous().cpu().numpy(),
                "streak": self.streak[:, :n].T.contiguous().cpu().numpy(), "p2c": self.p2c[:n].cpu().numpy(),
                "acc": self.acc.T.contiguous().cpu().numpy()}
