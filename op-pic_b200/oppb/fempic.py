"""FemPIC particle step on one B200 through the C ABI (include/oppb.h).

Host side of the library in Python for tests and the benchmark: it owns device buffers
(torch tensors used only as device memory and streams) and calls the CUDA kernels of
liboppb.so.  The layout follows the reference's CUDA backend: particle dats SoA
[dim][capacity] (opp_lib/src/cuda/opp_cuda_utils.cu:128-143), mesh dats uploaded SoA
and packed into the kernels' cell records once.

The step follows the generated main loop (apps_codegen/app_fempic_cg/fempic_opp.cpp:160-215):
  inject -> reset node charge -> push -> move (+ fused deposit) -> hole fill / cell sort.
The deposit of the final cell is fused into the move kernel; contributions are the same
as the separate deposit loop over the compacted set.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


# --------------------------------------------------------------------------- host mesh

class HostMesh:
    """Box tetrahedral mesh built by oppb_fempic_box_mesh (host AoS arrays, numpy views
    onto library-owned memory, copied so the Python object owns them)."""

    def __init__(self, nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
                 phi_inlet: float = 1.0, phi_fixed: float = 0.0, solve_field: bool = True):
        lib = L.load()
        m = L.FemPICMesh()
        rc = lib.oppb_fempic_box_mesh(nx, ny, nz, lx, ly, lz, C.byref(m))
        if rc != 0:
            raise RuntimeError(f"oppb_fempic_box_mesh failed ({rc})")
        try:
            self.cg_iters = 0
            self.cg_resid = 0.0
            if solve_field:
                it, res = C.c_int32(0), C.c_double(0)
                pot = np.zeros(m.n_nodes)
                rc = lib.oppb_fempic_solve_field(C.byref(m), phi_inlet, phi_fixed, 1e-12, 100000,
                                                 pot.ctypes.data_as(L.c_dp), C.byref(it), C.byref(res))
                if rc != 0:
                    raise RuntimeError(f"field solve did not converge (resid {res.value})")
                self.cg_iters, self.cg_resid, self.n_pot = it.value, res.value, pot
            self.n_nodes, self.n_cells, self.n_ifaces = m.n_nodes, m.n_cells, m.n_ifaces
            nn, nc, nf = m.n_nodes, m.n_cells, m.n_ifaces

            def take(ptr, shape, dtype):
                n = int(np.prod(shape))
                return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True).reshape(shape)

            self.n_pos = take(m.n_pos, (nn, 3), np.float64)
            self.n_vol = take(m.n_vol, (nn,), np.float64)
            self.n_type = take(m.n_type, (nn,), np.int32)
            self.c2n = take(m.c2n, (nc, 4), np.int32)
            self.c2c = take(m.c2c, (nc, 4), np.int32)
            self.c_det = take(m.c_det, (nc, 16), np.float64)
            self.c_vol = take(m.c_vol, (nc,), np.float64)
            self.c_sd = take(m.c_sd, (nc, 4, 3), np.float64)
            self.c_ef = take(m.c_ef, (nc, 3), np.float64)
            self.c_centroid = take(m.c_centroid, (nc, 3), np.float64)
            self.if2c = take(m.if2c, (nf,), np.int32)
            self.if2n = take(m.if2n, (nf, 3), np.int32)
            self.if_u = take(m.if_u, (nf, 3), np.float64)
            self.if_v = take(m.if_v, (nf, 3), np.float64)
            self.if_norm = take(m.if_norm, (nf, 3), np.float64)
            self.if_area = take(m.if_area, (nf,), np.float64)
            self.if_n_pos = take(m.if_n_pos, (nf, 9), np.float64)
        finally:
            lib.oppb_fempic_mesh_free(C.byref(m))
        self.dims = (nx, ny, nz, lx, ly, lz)

    def inject_distribution(self, total: int) -> np.ndarray:
        """Cumulative per-face counts (oppb_fempic_inject_distribution)."""
        out = np.zeros(self.n_ifaces, np.int32)
        fm = L.FemPICMesh()
        fm.n_ifaces = self.n_ifaces
        fm.if_area = self.if_area.ctypes.data_as(L.c_dp)
        rc = L.load().oppb_fempic_inject_distribution(C.byref(fm), total, out.ctypes.data_as(L.c_ip))
        if rc != 0:
            raise RuntimeError("oppb_fempic_inject_distribution failed")
        return out


def injection_randoms(seed: int, step: int, count: int, sigma: float) -> np.ndarray:
    """Seeded per-step injection table, AoS [count][5]: a, b ~ U[0,1) (position in the inlet
    triangle, folded as in inject_ions_kernel) and the thermal velocity ~ N(0, sigma^2)^3."""
    rng = np.random.default_rng([seed, step])
    out = np.empty((count, 5))
    out[:, 0:2] = rng.random((count, 2))
    out[:, 2:5] = sigma * rng.standard_normal((count, 3))
    return out


# ------------------------------------------------------------------------- device side

def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_ptr(stream: torch.cuda.Stream | None) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


class DeviceMesh:
    """Cell dats uploaded in the reference's device layout (SoA) and packed into the
    kernel records by oppb_tet_mesh_pack.  Also holds the inlet."""

    def __init__(self, hm: HostMesh, device: torch.device, mixed: bool = True, dist: np.ndarray | None = None):
        self.device = device
        nc, nn = hm.n_cells, hm.n_nodes
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dt)  # noqa: E731
        soa_det = t(hm.c_det.T, torch.float64)
        soa_vol = t(hm.c_vol, torch.float64)
        soa_c2c = t(hm.c2c.T, torch.int32)
        soa_c2n = t(hm.c2n.T, torch.int32)
        soa_ef = t(hm.c_ef.T, torch.float64)
        soa_npos = t(hm.n_pos.T, torch.float64)
        self.det = torch.empty(nc * 16, dtype=torch.float64, device=device)
        self.nav = torch.zeros(nc * 4, dtype=torch.float64, device=device)
        self.c2n = torch.empty(nc * 4, dtype=torch.int32, device=device)
        self.ef = torch.empty(nc * 4, dtype=torch.float64, device=device)
        self.geo32 = torch.empty(nc * 16, dtype=torch.float32, device=device) if mixed else None
        self.nav32 = torch.zeros(nc * 8, dtype=torch.float32, device=device) if mixed else None
        self.s = L.TetMesh(nc, nn, _ptr(self.det), _ptr(self.nav), _ptr(self.c2n), _ptr(self.ef),
                           _ptr(self.geo32), _ptr(self.nav32))
        invalid = torch.zeros(1, dtype=torch.int32, device=device)
        L.check("oppb_tet_mesh_pack", L.load().oppb_tet_mesh_pack(
            C.byref(self.s), nc, _ptr(soa_det), _ptr(soa_vol), _ptr(soa_c2c), _ptr(soa_c2n), _ptr(soa_ef),
            _ptr(soa_npos), nn, _ptr(invalid), _stream_ptr(None)))
        if int(invalid.item()) != 0:
            raise ValueError(f"mesh maps hold {int(invalid.item())} out-of-range entries")
        self.n_cells, self.n_nodes = nc, nn
        # Inlet: dist, if2c, geom[12] = u, v, normal, node0.
        geom = np.concatenate([hm.if_u, hm.if_v, hm.if_norm, hm.if_n_pos[:, 0:3]], axis=1)
        self.if_geom = t(geom, torch.float64)
        self.if2c = t(hm.if2c, torch.int32)
        self.dist = t(dist if dist is not None else np.zeros(hm.n_ifaces, np.int32), torch.int32)
        self.inlet = L.Inlet(hm.n_ifaces, _ptr(self.dist), _ptr(self.if2c), _ptr(self.if_geom))


class DirectHopGrid:
    """The direct-hop seed's structured grid (include/oppb_dh.h), built on the device once:
    grid spacing h, bounding box of the nodes widened by `expansion` per axis (default 4h,
    the FemPIC app's choice, apps_codegen/app_fempic_cg/fempic_opp.cpp:69-76), map of every
    box to its mesh cell (OPPB_REMOVED_CELL where none).  Role of opp_init_direct_hop_cg."""

    def __init__(self, hm: HostMesh, mesh: DeviceMesh, spacing: float, expansion=None):
        lib = L.load()
        exp = np.full(3, 4.0 * spacing) if expansion is None else \
            np.ascontiguousarray(np.broadcast_to(np.asarray(expansion, np.float64), (3,)))
        n_pos = np.ascontiguousarray(hm.n_pos, np.float64)
        self.g = L.DhGrid()
        L.check("oppb_dh_grid_init", lib.oppb_dh_grid_init(n_pos.ctypes.data, hm.n_nodes, float(spacing),
                                                           exp.ctypes.data, C.byref(self.g)))
        self.map = torch.empty(int(self.g.size), dtype=torch.int32, device=mesh.device)
        self.g.map = self.map.data_ptr()
        npos_soa = torch.from_numpy(np.ascontiguousarray(hm.n_pos.T)).to(mesh.device)
        need = C.c_size_t(0)
        sp = _stream_ptr(None)
        rc = lib.oppb_dh_build(C.byref(mesh.s), npos_soa.data_ptr(), C.byref(self.g), None, 0, C.byref(need), sp)
        if rc != L.OPPB_ERR_WORKSPACE:
            L.check("oppb_dh_build", rc)
        ws = torch.empty(int(need.value), dtype=torch.uint8, device=mesh.device)
        L.check("oppb_dh_build", lib.oppb_dh_build(C.byref(mesh.s), npos_soa.data_ptr(), C.byref(self.g),
                                                   ws.data_ptr(), ws.numel(), C.byref(need), sp))
        torch.cuda.current_stream(mesh.device).synchronize()  # the workspace is freed on return
        self.spacing = float(spacing)
        self.expansion = exp
        self.dims = tuple(int(d) for d in self.g.dims)
        self.size = int(self.g.size)
        self.box = np.array(list(self.g.min) + list(self.g.max))


class ParticleSet:
    """Particle dats p_position, p_velocity, p_lc, p2c in SoA [dim][capacity] with swap
    buffers for the sort, the removal bitmap and the move status word."""

    DATS = (("pos", 3, torch.float64), ("vel", 3, torch.float64), ("lc", 4, torch.float64), ("p2c", 1, torch.int32))

    def __init__(self, device: torch.device, capacity: int = 0, alloc_mult: float = 2.0):
        self.device = device
        self.size = 0
        self.capacity = 0
        self.alloc_mult = alloc_mult
        self.status = torch.zeros(32 // 4, dtype=torch.int32, device=device)
        self._alloc(capacity)

    def _alloc(self, cap: int) -> None:
        old = {n: getattr(self, n, None) for n, _, _ in self.DATS}
        for name, dim, dt in self.DATS:
            fill = L.REMOVED_CELL if name == "p2c" else 0
            buf = torch.full((dim, max(cap, 1)), fill, dtype=dt, device=self.device)
            if old[name] is not None and self.size > 0:
                buf[:, : self.size].copy_(old[name][:, : self.size])
            setattr(self, name, buf)
            setattr(self, name + "_swap", torch.empty_like(buf))
        self.bits = torch.zeros((max(cap, 1) + 31) // 32, dtype=torch.int32, device=self.device)
        self.capacity = cap

    def increase(self, count: int) -> None:
        """opp_increase_particle_count_core semantics (capacity = size + count*alloc_mult),
        growing on the device (no host round trip)."""
        new_size = self.size + count
        if new_size > self.capacity:
            self._alloc(int(self.size + count * self.alloc_mult))

    def view(self) -> L.Particles:
        return L.Particles(self.size, self.capacity, _ptr(self.pos), _ptr(self.vel), _ptr(self.lc), _ptr(self.p2c),
                           _ptr(self.bits))

    def dat_list(self):
        arr = (L.Dat * len(self.DATS))()
        for k, (name, dim, dt) in enumerate(self.DATS):
            arr[k] = L.Dat(_ptr(getattr(self, name)), _ptr(getattr(self, name + "_swap")), dim,
                           8 if dt == torch.float64 else 4)
        return arr

    def swap_after_sort(self) -> None:
        for name, _, _ in self.DATS:
            a, b = getattr(self, name), getattr(self, name + "_swap")
            setattr(self, name, b)
            setattr(self, name + "_swap", a)

    def host_aos(self) -> dict:
        """Copy [0,size) to host AoS numpy (the seq backend's layout)."""
        n = self.size
        return {name: getattr(self, name)[:, :n].T.contiguous().cpu().numpy() if dim > 1
                else getattr(self, name)[0, :n].cpu().numpy() for name, dim, _ in self.DATS}

    def status_host(self) -> L.MoveStatus:
        raw = self.status.cpu().numpy().tobytes()
        return L.MoveStatus.from_buffer_copy(raw)


FILL_MODES = ("HoleFill_All", "Sort_All", "Shuffle_All", "Sort_Periodic", "Shuffle_Periodic")


@dataclass
class StepTimes:
    move_ms: float = 0.0
    compact_ms: float = 0.0
    push_ms: float = 0.0
    inject_ms: float = 0.0


class FemPIC:
    """The FemPIC particle step on one GPU.

    precision: 'f64' (bit-identical to the seq backend) or 'mixed' (FP32 push and tests
    with FP64 re-check; bit-identical cell decisions for the same positions).
    fill: 'HoleFill_All' | 'Sort_All' | 'Sort_Periodic' | 'Shuffle_All' | 'Shuffle_Periodic' as the
    reference's opp_fill (the shuffles sort by random keys, oppb_shuffle).
    """

    def __init__(self, hm: HostMesh, device: torch.device | str = "cuda", inject_per_step: int = 2000,
                 ion_velocity: float = 1.0, qm: float = 1.0, dt: float = 0.01, precision: str = "f64",
                 fill: str = "HoleFill_All", fill_period: int = 10, alloc_mult: float = 2.0,
                 capacity: int = 0, max_hops: int = 4096, band: float = 1e-5, fused_deposit: bool = True,
                 fused_push: bool = True, direct_hop: float | None = None, dh_expansion=None,
                 field=None, spwt: float = 1.0, phi_inlet: float = 1.0, phi_fixed: float = 0.0):
        if fill not in FILL_MODES:  # opp_finalize_particle_move_core aborts on an undefined fill type
            raise ValueError(f"opp_fill {fill!r} is not one of {FILL_MODES}")
        if not torch.cuda.is_available():
            raise RuntimeError("FemPIC needs a CUDA device (there is no CPU fallback)")
        self.device = torch.device(device)
        self.hm = hm
        self.inject_per_step = inject_per_step
        self.dist_host = hm.inject_distribution(inject_per_step)
        # The mixed path's FP32 records are packed for both precisions: the FP64 move can walk on
        # them (oppb_tuning.move_walk32).
        self.mesh = DeviceMesh(hm, self.device, mixed=True, dist=self.dist_host)
        self.parts = ParticleSet(self.device, capacity, alloc_mult)
        self.ion_velocity, self.qm, self.dt = ion_velocity, qm, dt
        if precision not in ("f64", "mixed"):
            raise ValueError(precision)
        self.precision = precision
        self.fill, self.fill_period = fill, fill_period
        self.max_hops, self.band = max_hops, band
        self.fused_deposit = fused_deposit
        # push as the prologue of the move kernel (one launch); needs the deposit fused too
        self.fused_push = fused_push and (fused_deposit or precision == "mixed")
        self.node_charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=self.device)
        self.iter = 0
        self._ws = torch.empty(0, dtype=torch.uint8, device=self.device)
        self._dep_ws = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.lib = L.load()
        self.last = {}
        self._pipe = None  # run_steps' copy stream, events and double buffers, made once
        # Global move: every walk starts from the cell of the structured grid's box that the
        # particle is in (opp_global_move with grid_spacing = direct_hop).
        self.dh = DirectHopGrid(hm, self.mesh, direct_hop, dh_expansion) if direct_hop else None
        # Field phase (field: oppb.field.FieldConstants): after the compaction, as the generated
        # main loop (fempic_opp.cpp:195-215): compute_node_charge_density, compute_phi (the
        # Newton step with phi_inlet / phi_fixed on the Dirichlet nodes), opp_reset_dat(c_ef)
        # and compute_electric_field into the move's packed field, which the next step's push
        # and injection read.  Replayed as one CUDA graph per node-charge buffer.
        self.field_consts = field
        self.field = None
        self.field_enabled = True  # the field phase can be paused (e.g. to fill with the set-up field)
        if field is not None:
            from .field import FieldDevice, boundary_potential

            self.field = FieldDevice(hm, self.device, boundary_potential(hm.n_type, phi_inlet, phi_fixed))
            self.n_vol = torch.from_numpy(np.ascontiguousarray(hm.n_vol)).to(self.device)
            self.spwt = float(spwt)
            self._field_graphs = {}
        self._pipeline(5, inject_per_step)
        # Graph-captured steps (include/oppb_graph.h): the device count, its sync state, the
        # captured graphs by (steps, phase, buffers, capacity) and a scratch count for warm-ups.
        self.count_dev = torch.zeros(4, dtype=torch.int32, device=self.device)  # oppb_set_count
        self._count_synced = False
        self._graphs = {}
        self._gio = {}  # run_graph_host's staging buffers and events

    # workspace shared by hole fill and sort (grown on demand)
    def _workspace(self, nbytes: int) -> torch.Tensor:
        if self._ws.numel() < nbytes:
            self._ws = torch.empty(int(nbytes * 1.25) + 256, dtype=torch.uint8, device=self.device)
        return self._ws

    def inject(self, rnd_soa: torch.Tensor, stream=None) -> None:
        """rnd_soa: device float64 [5][count] (a, b, thermal vx, vy, vz)."""
        count = rnd_soa.shape[1]
        p = self.parts
        p.increase(count)
        start = p.size
        p.size += count
        v = p.view()
        L.check("oppb_inject_f64", self.lib.oppb_inject_f64(
            C.byref(self.mesh.s), C.byref(self.mesh.inlet), C.byref(v), start, count, _ptr(rnd_soa),
            rnd_soa.stride(0), rnd_soa.shape[0], self.ion_velocity, self.qm, self.dt, _stream_ptr(stream)))

    def zero_node_charge(self, stream=None) -> None:
        """opp_reset_dat(n_charge_den) with the library's fill kernel (oppb_fill)."""
        L.check("oppb_fill", self.lib.oppb_fill(_ptr(self.node_charge), self.node_charge.numel(), 8, 0,
                                                _stream_ptr(stream)))

    def push(self, stream=None) -> None:
        v = self.parts.view()
        fn = self.lib.oppb_push_mixed if self.precision == "mixed" else self.lib.oppb_push_f64
        L.check("oppb_push", fn(C.byref(self.mesh.s), C.byref(v), self.qm, self.dt, _stream_ptr(stream)))

    def _deposit_ws(self) -> torch.Tensor:
        nbytes = self.lib.oppb_deposit_workspace_bytes(self.mesh.n_nodes)
        if self._dep_ws.numel() < nbytes:
            self._dep_ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._dep_ws

    def field_phase(self, stream=None) -> None:
        """Node charge density, potential and cell field from node_charge (in place, as the
        reference scales n_charge_den), replayed from a CUDA graph."""
        key = self.node_charge.data_ptr()
        g = self._field_graphs.get(key)
        if g is None:
            state = (self.field.d.clone(), self.field.f1.clone(), self.node_charge.clone())
            g = self.field.capture(self.node_charge, self.n_vol, self.spwt, self.field_consts, self.mesh.ef, 4)
            self.field.d.copy_(state[0])  # capture and its warm-up leave the state as it was
            self.field.f1.copy_(state[1])
            self.node_charge.copy_(state[2])
            self._field_graphs[key] = g
        if stream is not None:
            with torch.cuda.stream(stream):
                g.replay()
        else:
            g.replay()

    def _move_ex(self, push: bool, stream=None) -> None:
        """The move through oppb_move_ex (the direct-hop seed is only reached there)."""
        v = self.parts.view()
        ws = self._deposit_ws()
        mixed = self.precision == "mixed"
        o = L.MoveOptions(precision=L.PRECISION_MIXED if mixed else L.PRECISION_F64,
                          deposit=int(mixed or self.fused_deposit), push=int(push), qm=self.qm, dt=self.dt,
                          band=self.band, dh=C.pointer(self.dh.g) if self.dh is not None else None)
        L.check("oppb_move_ex", self.lib.oppb_move_ex(C.byref(self.mesh.s), C.byref(v), C.byref(o),
                                                      _ptr(self.node_charge), _ptr(self.parts.status),
                                                      self.max_hops, _ptr(ws), ws.numel(), _stream_ptr(stream)))

    def move(self, stream=None) -> None:
        """Move (+ fused deposit into node_charge, which the caller zeroes)."""
        if self.dh is not None:
            return self._move_ex(False, stream)
        v = self.parts.view()
        st = _ptr(self.parts.status)
        sp = _stream_ptr(stream)
        ws = self._deposit_ws()
        if self.precision == "mixed":
            rc = self.lib.oppb_move_deposit_mixed(C.byref(self.mesh.s), C.byref(v), _ptr(self.node_charge), st,
                                                  self.max_hops, self.band, _ptr(ws), ws.numel(), sp)
        elif self.fused_deposit:
            rc = self.lib.oppb_move_deposit_f64(C.byref(self.mesh.s), C.byref(v), _ptr(self.node_charge), st,
                                                self.max_hops, _ptr(ws), ws.numel(), sp)
        else:
            rc = self.lib.oppb_move_f64(C.byref(self.mesh.s), C.byref(v), st, self.max_hops, sp)
        L.check("oppb_move", rc)

    def push_move(self, stream=None) -> None:
        """Push + move + deposit in one launch (the push is the move kernel's prologue);
        bit-identical to push() followed by move()."""
        if self.dh is not None:
            return self._move_ex(True, stream)
        v = self.parts.view()
        st = _ptr(self.parts.status)
        sp = _stream_ptr(stream)
        ws = self._deposit_ws()
        if self.precision == "mixed":
            rc = self.lib.oppb_push_move_deposit_mixed(C.byref(self.mesh.s), C.byref(v), _ptr(self.node_charge), st,
                                                       self.max_hops, self.band, self.qm, self.dt, _ptr(ws),
                                                       ws.numel(), sp)
        else:
            rc = self.lib.oppb_push_move_deposit_f64(C.byref(self.mesh.s), C.byref(v), _ptr(self.node_charge), st,
                                                     self.max_hops, self.qm, self.dt, _ptr(ws), ws.numel(), sp)
        L.check("oppb_push_move_deposit", rc)

    def deposit(self, stream=None) -> None:
        v = self.parts.view()
        ws = self._deposit_ws()
        L.check("oppb_deposit_f64", self.lib.oppb_deposit_f64(C.byref(self.mesh.s), C.byref(v),
                                                              _ptr(self.node_charge), _ptr(ws), ws.numel(),
                                                              _stream_ptr(stream)))

    def organize_kind(self) -> str:
        """What a compaction at the current iteration does ('holefill', 'sort' or 'shuffle'):
        opp_finalize_particle_move_core's rule (opp_lib/src/core/opp_particle_organize_core.cpp:49-95)."""
        periodic = self.fill in ("Sort_Periodic", "Shuffle_Periodic")
        if self.fill == "HoleFill_All" or (periodic and self.iter % self.fill_period != 0):
            return "holefill"
        return "sort" if self.fill.startswith("Sort") else "shuffle"

    def sort_now(self) -> bool:
        return self.organize_kind() == "sort"

    def shuffle_seed(self) -> int:
        """Seed of this iteration's shuffle keys (the reference seeds its RandomFunctor with 123,
        opp_lib/src/cuda/opp_particle_sorter.cu:195-201; here 123 and the iteration)."""
        return (123 << 32) | (self.iter & 0xFFFFFFFF) | (1 << 63)

    def finalize(self, remove_count: int, stream=None) -> str:
        """opp_finalize_particle_move: hole fill or cell sort, then size -= removed."""
        if remove_count <= 0:
            return "none"
        p = self.parts
        dats = p.dat_list()
        sp = _stream_ptr(stream)
        kind = self.organize_kind()
        if kind == "sort":
            nbytes = self.lib.oppb_sort_workspace_bytes(p.size, self.mesh.n_cells)
            ws = self._workspace(nbytes)
            L.check("oppb_sort_by_cell", self.lib.oppb_sort_by_cell(
                p.size, self.mesh.n_cells, p.capacity, len(p.DATS), dats, 3, None, _ptr(ws), ws.numel(), sp))
            p.swap_after_sort()
        elif kind == "shuffle":
            nbytes = self.lib.oppb_sort_workspace_bytes(p.size, self.mesh.n_cells)
            ws = self._workspace(nbytes)
            L.check("oppb_shuffle", self.lib.oppb_shuffle(
                p.size, self.mesh.n_cells, p.capacity, len(p.DATS), dats, 3, self.shuffle_seed(), None, _ptr(ws),
                ws.numel(), sp))
            p.swap_after_sort()
        else:
            nbytes = self.lib.oppb_hole_fill_workspace_bytes(p.size, remove_count)
            ws = self._workspace(nbytes)
            L.check("oppb_hole_fill", self.lib.oppb_hole_fill(
                p.size, remove_count, _ptr(p.bits), p.capacity, len(p.DATS), dats, _ptr(ws), ws.numel(), sp))
        p.size -= remove_count
        return kind

    def step(self, rnd_soa: torch.Tensor, stream=None, timers: StepTimes | None = None) -> dict:
        """One FemPIC particle step.  Reads the move status once (the remove count that
        sizes the compaction), as the reference does after its move."""
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if timers is not None else None
        s = stream if stream is not None else torch.cuda.current_stream()
        if ev: ev[0].record(s)
        self.inject(rnd_soa, stream)
        self.zero_node_charge(stream)
        if ev: ev[1].record(s)
        n_before = self.parts.size
        if self.fused_push:
            if ev: ev[2].record(s)
            self.push_move(stream)  # push time is counted in move_ms
        else:
            self.push(stream)
            if ev: ev[2].record(s)
            self.move(stream)  # unfused FP64 deposit runs after the compaction, as the reference loop order
        if ev: ev[3].record(s)
        st = self.parts.status_host()
        if st.error:
            raise L.OppbError(f"move (particle {st.error_index})", st.error)
        kind = self.finalize(st.remove_count, stream)
        self._count_synced = False
        if not self.fused_deposit and self.precision == "f64":
            self.deposit(stream)
        if self.field is not None and self.field_enabled:
            self.field_phase(stream)
        if ev:
            ev[4].record(s)
            ev[4].synchronize()
            timers.inject_ms += ev[0].elapsed_time(ev[1])
            timers.push_ms += ev[1].elapsed_time(ev[2])
            timers.move_ms += ev[2].elapsed_time(ev[3])
            timers.compact_ms += ev[3].elapsed_time(ev[4])
        out = {"iter": self.iter, "size_before_move": n_before, "removed": st.remove_count, "size": self.parts.size,
               "visits": int(st.total_visits), "max_visits": st.max_visits, "rechecks": st.recheck_count,
               "compaction": kind}
        self.last = out
        self.iter += 1
        return out


    def _pipeline(self, rows: int, cols: int) -> dict:
        """run_steps' state, kept between calls so that no call allocates or creates a stream
        once it exists: the copy stream, its events, two device tables of at least
        [rows][cols] and the node-charge buffer that alternates with node_charge."""
        p = self._pipe
        if p is None:
            ev = lambda: torch.cuda.Event()  # noqa: E731
            p = self._pipe = {"copy": torch.cuda.Stream(device=self.device), "alt": torch.empty_like(self.node_charge),
                              "tables": [], "table_ready": [ev(), ev()], "table_free": [ev(), ev()],
                              "charge_ready": [ev(), ev()], "charge_free": [ev(), ev()]}
        t = p["tables"]
        if not t or t[0].shape[0] < rows or t[0].shape[1] < cols:
            rows, cols = max(rows, t[0].shape[0] if t else 0), max(cols, t[0].shape[1] if t else 0)
            p["tables"] = [torch.empty((rows, cols), dtype=torch.float64, device=self.device) for _ in range(2)]
        return p

    def run_steps(self, host_tables: list[torch.Tensor], charges_out: list[torch.Tensor] | None = None) -> list[dict]:
        """len(host_tables) steps fed from host memory, with the node charges of every step
        copied back to the host.  host_tables: pinned CPU float64 [5][count] tables (the
        step's injection randoms; count may differ between steps); charges_out: pinned CPU
        float64 [n_nodes] tensors, one per step (or None).  Copies run on a second stream and
        overlap the steps: the next step's table goes up while the current step computes,
        and a step's charges come down (from one of two alternating node-charge buffers)
        while the next step computes.  Returns the per-step records of step(); every copy
        has completed on return, and node_charge holds the last step's charges."""
        n = len(host_tables)
        if n == 0:
            return []
        if charges_out is not None and len(charges_out) != n:
            raise ValueError("charges_out needs one tensor per step")
        cur = torch.cuda.current_stream(self.device)
        p = self._pipeline(max(t.shape[0] for t in host_tables), max(t.shape[1] for t in host_tables))
        copy = p["copy"]
        table_ready, table_free = p["table_ready"], p["table_free"]
        charge_ready, charge_free = p["charge_ready"], p["charge_free"]
        charges = [self.node_charge, p["alt"]]
        tables = [None, None]

        def upload(k: int, b: int) -> None:  # on the copy stream, into buffer b once step k-2 has read it
            rows, cols = host_tables[k].shape
            tables[b] = p["tables"][b][:rows, :cols]
            with torch.cuda.stream(copy):
                copy.wait_event(table_free[b])
                tables[b].copy_(host_tables[k], non_blocking=True)
                table_ready[b].record(copy)

        for e in table_free + charge_free:
            e.record(cur)
        upload(0, 0)
        out = []
        for k in range(n):
            b = k % 2
            if k + 1 < n:  # prefetch the next table into the other buffer
                upload(k + 1, 1 - b)
            cur.wait_event(table_ready[b])
            cur.wait_event(charge_free[b])  # the copy of this buffer's previous charges is done
            self.node_charge = charges[b]
            out.append(self.step(tables[b]))
            table_free[b].record(cur)
            charge_ready[b].record(cur)
            if charges_out is not None:
                with torch.cuda.stream(copy):
                    copy.wait_event(charge_ready[b])
                    charges_out[k].copy_(charges[b], non_blocking=True)
                    charge_free[b].record(copy)
            else:
                charge_free[b].record(cur)
        p["alt"] = charges[n % 2]  # the buffer that does not hold the last step's charges
        copy.synchronize()
        cur.wait_stream(copy)
        return out

    # ------------------------------------------------------------ graph-captured steps

    def _bufs(self) -> tuple:
        p = self.parts
        return tuple(getattr(p, n) for n, _, _ in p.DATS) + tuple(getattr(p, n + "_swap") for n, _, _ in p.DATS)

    def _set_bufs(self, bufs: tuple) -> None:
        p, k = self.parts, len(self.parts.DATS)
        for j, (n, _, _) in enumerate(p.DATS):
            setattr(p, n, bufs[j])
            setattr(p, n + "_swap", bufs[k + j])

    def _graph_phase(self) -> int:
        return self.iter % self.fill_period if self.fill.endswith("Periodic") else 0

    def _step_dev(self, table: torch.Tensor, bound: int, records: torch.Tensor, n_records: int, stream=None,
                  count=None, field: bool = True, charge_out: torch.Tensor | None = None) -> None:
        """One step on the device count (no host read): the launches of step() with the fused
        push, sized from `bound`.  count: the oppb_set_count tensor (default self.count_dev);
        charge_out: a device buffer that receives the step's node charges (a copy)."""
        p, m, lib = self.parts, self.mesh, self.lib
        cnt = _ptr(self.count_dev if count is None else count)
        st = _ptr(p.status)
        sp = _stream_ptr(stream)
        n_inj = int(table.shape[1])
        self.zero_node_charge(stream)
        v = p.view()
        v.size = bound
        L.check("oppb_inject_dev", lib.oppb_inject_dev(
            C.byref(m.s), C.byref(m.inlet), C.byref(v), cnt, n_inj, _ptr(table), table.stride(0), table.shape[0],
            self.ion_velocity, self.qm, self.dt, sp))
        ws = self._deposit_ws()
        o = L.MoveOptions(precision=L.PRECISION_MIXED if self.precision == "mixed" else L.PRECISION_F64,
                          deposit=1, push=1, qm=self.qm, dt=self.dt, band=self.band, dh=None, set_count=cnt,
                          pending=n_inj)
        L.check("oppb_move_ex", lib.oppb_move_ex(C.byref(m.s), C.byref(v), C.byref(o), _ptr(self.node_charge), st,
                                                 self.max_hops, _ptr(ws), ws.numel(), sp))
        dats = p.dat_list()
        kind = self.organize_kind()
        cws = self._ws
        if kind == "sort":
            L.check("oppb_sort_by_cell_dev", lib.oppb_sort_by_cell_dev(
                bound, cnt, n_inj, st, m.n_cells, p.capacity, len(p.DATS), dats, 3, _ptr(cws), cws.numel(), sp))
            p.swap_after_sort()
        elif kind == "shuffle":
            L.check("oppb_shuffle_dev", lib.oppb_shuffle_dev(
                bound, cnt, n_inj, st, m.n_cells, p.capacity, len(p.DATS), dats, 3, self.shuffle_seed(), _ptr(cws),
                cws.numel(), sp))
            p.swap_after_sort()
        else:
            L.check("oppb_hole_fill_dev", lib.oppb_hole_fill_dev(
                bound, cnt, n_inj, st, _ptr(p.bits), p.capacity, len(p.DATS), dats, _ptr(cws), cws.numel(), sp))
        L.check("oppb_step_end_dev", lib.oppb_step_end_dev(cnt, n_inj, st, _ptr(records), n_records, sp))
        if charge_out is not None:
            charge_out.copy_(self.node_charge)
        if field and self.field is not None and self.field_enabled:
            self.field.launch(self.node_charge, self.n_vol, self.spwt, self.field_consts, self.mesh.ef, 4)
        self.iter += 1

    def _sync_count(self) -> None:
        """Device count := host count (after host-sized steps)."""
        if not self._count_synced:
            self.count_dev.copy_(torch.tensor([self.parts.size, 0, 0, 0], dtype=torch.int32))
            self._count_synced = True

    def capture_steps(self, steps: int, n_inject: int | None = None, slack: float = 0.02,
                      keep_charges: bool = False) -> StepGraph:
        """Captures `steps` whole steps, from the current iteration and particle buffers, as one
        CUDA graph.  The capacity grows first when the count could exceed it (every particle
        injected, none removed, plus `slack`).  keep_charges: every step also copies its node
        charges into the graph's `charges[k]`."""
        if not self.fused_push:
            raise ValueError("graph-captured steps need the fused push (fused_push=True)")
        if self.dh is not None:
            raise ValueError("graph-captured steps walk from the previous cell (no direct-hop seed)")
        n_inj = self.inject_per_step if n_inject is None else int(n_inject)
        p = self.parts
        bound = int((p.size + steps * n_inj) * (1.0 + slack)) + 1
        if bound > p.capacity:
            p._alloc(max(bound, int(p.size + steps * n_inj * p.alloc_mult)))
            self._graphs.clear()
        bound = min(bound, p.capacity)
        ws_bytes = max(self.lib.oppb_hole_fill_dev_workspace_bytes(bound),
                       self.lib.oppb_sort_dev_workspace_bytes(bound))
        self._workspace(ws_bytes)
        self._deposit_ws()
        tables = [torch.zeros((5, n_inj), dtype=torch.float64, device=self.device) for _ in range(steps)]
        records = torch.zeros((steps, 8), dtype=torch.int32, device=self.device)
        charges = torch.zeros((steps, self.node_charge.numel()), dtype=torch.float64, device=self.device) \
            if keep_charges else None
        # Warm-up: one launch of every kernel the capture uses (the first launch of a kernel
        # loads it), on a scratch count of -n_inj: the injection starts below 0 and writes
        # nothing, and every later launch sees zero particles.
        scratch = torch.zeros(4, dtype=torch.int32, device=self.device)
        saved = (self._bufs(), self.iter, p.size, self.node_charge.clone(), p.status.clone())
        for k in range(min(steps, max(1, self.fill_period if self.fill.endswith("Periodic") else 1))):
            scratch.fill_(0)
            scratch[0] = -n_inj
            self._step_dev(tables[0], bound, records, steps, count=scratch, field=False)
        if self.field is not None and self.field_enabled:
            self.field.warm(self.node_charge, self.n_vol, self.spwt, self.field_consts, self.mesh.ef, 4)
        self.node_charge.copy_(saved[3])
        p.status.copy_(saved[4])
        self._set_bufs(saved[0])
        self.iter, p.size = saved[1], saved[2]
        torch.cuda.synchronize(self.device)
        self._sync_count()
        launches0 = self.lib.oppb_kernel_launches()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                for k in range(steps):
                    self._step_dev(tables[k], bound, records, steps, charge_out=None if charges is None else charges[k])
        torch.cuda.current_stream(self.device).wait_stream(s)
        launches = int(self.lib.oppb_kernel_launches() - launches0)
        bufs_after = self._bufs()
        self._set_bufs(saved[0])
        self.iter, p.size = saved[1], saved[2]
        return StepGraph(g, steps, bound, tables, records, saved[0], bufs_after, p.capacity, launches, charges,
                         self.node_charge.data_ptr())

    def _graph_key(self, steps: int, n_inj: int, keep_charges: bool) -> tuple:
        return (steps, n_inj, self._graph_phase(), StepGraph.ptrs(self._bufs()), self.parts.capacity,
                self.node_charge.data_ptr(), keep_charges)

    def graph_for(self, steps: int, n_inject: int | None = None, keep_charges: bool = False) -> StepGraph:
        """The captured graph for the next `steps` steps from here (captured when none fits)."""
        n_inj = self.inject_per_step if n_inject is None else int(n_inject)
        g = self._graphs.get(self._graph_key(steps, n_inj, keep_charges))
        if g is None or self.parts.size + steps * n_inj > g.bound:
            g = self.capture_steps(steps, n_inj, keep_charges=keep_charges)
            self._graphs[self._graph_key(steps, n_inj, keep_charges)] = g
        return g

    def replay(self, g: StepGraph, stream=None) -> list[dict]:
        """Runs the steps of g (its tables as they are), then reads the count and the step records
        back once.  Raises on a device error of any of the steps."""
        if StepGraph.ptrs(g.bufs_before) != StepGraph.ptrs(self._bufs()) or g.capacity != self.parts.capacity or \
                g.node_charge_ptr != self.node_charge.data_ptr():
            raise ValueError("the graph was captured for other particle or node-charge buffers")
        self._sync_count()
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(s):
            g.graph.replay()
        return self.replay_finish(g)

    def replay_finish(self, g: StepGraph) -> list[dict]:
        """After g.graph.replay() on the current stream (the device count in sync): reads the
        count and the step records back and advances the host's view of the set."""
        cnt = L.SetCount.from_buffer_copy(self.count_dev.cpu().numpy().tobytes())
        raw = g.records.cpu().numpy().tobytes()
        recs = [L.StepRecord.from_buffer_copy(raw[32 * k:32 * (k + 1)]) for k in range(g.steps)]
        first = (cnt.steps - g.steps) % g.steps  # the ring position of this replay's first step
        recs = [recs[(first + k) % g.steps] for k in range(g.steps)]
        out = []
        for k, r in enumerate(recs):
            out.append({"iter": self.iter + k, "size_before_move": r.size_before_move, "removed": r.removed,
                        "size": r.size, "visits": int(r.total_visits), "max_visits": r.max_visits,
                        "rechecks": r.recheck_count, "error": r.error})
        self.parts.size = cnt.size
        self.iter += g.steps
        self._set_bufs(g.bufs_after)
        if cnt.error:
            self.count_dev[1:3] = 0
            raise L.OppbError(f"graph-captured step {cnt.error_step}", cnt.error)
        self.last = out[-1]
        return out

    def run_graph(self, tables: list[torch.Tensor]) -> list[dict]:
        """len(tables) steps from one graph replay; tables: device float64 [5][count] injection
        tables (copied into the graph's own tables first)."""
        g = self.graph_for(len(tables), int(tables[0].shape[1]))
        for dst, src in zip(g.tables, tables):
            if dst.data_ptr() != src.data_ptr():
                dst.copy_(src)
        return self.replay(g)

    def run_graph_host(self, host_tables: list[torch.Tensor], charges_out: list[torch.Tensor] | None = None,
                       steps_per_graph: int | None = None) -> list[dict]:
        """run_steps' contract (host tables in, every step's node charges out) on graph-captured
        steps: the steps go in chunks of steps_per_graph (default: the fill period of a
        periodic fill, else 10), each one replay of a captured graph that also copies every
        step's node charges aside; the count and the step records come back once per chunk.
        host_tables: pinned CPU float64 [5][count] tables, one count for all steps;
        charges_out: pinned CPU float64 [n_nodes] tensors, one per step (or None).  A second
        stream moves the next chunk's tables up and the last chunk's charges down while a
        chunk runs.  Returns the per-step records; every copy has completed on return, and
        node_charge holds the last step's charges."""
        n = len(host_tables)
        if n == 0:
            return []
        if charges_out is not None and len(charges_out) != n:
            raise ValueError("charges_out needs one tensor per step")
        rows, n_inj = host_tables[0].shape
        if any(t.shape != host_tables[0].shape for t in host_tables):
            raise ValueError("graph-captured steps inject the same count every step")
        S = steps_per_graph or (self.fill_period if self.fill.endswith("Periodic") else 10)
        chunks = [list(range(c, min(c + S, n))) for c in range(0, n, S)]
        cur = torch.cuda.current_stream(self.device)
        p = self._pipeline(rows, n_inj)
        copy = p["copy"]
        io = self._graph_io(S, rows, n_inj)
        t_ready, t_free, c_ready, c_free = io["table_ready"], io["table_free"], io["charge_ready"], io["charge_free"]
        for e in t_free + c_free:
            e.record(cur)

        def upload(c: int) -> None:  # chunk c's tables into staging set c % 2, on the copy stream
            b = c % 2
            with torch.cuda.stream(copy):
                copy.wait_event(t_free[b])
                for k, j in enumerate(chunks[c]):
                    io["tables"][b][k].copy_(host_tables[j], non_blocking=True)
                t_ready[b].record(copy)

        upload(0)
        out = []
        for c, idx in enumerate(chunks):
            b = c % 2
            g = self.graph_for(len(idx), n_inj, keep_charges=True)
            if c + 1 < len(chunks):
                upload(c + 1)
            cur.wait_event(t_ready[b])
            for k in range(len(idx)):
                g.tables[k].copy_(io["tables"][b][k])
            t_free[b].record(cur)
            self._sync_count()
            g.graph.replay()
            cur.wait_event(c_free[b])  # the previous download from this staging set is done
            io["charges"][b][:len(idx)].copy_(g.charges)
            c_ready[b].record(cur)
            if charges_out is not None:
                with torch.cuda.stream(copy):
                    copy.wait_event(c_ready[b])
                    for k, j in enumerate(idx):
                        charges_out[j].copy_(io["charges"][b][k], non_blocking=True)
                    c_free[b].record(copy)
            else:
                c_free[b].record(cur)
            out.extend(self.replay_finish(g))
        copy.synchronize()
        cur.wait_stream(copy)
        return out

    def _graph_io(self, steps: int, rows: int, cols: int) -> dict:
        """run_graph_host's device staging (two sets of `steps` injection tables and of `steps`
        node-charge buffers) and its events, made once per shape."""
        key = (steps, rows, cols)
        io = self._gio.get(key)
        if io is None:
            ev = lambda: torch.cuda.Event()  # noqa: E731
            nn = self.node_charge.numel()
            io = self._gio[key] = {
                "tables": [torch.empty((steps, rows, cols), dtype=torch.float64, device=self.device) for _ in range(2)],
                "charges": [torch.empty((steps, nn), dtype=torch.float64, device=self.device) for _ in range(2)],
                "table_ready": [ev(), ev()], "table_free": [ev(), ev()],
                "charge_ready": [ev(), ev()], "charge_free": [ev(), ev()]}
        return io


class StepGraph:
    """Whole FemPIC steps captured as one CUDA graph (include/oppb_graph.h): per step the node
    charge reset, inject, push + move + deposit, hole fill / sort / shuffle, the step record and,
    when on, the field phase, all sized from the device count.  `tables` are the device
    injection tables the graph reads (step k reads tables[k]); `records` receive the steps'
    oppb_step_record.  Valid while the particle count stays within `bound`, the particle
    buffers and capacity are those of the capture and the step phase (iteration modulo the fill
    period) is the same."""

    def __init__(self, graph, steps: int, bound: int, tables, records, bufs_before, bufs_after, capacity: int,
                 launches: int, charges=None, node_charge_ptr: int = 0):
        self.graph, self.steps, self.bound = graph, steps, bound
        self.tables, self.records = tables, records
        self.bufs_before, self.bufs_after, self.capacity = bufs_before, bufs_after, capacity
        self.launches = launches  # library kernels per replay
        self.charges = charges  # [steps][n_nodes] per-step node charges (keep_charges), else None
        self.node_charge_ptr = node_charge_ptr

    @staticmethod
    def ptrs(bufs) -> tuple:
        return tuple(t.data_ptr() for t in bufs)


def randoms_to_device(rnd_aos: np.ndarray, device) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(rnd_aos.T)).to(device)
