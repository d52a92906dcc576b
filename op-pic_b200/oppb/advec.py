"""NESO-advection particle path on the B200 backend (include/oppb_advec.h): one instance or a
batch of independent instances of different sizes advanced by one persistent launch per step.

Host-side set-up mirrors the reference app where the particle path needs it:
  AdvecMesh   init_mesh of apps_codegen/app_neso_advection_mdir_cg/advec_misc.h: nx x ny square
              cells, index x + nx*y (VOXEL), periodic 4-neighbour map c2c in CellMap order
              xd_y, xu_y, x_yd, x_yu (VOXEL_MAP, advec_defs.h:46-54), lower-left corners c_pos_ll
  particles   init_particles' construction: positions uniform inside every cell (cell order),
              normal velocities, move direction (1, 1); seeded numpy generator
  AdvecBatch  device buffers of many instances concatenated, the instance table, the step
              launch and its CUDA-graph capture; the global move (opp_global_move with
              opp_init_direct_hop_cg, advec_opp.cpp:97-103) as each instance's direct-hop grid
  shard_instances  the split of an ensemble over GPUs: instances are independent, so each
              rank advances its own subset in its own persistent launch, with no collective
              on the data path
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from oppb import _lib as L


class AdvecMesh:
    def __init__(self, nx: int, ny: int, cell_width: float = 1.0):
        self.nx, self.ny, self.cell_width = nx, ny, cell_width
        self.n_cells = nx * ny
        y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        x, y = x.ravel(), y.ravel()  # index = x + nx*y, ascending

        def vox(a, b):
            a = np.where(a < 0, nx - 1, np.where(a >= nx, 0, a))
            b = np.where(b < 0, ny - 1, np.where(b >= ny, 0, b))
            return (a + nx * b).astype(np.int32)

        self.c2c = np.stack([vox(x - 1, y), vox(x + 1, y), vox(x, y - 1), vox(x, y + 1)], axis=1).astype(np.int32)
        self.c_pos_ll = np.stack([x * cell_width, y * cell_width], axis=1).astype(np.float64)
        self.extents = (nx * cell_width, ny * cell_width)


def particles(mesh: AdvecMesh, ppc: int, v_sd: float, seed: int, v_clip: float | None = None):
    """ppc particles per cell in cell order, positions uniform in the cell, velocities
    N(0, v_sd^2) per axis (clipped to +-v_clip), mdir (1, 1).  Returns AoS pos, vel, mdir, p2c."""
    rng = np.random.default_rng(seed)
    p2c = np.repeat(np.arange(mesh.n_cells, dtype=np.int32), ppc)
    pos = mesh.c_pos_ll[p2c] + rng.uniform(0.0, mesh.cell_width, (len(p2c), 2))
    vel = rng.normal(0.0, v_sd, (len(p2c), 2))
    if v_clip is not None:
        np.clip(vel, -v_clip, v_clip, out=vel)
    mdir = np.ones((len(p2c), 2), np.int32)
    return pos, vel, mdir, p2c


WORK_ITEM = 256  # particles per work item of the persistent launch


def shard_instances(weights, n_ranks: int) -> list[list[int]]:
    """Longest-processing-time-first split of independent instances over n_ranks GPUs:
    instances in decreasing weight (ties: lower index first) each go to the rank with the
    least weight so far (ties: lower rank).  The weight is the instance's particle count, the
    work of a step.  Deterministic, so every rank computes the same split from the same
    list.  Returns the instance indices of every rank in increasing order; the largest load
    is within the largest weight of the mean."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    loads = [0] * n_ranks
    out: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in sorted(range(len(weights)), key=lambda i: (-weights[i], i)):
        r = min(range(n_ranks), key=lambda r: (loads[r], r))
        out[r].append(i)
        loads[r] += weights[i]
    return [sorted(o) for o in out]


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def _stream(stream) -> int | None:
    return None if stream is None else stream.cuda_stream


class AdvecBatchDevice:
    """Device state of a batch of instances: particle dats of all instances concatenated
    (SoA [2][capacity]), packed cell records, the instance table and work-item prefix.
    There is no CPU fallback."""

    def __init__(self, meshes: list[AdvecMesh], counts: list[int], dts: list[float], device, grid: bool = True):
        """grid: verify each instance's packed cells against the periodic grid of the app's
        init_mesh (oppb_advec_check_grid) and, where they match bit for bit, let the move
        compute corners and neighbours instead of reading the records."""
        if not torch.cuda.is_available():
            raise RuntimeError("AdvecBatchDevice needs a CUDA device (there is no CPU fallback)")
        self.device = torch.device(device)
        self.lib = L.load()
        self.meshes, self.counts = meshes, list(counts)
        n_total = int(sum(counts))
        self.capacity = max(n_total, 1)
        cap = self.capacity
        self.pos = torch.zeros((2, cap), dtype=torch.float64, device=self.device)
        self.vel = torch.zeros((2, cap), dtype=torch.float64, device=self.device)
        self.mdir = torch.ones((2, cap), dtype=torch.int32, device=self.device)
        self.p2c = torch.zeros(cap, dtype=torch.int32, device=self.device)
        self.status = torch.zeros(8, dtype=torch.int32, device=self.device)
        self.counter = torch.zeros(8, dtype=torch.int32, device=self.device)
        total_cells = sum(m.n_cells for m in meshes)
        self.cells = torch.zeros(total_cells * 4, dtype=torch.float64, device=self.device)
        table = (L.AdvecInstance * len(meshes))()
        prefix = [0]
        self.part_offsets, self.cell_offsets = [], []
        po = co = 0
        for k, (m, n, dt) in enumerate(zip(meshes, counts, dts)):
            table[k] = L.AdvecInstance(po, n, co, m.n_cells, 0, dt, m.cell_width, (C.c_double * 2)(*m.extents))
            self.part_offsets.append(po)
            self.cell_offsets.append(co)
            c2c = torch.from_numpy(np.ascontiguousarray(m.c2c.T)).to(self.device)
            ll = torch.from_numpy(np.ascontiguousarray(m.c_pos_ll.T)).to(self.device)
            L.check("oppb_advec_pack_cells",
                    self.lib.oppb_advec_pack_cells(_ptr(self.cells), co, m.n_cells, m.n_cells, _ptr(ll), _ptr(c2c),
                                                   None))
            prefix.append(prefix[-1] + (n + WORK_ITEM - 1) // WORK_ITEM)
            po += n
            co += m.n_cells
        self.grid_nx = [0] * len(meshes)
        if grid:
            mism = torch.zeros(max(1, len(meshes)), dtype=torch.int32, device=self.device)
            for k, m in enumerate(meshes):
                L.check("oppb_advec_check_grid", self.lib.oppb_advec_check_grid(
                    _ptr(self.cells), self.cell_offsets[k], m.n_cells, m.nx, m.cell_width, _ptr(mism) + 4 * k, None))
            for k, bad in enumerate(mism.cpu().tolist()[:len(meshes)]):
                if bad == 0:
                    self.grid_nx[k] = meshes[k].nx
                    table[k].grid_nx = meshes[k].nx
        self.instances = torch.frombuffer(bytearray(bytes(table)), dtype=torch.uint8).to(self.device)
        self.tile_prefix = torch.tensor(prefix, dtype=torch.int32, device=self.device)
        self.batch = L.AdvecBatch(len(meshes), prefix[-1], _ptr(self.instances), _ptr(self.tile_prefix),
                                  _ptr(self.cells), cap, _ptr(self.pos), _ptr(self.vel), _ptr(self.mdir),
                                  _ptr(self.p2c), _ptr(self.counter))
        self.n_total = n_total
        self.dh_grids: list = []  # per instance (L.DhGrid, map tensor), once enable_direct_hop ran
        self._dh_table = None

    def enable_direct_hop(self, grid_spacing, expansion=None) -> None:
        """The app's global move: every instance gets the direct-hop grid of its mesh
        (BoundingBox(c_pos_ll, 2, expansion), expansion (2 cell widths, 2 cell widths, 0) as in
        advec_opp.cpp, the map built on the GPU) and its walks start from the grid's seed.
        grid_spacing: one value for all instances, or one per instance."""
        spacings = list(grid_spacing) if np.ndim(grid_spacing) else [grid_spacing] * len(self.meshes)
        if len(spacings) != len(self.meshes):
            raise ValueError("one grid spacing per instance")
        dh = (L.AdvecDh * len(self.meshes))()
        self.dh_grids = []
        ws = None
        for k, (m, spacing) in enumerate(zip(self.meshes, spacings)):
            ex = (C.c_double * 3)(*(expansion if expansion is not None else (2 * m.cell_width, 2 * m.cell_width, 0.0)))
            ll = np.ascontiguousarray(m.c_pos_ll, dtype=np.float64)
            g = L.DhGrid()
            L.check("oppb_dh_grid_init_2d", self.lib.oppb_dh_grid_init_2d(ll.ctypes.data, m.n_cells, spacing, ex,
                                                                          C.byref(g)))
            gmap = torch.empty(int(g.size), dtype=torch.int32, device=self.device)
            g.map = gmap.data_ptr()
            cells = self.cells.data_ptr() + 32 * self.cell_offsets[k]
            need = C.c_size_t(0)
            for _ in range(2):  # the first call may only size the workspace
                rc = self.lib.oppb_dh_build_quad(cells, m.n_cells, m.cell_width, C.byref(g), _ptr(ws),
                                                 0 if ws is None else ws.numel(), C.byref(need), None)
                if rc != L.OPPB_ERR_WORKSPACE:
                    break
                ws = torch.empty(int(need.value), dtype=torch.uint8, device=self.device)
            L.check("oppb_dh_build_quad", rc)
            dh[k] = L.AdvecDh(g.map, (C.c_double * 2)(g.min[0], g.min[1]), g.inv_spacing,
                              (L.c_i64 * 2)(g.dims[0], g.dims[1]))
            self.dh_grids.append((g, gmap))
        self._dh_table = torch.frombuffer(bytearray(bytes(dh)), dtype=torch.uint8).to(self.device)
        self.batch.dh = self._dh_table.data_ptr()
        torch.cuda.synchronize(self.device)

    def disable_direct_hop(self) -> None:
        """Walks start from p2c again."""
        self.batch.dh = None
        self._dh_table = None
        self.dh_grids = []

    def set_instance(self, k: int, pos, vel, mdir, p2c) -> None:
        """Upload one instance's host AoS particles."""
        a, n = self.part_offsets[k], self.counts[k]
        assert len(p2c) == n
        self.pos[:, a:a + n] = torch.from_numpy(np.ascontiguousarray(pos.T)).to(self.device)
        self.vel[:, a:a + n] = torch.from_numpy(np.ascontiguousarray(vel.T)).to(self.device)
        self.mdir[:, a:a + n] = torch.from_numpy(np.ascontiguousarray(mdir.T)).to(self.device)
        self.p2c[a:a + n] = torch.from_numpy(np.ascontiguousarray(p2c, dtype=np.int32)).to(self.device)

    def fill_instance(self, k: int, ppc: int, v_sd: float, v_clip: float, seed: int) -> None:
        """particles()'s construction drawn on the device (torch generator) for instance k."""
        m, a, n = self.meshes[k], self.part_offsets[k], self.counts[k]
        assert n == m.n_cells * ppc
        g = torch.Generator(device=self.device)
        g.manual_seed(seed)
        cells = torch.arange(m.n_cells, dtype=torch.int32, device=self.device).repeat_interleave(ppc)
        self.p2c[a:a + n] = cells
        cw = m.cell_width
        self.pos[0, a:a + n] = (cells % m.nx).to(torch.float64) * cw
        self.pos[1, a:a + n] = (cells // m.nx).to(torch.float64) * cw
        u = torch.empty((2, n), dtype=torch.float64, device=self.device).uniform_(0.0, cw, generator=g)
        self.pos[:, a:a + n] += u
        self.vel[:, a:a + n].normal_(0.0, v_sd, generator=g).clamp_(-v_clip, v_clip)
        self.mdir[:, a:a + n] = 1

    def zero_status(self) -> None:
        self.status.zero_()

    def step(self, max_hops: int = 4096, stream=None) -> None:
        """update_pos + move of every instance, one persistent launch; status accumulates."""
        L.check("oppb_advec_step", self.lib.oppb_advec_step(C.byref(self.batch), _ptr(self.status), max_hops,
                                                            _stream(stream)))

    def update_pos(self, stream=None) -> None:
        L.check("oppb_advec_update_pos", self.lib.oppb_advec_update_pos(C.byref(self.batch), _stream(stream)))

    def move(self, max_hops: int = 4096, stream=None) -> None:
        L.check("oppb_advec_move", self.lib.oppb_advec_move(C.byref(self.batch), _ptr(self.status), max_hops,
                                                            _stream(stream)))

    def capture(self, steps: int, max_hops: int = 4096) -> torch.cuda.CUDAGraph:
        """A CUDA graph of `steps` consecutive step() launches.  Make one step() call first:
        it sizes the persistent grid (an occupancy query) outside the capture."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(g, stream=s):
            for _ in range(steps):
                self.step(max_hops, stream=s)
        torch.cuda.current_stream().wait_stream(s)
        return g

    def status_host(self) -> L.MoveStatus:
        return L.MoveStatus.from_buffer_copy(self.status.cpu().numpy().tobytes())

    def host_instance(self, k: int) -> dict:
        a, n = self.part_offsets[k], self.counts[k]
        return {"pos": self.pos[:, a:a + n].T.contiguous().cpu().numpy(),
                "mdir": self.mdir[:, a:a + n].T.contiguous().cpu().numpy(),
                "p2c": self.p2c[a:a + n].cpu().numpy()}

    def instance_batches(self) -> list:
        """One single-instance batch per instance over the same buffers (for launching the
        instances one by one).  Returns (batch, keep-alive tensors) pairs."""
        import ctypes as C_

        out = []
        raw = self.instances.cpu().numpy().tobytes()
        size = C_.sizeof(L.AdvecInstance)
        for k, n in enumerate(self.counts):
            inst = torch.frombuffer(bytearray(raw[k * size:(k + 1) * size]), dtype=torch.uint8).to(self.device)
            pre = torch.tensor([0, (n + WORK_ITEM - 1) // WORK_ITEM], dtype=torch.int32, device=self.device)
            b = L.AdvecBatch(1, int(pre[1].item()), _ptr(inst), _ptr(pre), _ptr(self.cells), self.capacity,
                             _ptr(self.pos), _ptr(self.vel), _ptr(self.mdir), _ptr(self.p2c), _ptr(self.counter))
            if self._dh_table is not None:
                b.dh = self._dh_table.data_ptr() + k * C_.sizeof(L.AdvecDh)
            out.append((b, (inst, pre)))
        return out

    def step_batch(self, batch, max_hops: int = 4096, stream=None) -> None:
        L.check("oppb_advec_step", self.lib.oppb_advec_step(C.byref(batch), _ptr(self.status), max_hops,
                                                            _stream(stream)))
