"""The launch choices of the FemPIC path, picked by timing them on the live state.

The move + deposit launch has six choices (oppb_tuning): the FP64 move's lanes per particle
(one, 32 particles per warp, or a lane pair, 16 per warp), for the pair kernel the CTAs per
SM it is compiled for (8 at 32 registers a thread, 5 at 48), for the one-lane kernel whether
the cell records are staged into shared memory by bulk asynchronous copies; the deposit
strategy (warp-matched FP64 atomics, or a per-CTA shared-memory node table), how many
node-sum copies the atomics are spread over, and the block shape of the one-lane kernels
(128, 256 or 512 threads).  The cell sort has two (particle-dat columns moved per launch,
gather by destination or scatter by source).  tune_move, tune_lanes, tune_block and tune_sort
time every candidate on the simulation's current particle state, restoring a snapshot of the
particle dats before each trial so that every candidate sees the same input, then keep the
fastest as the process-wide tuning.  The choice of a trial is the median of its repetitions.
tune_sort_period times whole sort cycles (the steps between two cell sorts) for candidate
Sort_Periodic periods from a snapshot of the state and reports the cost per particle-step of
each; results stay bit-exact for any period (the oracle runs the same one).
"""
from __future__ import annotations

import ctypes as C
import statistics
from dataclasses import dataclass, field
from typing import Callable

import torch

from oppb import _lib as L

MOVE_CANDIDATES = [(dep, rep) for dep in (L.DEPOSIT_WARP_ATOMIC, L.DEPOSIT_CTA_TABLE) for rep in (1, 4, 8, 16)]
# (move_lanes, move_occupancy, move_stage, move_walk32)
LANE_CANDIDATES = [(1, 8, 0, 0), (1, 8, 0, 1), (1, 8, 0, 2), (1, 8, 1, 0), (2, 8, 0, 0), (2, 5, 0, 0)]
BLOCK_CANDIDATES = [256, 128, 512]  # threads per CTA of the one-lane move kernels
SORT_CANDIDATES = [(16, 0), (10, 0), (5, 0), (16, 1), (10, 1)]  # (columns per launch, scatter form)
PERIOD_CANDIDATES = [5, 10, 20]
MARGIN = 0.01  # a move-launch candidate replaces the default only when more than 1 % faster


@dataclass
class TuneResult:
    choice: object
    times_ms: dict = field(default_factory=dict)

    def report(self) -> dict:
        return {"choice": str(self.choice), "ms": {str(k): v for k, v in self.times_ms.items()}}


def pick(candidates, run: Callable[[object], float], reps: int = 3, margin: float = 0.0) -> TuneResult:
    """Times run(candidate) reps times per candidate (each call returns milliseconds) and returns
    the candidate with the smallest median; ties go to the earlier candidate.  With margin > 0
    the first candidate (the default) is kept unless the fastest beats it by more than that
    fraction, so that trial noise does not flip the choice."""
    if not candidates:
        raise ValueError("no candidates")
    res = TuneResult(choice=None)
    for c in candidates:
        res.times_ms[c] = statistics.median(run(c) for _ in range(reps))
    res.choice = min(candidates, key=lambda c: (res.times_ms[c], candidates.index(c)))
    first = candidates[0]
    if res.times_ms[res.choice] > res.times_ms[first] * (1.0 - margin):
        res.choice = first
    return res


class ParticleSnapshot:
    """Copies of the particle dats [0, size) and the move's outputs, restored before each trial."""

    def __init__(self, sim):
        self.sim = sim
        p = sim.parts
        n = p.size
        self.saved = {name: getattr(p, name)[:, :n].clone() for name, _, _ in p.DATS}

    def restore(self) -> None:
        p = self.sim.parts
        for name, t in self.saved.items():
            getattr(p, name)[:, :t.shape[1]].copy_(t)
        self.sim.zero_node_charge()


def snapshot_fits(sim, headroom: float = 1.25) -> bool:
    """Whether a ParticleSnapshot of sim (a copy of every particle dat over [0, size)) fits in
    the device's free memory with some headroom."""
    p = sim.parts
    nbytes = sum(getattr(p, name)[:, :p.size].numel() * getattr(p, name).element_size() for name, _, _ in p.DATS)
    free, _ = torch.cuda.mem_get_info(sim.device)
    return nbytes * headroom <= free


def _timed(fn) -> float:
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _tune_walk(sim, cands, apply, current, reps: int, with_push: bool | None) -> TuneResult:
    """Times each candidate of the move + deposit launch on sim's current state, pushed as a step
    pushes it: with the push as its prologue when with_push (default: when sim fuses the push),
    else the move launch alone after an untimed push.  apply(c) sets candidate c's tuning;
    current(t) reads a tuning's choice.  Sets the fastest; sim's state is left as found.  When
    the state's snapshot does not fit in device memory, nothing is timed and the current choice
    (or the first candidate) is kept."""
    before = L.Tuning()
    L.load().oppb_get_tuning(C.byref(before))
    if not snapshot_fits(sim):
        cur = current(before)
        return TuneResult(choice=cur if cur in cands else cands[0])
    snap = ParticleSnapshot(sim)
    fused = sim.fused_push if with_push is None else with_push

    def run(c) -> float:
        apply(c)
        snap.restore()
        if fused:
            return _timed(sim.push_move)
        sim.push()
        return _timed(sim.move)

    try:
        res = pick(cands, run, reps, margin=MARGIN)
    except Exception:
        L.load().oppb_set_tuning(C.byref(before))
        raise
    finally:
        snap.restore()
    apply(res.choice)
    return res


def tune_move(sim, candidates=None, reps: int = 3, with_push: bool | None = None) -> TuneResult:
    """Deposit strategy x node-sum copies for sim's move + deposit launch."""
    return _tune_walk(sim, candidates or MOVE_CANDIDATES, lambda c: L.set_tuning(deposit=c[0], replicas=c[1]),
                      lambda t: (t.deposit, t.replicas), reps, with_push)


def tune_lanes(sim, candidates=None, reps: int = 3, with_push: bool | None = None) -> TuneResult:
    """Lanes per particle, compiled occupancy, record staging and FP32 walk of the FP64 move +
    deposit launch (the mixed kernel has one lane per particle: nothing to tune there), with the
    deposit choice in force."""
    if sim.precision != "f64":
        return TuneResult(choice=(1, 8, 0, 0))
    return _tune_walk(sim, candidates or LANE_CANDIDATES,
                      lambda c: L.set_tuning(move_lanes=c[0], move_occupancy=c[1], move_stage=c[2], move_walk32=c[3]),
                      lambda t: (t.move_lanes, t.move_occupancy, t.move_stage, t.move_walk32), reps, with_push)


def block_shape_applies(t: L.Tuning, precision: str) -> bool:
    """Whether oppb_tuning.move_block shapes the launch: the one-lane kernels with the
    warp-grouped deposit (the CTA table is sized for 256 threads, the exact deposit, the
    lane-pair, staged and FP32-walk kernels run 256)."""
    if t.deposit != L.DEPOSIT_WARP_ATOMIC:
        return False
    return precision != "f64" or (t.move_lanes in (0, 1) and t.move_stage == 0 and t.move_walk32 == 0)


def tune_block(sim, candidates=None, reps: int = 3, with_push: bool | None = None) -> TuneResult:
    """Threads per CTA of the one-lane move + deposit launch (2048 / block CTAs per SM, 32
    registers a thread either way), with the deposit and lane choices in force; nothing is timed
    when those choices do not use the one-lane warp-deposit kernel."""
    t = L.Tuning()
    L.load().oppb_get_tuning(C.byref(t))
    if not block_shape_applies(t, sim.precision):
        return TuneResult(choice=t.move_block or 256)
    return _tune_walk(sim, candidates or BLOCK_CANDIDATES, lambda c: L.set_tuning(move_block=c),
                      lambda t: t.move_block, reps, with_push)


class StateSnapshot:
    """The whole particle state of a FemPIC sim (count, iteration, dats over [0, size), the
    buffer roles), restored before each trial of a multi-step measurement."""

    def __init__(self, sim):
        self.sim = sim
        p = sim.parts
        self.size, self.iter, self.period = p.size, sim.iter, sim.fill_period
        self.bufs = sim._bufs()
        self.saved = {name: getattr(p, name)[:, :p.size].clone() for name, _, _ in p.DATS}

    def restore(self) -> None:
        sim, p = self.sim, self.sim.parts
        sim._set_bufs(self.bufs)
        for name, t in self.saved.items():
            getattr(p, name)[:, :t.shape[1]].copy_(t)
        p.size, sim.iter, sim.fill_period = self.size, self.iter, self.period
        sim._count_synced = False
        sim.zero_node_charge()


def state_snapshot_fits(sim, steps: int, headroom: float = 1.25) -> bool:
    """Whether a StateSnapshot fits, and the state can grow by `steps` injections within capacity."""
    p = sim.parts
    return snapshot_fits(sim, headroom) and p.size + steps * sim.inject_per_step <= p.capacity


def tune_sort_period(sim, tables, candidates=None) -> TuneResult:
    """Cost of a Sort_Periodic cycle per particle-step for each candidate period P: from a
    snapshot of the state, P steps (hole fills, then the cell sort on the cycle's last step),
    timed over the move + compaction launches as the bench times its steps; tables: device
    injection tables, used in turn.  times_ms holds nanoseconds per particle-step (the
    comparison the choice is made on).  The period is reported, not set: sim.fill_period and
    the state are left as found."""
    cands = candidates or PERIOD_CANDIDATES
    if not sim.fill.startswith("Sort") or not state_snapshot_fits(sim, max(cands)):
        return TuneResult(choice=sim.fill_period)
    snap = StateSnapshot(sim)
    s = torch.cuda.current_stream()

    def run(period) -> float:
        snap.restore()
        sim.fill_period = period
        sim.iter = period * (1 + sim.iter // period) - period + 1  # the cycle ends with the sort step
        ps, t = 0, 0.0
        for k in range(period):
            sim.inject(tables[k % len(tables)])
            sim.zero_node_charge()
            n = sim.parts.size
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(s)
            sim.push_move() if sim.fused_push else (sim.push(), sim.move())
            e[1].record(s)
            st = sim.parts.status_host()
            if st.error:
                raise L.OppbError("move", st.error)
            e[2].record(s)
            sim.finalize(st.remove_count)
            e[3].record(s)
            e[3].synchronize()
            sim.iter += 1
            ps += n
            t += e[0].elapsed_time(e[1]) + e[2].elapsed_time(e[3])
        return 1e6 * t / ps  # ns per particle-step

    try:
        res = pick(cands, run, reps=1)
    finally:
        snap.restore()
    return res


def time_move(sim, deposit: int, replicas: int = 1, reps: int = 3, with_push: bool | None = None) -> float:
    """Median milliseconds of sim's move + deposit launch with the given deposit strategy, timed as
    tune_move times its candidates (NaN when the state's snapshot does not fit in device memory);
    the tuning and sim's state are left as found."""
    before = L.Tuning()
    L.load().oppb_get_tuning(C.byref(before))
    try:
        return tune_move(sim, [(deposit, replicas)], reps, with_push).times_ms.get((deposit, replicas), float("nan"))
    finally:
        L.load().oppb_set_tuning(C.byref(before))


def tune_sort(sim, candidates=None, reps: int = 3) -> TuneResult:
    """Columns per launch and form (gather by destination, or scatter by source) of the cell
    sort's dat move, timed on sim's current (unsorted) state; the sort writes into the swap
    buffers only, so the state is not changed."""
    p = sim.parts
    lib = sim.lib
    nbytes = lib.oppb_sort_workspace_bytes(p.size, sim.mesh.n_cells)
    ws = sim._workspace(nbytes)
    dats = p.dat_list()

    def run(c) -> float:
        L.set_tuning(sort_gather_cols=c[0], sort_scatter=c[1])
        return _timed(lambda: L.check("oppb_sort_by_cell", lib.oppb_sort_by_cell(
            p.size, sim.mesh.n_cells, p.capacity, len(p.DATS), dats, 3, None, ws.data_ptr(), ws.numel(), None)))

    res = pick(candidates or SORT_CANDIDATES, run, reps)
    L.set_tuning(sort_gather_cols=res.choice[0], sort_scatter=res.choice[1])
    return res
