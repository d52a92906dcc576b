#!/usr/bin/env python3
"""FemPIC particle hot path benchmark (move + deposit, with the removal compaction and
periodic cell sort) on the electrostatic tet-mesh workload:

  box 1 x 1 x 4 cut into 48 x 48 x 192 hexahedra x 6 tets = 2,654,208 cells, 463,393 nodes;
  250,000 ions injected per step through the z=0 face (drift 1.0 along +z, Maxwellian
  sigma 0.1), dt 0.01, unit charge/mass, static FEM field; particles removed on leaving
  the box; opp_fill = Sort_Periodic with period 10; 300 fill steps to reach the steady
  state (~5e7 particles), then W warm-up and K timed steps.

Both precisions run on the same seeded inputs: plain FP64 (bit-identical to the seq
backend) and mixed (FP32 push and barycentric tests, FP64 re-check in |lambda| < 1e-5,
FP64 node totals).  value = mixed particle-steps/s = sum N_alive(start of move) /
sum t(move+deposit+compaction), device time (CUDA events), summed over ranks ÷ max-rank
time.  Particle dats (~4 GB) exceed L2, so no flush is needed between steps.

--impl reference times the reference's own CPU implementation of the same path (the
compiled OP-PIC omp/seq backend when oracle/_ref holds it, else the C oracle) on a
bounded sample of the workload, on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT / "op-pic_b200", ROOT):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "particle-steps/s (move+deposit) mixed vs plain FP64 on 1 B200; % HBM roofline"
UNIT = "particle-steps/s"
CFG = dict(nx=48, ny=48, nz=192, lx=1.0, ly=1.0, lz=4.0, inject=250_000, sigma=0.1, dt=0.01, qm=1.0,
           v_ion=1.0, fill="Sort_Periodic", period=10, fill_steps=300, seed=0, capacity=90_000_000)
WORKLOAD = ("FemPIC electrostatic tet-mesh PIC, 48x48x192 hexes x 6 = 2,654,208 tets, 463,393 nodes; "
            "250,000 ions/step; steady state after 300 fill steps; Sort_Periodic period 10")
# Algorithmic bytes per move+deposit launch: per particle read pos 24 + p2c 4, write p2c 4 + p_lc 32;
# per cell the record read once (FP64: det 128 + nav {coef, c2c, pad} 32 + c2n 16; mixed: the
# 64-B f32 record {3 lambda rows, origin} + c2c 16 + c2n 16); per node one FP64 read-modify-write.
BYTES_PER_PARTICLE = 64
BYTES_PER_CELL = {"f64": 168, "mixed": 96}
BYTES_PER_NODE = 16
# DRAM bytes per particle of one move+deposit launch (dram__bytes_read.sum + dram__bytes_write.sum),
# from an ncu capture of full-size launches of this workload: profiles/move_mixed_kernel_fempic_48x48x192.txt
# and profiles/move_f64_kernel_fempic_48x48x192.txt.
MEASURED_DRAM_BYTES_PER_PARTICLE = {"f64": 73.0, "mixed": 70.0}
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum of full-size launches, per particle x particles"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- our arm

def mixed_vs_f64(sim, charges: bool = False):
    """One move + deposit of the mixed kernel and one of the FP64 kernel from the same pushed
    particle state (the steady state after the timed steps, pushed once and restored between
    the two): cells, lambdas and node charges of the mixed form against the FP64 form.  The
    state the timed steps left is put back afterwards.  charges: also return the two node-charge
    vectors."""
    import ctypes as C

    import torch

    from oppb import _lib as L
    from oppb.autotune import ParticleSnapshot

    before = ParticleSnapshot(sim)
    sim.push()  # the walks of a step: both moves start from the same pushed state
    snap = ParticleSnapshot(sim)
    p, n = sim.parts, sim.parts.size
    out = {}
    for name in ("mixed", "f64"):
        snap.restore()
        if name == "mixed":
            sim.move()
        else:
            v, ws = p.view(), sim._deposit_ws()
            L.check("oppb_move_deposit_f64", sim.lib.oppb_move_deposit_f64(
                C.byref(sim.mesh.s), C.byref(v), sim.node_charge.data_ptr(), p.status.data_ptr(), sim.max_hops,
                ws.data_ptr(), ws.numel(), None))
        torch.cuda.synchronize()
        st = p.status_host()
        if st.error:
            raise L.OppbError(f"{name} move", st.error)
        out[name] = (p.p2c[0, :n].clone(), p.lc[:, :n].clone(), sim.node_charge.clone(), st.remove_count)
    before.restore()  # the state the timed steps left, for the steps that follow
    (c_m, l_m, q_m, r_m), (c_f, l_f, q_f, r_f) = out["mixed"], out["f64"]
    kept = c_f != L.REMOVED_CELL
    dq = (q_m - q_f).abs()
    big = q_f.abs() >= 1.0
    rep = {"what": "one mixed and one FP64 move + deposit from the same pushed steady state",
            "particles": n, "cells_differing": int((c_m != c_f).sum()), "removed": [int(r_m), int(r_f)],
            "lambda_max_abs_diff": float((l_m - l_f)[:, kept].abs().max()),
            "node_charge_normwise_rel": float(dq.max() / q_f.abs().max()),
            "node_charge_max_err_over_max_q_or_1": float((dq / q_f.abs().clamp(min=1.0)).max()),
            "node_charge_mean_rel_where_q_ge_1": float((dq[big] / q_f.abs()[big]).mean()),
            "node_charge_max_abs": float(q_f.abs().max())}
    return (rep, q_m, q_f) if charges else rep


HBM_SPEC_GBS = 8000.0  # B200 HBM3e data-sheet bandwidth (DGX figure), for context beside the measured copy peak


def run_precision(hm, dev, precision: str, steps: int, warmup: int, seed: int, sampler=None,
                  e2e_steps: int = 0, cpu_sample: bool = False) -> dict:
    import numpy as np
    import torch
    import torch.distributed as dist

    from oppb import _lib as L
    from oppb.fempic import FemPIC, injection_randoms

    sim = FemPIC(hm, dev, inject_per_step=CFG["inject"], ion_velocity=CFG["v_ion"], qm=CFG["qm"], dt=CFG["dt"],
                 precision=precision, fill=CFG["fill"], fill_period=CFG["period"], capacity=CFG["capacity"])
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rnd_buf = torch.empty((5, CFG["inject"]), dtype=torch.float64, device=dev)

    def device_randoms(out):
        out[0:2].uniform_(0.0, 1.0, generator=gen)
        out[2:5].normal_(0.0, CFG["sigma"], generator=gen)
        return out

    t0 = time.time()
    for _ in range(CFG["fill_steps"]):
        sim.step(device_randoms(rnd_buf))
    torch.cuda.synchronize()
    log(f"[{precision}] fill {CFG['fill_steps']} steps in {time.time() - t0:.1f}s, size {sim.parts.size}")
    for _ in range(warmup):
        sim.step(device_randoms(rnd_buf))
    # Launch choices (FP64 move lanes per particle, occupancy and record staging, deposit
    # strategy, node-sum copies, block shape, the sort's dat move) timed on this state before
    # the timed steps; the state is restored after each trial.  The sort interval's trials
    # (whole sort cycles) are reported; the timed steps keep the workload's period.
    from oppb.autotune import tune_block, tune_lanes, tune_move, tune_sort, tune_sort_period
    tuned = {"lanes": tune_lanes(sim, with_push=False).report(), "move": tune_move(sim, with_push=False).report()}
    tuned["block"] = tune_block(sim, with_push=False).report()
    tuned["sort"] = tune_sort(sim).report()
    period_tables = [device_randoms(torch.empty_like(rnd_buf)) for _ in range(4)]
    sp = tune_sort_period(sim, period_tables)
    tuned["sort_interval"] = {"ns_per_particle_step": {str(k): v for k, v in sp.times_ms.items()},
                              "best": sp.choice, "used": CFG["period"]}
    del period_tables
    # The deterministic deposit (integer fixed-point node sums) on the same state, for the record.
    from oppb.autotune import time_move
    t_exact = time_move(sim, L.DEPOSIT_EXACT, with_push=False)
    tuned["deterministic_deposit_ms"] = t_exact if t_exact == t_exact else None  # NaN: not measured
    log(f"[{precision}] autotune lanes {tuned['lanes']['choice']} move {tuned['move']['choice']} "
        f"block {tuned['block']['choice']} "
        f"sort cols {tuned['sort']['choice']} sort interval {tuned['sort_interval']}")
    # Inputs of the timed steps generated before timing (device-resident).
    tables = [device_randoms(torch.empty_like(rnd_buf)) for _ in range(min(steps, 16))]
    torch.cuda.synchronize()

    s = torch.cuda.current_stream()
    E = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rec = []
    lib = L.load()
    launches0 = lib.oppb_kernel_launches()
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    if dist.is_initialized():  # every rank enters the timed steps together
        dist.barrier()
        torch.cuda.synchronize()
    # Profiler range = the timed steps (for `ncu --profile-from-start off`); no effect otherwise.
    torch.cuda.profiler.start()
    ev_all0, ev_all1 = E(), E()
    ev_all0.record(s)
    for k in range(steps):
        ev = [E() for _ in range(5)]
        sim.inject(tables[k % len(tables)])
        sim.zero_node_charge()
        ev[4].record(s)
        sim.push()
        n_alive = sim.parts.size
        ev[0].record(s)
        sim.move()
        ev[1].record(s)
        st = sim.parts.status_host()
        if st.error:
            raise L.OppbError("move", st.error)
        ev[2].record(s)
        kind = sim.finalize(st.remove_count)
        ev[3].record(s)
        sim.iter += 1
        rec.append((n_alive, ev, kind, st.total_visits, st.recheck_count, st.remove_count))
    ev_all1.record(s)
    torch.cuda.synchronize()
    if dist.is_initialized():
        dist.barrier()
    torch.cuda.profiler.stop()
    clocks = sampler.stop() if sampler else None
    launches = lib.oppb_kernel_launches() - launches0
    total_ms = ev_all0.elapsed_time(ev_all1)
    t_move = [r[1][0].elapsed_time(r[1][1]) for r in rec]
    t_comp = [r[1][2].elapsed_time(r[1][3]) for r in rec]
    t_push = [r[1][4].elapsed_time(r[1][0]) for r in rec]
    n = [r[0] for r in rec]
    ps = sum(n)
    out = {
        "precision": precision,
        "particle_steps": ps,
        "t_move_ms": sum(t_move),
        "t_compact_ms": sum(t_comp),
        "value": ps / ((sum(t_move) + sum(t_comp)) / 1e3),
        "move_only": ps / (sum(t_move) / 1e3),
        "whole_step": ps / (total_ms / 1e3),
        "ms_per_step": total_ms / steps,
        "mean_particles": ps / steps,
        "visits_per_particle": sum(int(r[3]) for r in rec) / ps,
        "recheck_frac": sum(r[4] for r in rec) / max(1, sum(int(r[3]) for r in rec)),
        "removed_per_step": sum(r[5] for r in rec) / steps,
        "sorts": sum(1 for r in rec if r[2] == "sort"),
        "launches": int(launches),
        "clocks": clocks,
        "autotune": tuned,
    }
    if precision == "mixed":
        out["vs_f64"] = mixed_vs_f64(sim)
    # Roofline of the move(+deposit) kernel: algorithmic bytes / mean launch time.
    bytes_per_launch = [BYTES_PER_PARTICLE * r[0] + BYTES_PER_CELL[precision] * hm.n_cells
                        + BYTES_PER_NODE * hm.n_nodes for r in rec]
    out["move_gbs"] = sum(bytes_per_launch) / (sum(t_move) / 1e3) / 1e9
    out["move_bytes_per_launch"] = sum(bytes_per_launch) / steps
    out["move_ms_per_launch"] = sum(t_move) / steps
    # Move time against the steps since the last cell sort (0 = the first move after a sort):
    # particles leave their sorted neighbours as they hop, so a warp's lanes spread over more
    # cells until the next sort.
    by_phase, phase = {}, None
    for r, t in zip(rec, t_move):
        if phase is not None:
            by_phase.setdefault(phase, []).append(t)
            phase += 1
        if r[2] == "sort":
            phase = 0
    out["move_ms_since_sort"] = {str(k): sum(v) / len(v) for k, v in sorted(by_phase.items())}
    out["push_ms_per_launch"] = sum(t_push) / steps
    out["push_inclusive"] = ps / ((sum(t_push) + sum(t_move) + sum(t_comp)) / 1e3)

    # The push fused into the move kernel as its prologue (one launch per step): push +
    # move + deposit + compaction, device time, on the following steps.
    n_fused = min(steps, 20)
    ps_f, t_f = 0, 0.0
    for k in range(n_fused):
        ev = [E() for _ in range(4)]
        sim.inject(tables[k % len(tables)])
        sim.zero_node_charge()
        n_alive = sim.parts.size
        ev[0].record(s)
        sim.push_move()
        ev[1].record(s)
        st = sim.parts.status_host()
        if st.error:
            raise L.OppbError("push_move", st.error)
        ev[2].record(s)
        sim.finalize(st.remove_count)
        ev[3].record(s)
        sim.iter += 1
        torch.cuda.synchronize()
        ps_f += n_alive
        t_f += ev[0].elapsed_time(ev[1]) + ev[2].elapsed_time(ev[3])
    out["push_inclusive_fused"] = ps_f / (t_f / 1e3)
    out["fused_steps"] = n_fused

    # Whole steps replayed from CUDA graphs (include/oppb_graph.h): one graph = one sort cycle
    # of steps (inject, push + move + deposit, hole fill / sort, step record), the particle
    # count kept on the device; one readback of the count and the records per replay.  The
    # tables are refilled between replays, outside the timed replay.
    G = CFG["period"]
    reps = max(2, min(steps, 40) // G)
    g = sim.graph_for(G)
    for t in g.tables:
        device_randoms(t)
    sim.replay(g)  # the first replay of each buffer parity (a sort swaps the buffers) is untimed
    g = sim.graph_for(G)
    for t in g.tables:
        device_randoms(t)
    sim.replay(g)
    ps_g, t_g, l_g = 0, 0.0, 0
    for _ in range(reps):
        g = sim.graph_for(G)
        for t in g.tables:
            device_randoms(t)
        e0, e1 = E(), E()
        torch.cuda.profiler.start()  # profiler range: the replays (for `ncu --profile-from-start off`)
        e0.record(s)
        g.graph.replay()
        e1.record(s)
        torch.cuda.profiler.stop()
        recs = sim.replay_finish(g)
        ps_g += sum(r["size_before_move"] for r in recs)
        t_g += e0.elapsed_time(e1)
        l_g += g.launches
    out["graph_step"] = {"value": ps_g / (t_g / 1e3), "unit": UNIT, "ms_per_step": t_g / (reps * G),
                         "steps_per_graph": G, "replays": reps, "launches_per_replay": g.launches,
                         "gpu_launches": l_g, "captured_graphs": len(sim._graphs),
                         "what": "whole steps (inject, push + move + deposit, hole fill / cell sort) replayed "
                                 "from one CUDA graph per sort cycle, particle count on the device, device time"}

    if e2e_steps:
        # End to end through the public API (FemPIC.run_steps): every step's injection table
        # goes up from pinned host memory and its node charges (plus the move status) come
        # back; the copies run on a second stream and overlap the neighbouring steps.  The
        # same steps through FemPIC.run_graph_host (graph replays of one sort cycle, the count
        # read back once a replay) are reported beside it.
        host_tables = [torch.from_numpy(np.ascontiguousarray(injection_randoms(seed + 7, k, CFG["inject"],
                                                                                CFG["sigma"]).T)).pin_memory()
                       for k in range(e2e_steps)]
        charges_out = [torch.empty(hm.n_nodes, dtype=torch.float64).pin_memory() for _ in range(e2e_steps)]

        def timed(call) -> tuple[float, list]:
            torch.cuda.synchronize()
            e0, e1 = E(), E()
            e0.record(s)
            recs = call(host_tables, charges_out)
            e1.record(s)
            e1.synchronize()
            return e0.elapsed_time(e1), recs

        for _ in range(max(1, warmup)):  # untimed warm-up calls of the same API, 3 steps each
            sim.run_steps(host_tables[:3], charges_out[:3])
        t_e2e, recs = timed(sim.run_steps)
        # The graph path's warm-up captures its graphs for both buffer parities of a sort cycle.
        per = CFG["period"]
        k = 2 * per if e2e_steps >= 2 * per else e2e_steps
        sim.run_graph_host(host_tables[:k], charges_out[:k])
        t_graph, recs_graph = timed(sim.run_graph_host)
        n_e2e = sum(r["size_before_move"] for r in recs)
        n_graph = sum(r["size_before_move"] for r in recs_graph)
        out["e2e"] = {"value": n_e2e / (t_e2e / 1e3), "unit": UNIT,
                      "h2d_bytes_per_step": int(host_tables[0].numel() * 8),
                      "d2h_bytes_per_step": int(charges_out[0].numel() * 8 + 32), "steps": e2e_steps,
                      "what": "whole step (inject, push + move + deposit, compaction) through FemPIC.run_steps",
                      "graph_replays": {"value": n_graph / (t_graph / 1e3), "unit": UNIT,
                                        "what": "the same steps through FemPIC.run_graph_host: replays of one sort "
                                                "cycle, the count and step records read back once a replay"}}

    if cpu_sample:
        # One more step up to the push, then a contiguous slice of the particles as the
        # CPU sample (positions after the push, cells before the move).
        sim.inject(tables[0])
        sim.zero_node_charge()
        sim.push()
        m = sim.parts.size
        k = min(m, 1_000_000)
        a = (m - k) // 2
        out["cpu_sample_state"] = {
            "pos": sim.parts.pos[:, a:a + k].T.contiguous().cpu().numpy(),
            "p2c": sim.parts.p2c[0, a:a + k].contiguous().cpu().numpy(),
        }
    del sim
    torch.cuda.empty_cache()
    return out


def cpu_baseline_port(hm, sample: dict, budget_s: float = 8.0) -> dict:
    """The C oracle (single thread) on the sampled particles: move + deposit, repeated."""
    import numpy as np

    from oracle import oracle as O

    pos, p2c0 = sample["pos"], sample["p2c"]
    n = len(p2c0)
    ps, t = 0, 0.0
    while t < budget_s:
        p2c = p2c0.copy()
        lc = np.zeros((n, 4))
        q = np.zeros(hm.n_nodes)
        t0 = time.perf_counter()
        O.move(pos, lc, p2c, hm.c2c, hm.c_vol, hm.c_det, n=n)
        keep = p2c != O.REMOVED
        O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c[keep]), hm.c2n, q)
        t += time.perf_counter() - t0
        ps += n
    return {"value": ps / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} steady-state particles (contiguous slice after the push), FP64 move + deposit, "
                      f"C oracle single thread, {ps // n} repetitions"}


def replica_sum(v: float, dev) -> float:
    """Sum of v over the ranks of the default process group (v itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_job_value(particle_steps: float, seconds: float, ms_per_step: float, dev) -> tuple[float, float]:
    """Whole-job throughput of independent replicas, one per rank: the particle-steps of all
    ranks over the slowest rank's time (the max over ranks), and that rank's ms per step."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return particle_steps / seconds, ms_per_step
    ps = torch.tensor([particle_steps], dtype=torch.float64, device=dev)
    tm = torch.tensor([seconds, ms_per_step], dtype=torch.float64, device=dev)
    dist.all_reduce(ps, op=dist.ReduceOp.SUM)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    return float(ps.item()) / float(tm[0].item()), float(tm[1].item())


def arm_ours(args) -> dict:
    import torch
    import torch.distributed as dist

    from oppb.fempic import HostMesh

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    t0 = time.time()
    hm = HostMesh(CFG["nx"], CFG["ny"], CFG["nz"], CFG["lx"], CFG["ly"], CFG["lz"])
    log(f"mesh {hm.n_cells} cells built in {time.time() - t0:.1f}s (CG iters {hm.cg_iters})")
    seed = CFG["seed"] + 1000 * rank  # independent replicas per rank
    if world > 1:
        dist.barrier()
    f64 = mixed = None
    if args.precision in ("both", "f64"):
        f64 = run_precision(hm, dev, "f64", args.steps, args.warmup, seed,
                            cpu_sample=(rank == 0 and args.cpu_baseline),
                            sampler=ClockSampler(local) if args.precision == "f64" else None)
    if world > 1:
        dist.barrier()
    if args.precision in ("both", "mixed"):
        mixed = run_precision(hm, dev, "mixed", args.steps, args.warmup, seed, sampler=ClockSampler(local),
                              e2e_steps=args.e2e_steps)
    if f64 is None or mixed is None:  # single-precision profiling runs: a short line, no ratio
        r = f64 or mixed
        if rank == 0:
            print(json.dumps({"precision": r["precision"], "value": r["value"], "move_only": r["move_only"],
                              "move_ms_per_launch": r["move_ms_per_launch"], "move_gbs": r["move_gbs"],
                              "mean_particles": r["mean_particles"], "visits_per_particle": r["visits_per_particle"],
                              "clocks": r["clocks"], "autotune": r["autotune"],
                              "move_ms_since_sort": r["move_ms_since_sort"], "vs_f64": r.get("vs_f64")}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return {}

    res = {}
    for r in (f64, mixed):
        t = (r["t_move_ms"] + r["t_compact_ms"]) / 1e3
        r["job_value"], r["job_ms_per_step"] = replica_job_value(r["particle_steps"], t, r["ms_per_step"], dev)
    if "e2e" in mixed:
        e = mixed["e2e"]
        e["value"] = replica_sum(e["value"], dev)
    res["f64"], res["mixed"] = f64, mixed
    advec = None
    if args.advec:  # the ensemble is split over the ranks (before the process group goes)
        if world > 1:
            dist.barrier()
        advec = run_advec(dev, min(args.steps, 20), args.warmup, args.cpu_baseline, rank, world)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return {}
    peaks = measured_peaks()
    line = {
        "metric": METRIC,
        "value": mixed["job_value"],
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mixed["job_ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic",
        "config": workload_config(),
        "parallelism": f"replicas x{world}",
        "mean_particles": round(mixed["mean_particles"]),
        "plain_fp64": {"value": f64["job_value"], "move_only": f64["move_only"], "whole_step": f64["whole_step"],
                       "ms_per_step": f64["ms_per_step"], "move_ms_per_launch": f64["move_ms_per_launch"],
                       "move_gbs": f64["move_gbs"], "frac_of_hbm": f64["move_gbs"] / peaks["hbm_gbs"],
                       "visits_per_particle": f64["visits_per_particle"], "mean_particles": f64["mean_particles"],
                       "move_ms_since_sort": f64["move_ms_since_sort"]},
        "mixed": {"value": mixed["job_value"], "move_only": mixed["move_only"], "whole_step": mixed["whole_step"],
                  "move_ms_per_launch": mixed["move_ms_per_launch"], "recheck_frac": mixed["recheck_frac"],
                  "visits_per_particle": mixed["visits_per_particle"],
                  "move_ms_since_sort": mixed["move_ms_since_sort"], "vs_f64": mixed["vs_f64"]},
        "push_inclusive": {"unit": UNIT, "what": "push + move + deposit + compaction, device time",
                           "mixed_unfused": mixed["push_inclusive"], "mixed_fused": mixed["push_inclusive_fused"],
                           "f64_unfused": f64["push_inclusive"], "f64_fused": f64["push_inclusive_fused"],
                           "fused_steps": mixed["fused_steps"]},
        "graph_step": {"mixed": mixed["graph_step"], "f64": f64["graph_step"]},
        "mixed_over_plain": mixed["job_value"] / f64["job_value"],
        "autotune": {"what": "move launch (FP64 lanes per particle, occupancy and record staging; deposit "
                             "strategy and node-sum copies; block shape) and the sort's dat move (columns per "
                             "launch, gather or scatter), median of 3 timed trials on the warmed-up state; "
                             "sort interval: one timed sort cycle per candidate period from the same state",
                     "f64": f64["autotune"], "mixed": mixed["autotune"]},
        "roofline": {"bound": "hbm", "kernel": "move_mixed_kernel (move + fused deposit)",
                     "achieved": mixed["move_gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": mixed["move_gbs"] / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "frac_of_spec": mixed["move_gbs"] / HBM_SPEC_GBS, "spec_gbs": HBM_SPEC_GBS,
                     "bytes_per_launch": mixed["move_bytes_per_launch"],
                     "traffic": MEASURED_DRAM_BYTES_PER_PARTICLE["mixed"] * mixed["mean_particles"],
                     "traffic_source": TRAFFIC_SOURCE},
        "gpu_launches": mixed["launches"],
        "clocks": mixed["clocks"],
    }
    if "e2e" in mixed:
        line["e2e"] = mixed["e2e"]
    if args.cpu_baseline and "cpu_sample_state" in f64:
        line["cpu_baseline"] = cpu_baseline_port(hm, f64["cpu_sample_state"], args.cpu_seconds)
    if args.field and world == 1:
        line["field_phase"] = run_field_phase(hm, dev, min(args.steps, 20), args.warmup, seed, args.cpu_baseline)
    if args.dh and world == 1:
        line["direct_hop"] = run_direct_hop(hm, dev, min(args.steps, 20), args.warmup, seed, args.cpu_baseline)
    if args.cabana and world == 1:
        line["cabanapic"] = run_cabana(dev, min(args.steps, 20), args.warmup, args.cpu_baseline, args.cpu_seconds)
        line["gpu_launches_cabanapic"] = line["cabanapic"]["gpu_launches"]
    if advec is not None:
        line["advec_ensemble"] = advec
    return line


# ------------------------------------------------------------ direct-hop (global move)

DH_SPACING = 1.0 / 48  # one grid box per hexahedron of the 48x48x192 mesh


def run_direct_hop(hm, dev, steps: int, warmup: int, seed: int, cpu: bool) -> dict:
    """The global move (direct-hop seed, include/oppb_dh.h) on the bench workload: the GPU
    build of the structured map over the 2,654,208 cells, then the mixed step with every walk
    started from the grid's cell: push + move + deposit + compaction per step, device time,
    after the same 300-step fill.  cpu: the reference's map search (all cells per query)
    timed by the oracle on sampled boxes and scaled to the grid."""
    import numpy as np
    import torch

    from oppb import _lib as L
    from oppb.fempic import DirectHopGrid, FemPIC

    sim = FemPIC(hm, dev, inject_per_step=CFG["inject"], ion_velocity=CFG["v_ion"], qm=CFG["qm"], dt=CFG["dt"],
                 precision="mixed", fill=CFG["fill"], fill_period=CFG["period"], capacity=CFG["capacity"])
    builds = []
    for _ in range(3):  # the first build pays the module's first launches
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        grid = DirectHopGrid(hm, sim.mesh, DH_SPACING)
        builds.append(time.perf_counter() - t0)
    sim.dh = grid
    gmap = grid.map.cpu().numpy()
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rnd = torch.empty((5, CFG["inject"]), dtype=torch.float64, device=dev)

    def device_randoms(out):
        out[0:2].uniform_(0.0, 1.0, generator=gen)
        out[2:5].normal_(0.0, CFG["sigma"], generator=gen)
        return out

    for _ in range(CFG["fill_steps"] + warmup):
        sim.step(device_randoms(rnd))
    tables = [device_randoms(torch.empty_like(rnd)) for _ in range(min(steps, 16))]
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    E = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ps, t_ms, visits = 0, 0.0, 0
    l0 = L.load().oppb_kernel_launches()
    for k in range(steps):
        ev = [E() for _ in range(4)]
        sim.inject(tables[k % len(tables)])
        sim.zero_node_charge()
        n_alive = sim.parts.size
        ev[0].record(s)
        sim.push_move()
        ev[1].record(s)
        st = sim.parts.status_host()
        if st.error:
            raise L.OppbError("push_move (direct hop)", st.error)
        ev[2].record(s)
        sim.finalize(st.remove_count)
        ev[3].record(s)
        sim.iter += 1
        torch.cuda.synchronize()
        ps += n_alive
        visits += int(st.total_visits)
        t_ms += ev[0].elapsed_time(ev[1]) + ev[2].elapsed_time(ev[3])
    launches = L.load().oppb_kernel_launches() - l0
    out = {"what": "mixed push + move + deposit + compaction with the global move on (every walk starts from "
                   "the structured grid's cell), device time; grid spacing = hex size",
           "unit": UNIT, "value": ps / (t_ms / 1e3), "steps": steps, "mean_particles": ps / steps,
           "visits_per_particle": visits / ps, "gpu_launches": int(launches),
           "grid": {"spacing": DH_SPACING, "dims": list(grid.dims), "boxes": grid.size,
                    "boxes_with_cell": int((gmap != L.REMOVED_CELL).sum()),
                    "build_s": min(builds[1:]), "first_build_s": builds[0],
                    "build_what": "host bounding box + box counts, node upload, GPU binning and query "
                                  "(one stream sync to size the workspace)"}}
    del sim, grid
    torch.cuda.empty_cache()
    if cpu:
        from oracle import oracle as O

        dh = O.DirectHop(hm.n_pos, DH_SPACING, (4 * DH_SPACING,) * 3)
        rng = np.random.default_rng(seed)
        inside = np.flatnonzero(gmap != L.REMOVED_CELL)
        outside = np.flatnonzero(gmap == L.REMOVED_CELL)
        k_in, k_out = 24, 4
        t0 = time.perf_counter()
        dh.boxes(hm, rng.choice(inside, k_in, replace=False))
        t_in = (time.perf_counter() - t0) / k_in
        t0 = time.perf_counter()
        dh.boxes(hm, rng.choice(outside, k_out, replace=False))
        t_out = (time.perf_counter() - t0) / k_out
        est = t_in * len(inside) + t_out * len(outside)
        out["grid"]["cpu_baseline"] = {
            "value": est, "unit": "s (estimated map build)", "cores": 1, "kind": "port",
            "sample": f"C oracle (the reference's search over all cells per query) on {k_in} boxes with a cell and "
                      f"{k_out} without, scaled by the grid's {len(inside)} and {len(outside)} boxes"}
    return out


# ------------------------------------------------------------------ field phase

# Electron model of the field-phase leg in the workload's units: unit charge and permittivity,
# n0 = 1 and spwt so that the steady state's ion density (~5.7e7 particles in a volume of 4)
# is about n0, kTe = 100 so that exp((D - phi0) / kTe) stays O(1) while F1 accumulates over
# the timed steps (the reference never resets F1; over hundreds of steps D grows until the
# exponential overflows, so the leg fills with the set-up field and turns the phase on after).
FIELD = dict(n0=1.0, phi0=0.0, kte=100.0, qe=1.0, eps0=1.0, spwt=4.0 / 5.7e7)


def run_field_phase(hm, dev, steps: int, warmup: int, seed: int, cpu: bool) -> dict:
    """The mixed step with the field phase on (compute_node_charge_density, compute_phi's
    Newton step with the cooperative CG, compute_electric_field into the move's field, one
    CUDA graph per step), after the same 300-step fill with the set-up field: time of the
    field phase alone and of the whole step.  cpu: the oracle's compute_phi (C, one core) on
    the same state."""
    import numpy as np
    import torch

    from oppb import _lib as L
    from oppb.fempic import FemPIC
    from oppb.field import FieldConstants

    consts = FieldConstants(**{k: v for k, v in FIELD.items() if k != "spwt"})
    t0 = time.perf_counter()
    sim = FemPIC(hm, dev, inject_per_step=CFG["inject"], ion_velocity=CFG["v_ion"], qm=CFG["qm"], dt=CFG["dt"],
                 precision="mixed", fill=CFG["fill"], fill_period=CFG["period"], capacity=CFG["capacity"],
                 field=consts, spwt=FIELD["spwt"])
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    rnd = torch.empty((5, CFG["inject"]), dtype=torch.float64, device=dev)

    def device_randoms(out):
        out[0:2].uniform_(0.0, 1.0, generator=gen)
        out[2:5].normal_(0.0, CFG["sigma"], generator=gen)
        return out

    sim.field_enabled = False
    for _ in range(CFG["fill_steps"]):
        sim.step(device_randoms(rnd))
    sim.field_enabled = True
    for _ in range(warmup):
        sim.step(device_randoms(rnd))
    tables = [device_randoms(torch.empty_like(rnd)) for _ in range(min(steps, 16))]
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    E = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ps, t_step, t_field, iters, pmax = 0, 0.0, 0.0, [], 0.0
    l0 = L.load().oppb_kernel_launches()
    for k in range(steps):
        e0, e1 = E(), E()
        n_before = sim.parts.size
        e0.record(s)
        sim.step(tables[k % len(tables)])  # includes the field phase at its end
        e1.record(s)
        torch.cuda.synchronize()
        ps += n_before + CFG["inject"]
        t_step += e0.elapsed_time(e1)
        st = sim.field.status_host()
        if not st.converged:
            raise RuntimeError(f"field solve did not converge ({st.iterations} iterations)")
        iters.append(st.iterations)
        pmax = max(pmax, float(sim.field.potential.abs().max()))
    # The field phase alone, replayed on the last step's node charge (recovered from the
    # density the step left: charge = density * n_vol / spwt, to rounding); the Newton state
    # advances with each replay, as it would step to step.
    reps = 10
    charge = sim.node_charge * sim.n_vol / FIELD["spwt"]
    saved = (sim.field.d.clone(), sim.field.f1.clone(), charge)
    f0, f1 = E(), E()
    torch.cuda.synchronize()
    f0.record(s)
    for _ in range(reps):
        sim.node_charge.copy_(saved[2])
        sim.field_phase()
    f1.record(s)
    f1.synchronize()
    t_field = f0.elapsed_time(f1) / reps
    launches = L.load().oppb_kernel_launches() - l0
    out = {"what": "mixed step with the field phase (node charge density, Newton step of the Poisson-Boltzmann "
                   "potential with cooperative CG, cell field), device time; the field phase is one CUDA graph",
           "unit": UNIT, "whole_step_value": ps / (t_step / 1e3), "steps": steps,
           "field_ms": t_field, "field_what": "graph replay of the field phase on the last step's charge "
                                              "(node copy of 3.7 MB included)",
           "cg_iterations": {"mean": float(np.mean(iters)), "min": int(min(iters)), "max": int(max(iters))},
           "max_abs_potential": pmax, "visits_per_particle_last": sim.last["visits"] / max(1, sim.last["size_before_move"]),
           "nodes": hm.n_nodes, "unknowns": sim.field.neq, "nnz": sim.field.nnz, "setup_s": setup_s,
           "constants": FIELD, "gpu_launches": int(launches)}
    # The field from mixed node charges against the field from FP64 ones: both charge vectors
    # come from one move + deposit of each kernel on the same pushed state, and each field
    # phase starts from the same Newton state.
    rep, q_m, q_f = mixed_vs_f64(sim, charges=True)
    d0, f10 = sim.field.d.clone(), sim.field.f1.clone()
    res = {}
    for name, q in (("mixed", q_m), ("f64", q_f)):
        sim.field.d.copy_(d0)
        sim.field.f1.copy_(f10)
        sim.node_charge.copy_(q)
        sim.field_phase()
        torch.cuda.synchronize()
        res[name] = (sim.field.potential.clone(), sim.mesh.ef.view(-1, 4)[:, :3].clone())
    sim.field.d.copy_(d0)
    sim.field.f1.copy_(f10)
    (pm, em), (pf, ef_) = res["mixed"], res["f64"]
    out["mixed_vs_f64"] = {
        "what": "field phase on the node charges of one mixed and one FP64 move + deposit from the same pushed "
                "state, both from the same Newton state (CG stops at 1e-10 relative residual)",
        "node_charge_normwise_rel": rep["node_charge_normwise_rel"], "cells_differing": rep["cells_differing"],
        "potential_normwise_rel": float((pm - pf).abs().max() / pf.abs().max()),
        "field_normwise_rel": float((em - ef_).abs().max() / ef_.abs().max())}
    if cpu:
        from oracle import field as F

        fs = F.FieldSystem(hm.n_pos, hm.n_type, sim.field.d_bnd.cpu().numpy(), hm.c2n)
        fs.d[:fs.neq] = saved[0][:fs.neq].cpu().numpy()
        fs.f1[:fs.neq] = saved[1][:fs.neq].cpu().numpy()
        den = saved[2].cpu().numpy()
        t0 = time.perf_counter()  # density scaling + compute_phi, as one field phase minus the cell field
        _, it, _ = fs.solve(F.node_charge_density(den, hm.n_vol, FIELD["spwt"]),
                            F.FieldConsts(**{k: v for k, v in FIELD.items() if k != "spwt"}))
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": t * 1e3, "unit": "ms per compute_phi", "cores": 1, "kind": "port",
                               "sample": f"C oracle (Jacobi CG, {it} iterations) on the same state; the reference "
                                         f"solves with PETSc KSPCG, absent here"}
    del sim
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------- CabanaPIC (second workload)

CAB = dict(nx=32, ny=32, nz=256, lx=1.0, ly=1.0, lz=8.0, nppc=400, v0=0.2, sigma=0.01, courant=0.5, seed=3)
CAB_WORKLOAD = ("CabanaPIC two-stream move + current deposit: 32x32x256 periodic hexes (262,144 cells + ghost "
                "layer), 400 particles per cell (2 counter-streaming species x 200), u_z = +-0.2c gamma + "
                "N(0, 0.01c), dt = 0.5 Courant; synthetic fixed interpolated fields")
# Per call: read pos 24 + vel 24 + weight 8 + p2c 4, write pos 24 + vel 24 B per particle; per cell
# the interp record 160 B + faces 32 B read and the 12 accumulators read + written (192 B).
CAB_BYTES_PER_PARTICLE = 108
CAB_BYTES_PER_CELL = 384
# DRAM bytes per particle of one full-size launch (ncu, profiles/cabana_move_deposit_kernel_twostream_32x32x256.txt).
CAB_MEASURED_DRAM_BYTES_PER_PARTICLE = 122.0


CAB_OCCUPANCY_CANDIDATES = [4, 0, 5]  # CTAs per SM the move + deposit kernel is compiled for (0: compiler's)


def _cabana_leg(dev, mesh, deck, n, precision: str, steps: int, warmup: int):
    """warmup untimed calls, the occupancy trials (3 calls per candidate, each from the same
    saved state, restored afterwards; the default kept unless another is more than 1 % faster),
    then steps timed move_deposit calls of one form; the device state is kept."""
    import torch

    from oppb import _lib as L
    from oppb.autotune import MARGIN, pick
    from oppb.cabana import CabanaDevice, synthetic_interp

    cd = CabanaDevice(mesh, dev, n, precision=precision)
    cd.set_interp(synthetic_interp(mesh, CAB["seed"]))
    cd.fill_two_stream(mesh, deck, CAB["v0"], CAB["sigma"], CAB["seed"])
    lib = L.load()
    for _ in range(warmup):
        cd.move_deposit(deck)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()

    # Every trial starts from the same particle state (the dats a call changes, restored).
    names = [x for x in ("pos", "vel", "vel32", "streak", "p2c") if getattr(cd, x) is not None]
    saved = {x: getattr(cd, x).clone() for x in names}

    def trial(occ) -> float:
        L.set_tuning(cabana_occupancy=occ)
        for x in names:
            getattr(cd, x).copy_(saved[x])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        cd.move_deposit(deck)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)

    tuned = pick(CAB_OCCUPANCY_CANDIDATES, trial, reps=3, margin=MARGIN)
    L.set_tuning(cabana_occupancy=tuned.choice)
    for x in names:
        getattr(cd, x).copy_(saved[x])
    del saved
    cd.occupancy_trials = tuned.report()
    t_ms, visits = [], 0
    l0 = lib.oppb_kernel_launches()
    torch.cuda.profiler.start()
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        cd.move_deposit(deck)
        e1.record(s)
        e1.synchronize()
        st = cd.status_host()
        if st.error:
            raise L.OppbError("cabana move_deposit", st.error)
        t_ms.append(e0.elapsed_time(e1))
        visits += int(st.total_visits)
    torch.cuda.profiler.stop()
    return cd, sum(t_ms) / 1e3, visits, lib.oppb_kernel_launches() - l0


def run_cabana(dev, steps: int, warmup: int, cpu: bool, cpu_seconds: float) -> dict:
    """move_deposit on the config-sized two-stream state: `warmup` untimed then `steps` timed
    calls (c_acc zeroed + kernel each, as the reference main loop between field updates), for
    the FP64 form (bit-identical to the reference) and the FP32-momentum form (FP64 position,
    FP32 momentum) from the same construction, with the second's departure from the first."""
    import torch

    from oppb.cabana import Deck, HexMesh

    mesh = HexMesh(CAB["nx"], CAB["ny"], CAB["nz"])
    deck = Deck(CAB["nx"], CAB["ny"], CAB["nz"], CAB["lx"], CAB["ly"], CAB["lz"], nppc=CAB["nppc"],
                courant_frac=CAB["courant"])
    n = len(mesh.interior) * CAB["nppc"]
    cd, t, visits, launches = _cabana_leg(dev, mesh, deck, n, "f64", steps, warmup)
    bytes_call = CAB_BYTES_PER_PARTICLE * n + CAB_BYTES_PER_CELL * mesh.n_cells
    peaks = measured_peaks()
    out = {"workload": CAB_WORKLOAD, "metric": "particle-steps/s (move + current deposit)", "unit": UNIT,
           "value": n * steps / t, "particles": n, "cells": mesh.n_cells, "steps": steps, "warmup": warmup,
           "ms_per_step": 1e3 * t / steps, "calls_per_particle": visits / (n * steps), "dtype": "f64",
           "gpu_launches": int(launches),
           "roofline": {"bound": "hbm", "achieved": bytes_call / (t / steps) / 1e9, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": bytes_call / (t / steps) / 1e9 / peaks["hbm_gbs"],
                        "bytes_per_launch": bytes_call, "traffic": CAB_MEASURED_DRAM_BYTES_PER_PARTICLE * n,
                        "traffic_source": TRAFFIC_SOURCE}}
    out["occupancy"] = cd.occupancy_trials
    cm, tm, _, _ = _cabana_leg(dev, mesh, deck, n, "mixed", steps, warmup)
    # Departure of the FP32-momentum form from the FP64 form after the same calls.
    u64, u32 = cd.vel[:, :n], cm.vel32[:, :n].double()
    du = float((u32 - u64).abs().max() / u64.abs().max())
    du_mean = float((u32 - u64).abs().mean() / u64.abs().mean())
    dacc = float((cm.acc - cd.acc).abs().max() / cd.acc.abs().max())
    cells = float((cm.p2c[:n] != cd.p2c[:n]).double().mean())
    bytes_mixed = bytes_call - 24 * n + 80 * mesh.n_cells  # momentum 12 B read + 12 B written, f32 record read
    out["fp32_momentum"] = {"what": "FP64 position, FP32 momentum (FP32 push from an FP32 field record); positions, "
                                    "cells and current deposit in FP64",
                            "value": n * steps / tm, "ms_per_step": 1e3 * tm / steps,
                            "speedup_over_f64": t / tm, "occupancy": cm.occupancy_trials,
                            "vs_f64_after_steps": {"momentum_max_rel": du, "momentum_mean_rel": du_mean,
                                                   "current_max_rel": dacc,
                                                   "cells_differing": cells, "calls": warmup + steps},
                            "roofline_frac": bytes_mixed / (tm / steps) / 1e9 / peaks["hbm_gbs"]}
    del cd, cm
    torch.cuda.empty_cache()
    if cpu:
        out["cpu_baseline"] = cabana_cpu_baseline(cpu_seconds)
    return out


def cabana_cpu_baseline(budget_s: float) -> dict:
    """The compiled reference omp build (oracle/_ref/cabana_ref_omp, all host threads) on a
    bounded sample of the same construction (8x8x64 cells, 400 per cell), else the C oracle."""
    import numpy as np

    from oppb.cabana import Deck, HexMesh, synthetic_interp, two_stream
    from oracle import cabana as OC
    from oracle import ref_runner as R

    mesh = HexMesh(8, 8, 64)
    deck = Deck(8, 8, 64, 0.25, 0.25, 2.0, nppc=CAB["nppc"], courant_frac=CAB["courant"])
    interp = synthetic_interp(mesh, CAB["seed"])
    pos, vel, streak, w, p2c = two_stream(mesh, deck, CAB["v0"], CAB["sigma"], CAB["seed"])
    n = len(p2c)
    if (R.REF_DIR / "cabana_ref_omp").exists():
        cores = len(os.sched_getaffinity(0))
        calls = 8
        res = OC.run_reference("omp", mesh.c2ngc, interp, pos, vel, streak, w, p2c, deck.qdt_2mc, deck.cdt_d,
                               deck.qsp, calls=calls, threads=cores)
        t = float(res["times"][1:].sum())
        return {"value": n * (calls - 1) / t, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"{n} particles (8x8x64 cells x {CAB['nppc']}), {calls - 1} timed calls after 1; "
                          f"compiled OP-PIC omp backend + generated CabanaPIC loops"}
    ps, t = 0, 0.0
    while t < budget_s:
        acc = np.zeros((mesh.n_cells, 12))
        t0 = time.perf_counter()
        OC.move_deposit(pos, vel, streak, w, p2c, mesh.c2ngc, interp, acc, deck.qdt_2mc, np.array(deck.cdt_d),
                        deck.qsp)
        t += time.perf_counter() - t0
        ps += n
    return {"value": ps / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} particles (8x8x64 cells x {CAB['nppc']}); C oracle single thread"}


# ------------------------------------------------- NESO-advection ensemble (third workload)

ADV = dict(instances=64, side_lo=64, side_hi=512, ppc_lo=10, ppc_hi=200, cell_width=1.0, dt=0.5, v_sd=0.5,
           v_clip=1.0, seed=5, graph_steps=10)
ADV_WORKLOAD = ("NESO-advection ensemble: 64 independent periodic square meshes, side ~ U{64..512} cells, "
                "10..200 particles per cell (seeded), |v dt| <= 0.5 cell per step; update_pos + move of every "
                "instance in one persistent launch per step, captured as a CUDA graph")
# Per step: read pos 16 + vel 16 + mdir 8 + p2c 4, write pos 16 + mdir 8 B per particle; 32 B per cell record.
ADV_BYTES_PER_PARTICLE = 68
ADV_BYTES_PER_CELL = 32
# DRAM bytes per particle of one launch (ncu, profiles/advec_kernel_neso_ensemble_64.txt): a
# 19.2M-particle, 8-instance capture, scaled by the particle count (traffic grows with it).
ADV_MEASURED_DRAM_BYTES_PER_PARTICLE = 69.7
ADV_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of an 8-instance, 19.2M-particle launch, "
                      "per particle x particles")


def run_advec(dev, steps: int, warmup: int, cpu: bool, rank: int = 0, world: int = 1) -> dict:
    """The ensemble three ways on the same state: CUDA-graph replay of the batched step, the
    batched step launched directly, and one launch per instance.  With world > 1 the
    instances are split over the ranks by shard_instances (longest processing time first by
    particle count); each rank advances its shard in its own persistent launch and the
    figures are all particle-steps over the slowest rank's time (strong scaling: the ensemble
    is the same at every N).  Every rank takes the same collective steps."""
    import numpy as np
    import torch

    from oppb import _lib as L
    from oppb.advec import AdvecBatchDevice, AdvecMesh, shard_instances

    rng = np.random.default_rng(ADV["seed"])
    sides = rng.integers(ADV["side_lo"], ADV["side_hi"] + 1, ADV["instances"])
    ppcs = rng.integers(ADV["ppc_lo"], ADV["ppc_hi"] + 1, ADV["instances"])
    weights = [int(sd) * int(sd) * int(pc) for sd, pc in zip(sides, ppcs)]
    shards = shard_instances(weights, world)
    mine = shards[rank]
    meshes = [AdvecMesh(int(sides[k]), int(sides[k]), ADV["cell_width"]) for k in mine]
    counts = [m.n_cells * int(ppcs[k]) for m, k in zip(meshes, mine)]
    n = sum(counts)
    lib = L.load()
    G = ADV["graph_steps"]
    graph_steps = max(1, steps // G) * G
    t_graph = t_direct = t_single = 0.0
    visits, launches, sweep, best = 0, 0, {}, None
    if mine:
        bd = AdvecBatchDevice(meshes, counts, [ADV["dt"]] * len(meshes), dev)
        for j, k in enumerate(mine):  # seeded by the global instance index: same state at any N
            bd.fill_instance(j, int(ppcs[k]), ADV["v_sd"], ADV["v_clip"], ADV["seed"] * 1000 + k)
        for _ in range(warmup):
            bd.step()
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        E = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

        def timed(fn, reps):
            bd.zero_status()
            torch.cuda.synchronize()
            e0, e1 = E(), E()
            e0.record(s)
            for _ in range(reps):
                fn()
            e1.record(s)
            e1.synchronize()
            st = bd.status_host()
            if st.error:
                raise L.OppbError("advec step", st.error)
            return e0.elapsed_time(e1) / 1e3, int(st.total_visits)

        # Autotune the particles in flight per thread (the kernel's work items per block pass)
        # on this state, then capture the graph with the fastest choice.
        for items in (1, 2, 4):
            L.set_tuning(advec_items=items)
            bd.step()
            t_k, _ = timed(bd.step, 3)
            sweep[items] = n * 3 / t_k
        best = max(sweep, key=sweep.get)
        L.set_tuning(advec_items=best)
        graph = bd.capture(G)
        l0 = lib.oppb_kernel_launches()
        t_graph, visits = timed(graph.replay, graph_steps // G)
        torch.cuda.profiler.start()
        t_direct, _ = timed(bd.step, graph_steps)
        torch.cuda.profiler.stop()
        launches = lib.oppb_kernel_launches() - l0
        singles = bd.instance_batches()
        t_single, _ = timed(lambda: [bd.step_batch(b) for b, _ in singles], graph_steps)
        del graph, bd, singles
        torch.cuda.empty_cache()
    ps = n * graph_steps
    value, ms_step = replica_job_value(ps, t_graph, 1e3 * t_graph / graph_steps, dev)
    direct, _ = replica_job_value(ps, t_direct, 0.0, dev)
    single, _ = replica_job_value(ps, t_single, 0.0, dev)
    n_all = int(round(replica_sum(float(n), dev)))
    cells = sum(m.n_cells for m in meshes)
    bytes_step = ADV_BYTES_PER_PARTICLE * n + ADV_BYTES_PER_CELL * cells
    peaks = measured_peaks()
    achieved = bytes_step / (t_graph / graph_steps) / 1e9 if t_graph > 0 else 0.0
    out = {"workload": ADV_WORKLOAD, "metric": "particle-steps/s (update_pos + move, all instances)", "unit": UNIT,
           "value": value, "particles": n_all, "instances": len(sides),
           "cells": int(sum(int(sd) * int(sd) for sd in sides)), "steps": graph_steps, "warmup": warmup,
           "ms_per_step": ms_step, "calls_per_particle": visits / max(1, ps),
           "direct_launch_value": direct, "per_instance_launch_value": single,
           "dtype": "f64", "gpu_launches": int(launches), "scaling": "strong" if world > 1 else "weak",
           "sharding": {"rule": "longest processing time first by particle count, no data-path collective",
                        "ranks": world, "instances_per_rank": [len(x) for x in shards],
                        "particles_per_rank": [sum(int(sides[k]) ** 2 * int(ppcs[k]) for k in x) for x in shards]},
           "autotune": {"advec_items": {str(k): v for k, v in sweep.items()}, "chosen": best},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": achieved / peaks["hbm_gbs"], "bytes_per_launch": bytes_step,
                        "traffic": ADV_MEASURED_DRAM_BYTES_PER_PARTICLE * n, "traffic_source": ADV_TRAFFIC_SOURCE,
                        "what": "rank 0's persistent launch over its shard"}}
    if cpu and rank == 0:
        out["cpu_baseline"] = advec_cpu_baseline()
    return out


def advec_cpu_baseline() -> dict:
    """The compiled reference omp build (oracle/_ref/advec_ref_omp, all host threads) on one
    256 x 256 instance with 100 particles per cell, else the C oracle on a 128 x 128 one."""
    from oppb.advec import AdvecMesh, particles
    from oracle import advec as OA
    from oracle import ref_runner as R

    if (R.REF_DIR / "advec_ref_omp").exists():
        m = AdvecMesh(256, 256, ADV["cell_width"])
        pos, vel, mdir, p2c = particles(m, 100, ADV["v_sd"], ADV["seed"], v_clip=ADV["v_clip"])
        cores = len(os.sched_getaffinity(0))
        steps = 6
        res = OA.run_reference("omp", m.nx, m.ny, m.cell_width, ADV["dt"], pos, vel, mdir, p2c, m.c2c, m.c_pos_ll,
                               steps, threads=cores)
        t = float(res["times"][1:].sum())
        return {"value": len(p2c) * (steps - 1) / t, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"one 256x256 instance, {len(p2c)} particles, {steps - 1} timed steps after 1; compiled "
                          f"OP-PIC omp backend + generated NESO-advection loops"}
    m = AdvecMesh(128, 128, ADV["cell_width"])
    pos, vel, mdir, p2c = particles(m, 100, ADV["v_sd"], ADV["seed"], v_clip=ADV["v_clip"])
    t0 = time.perf_counter()
    OA.steps(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, ADV["dt"], m.extents, m.cell_width, 5)
    t = time.perf_counter() - t0
    return {"value": len(p2c) * 5 / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one 128x128 instance, {len(p2c)} particles, 5 steps; C oracle single thread"}


# ------------------------------------------------------------------------ reference arm

def workload_config() -> dict:
    """The bench line's config: the workload alone, the same object in both arms."""
    return {"workload": WORKLOAD, "cells": 6 * CFG["nx"] * CFG["ny"] * CFG["nz"],
            "nodes": (CFG["nx"] + 1) * (CFG["ny"] + 1) * (CFG["nz"] + 1), "inject_per_step": CFG["inject"],
            "fill_steps": CFG["fill_steps"], "sort_period": CFG["period"],
            "l2": "inputs larger than L2 (particle dats ~4 GB), no flush"}


def arm_reference(args) -> dict:
    """The reference's own CPU path on the same workload: the compiled OP-PIC omp backend with
    the generated FemPIC loops (oracle/_ref/fempic_ref_omp) on every host thread.  The mesh is
    the same box, written as the app's text mesh files and loaded by the app's own loader
    (load_mesh, fempic_misc_mesh_loader.h); the injection distribution is the workload's; the
    field is the exact static field of the workload's Laplace problem; the randoms come from
    the harness's seeded generator.  Per step: inject -> push -> move (with its hole fill or
    cell sort, Sort_Periodic every 10 steps) -> deposit, all the reference's code; the fill
    steps reach the steady state, then W warm-up and K timed steps, timing move (+ compaction)
    and deposit with the harness's clock.  Nothing of this library is loaded.  Without the
    compiled reference it runs the C oracle port on the oracle's restatement of the loader."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return {}
    from oracle import ref_runner as R

    dims = (CFG["nx"], CFG["ny"], CFG["nz"], CFG["lx"], CFG["ly"], CFG["lz"])
    fill, w, k = CFG["fill_steps"], args.warmup, args.steps
    cores = len(os.sched_getaffinity(0))
    if R.available("omp"):
        out = R.run_box("omp", dims, CFG["inject"], fill + w + k, fill=CFG["fill"], period=CFG["period"],
                        alloc_mult=REF_ALLOC_MULTIPLE, threads=cores, seed=CFG["seed"], dt=CFG["dt"], qm=CFG["qm"],
                        ion_velocity=CFG["v_ion"], sigma=CFG["sigma"])
        recs = out["records"][fill + w:]
        t = float((recs["t_move"] + recs["t_deposit"]).sum())
        ps = float(recs["size_before_move"].sum())
        kind = "reference"
        sample = (f"the whole workload: {fill} fill steps + {w} warm-up + {k} timed steps at "
                  f"{CFG['inject']:,} ions per step; compiled OP-PIC omp backend + generated FemPIC loops, "
                  f"OMP_NUM_THREADS={cores}; mesh from the app's loader")
    else:
        ps, t, cores = reference_port(fill, w, k)
        kind = "port"
        sample = f"{fill} fill + {w} warm-up + {k} timed steps; C oracle, one thread"
    value = ps / t
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": k,
        "warmup": w, "ms_per_step": 1e3 * t / k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
        "mean_particles": round(ps / k),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# opp_allocation_multiple of the reference's FemPIC configuration (apps_codegen/app_fempic_cg/configs/coarse.param).
REF_ALLOC_MULTIPLE = 11.0


def reference_port(fill: int, warmup: int, steps: int) -> tuple[float, float, int]:
    """The C oracle (one thread) on the workload, its mesh from the oracle's restatement of the
    app's loader: (particle-steps, seconds of move + compaction + deposit, cores)."""
    from oracle import mesh as OM
    from oracle import oracle as O

    hm = OM.box_mesh(CFG["nx"], CFG["ny"], CFG["nz"], CFG["lx"], CFG["ly"], CFG["lz"])
    hm.c_ef = OM.static_field(hm, 1.0, 0.0, CFG["lz"])
    dist = OM.area_distribution(hm.if_area, CFG["inject"])
    orc = O.OracleFemPIC(hm, dist, ion_velocity=CFG["v_ion"], qm=CFG["qm"], dt=CFG["dt"], fill=CFG["fill"],
                         fill_period=CFG["period"], alloc_mult=2.0)
    rng = __import__("numpy").random.default_rng(CFG["seed"])

    def table():
        import numpy as np

        out = np.empty((CFG["inject"], 5))
        out[:, 0:2] = rng.random((CFG["inject"], 2))
        out[:, 2:5] = CFG["sigma"] * rng.standard_normal((CFG["inject"], 3))
        return out

    for _ in range(fill + warmup):
        orc.step(table())
    ps, t = 0, 0.0
    for _ in range(steps):
        orc.inject(table())
        orc.node_charge[:] = 0
        O.push(orc.p2c, hm.c_ef, orc.pos, orc.vel, orc.qm, orc.dt, n=orc.size)
        n_alive = orc.size
        t0 = time.perf_counter()
        rc, _, _ = O.move(orc.pos, orc.lc, orc.p2c, hm.c2c, hm.c_vol, hm.c_det, n=orc.size)
        orc.finalize(rc)
        O.deposit(orc.lc, orc.p2c, hm.c2n, orc.node_charge, n=orc.size)
        t += time.perf_counter() - t0
        orc.iter += 1
        ps += n_alive
    return ps, t, 1


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["oppb", "reference"], default="oppb")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--fill-steps", type=int, default=CFG["fill_steps"], help="steps to reach the steady state")
    ap.add_argument("--capacity", type=int, default=CFG["capacity"], help="particle set capacity")
    ap.add_argument("--precision", choices=["both", "f64", "mixed"], default="both")
    ap.add_argument("--no-cabana", dest="cabana", action="store_false",
                    help="skip the CabanaPIC move + current deposit measurement")
    ap.add_argument("--cabana-only", action="store_true",
                    help="run only the CabanaPIC measurement and print its object")
    ap.add_argument("--cabana-dims", default=None, help="nx,ny,nz of the CabanaPIC mesh (default 32,32,256)")
    ap.add_argument("--no-advec", dest="advec", action="store_false",
                    help="skip the NESO-advection ensemble measurement")
    ap.add_argument("--advec-only", action="store_true", help="run only the NESO-advection ensemble measurement")
    ap.add_argument("--advec-instances", type=int, default=None, help="ensemble size (default 64)")
    ap.add_argument("--advec-side-max", type=int, default=None, help="largest mesh side (default 512)")
    ap.add_argument("--no-field", dest="field", action="store_false",
                    help="skip the field-phase measurement")
    ap.add_argument("--field-only", action="store_true", help="run only the field-phase measurement")
    ap.add_argument("--no-dh", dest="dh", action="store_false",
                    help="skip the global-move (direct-hop) measurement")
    ap.add_argument("--dh-only", action="store_true", help="run only the global-move (direct-hop) measurement")
    ap.add_argument("--deposit", choices=["warp", "table"], default="warp",
                    help="deposit strategy: warp-run FP64 atomics or per-CTA shared node table")
    args = ap.parse_args()
    CFG["fill_steps"], CFG["capacity"] = args.fill_steps, args.capacity
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl != "reference":
        from oppb import _lib as L

        L.set_deposit_strategy(L.DEPOSIT_CTA_TABLE if args.deposit == "table" else L.DEPOSIT_WARP_ATOMIC)
    if args.cabana_dims:
        nx, ny, nz = (int(v) for v in args.cabana_dims.split(","))
        CAB.update(nx=nx, ny=ny, nz=nz, lx=nx / 32, ly=ny / 32, lz=nz / 32)
    if args.advec_instances:
        ADV["instances"] = args.advec_instances
    if args.advec_side_max:
        ADV["side_hi"] = max(args.advec_side_max, ADV["side_lo"])
    if args.advec_only and args.impl != "reference":
        import torch

        print(json.dumps(run_advec(torch.device("cuda:0"), args.steps, args.warmup, args.cpu_baseline)), flush=True)
        return
    if args.field_only and args.impl != "reference":
        import torch

        from oppb.fempic import HostMesh

        hm = HostMesh(CFG["nx"], CFG["ny"], CFG["nz"], CFG["lx"], CFG["ly"], CFG["lz"])
        print(json.dumps(run_field_phase(hm, torch.device("cuda:0"), args.steps, args.warmup, CFG["seed"],
                                         args.cpu_baseline)), flush=True)
        return
    if args.dh_only and args.impl != "reference":
        import torch

        from oppb.fempic import HostMesh

        hm = HostMesh(CFG["nx"], CFG["ny"], CFG["nz"], CFG["lx"], CFG["ly"], CFG["lz"])
        print(json.dumps(run_direct_hop(hm, torch.device("cuda:0"), args.steps, args.warmup, CFG["seed"],
                                        args.cpu_baseline)), flush=True)
        return
    if args.cabana_only and args.impl != "reference":
        import torch

        print(json.dumps(run_cabana(torch.device("cuda:0"), args.steps, args.warmup, args.cpu_baseline,
                                    args.cpu_seconds)), flush=True)
        return
    line = arm_reference(args) if args.impl == "reference" else arm_ours(args)
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
