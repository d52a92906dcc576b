"""The autotuner's choice rule without a GPU: the candidate with the smallest median time wins,
ties go to the earlier candidate, and every candidate is timed the requested number of times."""
from __future__ import annotations

import pytest

from oppb.autotune import (BLOCK_CANDIDATES, LANE_CANDIDATES, MOVE_CANDIDATES, PERIOD_CANDIDATES, SORT_CANDIDATES,
                            block_shape_applies, pick)


def test_pick_smallest_median():
    times = {"a": [5.0, 1.0, 5.0], "b": [3.0, 3.0, 3.0], "c": [4.0, 2.0, 9.0]}
    calls = {k: 0 for k in times}

    def run(c):
        calls[c] += 1
        return times[c][calls[c] - 1]

    res = pick(["a", "b", "c"], run, reps=3)
    assert res.choice == "b"  # medians 5, 3, 4
    assert res.times_ms == {"a": 5.0, "b": 3.0, "c": 4.0}
    assert all(v == 3 for v in calls.values())
    assert res.report()["choice"] == "b"


def test_pick_margin_keeps_the_default_within_noise():
    times = {"d": 2.000, "a": 1.995, "b": 2.5}
    assert pick(["d", "a", "b"], lambda c: times[c], reps=1, margin=0.01).choice == "d"
    assert pick(["d", "a", "b"], lambda c: times[c], reps=1).choice == "a"
    times["a"] = 1.9
    assert pick(["d", "a", "b"], lambda c: times[c], reps=1, margin=0.01).choice == "a"


def test_pick_ties_and_errors():
    assert pick([(1, 8), (0, 4)], lambda c: 1.0, reps=1).choice == (1, 8)
    with pytest.raises(ValueError):
        pick([], lambda c: 0.0)


def test_candidate_sets():
    assert len(set(MOVE_CANDIDATES)) == len(MOVE_CANDIDATES) == 8
    assert all(1 <= c <= 16 and f in (0, 1) for c, f in SORT_CANDIDATES) and SORT_CANDIDATES[0] == (16, 0)
    assert LANE_CANDIDATES[0] == (1, 8, 0, 0)
    assert all(lanes in (1, 2) and occ in (5, 8) and stage in (0, 1) and w in (0, 1, 2)
               for lanes, occ, stage, w in LANE_CANDIDATES)
    assert (1, 8, 0, 1) in LANE_CANDIDATES
    assert 10 in PERIOD_CANDIDATES
    assert BLOCK_CANDIDATES[0] == 256 and sorted(BLOCK_CANDIDATES) == [128, 256, 512]


def test_tuning_fields_validated():
    """oppb_set_tuning accepts the documented values of every field and refuses others."""
    from oppb import _lib as L

    L.set_tuning(move_lanes=2, move_occupancy=5, sort_scatter=1, move_stage=1, move_block=512)
    t = L.Tuning()
    L.load().oppb_get_tuning(t)
    assert (t.move_lanes, t.move_occupancy, t.sort_scatter, t.move_stage, t.move_block) == (2, 5, 1, 1, 512)
    for kw in (dict(move_lanes=3), dict(move_occupancy=6), dict(sort_scatter=2), dict(move_stage=2),
               dict(move_block=64), dict(move_block=384), dict(move_block=1024), dict(cabana_occupancy=3),
               dict(cabana_occupancy=8), dict(move_walk32=3)):
        with pytest.raises(L.OppbError):
            L.set_tuning(**kw)
    L.set_tuning(move_block=0)  # 0 reads as the default
    L.load().oppb_get_tuning(t)
    assert t.move_block == 256
    L.set_tuning(cabana_occupancy=5)
    L.load().oppb_get_tuning(t)
    assert t.cabana_occupancy == 5
    L.set_tuning(cabana_occupancy=4)
    L.set_tuning(move_lanes=1, move_occupancy=8, sort_scatter=0, move_stage=0, move_block=256)


def test_block_shape_applies_to_the_one_lane_warp_deposit():
    """move_block shapes the one-lane kernels with the warp-grouped deposit only."""
    from oppb import _lib as L

    t = L.Tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=1, move_stage=0, move_block=128)
    assert block_shape_applies(t, "f64") and block_shape_applies(t, "mixed")
    assert not block_shape_applies(L.Tuning(deposit=L.DEPOSIT_CTA_TABLE, move_lanes=1), "mixed")
    assert not block_shape_applies(L.Tuning(deposit=L.DEPOSIT_EXACT, move_lanes=1), "f64")
    assert not block_shape_applies(L.Tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=2), "f64")
    assert not block_shape_applies(L.Tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=1, move_stage=1), "f64")
    assert not block_shape_applies(L.Tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=1, move_walk32=1), "f64")
    assert block_shape_applies(L.Tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=2), "mixed")


def test_snapshot_fits_counts_live_columns(monkeypatch):
    """snapshot_fits compares the bytes of every particle dat over [0, size) (with headroom)
    against the free device memory the driver reports."""
    import types

    import torch

    from oppb import autotune as A

    class Parts:
        DATS = (("pos", 3, torch.float64), ("p2c", 1, torch.int32))
        size = 1000
        pos = torch.zeros(3, 4000, dtype=torch.float64)
        p2c = torch.zeros(1, 4000, dtype=torch.int32)

    sim = types.SimpleNamespace(parts=Parts(), device="cpu")
    need = 1000 * (3 * 8 + 4)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (int(need * 1.25), 1 << 40))
    assert A.snapshot_fits(sim)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (need, 1 << 40))
    assert not A.snapshot_fits(sim)
