"""Autotuner selection logic on the host (CPU only).

A fake context stands in for the GPU: its plans report a synthetic device time for the
tuning currently set, and its set_tuning applies the library's range checks
(rtnn_set_tuning, api.cu). The tests check what rtnn_b200/autotune.py decides from those
times, not the times themselves.
"""
import numpy as np
import pytest
import torch

import rtnn_b200
from rtnn_b200 import autotune as at

# the library's default tuning (api.cu)
DEFAULT = dict(cell_ratio=0.5, min_cell_ratio=0.0625, points_per_cell=0.0, cell_budget=16.0,
               warps_per_block=4, blocks_per_sm=0, width_margin=1.1, fallback_passes=4,
               lane_walk_ratio=0.0, gap_ratio=2.0, pending_slots=16, query_warps=2,
               buckets_per_halving=1.0, width_model=0, width_clip=0)


class _Tuning(dict):
    def as_dict(self):
        return dict(self)


class _Plan:
    def __init__(self, ctx, kw):
        self.ctx, self.kw = ctx, kw

    def execute(self, points, queries=None, out=None, stats=None):
        self.ctx.executes += 1
        if stats is not None:
            stats.ms_total = self.ctx.cost(self.ctx.tun, self.ctx.model)
        return out

    def close(self):
        pass


class FakeCtx:
    def __init__(self, cost):
        self.cost = cost
        self.tun = dict(DEFAULT)
        self.model = None
        self.executes = 0
        self.rejected = 0

    def tuning(self):
        return _Tuning(self.tun)

    def set_tuning(self, **kw):
        ok = (0 < kw["cell_ratio"] <= 64 and 0 < kw["min_cell_ratio"] <= kw["cell_ratio"] and
              kw["points_per_cell"] >= 0 and 1 <= kw["warps_per_block"] <= 8 and
              8 <= kw["pending_slots"] <= 256 and kw["query_warps"] <= 4 and
              kw["fallback_passes"] <= 6 and 0 <= kw["buckets_per_halving"] <= 8 and
              kw["width_model"] <= 2 and kw["width_clip"] <= 16)
        if not ok:
            self.rejected += 1
            raise rtnn_b200.RtnnError(1, "tuning values out of range")
        self.tun = dict(kw)

    def plan(self, offsets, qoffsets=None, use_graph=True, **kw):
        return _Plan(self, kw)

    def get_model(self):
        return self.model

    def set_model(self, m):
        self.model = m


POINTS = torch.zeros((64, 3))
OFFSETS = np.array([0, 64], np.uint64)


def separable(t, model):
    return (1.0 + abs(t["points_per_cell"] - 1.0) + abs(t["cell_ratio"] - 0.25) +
            (0.0 if t["warps_per_block"] == 2 else 0.5) + 0.1 * abs(t["gap_ratio"] - 4.0) +
            abs(t["pending_slots"] - 32) / 64 + (0.0 if t["query_warps"] == 1 else 0.3) +
            0.2 * t["lane_walk_ratio"])


def test_descent_reaches_the_optimum_of_a_separable_cost():
    ctx = FakeCtx(separable)
    best = at.autotune(ctx, POINTS, OFFSETS, mode="knn", radius=0.2, k=8, use_cache=False)
    expect = dict(points_per_cell=1.0, cell_ratio=0.25, warps_per_block=2, gap_ratio=4.0,
                  pending_slots=32, query_warps=1, lane_walk_ratio=0.0)
    assert {n: best[n] for n in expect} == expect
    assert ctx.tun == best                     # left set on the context
    assert ctx.cost(ctx.tun, None) == pytest.approx(1.0)


def test_presets_escape_what_one_knob_at_a_time_cannot():
    # only the fine-cell regime as a whole is fast: no single knob change from the
    # defaults improves, so plain descent stays put and the preset finds it
    def joint(t, model):
        fine = t["cell_ratio"] == 0.125 and t["points_per_cell"] == 0.125
        return 1.0 if fine else 5.0
    ctx = FakeCtx(joint)
    plain = at.autotune(ctx, POINTS, OFFSETS, use_cache=False, knobs=at.CELL_KNOBS)
    assert joint(plain, None) == 5.0
    ctx = FakeCtx(joint)
    best = at.autotune(ctx, POINTS, OFFSETS, use_cache=False, knobs=at.CELL_KNOBS,
                       presets=at.GRID_PRESETS)
    assert (best["cell_ratio"], best["points_per_cell"]) == (0.125, 0.125)


def test_rejected_settings_are_skipped():
    ctx = FakeCtx(lambda t, m: 1.0 + abs(t["pending_slots"] - 300))
    best = at.autotune(ctx, POINTS, OFFSETS, use_cache=False,
                       knobs=[("pending_slots", [4, 8, 300, 256])])
    assert best["pending_slots"] == 256        # 300 is closest but out of range
    assert ctx.rejected == 2


def test_cache_skips_the_search(tmp_path, monkeypatch):
    monkeypatch.setenv("RTNN_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    ctx = FakeCtx(separable)
    first = at.autotune(ctx, POINTS, OFFSETS, mode="knn", radius=0.2, k=8)
    n = ctx.executes
    ctx2 = FakeCtx(separable)
    again = at.autotune(ctx2, POINTS, OFFSETS, mode="knn", radius=0.2, k=8)
    assert again == first and ctx2.tun == first and ctx2.executes == 0 and n > 0
    # another workload signature is searched again
    at.autotune(ctx2, POINTS, OFFSETS, mode="knn", radius=0.2, k=16)
    assert ctx2.executes > 0


def test_learned_keeps_the_model_of_the_winning_preset():
    # the model trained at a grid and bucket kind only pays there; the second preset's grid
    # with per-tile widths and its own model is fastest, and its margin optimum is 1.25
    def cost(t, model):
        c = 1.0 + abs(t["width_margin"] - 1.25)
        if model != ("model", t["cell_ratio"], t["width_model"]):
            c += 10.0
        c += 0.0 if t["width_model"] == 1 else 0.5
        return c + (0.0 if t["cell_ratio"] == 0.25 else 1.0)

    ctx = FakeCtx(cost)
    trained = []

    def train(c):
        c.set_model(("model", c.tun["cell_ratio"], c.tun["width_model"]))
        trained.append((c.tun["cell_ratio"], c.tun["width_model"]))
        return {"preset": c.tun["cell_ratio"], "kind": c.tun["width_model"]}

    tun, info = at.autotune_learned(ctx, POINTS, OFFSETS, mode="knn", radius=0.2, k=8,
                                    train=train)
    assert trained == [(p["cell_ratio"], kind) for p in at.GRID_PRESETS for kind in (0, 1)]
    assert tun["cell_ratio"] == 0.25 and tun["width_model"] == 1
    assert {n: info[n] for n in ("preset", "kind", "widths")} == {"preset": 0.25, "kind": 1,
                                                                  "widths": "on"}
    assert info["ms_on"] < info["ms_off"]
    assert ctx.model == ("model", 0.25, 1) and ctx.tun == tun
    assert tun["width_margin"] == 1.25


def test_learned_switches_widths_off_where_they_cannot_pay():
    # every narrowed setting costs more than the full radius (widths saturated at r): the
    # tuning that comes back is the starting one with the widths off (width_model 2)
    def cost(t, model):
        return 1.0 if t["width_model"] == 2 else 2.0 + abs(t["width_margin"] - 1.1)

    ctx = FakeCtx(cost)
    start = dict(DEFAULT, cell_ratio=0.125, points_per_cell=0.125, min_cell_ratio=0.01)
    ctx.set_tuning(**start)
    tun, info = at.autotune_learned(ctx, POINTS, OFFSETS, mode="radius", radius=2.0, k=64,
                                    train=lambda c: {"samples": 1})
    assert tun == {**start, "width_model": at.OFF} and ctx.tun == tun
    assert info["widths"] == "off" and info["ms_off"] < info["ms_on"]


def test_grid_of_takes_the_cell_settings():
    t = dict(DEFAULT, cell_ratio=0.125, points_per_cell=0.125, min_cell_ratio=0.01, query_warps=1)
    assert at.grid_of(t) == dict(cell_ratio=0.125, min_cell_ratio=0.01, points_per_cell=0.125,
                                 query_warps=1)
