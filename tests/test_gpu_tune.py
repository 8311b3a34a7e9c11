"""The autotuner and the tile-schedule knobs: every setting gives the same results, and the
tuner's choice is one of the candidates and no slower than the default it started from."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def test_knob_values_are_checked(ctx):
    for knob, bad in ((wk.KNOB_LANES, 3), (wk.KNOB_BATCH_LANES, 16), (wk.KNOB_SLICE_ROWS, 4),
                      (wk.KNOB_BATCH_SLICE_ROWS, 1 << 25), (wk.KNOB_BATCH_FLAT, 1 << 16),
                      (wk.KNOB_BATCH_FLAT, -1), (9, 4)):
        with pytest.raises(wk.WukongError) as e:
            ctx.tune_set(knob, bad)
        assert e.value.code == wk.E_BADARG


@pytest.mark.parametrize("lanes,slice_rows", [(2, 128), (8, 32), (4, 16384), (2, 8), (1, 128), (1, 8)])
def test_every_setting_gives_the_oracle_results(ctx, graph20, lanes, slice_rows):
    v = graph20["vocab"]
    o = graph20["oracle"]
    old = [ctx.tune_get(k) for k in range(6)]
    try:
        ctx.tune_set(wk.KNOB_LANES, lanes)
        ctx.tune_set(wk.KNOB_BATCH_LANES, lanes)
        ctx.tune_set(wk.KNOB_SLICE_ROWS, slice_rows)
        ctx.tune_set(wk.KNOB_BATCH_SLICE_ROWS, slice_rows)
        for q in (workloads.heavy_star(v), workloads.heavy_triangle(v)):
            got, _ = ctx.execute(q, wk.MODE_GRAPH)
            _, want, _ = o.run(q.flat(), q.nvars)
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
        qs = workloads.light_queries(v, graph20["instances"], 300, seed=41)
        for q, (t, st) in zip(qs, ctx.batch(qs)):
            _, want, _ = o.run(q.flat(), q.nvars)
            assert st == 0 and np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))
    finally:
        for k, val in enumerate(old):
            ctx.tune_set(k, val)


def test_autotune_picks_a_candidate_and_keeps_results(ctx, graph20):
    v = graph20["vocab"]
    o = graph20["oracle"]
    qs = workloads.light_queries(v, graph20["instances"], 2000, seed=42)
    heavy = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
    old = [ctx.tune_get(k) for k in range(6)]
    try:
        r = ctx.autotune(qs + heavy, iters=3)
        assert r["batch_lanes"] in (1, 2, 4, 8) and r["lanes"] in (1, 2, 4, 8)
        assert r["batch_slice_rows"] in (8, 16, 32, 128, 512)
        assert r["slice_rows"] in (8, 16, 32, 128, 512)
        assert r["candidates"] == 4 * 5 + max(len(q.patterns) for q in qs) + 4 + 5
        assert 0 <= r["batch_flat"] < 64 and ctx.tune_get(wk.KNOB_BATCH_FLAT) == r["batch_flat"]
        assert ctx.tune_get(wk.KNOB_BATCH_LANES) == r["batch_lanes"]
        assert ctx.tune_get(wk.KNOB_SLICE_ROWS) == r["slice_rows"]
        assert 0 < r["batch_ms_tuned"] <= 1.25 * r["batch_ms_default"]
        assert 0 < r["single_ms_tuned"] <= 1.25 * r["single_ms_default"]
        res = ctx.batch(qs)
        for i in range(0, len(qs), 37):
            _, want, _ = o.run(qs[i].flat(), qs[i].nvars)
            assert np.array_equal(oracle.sorted_rows(res[i][0]), oracle.sorted_rows(want))
        for q in heavy:
            got, _ = ctx.execute(q, wk.MODE_GRAPH)
            _, want, _ = o.run(q.flat(), q.nvars)
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    finally:
        for k, val in enumerate(old):
            ctx.tune_set(k, val)
