"""Serving: continuous batching over an open-loop arrival stream.

Each query's result must be the same alone (the oracle) and in the mix: light and index-start
queries arrive while others are on the GPU, are admitted as slots and memory free up, and share
the device (lights in iterations, index-start queries on lanes beside them).
"""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def _mix(graph, n_light, seed):
    v = graph["vocab"]
    qs = workloads.light_queries(v, graph["instances"], n_light, seed=seed)
    rng = np.random.default_rng(seed)
    for i in rng.choice(len(qs), size=max(1, n_light // 50), replace=False):
        qs[i] = workloads.heavy_star(v) if i % 2 else workloads.heavy_triangle(v)
    qs[3] = wk.Query([(-1, v["p_takes"], wk.OUT, -2)])   # fails at dispatch (UNKNOWN_SUB)
    return qs


def _check(o, qs, res, blind=False):
    for q, (t, st, ta, td, rows) in zip(qs, res):
        wst, want, _ = o.run(q.flat(), q.nvars)
        assert st == wst
        assert td >= ta
        if st == 0:
            assert rows == want.shape[0]
            if not blind:
                assert t.shape == want.shape
                assert np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))


@pytest.mark.parametrize("qps", [20_000, 500_000])
def test_open_loop_results_match_oracle(ctx, graph20, qps):
    qs = _mix(graph20, 800, seed=21)
    rng = np.random.default_rng(7)
    arrivals = np.cumsum(rng.exponential(1e6 / qps, size=len(qs)))
    res = ctx.serve(qs, arrivals)
    _check(graph20["oracle"], qs, res)
    lat = np.array([r[3] - r[2] for r in res if r[1] == 0])
    assert (lat > 0).all()


def test_small_slots_and_arenas_force_queueing_and_growth(ctx, graph20):
    """Few slots (queueing, slot reuse) and a tiny arena (growth + rerun of an iteration)."""
    qs = _mix(graph20, 300, seed=22)
    arrivals = np.zeros(len(qs))   # everything arrives at once
    res = ctx.serve(qs, arrivals, max_inflight=16, arena_bytes=4096, max_heavy_inflight=1)
    _check(graph20["oracle"], qs, res)


def test_two_lanes_and_a_tight_working_set_cap(ctx, graph20):
    """Two index-start queries at once; a cap that admits only a few queries at a time."""
    qs = _mix(graph20, 400, seed=24)
    arrivals = np.linspace(0, 500, len(qs))
    res = ctx.serve(qs, arrivals, max_heavy_inflight=2, working_set_cap_bytes=64 << 20,
                    lane_table_bytes=16 << 20, min_proj_bytes=1 << 20, light_ctas_per_sm=1)
    _check(graph20["oracle"], qs, res)


def test_blind_mode_returns_row_counts(ctx, graph20):
    qs = _mix(graph20, 400, seed=25)
    res = ctx.serve(qs, np.linspace(0, 1000, len(qs)), blind=1)
    _check(graph20["oracle"], qs, res, blind=True)
    assert all(r[0] is None for r in res)


def test_same_alone_and_in_mix(ctx, graph20):
    qs = _mix(graph20, 200, seed=23)
    mixed = ctx.serve(qs, np.linspace(0, 2000, len(qs)))
    for i in range(0, len(qs), 17):
        alone = ctx.serve([qs[i]], [0.0])[0]
        assert alone[1] == mixed[i][1]
        if alone[1] == 0:
            assert np.array_equal(alone[0], mixed[i][0])   # identical rows, identical order
