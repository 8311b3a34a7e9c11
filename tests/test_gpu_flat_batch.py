"""Batch levels through the flat passes (knob 5): the same tables, row for row, as the tile
launch, for plain and skewed batches, failing plans, index-start queries mixed in, overflow
reruns and the pipelined stream."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


@pytest.fixture
def flat_knob(ctx):
    old = ctx.tune_get(wk.KNOB_BATCH_FLAT)
    yield ctx
    ctx.tune_set(wk.KNOB_BATCH_FLAT, old)


def _queries(graph, n, seed):
    v = graph["vocab"]
    qs = workloads.light_queries(v, graph["instances"], n, seed=seed)
    qs[7] = wk.Query([(-1, v["p_takes"], wk.OUT, -2)])   # UNKNOWN_SUB at dispatch
    qs[11] = workloads.heavy_star(v)
    qs[13] = workloads.heavy_triangle(v)
    return qs


ALL_LEVELS = 0xFFFF   # knob 5 is a mask over batch levels; bit k sends level k to the flat passes


@pytest.mark.parametrize("n,seed,mask", [(1, 91, ALL_LEVELS), (64, 92, ALL_LEVELS),
                                         (3000, 93, ALL_LEVELS), (3000, 95, 0b101), (3000, 96, 0b10)])
def test_flat_levels_equal_tile_levels(flat_knob, graph20, n, seed, mask):
    ctx = flat_knob
    o = graph20["oracle"]
    qs = _queries(graph20, max(n, 16), seed)[:n] if n > 16 else workloads.light_queries(
        graph20["vocab"], graph20["instances"], n, seed=seed)
    ctx.tune_set(wk.KNOB_BATCH_FLAT, 0)
    tile = ctx.batch(qs)
    ctx.tune_set(wk.KNOB_BATCH_FLAT, mask)
    flat = ctx.batch(qs)
    for q, (t0, s0), (t1, s1) in zip(qs, tile, flat):
        st, want, _ = o.run(q.flat(), q.nvars)
        assert s0 == s1 == st
        if st == 0:
            assert np.array_equal(t0, t1)   # identical rows in identical order
            assert np.array_equal(oracle.sorted_rows(t1), oracle.sorted_rows(want))


def test_flat_levels_stream_and_device_replay(flat_knob, graph20):
    ctx = flat_knob
    o = graph20["oracle"]
    ctx.tune_set(wk.KNOB_BATCH_FLAT, ALL_LEVELS)
    qs = _queries(graph20, 900, 94)
    got = ctx.batch(qs, stream_batch=256, cap_elems=1024)
    for q, (t, st) in zip(qs, got):
        wst, want, _ = o.run(q.flat(), q.nvars)
        assert st == wst
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))
    total = ctx.batch_device(qs)
    for _ in range(3):
        ctx.batch_replay()
    ctx.check()
    assert total == sum(t.shape[0] for t, st in got if st == 0)
