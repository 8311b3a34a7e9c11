"""Batched execution: every query's result equals the oracle's, alone and in the mix."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def _check_batch(ctx, o, qs):
    res = ctx.batch(qs)
    for q, (got, st) in zip(qs, res):
        wst, want, _ = o.run(q.flat(), q.nvars)
        assert st == wst
        if st == 0:
            assert got.shape == want.shape
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    return res


def test_light_batch(ctx, graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    qs = workloads.light_queries(v, graph20["instances"], 2000, seed=11)
    _check_batch(ctx, o, qs)


def test_mixed_batch_with_heavy_and_bad_plans(ctx, graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    unit = int(graph20["instances"][v["t_unit"]][2])
    qs = workloads.light_queries(v, graph20["instances"], 300, seed=12)
    qs[5] = workloads.heavy_star(v)
    qs[17] = workloads.heavy_triangle(v)
    qs[40] = wk.Query([(-1, v["p_takes"], wk.OUT, -2)])                    # UNKNOWN_SUB
    qs[41] = wk.Query([(unit, v["p_member_of"], wk.IN, -1)] * 2)           # FIRST_PATTERN_ERROR
    qs[42] = wk.Query([(unit, v["p_member_of"], wk.IN, -1)])               # one pattern
    qs[43] = wk.Query([(v["next_vid"] + 9, v["p_takes"], wk.OUT, -1), (-1, v["p_takes"], wk.IN, -2)])
    qs[44] = wk.Query([(v["t_course"], wk.TYPE_ID, wk.IN, -1)])           # index start only
    _check_batch(ctx, o, qs)


def test_result_same_alone_and_in_mix(ctx, graph20):
    """Each query's result is identical when run alone and when run inside a batch."""
    v = graph20["vocab"]
    qs = workloads.light_queries(v, graph20["instances"], 400, seed=13)
    mixed = ctx.batch(qs)
    for i in range(0, 400, 37):
        alone = ctx.batch([qs[i]])[0]
        single, _ = ctx.execute(qs[i], wk.MODE_RESIDENT)
        assert alone[1] == mixed[i][1] == 0
        assert np.array_equal(alone[0], mixed[i][0])            # same order, not just multiset
        assert np.array_equal(oracle.sorted_rows(single), oracle.sorted_rows(mixed[i][0]))


def test_batch_growth_and_replay(graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    with wk.Context(0) as c:
        c.upload_gstore(graph20["gstore"])
        qs = [workloads.heavy_star(v)] * 3 + workloads.light_queries(v, graph20["instances"], 50, seed=3)
        res = _check_batch(c, o, qs)
        total = c.batch_device(qs)
        assert total == sum(r[0].shape[0] for r in res if r[1] == 0)
        for _ in range(3):
            c.batch_replay()
        c.check()


def test_empty_batch_and_all_failed(ctx, graph20):
    assert ctx.batch([]) == []
    bad = [wk.Query([(-1, 5, wk.OUT, -2)])] * 3
    res = ctx.batch(bad)
    assert [r[1] for r in res] == [wk.UNKNOWN_SUB] * 3
