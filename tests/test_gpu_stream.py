"""Pipelined batches (wk_batch_execute_stream): the same tables as one batch at a time.

Batches of uneven size, plans that fail at dispatch, a batch in which every plan fails (nothing
reaches the device), index-start queries that grow the batch buffers mid-stream, and a host
buffer that is too small the first time.
"""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def _stream_queries(graph, n, seed):
    v = graph["vocab"]
    qs = workloads.light_queries(v, graph["instances"], n, seed=seed)
    qs[5] = wk.Query([(-1, v["p_takes"], wk.OUT, -2)])   # UNKNOWN_SUB at dispatch
    return qs


@pytest.mark.parametrize("batch", [128, 300, 1000, 4096])
def test_stream_equals_batches(ctx, graph20, batch):
    o = graph20["oracle"]
    qs = _stream_queries(graph20, 1000, seed=61)
    got = ctx.batch(qs, stream_batch=batch)
    for i, q in enumerate(qs):
        st, want, _ = o.run(q.flat(), q.nvars)
        assert got[i][1] == st, i
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(got[i][0]), oracle.sorted_rows(want)), i
    # identical rows in identical order to the one-batch-at-a-time path
    for s in range(0, len(qs), batch):
        one = ctx.batch(qs[s:s + batch])
        for a, b in zip(one, got[s:s + batch]):
            assert a[1] == b[1]
            if a[1] == 0:
                assert np.array_equal(a[0], b[0])


def test_stream_with_failing_batch_and_growth(ctx, graph20):
    v = graph20["vocab"]
    o = graph20["oracle"]
    bad = [wk.Query([(-1, v["p_takes"], wk.OUT, -2)])] * 64          # a batch where all fail
    light = workloads.light_queries(v, graph20["instances"], 192, seed=62)
    heavy = [workloads.heavy_star(v), workloads.heavy_triangle(v)] * 32   # grows the buffers
    qs = light[:64] + bad + heavy + light[64:]
    got = ctx.batch(qs, stream_batch=64, cap_elems=1024)   # the host buffer grows too
    for i, q in enumerate(qs):
        st, want, _ = o.run(q.flat(), q.nvars)
        assert got[i][1] == st, i
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(got[i][0]), oracle.sorted_rows(want)), i
