"""Skewed graph (degreeFrom targets and course choices Zipf-distributed, s = 1.1): hub vertices
with long neighbour lists and uneven tables through every path: single queries (tile launch
and flat pipeline), batches, a pipelined stream and serving, all against the oracle."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zipf_graph(built):
    tr, v = wk.synth_generate(30, seed=3, zipf=True, zipf_s=1.1)
    g = wk.GStore(tr)
    o = oracle.OracleStore(tr)
    inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    with wk.Context(0) as ctx:
        ctx.upload_gstore(g)
        yield {"ctx": ctx, "vocab": v, "oracle": o, "instances": inst}


def _hub_queries(v):
    # alumni of every organisation, then what they take: the hub organisations' lists are long
    return [wk.Query([(v["t_org"], wk.TYPE_ID, wk.IN, -1), (-1, v["p_degree_from"], wk.IN, -2),
                      (-2, v["p_takes"], wk.OUT, -3)]),
            workloads.heavy_star(v), workloads.heavy_triangle(v)]


def test_skewed_lists_are_long(zipf_graph):
    o = zipf_graph["oracle"]
    v = zipf_graph["vocab"]
    degs = [o.run(wk.Query([(int(org), v["p_degree_from"], wk.IN, -1)]).flat(), 1)[1].shape[0]
            for org in zipf_graph["instances"][v["t_org"]]]
    assert max(degs) > 10 * np.median(degs)   # hub organisations exist


@pytest.mark.parametrize("flat_rows", [0, 1])
def test_hub_queries_single(zipf_graph, flat_rows):
    ctx = zipf_graph["ctx"]
    o = zipf_graph["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, flat_rows)
    for q in _hub_queries(zipf_graph["vocab"]):
        _, want, _ = o.run(q.flat(), q.nvars)
        for mode in (wk.MODE_PLAIN, wk.MODE_GRAPH):
            got, _ = ctx.execute(q, mode)
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    ctx.tune_set(wk.KNOB_FLAT_ROWS, 65536)


@pytest.mark.parametrize("slice_rows", [8, 128, 4096])
def test_batch_stream_and_serving_on_skew(zipf_graph, slice_rows):
    ctx = zipf_graph["ctx"]
    o = zipf_graph["oracle"]
    v = zipf_graph["vocab"]
    ctx.tune_set(wk.KNOB_BATCH_SLICE_ROWS, slice_rows)
    qs = workloads.light_queries(v, zipf_graph["instances"], 600, seed=71)
    qs[::100] = _hub_queries(v) * 2
    want = [o.run(q.flat(), q.nvars) for q in qs]
    for got in (ctx.batch(qs), ctx.batch(qs, stream_batch=150)):
        for (st, w, _), (t, gst) in zip(want, got):
            assert gst == st
            if st == 0:
                assert np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(w))
    served = ctx.serve(qs, np.linspace(0, 3000, len(qs)))
    for (st, w, _), r in zip(want, served):
        assert r[1] == st
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(r[0]), oracle.sorted_rows(w))
    ctx.tune_set(wk.KNOB_BATCH_SLICE_ROWS, 128)
