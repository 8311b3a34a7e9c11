"""Answers of the reference's own CPU engine on the 20-organisation graph
(tests/golden/ref_engine_20orgs.json, made by tests/golden/make_ref_golden.py from
oracle/_ref/libwkref.so: the reference's sparql.hpp compiled unmodified from its tree).

CPU: the generator reproduces the graph byte for byte, the oracle reproduces every answer of the
reference engine (the pattern stage as sorted multisets, the final stage's DISTINCT / OFFSET /
LIMIT / projection row for row), and the library's host-side dispatch (wk_query_validate) gives
each query the status and column map the reference gave.  Where the reference engine library is
present the same queries are also run through it live.  GPU: the CUDA path reproduces every
digest, one query at a time and as one batch, and the device post-pattern stage reproduces the
reference's final stage.
"""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_engine_20orgs.json")


def _digest(rows):
    return hashlib.sha256(np.ascontiguousarray(rows.astype("<u4")).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _queries(golden):
    import wukong_b200 as wk
    return [(g, wk.Query(g["patterns"], nvars=g["nvars"])) for g in golden["queries"]]


def test_generator_is_frozen(built, graph20, golden):
    tr = graph20["triples"]
    assert tr.shape[0] == golden["graph"]["triples"]
    assert _digest(tr) == golden["graph"]["triples_sha256"]
    assert {k: int(x) for k, x in graph20["vocab"].items()} == golden["vocab"]


def test_oracle_reproduces_fixtures(graph20, golden):
    import oracle
    o = graph20["oracle"]
    for g, q in _queries(golden):
        st, rows, v2c = o.run(q.flat(), q.nvars)
        assert st == g["status"], g["name"]
        if st == 0:
            s = oracle.sorted_rows(rows)
            assert s.shape == (g["rows"], g["cols"]), g["name"]
            assert _digest(s) == g["sorted_sha256"], g["name"]
            assert v2c == g["v2c"], g["name"]


def test_host_dispatch_matches_fixtures(built, golden):
    import wukong_b200 as wk
    for g, q in _queries(golden):
        st, v2c, cols = wk.validate(q)
        assert st == g["status"], g["name"]
        if st == 0:
            assert v2c == g["v2c"], g["name"]
            assert cols == g["cols"], g["name"]


@pytest.mark.gpu
def test_gpu_matches_fixtures(ctx, golden):
    import oracle
    import wukong_b200 as wk
    for mode in (wk.MODE_PLAIN, wk.MODE_RESIDENT, wk.MODE_GRAPH):
        for g, q in _queries(golden):
            if g["status"]:
                with pytest.raises(wk.WukongError) as e:
                    ctx.execute(q, mode)
                assert e.value.code == g["status"], g["name"]
                continue
            t, v2c = ctx.execute(q, mode)
            s = oracle.sorted_rows(t)
            assert s.shape == (g["rows"], g["cols"]), (g["name"], mode)
            assert _digest(s) == g["sorted_sha256"], (g["name"], mode)
            assert v2c == g["v2c"], g["name"]


@pytest.mark.gpu
def test_gpu_batch_matches_fixtures(ctx, golden):
    import oracle
    qs = _queries(golden)
    res = ctx.batch([q for _, q in qs])
    for (g, _), (t, st) in zip(qs, res):
        assert st == g["status"], g["name"]
        if st == 0:
            assert _digest(oracle.sorted_rows(t)) == g["sorted_sha256"], g["name"]


def _final_cases(golden):
    import wukong_b200 as wk
    return [(g, wk.Query(g["patterns"], nvars=g["nvars"])) for g in golden["final"]]


def test_oracle_final_stage_reproduces_reference(graph20, golden):
    import oracle
    o = graph20["oracle"]
    for g, q in _final_cases(golden):
        st, rows, v2c = o.run(q.flat(), q.nvars)
        assert st == 0, g["name"]
        keep = [v2c[-r - 1] for r in g["required"]]
        got = oracle.final_process(rows, keep, distinct=g["distinct"], offset=g["offset"],
                                   limit=g["limit"])
        assert got.shape == (g["rows"], g["cols"]), g["name"]
        assert _digest(got) == g["table_sha256"], g["name"]   # row for row, in order


def test_reference_engine_live(graph20, golden):
    """Where oracle/_ref/libwkref.so was built (the reference tree was present), run the
    reference engine again on these queries and on more light queries, against the oracle."""
    import oracle
    import refengine
    import workloads
    if not refengine.available():
        pytest.skip("the reference engine library was not built here")
    o, tr, v = graph20["oracle"], graph20["triples"], graph20["vocab"]
    g = refengine.graph_from_store(o, tr, v)
    qs = [q for _, q in _queries(golden)]
    qs += workloads.light_queries(v, graph20["instances"], 200, seed=17)
    for q in qs:
        st, rows, v2c = g.run(q.flat(), q.nvars, required=refengine.bound_vars(q.flat()) or [-1])
        ost, orows, ov2c = o.run(q.flat(), q.nvars)
        assert st == ost
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(rows), oracle.sorted_rows(orows))
            assert list(v2c) == list(ov2c)


@pytest.mark.gpu
def test_gpu_final_stage_reproduces_reference(ctx, golden):
    """The device post-pattern stage on the device's own pattern-stage table.  Cases without
    DISTINCT depend on the table's row order, so they are kept to constant-start queries, whose
    order (row-major, then list order) is the same on the device and in the engine."""
    import wukong_b200 as wk
    for g, q in _final_cases(golden):
        if not g["distinct"] and g["patterns"][0][1] in (wk.PREDICATE_ID, wk.TYPE_ID):
            continue
        t, v2c = ctx.execute(q, wk.MODE_RESIDENT)
        tin = ctx.table(t, capacity=max(t.size, 1))
        out = tin.final_process([v2c[-r - 1] for r in g["required"]], distinct=g["distinct"],
                                offset=g["offset"], limit=g["limit"])
        got = out.download()
        assert got.shape == (g["rows"], g["cols"]), g["name"]
        assert _digest(got) == g["table_sha256"], g["name"]
        out.free()
        tin.free()


def test_oracle_bound_filter_reproduces_reference(built, golden):
    import oracle
    for g in golden["bound"]:
        t = np.array(g["table"], np.uint32).reshape(-1, g["cols"])
        got = oracle.bound_filter(t, g["bound_cols"])
        assert got.shape[0] == g["rows"], g["name"]
        assert _digest(got) == g["table_sha256"], g["name"]


@pytest.mark.gpu
def test_gpu_bound_filter_reproduces_reference(ctx, golden):
    for g in golden["bound"]:
        t = np.array(g["table"], np.uint32).reshape(-1, g["cols"])
        tin = ctx.table(t, capacity=max(t.size, 1))
        for _ in range(2):   # a second call on the same context gives the same rows
            out = tin.filter_bound(g["bound_cols"])
            got = out.download()
            assert got.shape == (g["rows"], g["cols"]), g["name"]
            assert _digest(got) == g["table_sha256"], g["name"]
            out.free()
        tin.free()


@pytest.mark.gpu
def test_gpu_bound_filter_large_and_refusals(ctx):
    """Many CTAs' chunks (order kept across them), and the refusals."""
    import oracle
    import wukong_b200 as wk
    rng = np.random.default_rng(5)
    t = rng.integers(1 << 17, 1 << 20, size=(300_000, 4), dtype=np.uint32)
    t[rng.random(t.shape) < 0.3] = 0xFFFFFFFF
    want = oracle.bound_filter(t, [1, 3])
    tin = ctx.table(t, capacity=t.size)
    out = tin.filter_bound([1, 3])
    assert np.array_equal(out.download(), want)
    with pytest.raises(wk.WukongError) as e:
        tin.filter_bound([4])
    assert e.value.code == wk.E_BADARG
    out.free()
    tin.free()
