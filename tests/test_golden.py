"""Frozen oracle outputs on the 20-organisation graph (tests/golden/oracle_20orgs.json, made by
tests/golden/make_golden.py).

CPU: the generator reproduces the graph byte for byte, the oracle reproduces every frozen
answer, and the library's host-side dispatch (wk_query_validate) gives each query the status
and column map the oracle engine gave.  GPU: the CUDA path reproduces every digest, one query
at a time and as one batch.
"""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "oracle_20orgs.json")


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
