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


@pytest.fixture(scope="module")
def oracle_versatile(graph20):
    import oracle
    return oracle.OracleStore(graph20["triples"], versatile=True)


def test_oracle_versatile_queries_reproduce_reference(oracle_versatile, golden):
    import oracle
    import wukong_b200 as wk
    for g in golden["versatile"]:
        q = wk.Query(g["patterns"], nvars=g["nvars"])
        st, rows, v2c = oracle_versatile.run(q.flat(), q.nvars)
        assert st == g["status"], g["name"]
        if st == 0:
            s = oracle.sorted_rows(rows)
            assert s.shape == (g["rows"], g["cols"]), g["name"]
            assert _digest(s) == g["sorted_sha256"], g["name"]
            assert list(v2c) == g["v2c"], g["name"]


def test_oracle_single_patterns_reproduce_reference(oracle_versatile, golden):
    for g in golden["patterns"]:
        t = np.array(g["table"], np.uint32).reshape(len(g["table"]), -1)
        st, rows, v2c = oracle_versatile.pattern(t, g["nvars"], g["pattern"], g["mt_tid"], g["mt_factor"])
        assert st == g["status"], g["name"]
        if st == 0:
            assert rows.shape == (g["rows"], g["cols"]), g["name"]
            assert _digest(rows) == g["table_sha256"], g["name"]   # row for row
            assert list(v2c) == g["v2c"], g["name"]


def test_non_versatile_store_refuses_unknown_predicates(graph20, golden):
    """Without the vertex-predicate lists the unknown-predicate patterns are unsupported, as in
    a reference build without VERSATILE; const_to_known needs no extra lists."""
    import wukong_b200 as wk
    o = graph20["oracle"]
    for g in golden["versatile"]:
        q = wk.Query(g["patterns"], nvars=g["nvars"])
        st, _, _ = o.run(q.flat(), q.nvars)
        if any(p[1] < 0 for p in g["patterns"]) and g["status"] == 0:
            assert st == wk.UNKNOWN_PATTERN, g["name"]


def test_reference_engine_live_zipf(built):
    """Where the reference engine library was built: on a 30-organisation graph whose
    degreeFrom targets and course choices follow Zipf (s = 1.1), the skewed shape of the scale
    configuration, the reference engine gives the oracle's status, rows and column map for the
    heavy star, the heavy triangle and 150 light queries."""
    import oracle
    import refengine
    import workloads
    import wukong_b200 as wk
    if not refengine.available():
        pytest.skip("the reference engine library was not built here")
    tr, v = wk.synth_generate(30, seed=5, zipf=True, zipf_s=1.1)
    o = oracle.OracleStore(tr)
    g = refengine.graph_from_store(o, tr, v)
    inst = {t: o.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    qs = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
    qs += workloads.light_queries(v, inst, 150, seed=41)
    nonempty = 0
    for q in qs:
        st, rows, v2c = g.run(q.flat(), q.nvars, required=refengine.bound_vars(q.flat()) or [-1])
        ost, orows, ov2c = o.run(q.flat(), q.nvars)
        assert st == ost
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(rows), oracle.sorted_rows(orows))
            assert list(v2c) == list(ov2c)
            nonempty += rows.shape[0] > 0
    assert nonempty >= 100


def test_reference_final_stage_live(graph20):
    """Where the reference engine library was built: the reference's own final stage
    (execute_sparql_query with required variables, DISTINCT, LIMIT and OFFSET) equals the
    oracle's restatement row for row, in order, on the heavy star, the heavy triangle and light
    queries, for seeded random choices of required variables (any subset, any order) and of
    DISTINCT / OFFSET / LIMIT. The device stage is checked against the same restatement."""
    import oracle
    import refengine
    import workloads
    if not refengine.available():
        pytest.skip("the reference engine library was not built here")
    o, tr, v = graph20["oracle"], graph20["triples"], graph20["vocab"]
    g = refengine.graph_from_store(o, tr, v)
    qs = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
    qs += workloads.light_queries(v, graph20["instances"], 40, seed=23)
    rng = np.random.default_rng(31)
    checked = 0
    for q in qs:
        st, rows, v2c = o.run(q.flat(), q.nvars)
        if st != 0:
            continue
        bound = refengine.bound_vars(q.flat())
        for _ in range(4):
            req = [int(x) for x in rng.permutation(bound)[:int(rng.integers(1, len(bound) + 1))]]
            distinct = bool(rng.integers(0, 2))
            n = rows.shape[0]
            offset = int(rng.choice([0, 0, 1, 3, n // 2, n + 2]))
            limit = int(rng.choice([-1, -1, 0, 1, 5, n]))
            rst, rtab, _ = g.run(q.flat(), q.nvars, required=req, distinct=distinct, limit=limit,
                                 offset=offset)
            assert rst == 0
            keep = [v2c[-r - 1] for r in req]
            want = oracle.final_process(rows, keep, distinct=distinct, offset=offset, limit=limit)
            assert rtab.shape == want.shape, (req, distinct, offset, limit)
            assert np.array_equal(rtab, want), (req, distinct, offset, limit)
            checked += 1
    assert checked >= 100


@pytest.mark.parametrize("versatile", [False, True])
def test_reference_engine_dispatch_live(built, versatile):
    """Where the reference engine library was built: seeded random plans (the dispatch test's
    generator) give the oracle's status, table and column map through the reference's own
    execute_sparql_query, on a store without and with the vertex-predicate lists."""
    import oracle
    import refengine
    import wukong_b200 as wk
    if not refengine.available() or not versatile:
        # the reference library is a VERSATILE build: it runs unknown predicates either way,
        # so only the versatile store can be compared with it
        pytest.skip("needs the reference engine library and a versatile store")
    V = 1 << 17
    tr = np.array([(V + 1, 5, V + 2), (V + 2, 6, V + 3), (V + 1, 1, 7), (V + 3, 5, V + 1),
                   (V + 2, 1, 7), (V + 3, 6, V + 2)], np.uint32)
    o = oracle.OracleStore(tr, versatile=True)
    g = refengine.graph_from_store(o, tr, None)
    rng = np.random.default_rng(29)
    consts = [V + 1, V + 2, V + 3, 7]
    for _ in range(400):
        nvars = int(rng.integers(1, 4))
        pats = []
        for k in range(int(rng.integers(1, 5))):
            def term():
                if rng.random() < 0.5:
                    return -int(rng.integers(1, nvars + 1))   # in range: the engine asserts otherwise
                return int(rng.choice(consts))
            pats.append((term(), int(rng.choice([5, 6, wk.TYPE_ID, -1])), int(rng.integers(0, 2)), term()))
        q = wk.Query(pats, nvars=nvars)
        st, tab, v2c = o.run(q.flat(), q.nvars)
        rst, rtab, rv2c = g.run(q.flat(), q.nvars, required=refengine.bound_vars(q.flat()) or [-1])
        if st == 0 and rst == 0 and len(refengine.bound_vars(q.flat())) != tab.shape[1]:
            continue   # a table replaced mid-plan: the projection is not the identity
        assert st == rst, (pats, st, rst)
        if st == 0:
            assert np.array_equal(oracle.sorted_rows(tab), oracle.sorted_rows(rtab)), pats
            assert list(v2c) == list(rv2c), pats


@pytest.fixture(scope="module")
def ctx_versatile(graph20):
    """A context holding the 20-organisation store built with the vertex-predicate lists."""
    import wukong_b200 as wk
    g = wk.GStore(graph20["triples"], versatile=True)
    c = wk.Context(0)
    c.upload_gstore(g)
    yield c
    c.close()
    g.close()


@pytest.mark.gpu
def test_gpu_versatile_queries_reproduce_reference(ctx_versatile, golden):
    import oracle
    import wukong_b200 as wk
    for mode in (wk.MODE_PLAIN, wk.MODE_RESIDENT, wk.MODE_GRAPH):
        for g in golden["versatile"]:
            q = wk.Query(g["patterns"], nvars=g["nvars"])
            if g["status"]:
                with pytest.raises(wk.WukongError) as e:
                    ctx_versatile.execute(q, mode)
                assert e.value.code == g["status"], (g["name"], mode)
                continue
            t, v2c = ctx_versatile.execute(q, mode)
            s = oracle.sorted_rows(t)
            assert s.shape == (g["rows"], g["cols"]), (g["name"], mode)
            assert _digest(s) == g["sorted_sha256"], (g["name"], mode)
            assert v2c == g["v2c"], (g["name"], mode)


@pytest.mark.gpu
def test_gpu_single_patterns_reproduce_reference(ctx_versatile, golden):
    """const_to_known, index_to_known (every mt slice) and the known-start versatile steps
    through their own entry points, row for row against the reference engine."""
    import wukong_b200 as wk
    c = ctx_versatile
    for g in golden["patterns"]:
        t = np.array(g["table"], np.uint32).reshape(len(g["table"]), -1)
        s, p, o, d, _ = g["pattern"]
        tin = c.table(t, capacity=t.size)
        out = c.table(capacity=1)
        name = g["name"]
        if name.startswith("c2k"):
            c.const_to_known(tin, -o - 1, s, p, d, out)
        elif name.startswith("i2k"):
            c.index_to_known(tin, -o - 1, s, d, out, g["mt_tid"], g["mt_factor"])
        elif name.startswith("kuu"):
            c.known_unknown_unknown(tin, -s - 1, d, out)
        elif name.startswith("kuc"):
            c.known_unknown_const(tin, -s - 1, o, d, out)
        got = out.download()
        assert g["status"] == 0 and got.shape == (g["rows"], g["cols"]), name
        assert _digest(got) == g["table_sha256"], name
        tin.free()
        out.free()


@pytest.mark.gpu
def test_gpu_constant_versatile_steps_and_refusals(ctx, ctx_versatile, golden):
    """The constant forms' entry points give the whole-query answers; a store without the
    vertex-predicate lists refuses unknown predicates; batches refuse versatile plans."""
    import oracle
    import wukong_b200 as wk
    byname = {g["name"]: g for g in golden["versatile"]}
    for name, call in (("v_const_unknown_unknown_out", "uu"), ("v_const_unknown_const", "uc")):
        g = byname[name]
        s, p, d, o = g["patterns"][0]
        out = ctx_versatile.table(capacity=1)
        if call == "uu":
            ctx_versatile.const_unknown_unknown(s, d, out)
        else:
            ctx_versatile.const_unknown_const(s, o, d, out)
        assert _digest(oracle.sorted_rows(out.download())) == g["sorted_sha256"], name
        out.free()
    q = wk.Query(byname["v_known_unknown_unknown"]["patterns"], nvars=3)
    with pytest.raises(wk.WukongError) as e:
        ctx.execute(q, wk.MODE_RESIDENT)
    assert e.value.code == wk.UNKNOWN_PATTERN
    res = ctx_versatile.batch([q])
    assert res[0][1] == wk.E_UNSUPPORTED


def _product_store_arrays(g):
    """The host GStore's arrays (wk_gstore_arrays) as RefGraph takes them."""
    slots, edges, segs = g.arrays()
    rows = np.array([[m.index, m.pid, m.dir, m.num_keys, m.num_buckets, m.bucket_start, m.num_edges,
                      m.edge_start, m.ext_start, m.ext_num] for m in segs], np.uint64)
    return slots.ctypes.data, slots.shape[0], edges.ctypes.data, rows


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_reference_engine_over_gstore_arrays(graph20, golden, which):
    """The reference engine reading a GStore in place (SlotGraph: the reference's ikey_t, its
    hash and its bucket walk over the slot array), once over the oracle's store and once over
    the library's own host-built store, answers like the oracle: light queries in parallel
    (row counts and statuses), the fixture queries, and the heavy star and triangle split over
    engine threads the way the reference splits an index start."""
    import refengine
    import workloads
    if not refengine.available():
        pytest.skip("the reference engine library was not built here")
    o, v = graph20["oracle"], graph20["vocab"]
    if which == "oracle":
        rg = refengine.RefGraph(o)
    else:
        rg = refengine.RefGraph(arrays=_product_store_arrays(graph20["gstore"]))
    qs = [q for _, q in _queries(golden)] + workloads.light_queries(v, graph20["instances"], 400, seed=29)
    rows, st = rg.run_many([q.flat() for q in qs], [q.nvars for q in qs], 4)
    orows, ost = o.run_many([q.flat() for q in qs], [q.nvars for q in qs], 4)
    assert np.array_equal(st, ost)
    assert np.array_equal(rows[st == 0].astype(np.int64), orows[st == 0].astype(np.int64))
    for q in (workloads.heavy_star(v), workloads.heavy_triangle(v)):
        want_st, want, _ = o.run(q.flat(), q.nvars)
        for f in (1, 3, 8):
            got_st, got_rows = rg.run_split(q.flat(), q.nvars, f)
            assert got_st == want_st == 0 and got_rows == want.shape[0]
