"""Whole-query parity: each query's sorted result multiset equals the oracle's."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu

MODES = [wk.MODE_PLAIN, wk.MODE_RESIDENT, wk.MODE_GRAPH]


def _same(ctx, o, q, mode):
    st, want, wv2c = o.run(q.flat(), q.nvars)
    assert st == 0
    got, v2c = ctx.execute(q, mode)
    assert v2c == wv2c
    assert got.shape == want.shape
    assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    return got


@pytest.mark.parametrize("mode", MODES)
def test_small_chain(ctx, graph20, mode):
    v, o = graph20["vocab"], graph20["oracle"]
    for unit in graph20["instances"][v["t_unit"]][:12]:
        got = _same(ctx, o, workloads.small_chain(v, int(unit)), mode)
        assert got.shape[1] == 2


@pytest.mark.parametrize("mode", MODES)
def test_heavy_queries(ctx, graph20, mode):
    v, o = graph20["vocab"], graph20["oracle"]
    for q in (workloads.heavy_star(v), workloads.heavy_triangle(v),
              workloads.heavy_star(v, v["t_person_c"])):
        for _ in range(2):   # replays (graph mode reuses the capture)
            _same(ctx, o, q, mode)


def test_light_queries(ctx, graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    qs = workloads.light_queries(v, graph20["instances"], 300, seed=5)
    for i, q in enumerate(qs):
        _same(ctx, o, q, wk.MODE_RESIDENT if i % 2 else wk.MODE_GRAPH)


def test_execute_host_and_enqueue(ctx, graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    q = workloads.heavy_star(v)
    st, want, _ = o.run(q.flat(), q.nvars)
    ctx.execute(q, wk.MODE_GRAPH)
    for _ in range(3):
        ctx.enqueue(q, wk.MODE_GRAPH)
    ctx.check()
    buf = np.zeros(want.size + 16, np.uint32)
    rows, cols = ctx.execute_host(q, buf, wk.MODE_GRAPH)
    got = buf[:rows * cols].reshape(rows, cols)
    assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    small = np.zeros(4, np.uint32)
    with pytest.raises(wk.WukongError) as e:
        ctx.execute_host(q, small)
    assert e.value.code == wk.E_CAPACITY


def test_dispatch_errors_match_oracle(ctx, graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    unit = int(graph20["instances"][v["t_unit"]][0])
    bad = [wk.Query([(-1, v["p_takes"], wk.OUT, -2)]),
           wk.Query([(unit, v["p_member_of"], wk.IN, -1), (unit, v["p_takes"], wk.OUT, -2)]),
           wk.Query([(v["t_unit"], v["p_takes"], wk.IN, -1)])]
    for q in bad:
        st, _, _ = o.run(q.flat(), q.nvars)
        with pytest.raises(wk.WukongError) as e:
            ctx.execute(q)
        assert e.value.code == st


def test_drop_in_reference_layout(graph20):
    """A store built by the reference's own construction rules (bucket sizing, extension
    extents, insertion order) runs unchanged on the GPU path."""
    v, o = graph20["vocab"], graph20["oracle"]
    slots, edges, segs = o.export()
    metas = (wk.SegMeta * len(segs))()
    for i, r in enumerate(segs):
        metas[i] = wk.SegMeta(int(r[0]), int(r[1]), int(r[2]), 0, *[int(x) for x in r[3:10]])
    with wk.Context(0) as c:
        c.upload_store(metas, slots, edges)
        for q in (workloads.heavy_star(v), workloads.heavy_triangle(v),
                  workloads.small_chain(v, int(graph20["instances"][v["t_unit"]][3]))):
            st, want, _ = o.run(q.flat(), q.nvars)
            got, _ = c.execute(q, wk.MODE_RESIDENT)
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))


def test_growth_from_tiny_buffers(graph20):
    """Outputs far larger than the configured buffers grow them and still match."""
    v, o = graph20["vocab"], graph20["oracle"]
    with wk.Context(0, rbuf_bytes=1024) as c:
        c.upload_gstore(graph20["gstore"])
        for mode in MODES:
            _same(c, o, workloads.heavy_star(v), mode)


def test_no_store(built):
    with wk.Context(0) as c:
        with pytest.raises(wk.WukongError) as e:
            c.execute(wk.Query([(1 << 17, 5, wk.OUT, -1)]))
        assert e.value.code == wk.E_NOSTORE
