"""The store built on the device (wk_store_build_device) against the host builder
(wk_gstore_build_ex), which the CPU suite checks against the oracle's restatement of the
reference's loader and init_gstore: the same slots, edges and segment table, byte for byte, at
the default load factor, at a full one (chained buckets), Zipf-skewed, versatile, and with
duplicate and filtered triples; then queries on the device-built store answer as the oracle."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def _host_arrays(tr, load, versatile):
    g = wk.GStore(tr, load_factor=load, versatile=versatile)
    slots, edges, segs = g.arrays()
    seg_list = [{f: getattr(segs[i], f) for f, _ in wk.SegMeta._fields_} for i in range(len(segs))]
    return g, slots.copy(), edges.copy(), seg_list


def _same_layout(ctx, tr, load=0.0, versatile=False):
    g, hs, he, hg = _host_arrays(tr, load, versatile)
    ctx.build_store(tr, load_factor=load, versatile=versatile)
    ds, de, dg = ctx.export_store()
    assert dg == hg
    assert de.shape == he.shape and np.array_equal(de, he)
    assert ds.shape == hs.shape and np.array_equal(ds, hs)
    g.close()


@pytest.mark.parametrize("orgs,load,zipf,versatile", [(20, 0.0, False, False), (6, 1.0, False, False),
                                                      (10, 0.0, True, False), (8, 0.0, False, True),
                                                      (5, 1.0, True, True)])
def test_device_build_matches_host_build(orgs, load, zipf, versatile):
    tr, _ = wk.synth_generate(orgs, seed=2, zipf=zipf)
    with wk.Context(0) as ctx:
        _same_layout(ctx, tr, load, versatile)


def test_device_build_duplicates_and_filtered_triples():
    """Repeated triples (the loader dedups), a PREDICATE_ID triple (never a key), a type-id
    object of another predicate (no IN key), in an order the sort has to fix."""
    tr, v = wk.synth_generate(4, seed=5)
    rng = np.random.default_rng(1)
    extra = np.concatenate([tr[rng.integers(0, len(tr), 3000)],
                            np.array([[tr[0, 0], 0, tr[1, 0]], [tr[2, 0], v["p_takes"], 5]], np.uint32)])
    mixed = np.concatenate([tr, extra])[rng.permutation(len(tr) + len(extra))]
    with wk.Context(0) as ctx:
        _same_layout(ctx, mixed)
        _same_layout(ctx, mixed, versatile=True)


def test_queries_on_device_built_store(graph20):
    v, o = graph20["vocab"], graph20["oracle"]
    with wk.Context(0) as ctx:
        ctx.build_store(graph20["triples"])
        qs = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
        qs += workloads.light_queries(v, graph20["instances"], 100, seed=13)
        for q in qs:
            st, want, _ = o.run(q.flat(), q.nvars)
            got, _ = ctx.execute(q, wk.MODE_RESIDENT)
            assert st == 0 and np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
        for q, (t, st) in zip(qs[2:], ctx.batch(qs[2:])):
            _, want, _ = o.run(q.flat(), q.nvars)
            assert st == 0 and np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))


def test_empty_and_refused_builds():
    with wk.Context(0) as ctx:
        ctx.build_store(np.zeros((0, 3), np.uint32))
        t, _ = ctx.execute(wk.Query([(1 << 17, 5, wk.OUT, -1)]), wk.MODE_PLAIN)
        assert t.shape[0] == 0
        with pytest.raises(wk.WukongError) as e:
            ctx.build_store(np.zeros((4, 3), np.uint32), load_factor=2.0)
        assert e.value.code == wk.E_BADARG


@pytest.mark.parametrize("load", [0.0, 1.0])
def test_upload_then_export_gives_the_uploaded_bytes(load):
    """The device copy keeps every one-entry list in its key's own pointer word (the entry with
    the pointer type 3, the original word kept aside); the export still gives back exactly the
    bytes that were uploaded, and queries still answer as the oracle does through every probe
    form and the flat passes."""
    tr, v = wk.synth_generate(12, seed=7)
    g, hs, he, hg = _host_arrays(tr, load, False)
    o = oracle.OracleStore(tr)
    with wk.Context(0) as ctx:
        ctx.upload_gstore(g)
        ds, de, dg = ctx.export_store()
        assert dg == hg and np.array_equal(de, he) and np.array_equal(ds, hs)
        inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
        qs = workloads.light_queries(v, inst, 300, seed=9)
        heavy = [workloads.heavy_star(v), workloads.heavy_triangle(v)]
        for lanes, flat_rows in ((1, 0), (1, 1), (2, 1), (8, 0)):
            ctx.tune_set(wk.KNOB_LANES, lanes)
            ctx.tune_set(wk.KNOB_BATCH_LANES, lanes)
            ctx.tune_set(wk.KNOB_FLAT_ROWS, flat_rows)
            ctx.tune_set(wk.KNOB_BATCH_FLAT, 63 if flat_rows else 0)
            for q, (t, st) in zip(qs + heavy, ctx.batch(qs) + [ctx.execute(h, wk.MODE_RESIDENT) for h in heavy]):
                ost, want, _ = o.run(q.flat(), q.nvars)
                assert ost == 0 and np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))
    g.close()
