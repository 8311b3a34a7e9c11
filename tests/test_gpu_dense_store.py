"""A dense key table (load factor 1.0: about seven keys per bucket) puts most keys past the
first sector and chains many buckets through slot 7.  Every probe path must still find every
key: single queries through the tile launch and the flat pipeline, batches through tile and flat
levels, against the oracle."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dense(built):
    tr, v = wk.synth_generate(20, seed=0)
    g = wk.GStore(tr, load_factor=1.0)
    o = oracle.OracleStore(tr)
    inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    with wk.Context(0) as ctx:
        ctx.upload_gstore(g)
        yield {"ctx": ctx, "gstore": g, "vocab": v, "oracle": o, "instances": inst}


def test_store_is_dense(dense):
    slots, _, _ = dense["gstore"].arrays()
    keys = slots[:, 0].reshape(-1, 8)
    occupied = keys[:, :7] != 0
    per_position = occupied.sum(0)
    assert per_position[2:].sum() > 0.3 * per_position.sum()   # most probes walk past slot 1
    assert (keys[:, 7] != 0).sum() > 100                       # chained buckets


@pytest.mark.parametrize("flat_rows", [0, 1])   # tile launch, flat pipeline
def test_heavy_queries(dense, flat_rows):
    ctx, v, o = dense["ctx"], dense["vocab"], dense["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, flat_rows)
    try:
        for q in (workloads.heavy_star(v), workloads.heavy_triangle(v)):
            st, want, _ = o.run(q.flat(), q.nvars)
            got, _ = ctx.execute(q, wk.MODE_RESIDENT)
            assert st == 0 and np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))
    finally:
        ctx.tune_set(wk.KNOB_FLAT_ROWS, 65536)


@pytest.mark.parametrize("mask", [0, 0xFFFF])   # tile levels, flat levels
def test_light_batch(dense, mask):
    ctx, v, o = dense["ctx"], dense["vocab"], dense["oracle"]
    qs = workloads.light_queries(v, dense["instances"], 1500, seed=61)
    ctx.tune_set(wk.KNOB_BATCH_FLAT, mask)
    try:
        for q, (t, st) in zip(qs, ctx.batch(qs)):
            wst, want, _ = o.run(q.flat(), q.nvars)
            assert st == wst
            if st == 0:
                assert np.array_equal(oracle.sorted_rows(t), oracle.sorted_rows(want))
    finally:
        ctx.tune_set(wk.KNOB_BATCH_FLAT, 0)
