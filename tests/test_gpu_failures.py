"""Failure handling without a GPU fault: errors are injected on the host (wk_debug_fail_next)
at the point where the context reads its device error word, so the host's handling runs as for
a real device-side error.  Every failure must come back as a status, and the context must give
correct results right afterwards."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu

OVERFLOW, TIMEOUT, CORRUPT = 1, 2, 4


def _fail_next(ctx, bits):
    assert wk.lib().wk_debug_fail_next(ctx.h, bits) == 0


def _same(got, want):
    return np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))


@pytest.mark.parametrize("mode", [wk.MODE_PLAIN, wk.MODE_RESIDENT, wk.MODE_GRAPH])
def test_query_errors_surface_and_context_recovers(ctx, graph20, mode):
    v = graph20["vocab"]
    q = workloads.heavy_star(v)
    _, want, _ = graph20["oracle"].run(q.flat(), q.nvars)
    for bits, code in ((TIMEOUT, wk.E_TIMEOUT), (CORRUPT, wk.E_CORRUPT)):
        _fail_next(ctx, bits)
        with pytest.raises(wk.WukongError) as e:
            ctx.execute(q, mode)
        assert e.value.code == code
        got, _ = ctx.execute(q, mode)   # the context is usable right away
        assert _same(got, want)
    _fail_next(ctx, OVERFLOW)           # an overflow is not an error: grow and rerun
    got, _ = ctx.execute(q, mode)
    assert _same(got, want)


def test_batch_and_serving_errors(ctx, graph20):
    v = graph20["vocab"]
    o = graph20["oracle"]
    qs = workloads.light_queries(v, graph20["instances"], 200, seed=81)
    _fail_next(ctx, TIMEOUT)
    with pytest.raises(wk.WukongError) as e:
        ctx.batch(qs)
    assert e.value.code == wk.E_TIMEOUT
    for q, (t, st) in zip(qs, ctx.batch(qs)):
        _, want, _ = o.run(q.flat(), q.nvars)
        assert st == 0 and _same(t, want)
    _fail_next(ctx, CORRUPT)
    with pytest.raises(wk.WukongError) as e:
        ctx.serve(qs, np.zeros(len(qs)))
    assert e.value.code == wk.E_CORRUPT
    for q, r in zip(qs, ctx.serve(qs, np.zeros(len(qs)))):
        _, want, _ = o.run(q.flat(), q.nvars)
        assert r[1] == 0 and _same(r[0], want)


def test_bad_injection_bits_are_refused(ctx):
    assert wk.lib().wk_debug_fail_next(ctx.h, 8) == wk.E_BADARG
