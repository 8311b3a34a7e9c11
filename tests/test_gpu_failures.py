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


def test_device_waits_run_out_and_context_recovers(ctx, graph20):
    """The real bounded waits, not a fake: with the spin limit at two polls (knob 6), a tile's
    look-back on a predecessor that has not published yet, or a CTA left without tiles that
    waits for the slice queue, gives up, sets the timeout bit and returns.  The call reports
    WK_E_TIMEOUT; with the default limit back the same context answers correctly."""
    v = graph20["vocab"]
    o = graph20["oracle"]
    persons = np.asarray(graph20["instances"][v["t_person_a"]], np.uint32).reshape(-1, 1)
    assert persons.shape[0] > 8 * 256   # many tiles, far fewer than the launch's CTAs
    want = o.step(0, persons, 0, v["p_takes"], wk.OUT)
    tin = ctx.table(persons, capacity=persons.size)
    out = ctx.table(capacity=want.size + 64)
    ctx.tune_set(wk.KNOB_SPIN_LIMIT, 2)
    try:
        codes = []
        for _ in range(5):
            codes.append(wk.lib().wk_step_known_to_unknown(ctx.h, tin.h, 0, v["p_takes"], wk.OUT, out.h))
            if codes[-1] == wk.E_TIMEOUT:
                break
        assert wk.E_TIMEOUT in codes, codes
        assert set(codes) <= {wk.SUCCESS, wk.E_TIMEOUT}, codes
    finally:
        ctx.tune_set(wk.KNOB_SPIN_LIMIT, 0)
    assert ctx.tune_get(wk.KNOB_SPIN_LIMIT) == 1 << 24
    ctx.known_to_unknown(tin, 0, v["p_takes"], wk.OUT, out)
    assert _same(out.download(), want)
    q = workloads.heavy_star(v)
    _, qwant, _ = o.run(q.flat(), q.nvars)
    got, _ = ctx.execute(q, wk.MODE_GRAPH)
    assert _same(got, qwant)
    for t in (tin, out):
        t.free()
