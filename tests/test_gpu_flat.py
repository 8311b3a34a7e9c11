"""The flat count / scan / expand pipeline for large single-query steps (wk_flat.cu).

The flat threshold (knob 4) decides which launch runs a step of an index-start plan or a
single step.  Every threshold, including ones that split a plan between the two launches on
the device, must give the oracle's tables; so must overflow reruns through the flat pipeline.
"""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


@pytest.fixture
def knobs(ctx):
    old = [ctx.tune_get(k) for k in range(5)]
    yield ctx
    for k, v in enumerate(old):
        ctx.tune_set(k, v)


def _heavy(v):
    return [workloads.heavy_star(v), workloads.heavy_star(v, v["t_person_b"]), workloads.heavy_triangle(v),
            wk.Query([(v["t_org"], wk.TYPE_ID, wk.IN, -1), (-1, wk.TYPE_ID, wk.OUT, -2),
                      (-2, wk.TYPE_ID, wk.IN, -3)]),                                  # type index k2u
            wk.Query([(v["p_takes"], wk.PREDICATE_ID, wk.IN, -1), (-1, v["p_takes"], wk.OUT, -2),
                      (-2, wk.TYPE_ID, wk.OUT, v["t_course"])])]                      # k2c


@pytest.mark.parametrize("threshold", [1, 2000, 20000, 0])
def test_index_plans_match_oracle_at_every_threshold(knobs, graph20, threshold):
    ctx = knobs
    o = graph20["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, threshold)
    for q in _heavy(graph20["vocab"]):
        st, want, _ = o.run(q.flat(), q.nvars)
        assert st == 0
        for mode in (wk.MODE_PLAIN, wk.MODE_RESIDENT, wk.MODE_GRAPH):
            got, _ = ctx.execute(q, mode)
            assert got.shape == want.shape, (threshold, mode)
            assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want)), (threshold, mode)


def test_flat_output_order_equals_tile_order(knobs, graph20):
    """Both launches write rows in row-major then edge order: identical tables, not only multisets."""
    ctx = knobs
    for q in _heavy(graph20["vocab"]):
        ctx.tune_set(wk.KNOB_FLAT_ROWS, 0)
        tile, _ = ctx.execute(q, wk.MODE_RESIDENT)
        ctx.tune_set(wk.KNOB_FLAT_ROWS, 1)
        flat, _ = ctx.execute(q, wk.MODE_RESIDENT)
        assert np.array_equal(tile, flat)


def test_single_steps_through_flat(knobs, graph20):
    ctx = knobs
    v = graph20["vocab"]
    o = graph20["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, 1)
    persons = np.asarray(graph20["instances"][v["t_person_a"]], np.uint32)
    courses = np.asarray(graph20["instances"][v["t_course"]], np.uint32)
    rng = np.random.default_rng(5)
    pairs = np.stack([rng.choice(persons, 4000), rng.choice(courses, 4000)], axis=1).astype(np.uint32)
    pairs[::97, 0] = 0xFFFFFFFF   # blank rows produce nothing
    tin = ctx.table(pairs, capacity=pairs.size)
    out = ctx.table(capacity=16)  # too small: the step grows it and reruns
    ctx.known_to_unknown(tin, 0, v["p_takes"], wk.OUT, out)
    want = o.step(0, pairs, 0, v["p_takes"], wk.OUT)
    assert np.array_equal(out.download(), want)
    ctx.known_to_known(tin, 0, 1, v["p_takes"], wk.OUT, out)
    want = o.step(1, pairs, 0, v["p_takes"], wk.OUT, ce=1)
    assert np.array_equal(out.download(), want)
    ctx.known_to_const(tin, 1, v["t_course"], wk.TYPE_ID, wk.OUT, out)
    want = o.step(2, pairs, 1, wk.TYPE_ID, wk.OUT, end_const=v["t_course"])
    assert np.array_equal(out.download(), want)
    empty = ctx.table(np.zeros((0, 2), np.uint32), capacity=8)
    ctx.known_to_unknown(empty, 0, v["p_takes"], wk.OUT, out)
    assert out.shape() == (0, 3)
    for t in (tin, out, empty):
        t.free()


def test_small_tables_overflow_and_rerun_in_flat(knobs, graph20):
    ctx = knobs
    v = graph20["vocab"]
    o = graph20["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, 1)
    with wk.Context(0, rbuf_bytes=4096) as c2:
        c2.upload_gstore(graph20["gstore"])
        c2.tune_set(wk.KNOB_FLAT_ROWS, 1)
        for q in _heavy(v):
            _, want, _ = o.run(q.flat(), q.nvars)
            for mode in (wk.MODE_RESIDENT, wk.MODE_GRAPH):
                got, _ = c2.execute(q, mode)
                assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))


@pytest.mark.parametrize("cols", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("rows", [1, 3, 1021, 6000])
def test_flat_expand_widths(knobs, graph20, cols, rows):
    """known_to_unknown through the flat passes at output widths 2-6: short lists (the courses
    a person takes) and long ones (the persons of a unit), blank rows, at row counts below, at
    and well past one expand window, the table equal to the oracle's row for row."""
    ctx = knobs
    v = graph20["vocab"]
    o = graph20["oracle"]
    ctx.tune_set(wk.KNOB_FLAT_ROWS, 1)
    rng = np.random.default_rng(100 * cols + rows)
    persons = np.asarray(graph20["instances"][v["t_person_a"]], np.uint32)
    units = np.asarray(graph20["instances"][v["t_unit"]], np.uint32)
    for start, pid, d in ((persons, v["p_takes"], wk.OUT), (units, v["p_member_of"], wk.IN)):
        tab = rng.integers(1 << 17, 1 << 20, size=(rows, cols), dtype=np.uint64).astype(np.uint32)
        cs = int(rng.integers(0, cols))
        tab[:, cs] = rng.choice(start, rows)
        tab[::13, cs] = 0xFFFFFFFF
        tin = ctx.table(tab, capacity=tab.size)
        out = ctx.table(capacity=16)
        ctx.known_to_unknown(tin, cs, pid, d, out)
        want = o.step(0, tab, cs, pid, d)
        got = out.download()
        tin.free()
        out.free()
        assert got.shape == want.shape, (cols, rows, pid)
        assert np.array_equal(got, want), (cols, rows, pid)
