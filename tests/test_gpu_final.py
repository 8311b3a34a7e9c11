"""The post-pattern stage on the device (wk_table_final_process) against the restatement of the
reference's final_process in oracle/: DISTINCT (sort by every column as signed 32-bit values,
first of each run equal on the required columns), OFFSET, LIMIT and projection, row for row."""
import numpy as np
import pytest

import oracle
import workloads
import wukong_b200 as wk

pytestmark = pytest.mark.gpu


def _run(ctx, table, keep, distinct, offset, limit):
    t = wk.Table(ctx, max(table.size, 1))
    t.upload(table)
    out = t.final_process(keep, distinct=distinct, offset=offset, limit=limit)
    got = out.download()
    t.free()
    out.free()
    return got


@pytest.mark.parametrize("seed", range(6))
def test_random_tables(ctx, seed):
    rng = np.random.default_rng(seed)
    rows = int(rng.choice([1, 2, 37, 1000, 20000, 70000]))
    cols = int(rng.integers(1, 6))
    # few distinct values per column, some of them past 2^31 (negative as the reference's ints)
    pool = np.array([0, 1, 2, 7, 300, 65536, 2**31 - 1, 2**31, 2**31 + 5, 2**32 - 1], dtype=np.uint64)
    table = pool[rng.integers(0, len(pool), size=(rows, cols))].astype(np.uint32)
    for _ in range(4):
        keep = [int(c) for c in rng.permutation(cols)[:int(rng.integers(1, cols + 1))]]
        distinct = bool(rng.integers(0, 2))
        offset = int(rng.choice([0, 0, 1, 5, rows // 2, rows + 3]))
        limit = int(rng.choice([-1, -1, 0, 1, 10, rows]))
        got = _run(ctx, table, keep, distinct, offset, limit)
        want = oracle.final_process(table, keep, distinct, offset, limit)
        assert got.shape == want.shape, (keep, distinct, offset, limit)
        assert np.array_equal(got, want), (keep, distinct, offset, limit)


def test_query_results(ctx, graph20):
    v = graph20["vocab"]
    for q in (workloads.heavy_star(v), workloads.heavy_triangle(v)):
        table, v2c = ctx.execute(q, wk.MODE_RESIDENT)
        keep = [v2c[1], v2c[0]]   # ?x2 then ?x1, as a SELECT would list them
        for distinct, offset, limit in ((True, 0, -1), (True, 3, 50), (False, 7, 100), (False, 0, -1)):
            got = _run(ctx, table, keep, distinct, offset, limit)
            assert np.array_equal(got, oracle.final_process(table, keep, distinct, offset, limit))


def test_empty_and_refusals(ctx):
    empty = np.zeros((0, 3), dtype=np.uint32)
    t = wk.Table(ctx, 8)
    t.upload(empty)
    out = t.final_process([1], distinct=True)
    assert out.shape() == (0, 3)   # left as it is, columns included
    out.free()
    t.upload(np.arange(12, dtype=np.uint32).reshape(4, 3))
    for keep, code in (([], wk.NO_REQUIRED_VAR), ([3], wk.E_BADARG), ([-1], wk.E_BADARG)):
        with pytest.raises(wk.WukongError) as e:
            t.final_process(keep)
        assert e.value.code == code
    t.free()


@pytest.mark.parametrize("cols,span", [(5, 2**32), (3, 2**22), (4, 3), (2, 1)])
def test_packed_key_chunks(ctx, cols, span):
    """Columns whose ranges need up to 32 bits each (five full-range columns: 160 bits, three
    64-bit key chunks), narrow ones that share one chunk, and constant ones that need none;
    offsets from each column's smallest value in signed order."""
    rng = np.random.default_rng(cols * 7 + 1)
    rows = 50_000
    base = rng.integers(0, 2**32 - span + 1, size=cols, dtype=np.uint64)
    table = (base + rng.integers(0, span, size=(rows, cols), dtype=np.uint64)).astype(np.uint32)
    table[rng.integers(0, rows, size=rows // 3)] = table[:rows // 3]   # repeated rows
    for keep in ([cols - 1], list(range(cols))[::-1], [0]):
        for offset, limit in ((0, -1), (11, 1000)):
            got = _run(ctx, table, keep, True, offset, limit)
            want = oracle.final_process(table, keep, True, offset, limit)
            assert np.array_equal(got, want), (keep, offset, limit)


def test_large_table_many_tiles_per_cta(ctx):
    """3 million rows: every sort CTA scatters several 2,048-row tiles per pass, with long runs
    of equal digits (a narrow column) and rows repeated across tiles."""
    rng = np.random.default_rng(91)
    rows = 3_000_000
    table = np.stack([rng.integers(0, 1 << 20, size=rows), rng.integers(0, 4, size=rows),
                      rng.integers(0, 1 << 26, size=rows)], axis=1).astype(np.uint32)
    table[rng.integers(0, rows, size=rows // 4)] = table[:rows // 4]
    got = _run(ctx, table, [0, 1], True, 0, -1)
    want = oracle.final_process(table, [0, 1], True, 0, -1)
    assert np.array_equal(got, want)


def _signed_sorted(table):
    """The rows in the reference's order: every column as a signed 32-bit value, first column
    most significant."""
    s = table.view(np.int32)
    order = np.lexsort([s[:, c] for c in range(table.shape[1] - 1, -1, -1)])
    return table[order]


@pytest.mark.parametrize("case", ["in_order", "last_pair_swapped", "descending"])
def test_tables_already_in_order(ctx, case):
    """A table already in the sort's order skips the sort; one that is out of order by a single
    pair at its very end, or reversed, does not."""
    rng = np.random.default_rng(11)
    rows = 50000
    pool = np.array([0, 3, 9, 2**17, 2**31 - 1, 2**31, 2**32 - 2, 2**32 - 1], dtype=np.uint64)
    table = _signed_sorted(pool[rng.integers(0, len(pool), size=(rows, 3))].astype(np.uint32))
    if case == "last_pair_swapped":
        k = rows - 2
        while np.array_equal(table[k], table[k + 1]):
            k -= 1
        table[[k, k + 1]] = table[[k + 1, k]]
    elif case == "descending":
        table = np.ascontiguousarray(table[::-1])
    for keep in ([0, 1], [1, 2], [2], [2, 0, 1]):
        got = _run(ctx, table, keep, True, 0, -1)
        want = oracle.final_process(table, keep, True, 0, -1)
        assert np.array_equal(got, want), (case, keep)


@pytest.mark.parametrize("cols", [3, 4])
@pytest.mark.parametrize("edge", [-1, 0, 1])
def test_order_check_at_tile_edges(ctx, cols, edge):
    """The order check stages rows in tiles of 8,192 // cols - 1 row pairs (plus the row after
    them): a table in order but for one pair of distinct rows swapped where a tile ends, where
    the next begins, or one further in, must still go through the sort."""
    rng = np.random.default_rng(12 + cols)
    rows = 30000
    table = _signed_sorted(rng.integers(0, 2**32, size=(rows, cols), dtype=np.uint64).astype(np.uint32))
    k = 3 * (8192 // cols - 1) + edge   # the swapped pair: rows k and k + 1
    assert not np.array_equal(table[k], table[k + 1])
    table[[k, k + 1]] = table[[k + 1, k]]
    keep = [cols - 1, 0]
    got = _run(ctx, table, keep, True, 0, -1)
    want = oracle.final_process(table, keep, True, 0, -1)
    assert np.array_equal(got, want), (cols, edge)
