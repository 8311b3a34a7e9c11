"""Per-step parity of the CUDA path against the oracle (bit-exact, through the C ABI)."""
import numpy as np
import pytest

import oracle
import wukong_b200 as wk

pytestmark = pytest.mark.gpu

BLANK = 0xFFFFFFFF


def _table(rng, start_vals, cols, cs):
    """Random table whose column cs holds start_vals; other columns random ids."""
    n = len(start_vals)
    t = rng.integers(1 << 17, 1 << 20, size=(n, cols), dtype=np.uint64).astype(np.uint32)
    if cols:
        t[:, cs] = start_vals
    return t


def _starts(graph, rng, n, kind):
    inst = graph["instances"]
    v = graph["vocab"]
    pools = {
        "person": np.concatenate([inst[v["t_person_a"]], inst[v["t_person_b"]], inst[v["t_person_c"]]]),
        "unit": inst[v["t_unit"]],
        "org": inst[v["t_org"]],
        "course": inst[v["t_course"]],
    }
    vals = rng.choice(pools[kind], size=n)
    # edge cases: missing vertices, blank, vertex 0, runs of equal consecutive values
    k = max(n // 20, 1)
    idx = rng.choice(n, size=min(4 * k, n), replace=False)
    vals[idx[:k]] = rng.integers(v["next_vid"], v["next_vid"] + 1000, size=len(idx[:k]))
    vals[idx[k:2 * k]] = BLANK
    vals[idx[2 * k:3 * k]] = 0
    if n > 10:
        vals[5:10] = vals[4]
    return vals.astype(np.uint32)


def _gpu_step(ctx, op, tab, cs, pid, d, ce=0, end_const=0):
    tin = ctx.table(tab)
    out = ctx.table(capacity=16)
    try:
        if op == 0:
            ctx.known_to_unknown(tin, cs, pid, d, out)
        elif op == 1:
            ctx.known_to_known(tin, cs, ce, pid, d, out)
        else:
            ctx.known_to_const(tin, cs, end_const, pid, d, out)
        return out.download()
    finally:
        tin.free()
        out.free()


@pytest.mark.parametrize("rows,cols", [(0, 1), (1, 1), (7, 2), (513, 3), (5000, 4), (40000, 2), (300, 31)])
def test_known_to_unknown(ctx, graph20, rows, cols):
    rng = np.random.default_rng(rows * 31 + cols)
    v, o = graph20["vocab"], graph20["oracle"]
    cs = cols // 2
    for kind, pid, d in [("person", v["p_member_of"], wk.OUT), ("person", v["p_takes"], wk.OUT),
                         ("unit", v["p_member_of"], wk.IN), ("org", v["p_degree_from"], wk.IN)]:
        if kind == "org" and rows > 5000:
            continue   # ~900 rows out per row in; keeps the oracle side to seconds
        tab = _table(rng, _starts(graph20, rng, rows, kind), cols, cs)
        want = o.step(0, tab, cs, pid, d)
        got = _gpu_step(ctx, 0, tab, cs, pid, d)
        assert got.shape == want.shape, (kind, pid, d)
        assert np.array_equal(got, want), (kind, pid, d)   # same rows in the same order


def test_known_to_unknown_type_index(ctx, graph20):
    """?t TYPE_ID IN ?x expands a type column through the type index (sparql.hpp:342-345)."""
    rng = np.random.default_rng(3)
    v, o = graph20["vocab"], graph20["oracle"]
    types = rng.integers(0, 12, size=200).astype(np.uint32)
    types[:5] = [v["t_unit"], v["t_org"], 1 << 17, BLANK, 0]
    tab = _table(rng, types, 2, 1)
    want = o.step(0, tab, 1, wk.TYPE_ID, wk.IN)
    got = _gpu_step(ctx, 0, tab, 1, wk.TYPE_ID, wk.IN)
    assert np.array_equal(oracle.sorted_rows(got), oracle.sorted_rows(want))


@pytest.mark.parametrize("rows", [0, 1, 100, 3000, 60000])
def test_known_to_known(ctx, graph20, rows):
    rng = np.random.default_rng(rows + 11)
    v, o, g = graph20["vocab"], graph20["oracle"], graph20["gstore"]
    persons = _starts(graph20, rng, rows, "person")
    units = np.zeros(rows, np.uint32)
    for i, p in enumerate(persons):
        u = g.get_triples(int(p), v["p_member_of"], wk.OUT) if p not in (0, BLANK) else []
        units[i] = u[0] if len(u) and rng.random() < 0.7 else rng.choice(graph20["instances"][v["t_unit"]])
    tab = np.stack([persons, units, rng.integers(0, 1 << 30, size=rows).astype(np.uint32)], axis=1)
    want = o.step(1, tab, 0, v["p_member_of"], wk.OUT, ce=1)
    got = _gpu_step(ctx, 1, tab, 0, v["p_member_of"], wk.OUT, ce=1)
    assert np.array_equal(got, want)
    if rows >= 100:
        assert 0 < got.shape[0] < rows


@pytest.mark.parametrize("rows", [0, 5, 2048, 50000])
def test_known_to_const(ctx, graph20, rows):
    rng = np.random.default_rng(rows + 5)
    v, o = graph20["vocab"], graph20["oracle"]
    tab = _table(rng, _starts(graph20, rng, rows, "person"), 2, 0)
    for pid, d, c in [(wk.TYPE_ID, wk.OUT, v["t_person_b"]),
                      (v["p_degree_from"], wk.OUT, int(graph20["instances"][v["t_org"]][3])),
                      (v["p_takes"], wk.OUT, 12345)]:
        want = o.step(2, tab, 0, pid, d, end_const=c)
        got = _gpu_step(ctx, 2, tab, 0, pid, d, end_const=c)
        assert np.array_equal(got, want), (pid, d, c)


def test_hub_lists(ctx, graph20):
    """Rows whose lists are long (an organisation's alumni) next to rows with empty lists."""
    v, o = graph20["vocab"], graph20["oracle"]
    orgs = graph20["instances"][v["t_org"]]
    starts = np.repeat(orgs[:4], 3).astype(np.uint32)
    tab = np.stack([starts, np.arange(len(starts), dtype=np.uint32)], axis=1)
    want = o.step(0, tab, 0, v["p_degree_from"], wk.IN)
    got = _gpu_step(ctx, 0, tab, 0, v["p_degree_from"], wk.IN)
    assert got.shape[0] > 1000
    assert np.array_equal(got, want)
    # membership deep inside a long list
    alumni = o.get_triples(int(orgs[0]), v["p_degree_from"], wk.IN)
    tab = np.stack([np.full(len(alumni), orgs[0], np.uint32), alumni[::-1]], axis=1)
    want = o.step(1, tab, 0, v["p_degree_from"], wk.IN, ce=1)
    got = _gpu_step(ctx, 1, tab, 0, v["p_degree_from"], wk.IN, ce=1)
    assert got.shape[0] == len(alumni) and np.array_equal(got, want)


def test_index_and_const_starts(ctx, graph20):
    v, o, g = graph20["vocab"], graph20["oracle"], graph20["gstore"]
    out = ctx.table(capacity=4)
    try:
        for t, d in [(v["t_person_a"], wk.IN), (v["p_takes"], wk.IN), (v["p_takes"], wk.OUT), (999, wk.IN)]:
            want = np.sort(o.get_index(t, d))
            ctx.index_to_unknown(t, d, out)
            got = out.download()
            assert got.shape[1] == 1
            assert np.array_equal(np.sort(got[:, 0]), want)
            # mt_factor slices concatenate to the whole list (sparql.hpp:213-224)
            parts = []
            for k in range(3):
                ctx.index_to_unknown(t, d, out, mt_tid=k, mt_factor=3)
                parts.append(out.download()[:, 0])
            assert np.array_equal(np.concatenate(parts), np.asarray(g.get_index(t, d)))
        unit = int(graph20["instances"][v["t_unit"]][0])
        for vid, pid, d in [(unit, v["p_member_of"], wk.IN), (unit, v["p_sub_org_of"], wk.OUT),
                            (unit, 4242, wk.OUT), (v["next_vid"] + 5, v["p_takes"], wk.OUT)]:
            ctx.const_to_unknown(vid, pid, d, out)
            assert np.array_equal(out.download()[:, 0], o.get_triples(vid, pid, d))
    finally:
        out.free()


def test_step_argument_errors(ctx, graph20):
    tin = ctx.table(np.zeros((4, 2), np.uint32))
    out = ctx.table(capacity=4)
    try:
        for f in (lambda: ctx.known_to_unknown(tin, 2, 5, wk.OUT, out),
                  lambda: ctx.known_to_unknown(tin, 0, 5, 3, out),
                  lambda: ctx.known_to_known(tin, 0, -1, 5, wk.OUT, out)):
            with pytest.raises(wk.WukongError) as e:
                f()
            assert e.value.code == wk.E_BADARG
    finally:
        tin.free()
        out.free()
