"""Host-side store builder and plan dispatch, checked against the oracle on CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def all_keys(tr):
    keys = set()
    for s, p, o in tr:
        keys.add((int(s), int(p), 1))
        if not (1 < o < (1 << 17)):
            keys.add((int(o), int(p), 0))
    return sorted(keys)


def test_synth_counts(graph20):
    tr, v = graph20["triples"], graph20["vocab"]
    # ~13.5k triples per organisation by the generator's distributions
    assert 20 * 11000 < tr.shape[0] < 20 * 16000
    assert tr[:, 0].min() >= (1 << 17)
    assert set(np.unique(tr[:, 1])) == {1, v["p_sub_org_of"], v["p_member_of"], v["p_takes"],
                                        v["p_degree_from"], v["p_author"]}
    # deterministic: same seed, same graph
    import wukong_b200 as wk
    tr2, _ = wk.synth_generate(20, seed=0)
    assert np.array_equal(tr, tr2)
    tr3, _ = wk.synth_generate(20, seed=1)
    assert not np.array_equal(tr[:1000], tr3[:1000])


def test_every_key_matches_oracle(graph20):
    g, o = graph20["gstore"], graph20["oracle"]
    keys = all_keys(graph20["triples"])
    rng = np.random.default_rng(0)
    pick = rng.choice(len(keys), size=min(len(keys), 30000), replace=False)
    for i in pick:
        vid, p, d = keys[i]
        assert np.array_equal(g.get_triples(vid, p, d), o.get_triples(vid, p, d)), (vid, p, d)


def test_index_lists_match_oracle_as_multisets(graph20):
    g, o, v = graph20["gstore"], graph20["oracle"], graph20["vocab"]
    for t in range(2, v["p_author"] + 1):
        for d in (0, 1):
            assert np.array_equal(np.sort(g.get_index(t, d)), np.sort(o.get_index(t, d))), (t, d)


def test_chained_buckets(built):
    """A full load factor forces slot-7 chains; every key must still be found."""
    import oracle
    import wukong_b200 as wk
    tr, _ = wk.synth_generate(3, seed=7)
    g = wk.GStore(tr, load_factor=1.0)
    slots, edges, segs = g.arrays()
    chains = sum(int(slots[b * 8 + 7, 0] != 0) for b in range(slots.shape[0] // 8))
    assert chains > 0
    o = oracle.OracleStore(tr)
    for vid, p, d in all_keys(tr)[::7]:
        assert np.array_equal(g.get_triples(vid, p, d), o.get_triples(vid, p, d))


def test_duplicates_and_separate_directions(built):
    import oracle
    import wukong_b200 as wk
    V = 1 << 17
    tr = np.array([(V + 1, 5, V + 2), (V + 1, 5, V + 2), (V + 1, 5, V + 3), (V + 4, 5, V + 2),
                   (V + 1, 1, 7)], np.uint32)
    g, o = wk.GStore(tr), oracle.OracleStore(tr)
    for st in (g, o):
        assert list(st.get_triples(V + 1, 5, 1)) == [V + 2, V + 3]    # dedup, ascending
        assert list(st.get_triples(V + 2, 5, 0)) == [V + 1, V + 4]
        assert list(st.get_triples(V + 1, 1, 1)) == [7]
        assert sorted(st.get_index(7, 0)) == [V + 1]                  # type index
        assert sorted(st.get_index(5, 0)) == [V + 1, V + 4]           # subjects of 5
        assert sorted(st.get_index(5, 1)) == [V + 2, V + 3]           # objects of 5
    empty = np.zeros((0, 3), np.uint32)
    g0 = wk.GStore(empty)
    assert g0.get_triples(V, 5, 1).size == 0
    assert g0.info()["keys"] == 0


def test_plan_dispatch_statuses(built):
    """GPUEngine::execute_one_pattern's dispatch, checked without a device against the oracle."""
    import oracle
    import wukong_b200 as wk
    V = 1 << 17
    tr = np.array([(V + 1, 5, V + 2), (V + 2, 6, V + 3), (V + 1, 1, 7)], np.uint32)
    o = oracle.OracleStore(tr)
    cases = {
        "ok_chain": ([(V + 1, 5, 1, -1), (-1, 6, 1, -2)], 0),
        "ok_index": ([(7, 1, 0, -1), (-1, 5, 1, -2)], 0),
        "index_bad_pred": ([(7, 5, 0, -1)], wk.OBJ_ERROR),
        "unknown_subject": ([(-1, 5, 1, -2)], wk.UNKNOWN_SUB),
        "const_not_first": ([(V + 1, 5, 1, -1), (V + 2, 6, 1, -2)], wk.FIRST_PATTERN_ERROR),
        "const_const": ([(V + 1, 5, 1, V + 2)], wk.UNKNOWN_PATTERN),
        "versatile": ([(V + 1, -2, 1, -1)], wk.UNKNOWN_PATTERN),
        "var_out_of_range": ([(V + 1, 5, 1, -9)], wk.VERTEX_INVALID),
    }
    for name, (pats, want) in cases.items():
        q = wk.Query(pats, nvars=2)
        rc, v2c, cols = wk.validate(q)
        assert rc == want, name
        st, tab, ov2c = o.run(q.flat(), q.nvars)
        assert st == want, name
        if want == 0:
            assert list(v2c) == list(ov2c), name
    rc, v2c, cols = wk.validate(wk.Query([(V + 1, 5, 1, -1), (-1, 6, 1, -2), (-1, 5, 1, -2)], nvars=2))
    assert rc == 0 and cols == 2 and v2c == [0, 1]


def test_capi_exports_every_declared_symbol(built):
    """The C ABI library loads and exports every function include/wukong_b200.h declares."""
    import wukong_b200 as wk
    hdr = open(os.path.join(ROOT, "include", "wukong_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(wk_[a-z0-9_]+)\s*\(", hdr))
    assert len(names) > 30
    L = C.CDLL(wk.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(wk.exported_symbols()) <= names


@pytest.mark.parametrize("versatile", [False, True])
def test_random_plans_dispatch_like_the_oracle(built, versatile):
    """Seeded random pattern lists (constants, variables bound or not, index starts, both
    directions, out-of-range variables, unknown predicates): the library's host-side dispatch
    (wk_query_validate_ex) gives the oracle's status and, on success, its column map, for a
    store without and with the vertex-predicate lists."""
    import oracle
    import wukong_b200 as wk
    V = 1 << 17
    tr = np.array([(V + 1, 5, V + 2), (V + 2, 6, V + 3), (V + 1, 1, 7), (V + 3, 5, V + 1),
                   (V + 2, 1, 7), (V + 3, 6, V + 2)], np.uint32)
    o = oracle.OracleStore(tr, versatile=versatile)
    rng = np.random.default_rng(11)
    consts = [V + 1, V + 2, V + 3, 7]
    seen = set()
    for _ in range(600):
        nvars = int(rng.integers(1, 4))
        pats = []
        for k in range(int(rng.integers(1, 5))):
            def term():
                if rng.random() < 0.5:
                    return -int(rng.integers(1, nvars + 2))   # may be past nvars
                return int(rng.choice(consts))
            s = term()
            p = int(rng.choice([5, 6, wk.TYPE_ID, wk.PREDICATE_ID, -1]))
            d = int(rng.integers(0, 2))
            pats.append((s, p, d, term()))
        q = wk.Query(pats, nvars=nvars)
        rc, v2c, cols = wk.validate(q, versatile=versatile)
        st, tab, ov2c = o.run(q.flat(), q.nvars)
        assert rc == st, (pats, nvars, rc, st)
        if st == 0:
            assert list(v2c) == list(ov2c), pats
            assert cols == tab.shape[1], pats
        seen.add(st)
    assert len(seen) >= 4   # the sample reaches several outcomes, success among them
    assert 0 in seen


def test_generator_library_matches_the_product(built):
    import wukong_b200 as wk
    """libwk_synth.so (the generator alone, used where the product must not be loaded) makes the
    same triples and vocabulary as the product library, uniform and Zipf-skewed."""
    for zipf in (False, True):
        a, va = wk.synth_generate(7, seed=3, zipf=zipf)
        b, vb = wk.synth_generate(7, seed=3, zipf=zipf, generator_only=True)
        assert va == vb
        assert np.array_equal(a, b)
