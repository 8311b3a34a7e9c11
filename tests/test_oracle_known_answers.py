"""Known-answer checks that pin the oracle and the product's host store builder.

The reference holds no golden vectors for the exploration step; its only known-answer store
test is tests/test_graph.cc (TestRDFGraph, :112-286): 20 mock subjects with predicates 11-20,
types 2-10 and VID_MIN = 1 << 17, loaded as separate pso and pos triple lists.  The assertions
below are that test's non-VERSATILE checks (neighbour lists with exact values, one type per
vertex, predicate index sizes, type index sizes), re-derived against both stores.
"""
import numpy as np
import pytest

VID_MIN = 1 << 17
OUT, IN, TYPE_ID = 1, 0, 1


def mock_triples():
    """test_graph.cc:133-158: pso and pos lists built side by side."""
    pso, pos = [], []
    for s in range(VID_MIN, VID_MIN + 20):
        for i in range(1, 4):
            pso.append((s, (s % 10) + 11, (s % VID_MIN) * 2 + VID_MIN + i))
            pos.append(((s % VID_MIN) * 3 + VID_MIN + i + 1, ((s + 1) % 10) + 11, s))
        pso.append((s, TYPE_ID, (s % 9) + 2))
    return np.array(pso, np.uint32), np.array(pos, np.uint32)


def stores(built):
    import oracle
    import wukong_b200 as wk
    pso, pos = mock_triples()
    return {"oracle": oracle.OracleStore(pso, pos), "product": wk.GStore(pso, pos)}


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_neighbours_with_predicate(built, which):
    st = stores(built)[which]
    for s in range(VID_MIN, VID_MIN + 20):
        e = st.get_triples(s, (s % 10) + 11, OUT)   # test_graph.cc:166-174
        assert e.size == 3
        assert list(e) == [(s % VID_MIN) * 2 + VID_MIN + i + 1 for i in range(3)]
        e = st.get_triples(s, ((s + 1) % 10) + 11, IN)   # :177-185
        assert e.size == 3
        assert list(e) == [(s % VID_MIN) * 3 + VID_MIN + i + 2 for i in range(3)]


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_types_and_indexes(built, which):
    st = stores(built)[which]
    for s in range(VID_MIN, VID_MIN + 20):   # :189-197
        e = st.get_triples(s, TYPE_ID, OUT)
        assert e.size == 1 and e[0] == (s % 9) + 2
    for p in range(11, 21):                  # :200-217
        assert st.get_triples(0, p, IN).size == 2
        assert st.get_triples(0, p, OUT).size == 2
    for t in range(2, 11):                   # :221-227
        assert st.get_triples(0, t, IN).size >= 2


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_missing_keys_are_empty(built, which):
    st = stores(built)[which]
    assert st.get_triples(VID_MIN + 5, 999, OUT).size == 0      # no such predicate
    assert st.get_triples(VID_MIN + 500, 11, OUT).size == 0     # no such vertex
    assert st.get_triples(VID_MIN, TYPE_ID, IN).size == 0      # type triples are never IN keys
    assert st.get_triples(0, 55, IN).size == 0                 # no such index


def test_kvstore_two_keys(built):
    """test_graph.cc:52-110 (TestKVStore): two keys, distinct slots, exact values, absent IN."""
    import oracle
    import wukong_b200 as wk
    tr = np.array([(1000 + VID_MIN, 20, 2000 + VID_MIN), (1001 + VID_MIN, 20, 2001 + VID_MIN)], np.uint32)
    for st in (oracle.OracleStore(tr), wk.GStore(tr)):
        assert list(st.get_triples(1000 + VID_MIN, 20, OUT)) == [2000 + VID_MIN]
        assert list(st.get_triples(1001 + VID_MIN, 20, OUT)) == [2001 + VID_MIN]
        assert st.get_triples(1001 + VID_MIN, 20, IN).size == 0
