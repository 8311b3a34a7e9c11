"""The dataset and plan readers (wk_load_id_dir, wk_plan_apply_fmt) against their restatements in
oracle/, and end to end: a dataset written as id_ files and read back builds the same store, and
a .fmt plan gives the query the planner would run."""
import os

import numpy as np
import pytest

import oracle
import wukong_b200 as wk


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)


def test_id_dir_reads_like_the_posix_loader(tmp_path, built):
    d = str(tmp_path)
    _write(os.path.join(d, "id_b.nt"), "7 8 9\n10 11 12\n")
    _write(os.path.join(d, "id_a.nt"), "1 2 3   4 5\n6\n13 14")          # incomplete last triple
    _write(os.path.join(d, "id_c.nt"), "20 21 22\n23 x 24\n25 26 27\n")  # stops at "x"
    _write(os.path.join(d, "id_d.nt"), "4294967295 0 1\n4294967296 1 2\n")   # past 2^32 - 1
    _write(os.path.join(d, "attr_a.nt"), "99 99 99\n")                   # not a data file
    _write(os.path.join(d, ".id_hidden"), "98 98 98\n")                   # dot entry
    _write(os.path.join(d, "str_index"), "97 97 97\n")
    got = wk.load_id_dir(d)
    want = oracle.read_id_dir(d)
    assert np.array_equal(got, want)
    assert got.tolist() == [[1, 2, 3], [4, 5, 6], [7, 8, 9], [10, 11, 12], [20, 21, 22],
                            [4294967295, 0, 1]]
    # trailing slash or not, the same files
    assert np.array_equal(wk.load_id_dir(d + "/"), got)


def test_id_dir_errors_and_empty(tmp_path, built):
    with pytest.raises(wk.WukongError) as e:
        wk.load_id_dir(str(tmp_path / "missing"))
    assert e.value.code == wk.E_BADARG
    assert wk.load_id_dir(str(tmp_path)).shape == (0, 3)


def test_dataset_round_trip_builds_the_same_store(tmp_path, built):
    tr, v = wk.synth_generate(3, seed=5)
    parts = np.array_split(tr, 3)
    for i, part in enumerate(parts):
        np.savetxt(os.path.join(str(tmp_path), "id_%02d.nt" % i), part, fmt="%d")
    back = wk.load_id_dir(str(tmp_path))
    assert np.array_equal(back, tr)
    a = wk.GStore(tr)
    b = wk.GStore(back)
    sa, ea, _ = a.arrays()
    sb, eb, _ = b.arrays()
    assert np.array_equal(sa, sb) and np.array_equal(ea, eb)


WRITTEN = [(-1, 5, -2), (-2, 6, 17), (3, 7, -1)]   # ?x p5 ?y . ?y p6 <17> . <3> p7 ?x


@pytest.mark.parametrize("fmt", [
    "1 >\n2 >\n3 >\n",
    "# plan\n\n{\n3 <\n1 >\n2 >\n}\n",
    "2 <\n1 <\n3 >\n",
    "1 <<\n1 >\n2\n3 >>\n",          # predicate-index starts; "2" keeps the previous direction
    "3 ?\n1>\n2 >  trailing words\n",   # an unknown direction leaves the pattern as written
    "1 >\n2 >\n3 >\n}\n9 >\n",       # "}" ends the group
])
def test_fmt_matches_restatement(fmt, built):
    q = wk.plan_fmt(WRITTEN, fmt)
    assert q.patterns == oracle.apply_fmt(WRITTEN, fmt, wk.PREDICATE_ID, wk.IN, wk.OUT)


def test_fmt_refusals(built):
    with pytest.raises(wk.WukongError) as e:      # fewer lines than patterns
        wk.plan_fmt(WRITTEN, "1 >\n2 >\n")
    assert e.value.code == wk.E_BADARG and oracle.apply_fmt(WRITTEN, "1 >\n2 >\n") is None
    for bad in ("1 >\n2 >\n4 >\n", "1 >\nabc\n3 >\n", "0 >\n1 >\n2 >\n"):   # names no pattern
        with pytest.raises(wk.WukongError) as e:
            wk.plan_fmt(WRITTEN, bad)
        assert e.value.code == wk.E_BADARG
        with pytest.raises(ValueError):
            oracle.apply_fmt(WRITTEN, bad)
    with pytest.raises(wk.WukongError) as e:
        wk.plan_fmt(WRITTEN, "1 >\nunion {\n2 >\n}\n3 >\n")
    assert e.value.code == wk.E_UNSUPPORTED


def test_fmt_plan_runs_like_the_hand_planned_query(graph20, built):
    v = graph20["vocab"]
    o = graph20["oracle"]
    # ?p memberOf ?u . ?p type PersonA, planned from the type index ("<" turns the type pattern
    # around) and from memberOf's predicate index ("<<" reuses a pattern as the index start)
    written = [(-1, v["p_member_of"], -2), (-1, wk.TYPE_ID, v["t_person_a"])]
    cases = [("2 <\n1 >\n", [(v["t_person_a"], wk.TYPE_ID, wk.IN, -1), (-1, v["p_member_of"], wk.OUT, -2)]),
             ("1 <<\n1 >\n2 >\n", [(v["p_member_of"], wk.PREDICATE_ID, wk.IN, -1),
                                    (-1, v["p_member_of"], wk.OUT, -2),
                                    (-1, wk.TYPE_ID, wk.OUT, v["t_person_a"])])]
    for fmt, hand in cases:
        q = wk.plan_fmt(written, fmt)
        assert q.patterns == hand
        st, t, _ = o.run(q.flat(), q.nvars)
        assert st == 0 and t.shape[0] > 0
