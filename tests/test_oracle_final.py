"""Known answers for the oracle's restatement of final_process (sparql.hpp:1419-1546), worked
out by hand from the reference's steps, so the device parity tests compare against a pinned
checker."""
import numpy as np

import oracle


def _t(rows):
    return np.array(rows, dtype=np.uint32).reshape(-1, len(rows[0]) if rows else 1)


def test_distinct_sorts_signed_and_keeps_first_of_each_run():
    # ids past 2^31 are negative in the reference's int table, so they sort first
    t = _t([[5, 1], [3, 2], [5, 1], [2**31, 2], [3, 9]])
    assert oracle.final_process(t, [0], distinct=True).tolist() == [[2**31], [3], [5]]
    assert oracle.final_process(t, [0, 1], distinct=True).tolist() == [[2**31, 2], [3, 2], [3, 9], [5, 1]]


def test_runs_are_judged_on_the_required_columns_only():
    # sorted by (c0, c1): (1,7) (1,8) (2,7); required column c1 only: neighbours 7, 8, 7 all
    # differ, so all three stay, in sorted order
    t = _t([[2, 7], [1, 8], [1, 7]])
    assert oracle.final_process(t, [1], distinct=True).tolist() == [[7], [8], [7]]


def test_offset_limit_projection_in_table_order():
    t = _t([[1, 10], [2, 20], [3, 30], [4, 40]])
    assert oracle.final_process(t, [1, 0], offset=1, limit=2).tolist() == [[20, 2], [30, 3]]
    assert oracle.final_process(t, [0], offset=9).shape == (0, 1)
    assert oracle.final_process(t, [0], limit=0).shape == (0, 1)


def test_empty_table_is_left_as_it_is():
    t = np.zeros((0, 3), dtype=np.uint32)
    assert oracle.final_process(t, [1], distinct=True).shape == (0, 3)
