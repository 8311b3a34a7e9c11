"""wk_step_known_to_unknown_noalloc: the known_to_unknown step with its scan scratch in a fixed
device array and no allocation, called through the C ABI.

Each case runs the existing entry point (wk_step_known_to_unknown) once and the no-alloc one
twice in a row: both no-alloc results must equal the existing one row for row (the second call
reuses the scratch the first one left behind), and the oracle's step as a multiset.  The
library's count of device allocations and the device's free memory do not move across the
no-alloc calls.  Limits are refused with WK_E_CAPACITY, and a refused call leaves the scratch
usable; a table left behind by a refused (overflowed) step is refused with WK_E_CORRUPT as an
input, by this entry point, by the allocating step and by the post-pattern stage alike.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
import wukong_b200 as wk

pytestmark = pytest.mark.gpu

MAX_ROWS = (16384 - 2) * 256


def _noalloc(ctx, tin, cs, pid, d, out):
    return wk.lib().wk_step_known_to_unknown_noalloc(ctx.h, tin.h, cs, pid, d, out.h)


def _err(ctx):
    return wk.lib().wk_last_error(ctx.h).decode()


def _cases(graph):
    v = graph["vocab"]
    inst = graph["instances"]
    persons = np.asarray(inst[v["t_person_a"]], np.uint32)
    courses = np.asarray(inst[v["t_course"]], np.uint32)
    pairs = np.stack([persons[:500], np.resize(courses, 500)], axis=1)
    return [
        ("persons takes", persons.reshape(-1, 1), 0, v["p_takes"], wk.OUT),
        ("courses taken by", courses.reshape(-1, 1), 0, v["p_takes"], wk.IN),
        ("second column", pairs, 1, v["p_takes"], wk.IN),
        # TYPE_ID / IN reads the type index: one row per type, long lists (slice queue)
        ("type index", np.array([[v["t_person_a"]], [v["t_course"]], [v["t_unit"]]], np.uint32),
         0, wk.TYPE_ID, wk.IN),
        ("absent vertices", np.arange(5, 400, dtype=np.uint32).reshape(-1, 1) + (1 << 30), 0,
         v["p_takes"], wk.OUT),
    ]


def test_noalloc_matches_existing_entry_point_twice(ctx, graph20):
    o = graph20["oracle"]
    for name, arr, cs, pid, d in _cases(graph20):
        tin = ctx.table(arr, capacity=arr.size)
        ref_t = ctx.table(capacity=1)
        ctx.known_to_unknown(tin, cs, pid, d, ref_t)   # existing entry point (may grow ref_t)
        ref = ref_t.download()
        want = o.step(0, arr, cs, pid, d)
        assert np.array_equal(oracle.sorted_rows(ref), oracle.sorted_rows(want)), name
        out = ctx.table(capacity=max(ref.size, 1) + 64)
        allocs = wk.device_allocs()
        for call in range(2):
            rc = _noalloc(ctx, tin, cs, pid, d, out)
            assert rc == 0, (name, call, rc, _err(ctx))
            got = out.download()
            assert got.shape == ref.shape, (name, call)
            assert np.array_equal(got, ref), (name, call)   # same rows in the same order
            # the device's free memory is taken after the first call: loading the library's
            # code and its fixed scratch array on first use is the driver's doing, not a call's
            torch.cuda.synchronize()
            if call == 0:
                free = torch.cuda.mem_get_info()[0]
        assert wk.device_allocs() == allocs, name   # the library allocated nothing
        assert torch.cuda.mem_get_info()[0] == free, name
        for t in (tin, ref_t, out):
            t.free()


def test_noalloc_refuses_what_it_cannot_hold(ctx, graph20):
    v = graph20["vocab"]
    persons = np.asarray(graph20["instances"][v["t_person_a"]], np.uint32).reshape(-1, 1)
    tin = ctx.table(persons, capacity=persons.size)
    small = ctx.table(capacity=8)   # far too small for the step's output
    rc = _noalloc(ctx, tin, 0, v["p_takes"], wk.OUT, small)
    assert rc == wk.E_CAPACITY
    assert "rows" in _err(ctx)
    # the refused step left `small` holding the row count it needed, past its capacity: an
    # overflowed table, which no call may read as input
    nxt = ctx.table(capacity=1 << 16)
    assert _noalloc(ctx, small, 1, v["p_takes"], wk.IN, nxt) == wk.E_CORRUPT
    assert wk.lib().wk_step_known_to_unknown(ctx.h, small.h, 1, v["p_takes"], wk.IN, nxt.h) == wk.E_CORRUPT
    keep = (C.c_int32 * 1)(0)
    assert wk.lib().wk_table_final_process(ctx.h, small.h, keep, 1, 1, 0, -1, nxt.h) == wk.E_CORRUPT
    nxt.free()
    big = np.full((MAX_ROWS + 1, 1), 1 << 30, np.uint32)
    tbig = ctx.table(big, capacity=big.size)
    out = ctx.table(capacity=1024)
    rc = _noalloc(ctx, tbig, 0, v["p_takes"], wk.OUT, out)
    assert rc == wk.E_CAPACITY
    assert "at most" in _err(ctx)
    # bad arguments are refused before any device work
    assert _noalloc(ctx, tin, 1, v["p_takes"], wk.OUT, out) == wk.E_BADARG
    assert wk.lib().wk_step_known_to_unknown_noalloc(ctx.h, tin.h, 0, v["p_takes"], 7, out.h) == wk.E_BADARG
    # a refused call leaves the scratch usable: the same step now fits and matches
    ref_t = ctx.table(capacity=1)
    ctx.known_to_unknown(tin, 0, v["p_takes"], wk.OUT, ref_t)
    ref = ref_t.download()
    fit = ctx.table(capacity=ref.size + 64)
    for _ in range(2):
        assert _noalloc(ctx, tin, 0, v["p_takes"], wk.OUT, fit) == 0, _err(ctx)
        assert np.array_equal(fit.download(), ref)
    for t in (tin, small, tbig, out, ref_t, fit):
        t.free()


def test_noalloc_symbol_is_exported(built):
    assert isinstance(wk.lib().wk_step_known_to_unknown_noalloc, C._CFuncPtr)
