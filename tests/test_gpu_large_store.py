"""A store of more than 2^29 buckets, whose slot numbers pass 2^32: every probe form finds the
keys that hash there.

Six thousand subjects each have one rdf:type edge, and a tiny load factor spreads their keys
over about 6.0e8 buckets of the rdf:type OUT segment (about 77 GB of slots), so about 11% of
them have a home bucket at or past 2^29.  rdf:type objects are type ids, which the IN direction
does not store as a normal segment, so that one segment is the only large one.  The rows are
known in advance (each subject's own type), so no oracle is needed."""
import numpy as np
import pytest

import wukong_b200 as wk

pytestmark = pytest.mark.gpu

N = 6000
BUCKETS = (1 << 29) + (1 << 26)   # the rdf:type OUT segment's buckets
NTYPES = 5


def _graph():
    subj = ((1 << 17) + 7 + 11 * np.arange(N, dtype=np.int64)).astype(np.uint32)
    types = (1000 + np.arange(N) % NTYPES).astype(np.uint32)
    tr = np.stack([subj, np.full(N, wk.TYPE_ID, np.uint32), types], axis=1)
    return subj, types, tr


@pytest.fixture(scope="module")
def big(built):
    import torch
    free, _ = torch.cuda.mem_get_info()
    if free < 90e9:
        pytest.skip("needs about 80 GB of free device memory")
    subj, types, tr = _graph()
    c = wk.Context(0)
    try:
        c.build_store(tr, load_factor=N / (7.0 * BUCKETS))
        assert c.store_bytes() >= BUCKETS * 8 * 16   # 16-byte slots, 8 a bucket
        yield c, subj, types
    finally:
        c.close()


# lanes 1: one thread per row; 2/4/8: the group probe; flat: the count pass
SETTINGS = [("lanes", 1), ("lanes", 2), ("lanes", 4), ("lanes", 8), ("flat", 0)]


def _apply(c, kind, lanes):
    c.tune_set(wk.KNOB_FLAT_ROWS, 1 if kind == "flat" else 1 << 30)
    c.tune_set(wk.KNOB_LANES, lanes if kind == "lanes" else 1)


@pytest.mark.parametrize("kind,lanes", SETTINGS)
def test_known_to_unknown_past_bucket_2_29(big, kind, lanes):
    c, subj, types = big
    old = [c.tune_get(k) for k in range(5)]
    # every subject, then ids that are no key (their probes walk to an empty slot)
    absent = ((1 << 17) + 8 + 11 * np.arange(500, dtype=np.int64)).astype(np.uint32)
    col = np.concatenate([subj, absent]).reshape(-1, 1)
    tin = c.table(col)
    out = c.table(capacity=16)
    try:
        _apply(c, kind, lanes)
        c.known_to_unknown(tin, 0, wk.TYPE_ID, wk.OUT, out)
        got = out.download()
    finally:
        for k, val in enumerate(old):
            c.tune_set(k, val)
        tin.free()
        out.free()
    want = np.stack([subj, types], axis=1)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kind,lanes", SETTINGS)
def test_known_to_known_past_bucket_2_29(big, kind, lanes):
    c, subj, types = big
    old = [c.tune_get(k) for k in range(5)]
    rng = np.random.default_rng(7)
    wrong = rng.random(N) < 0.5
    claimed = np.where(wrong, 1000 + (np.arange(N) + 1) % NTYPES, types).astype(np.uint32)
    tab = np.stack([subj, claimed], axis=1)
    tin = c.table(tab)
    out = c.table(capacity=16)
    try:
        _apply(c, kind, lanes)
        c.known_to_known(tin, 0, 1, wk.TYPE_ID, wk.OUT, out)
        got = out.download()
    finally:
        for k, val in enumerate(old):
            c.tune_set(k, val)
        tin.free()
        out.free()
    assert np.array_equal(got, tab[~wrong])
