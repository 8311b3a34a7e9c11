"""CHECKER OF THE ORACLE — test infrastructure only: ctypes wrapper of oracle/_ref/libwkref.so,
the reference's own CPU engine (src/core/engine/sparql.hpp and the headers it includes, compiled
unmodified from the reference tree by oracle/Makefile against oracle/refpin/stubs).

The golden-fixture script (tests/golden/make_ref_golden.py), tests and bench.py's reference arm
use it.  The library exists only where the reference tree was present when it was built (it
travels with the repository to a machine without that tree).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "_ref", "libwkref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.wkref_graph_new.restype = P
        L.wkref_graph_free.argtypes = [P]
        L.wkref_graph_put.argtypes = [P, C.c_uint32, C.c_uint32, C.c_int, P, C.c_uint64]
        L.wkref_query.argtypes = [P, P, C.c_int, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                  C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_int), P]
        L.wkref_free.argtypes = [P]
        L.wkref_graph_from_store.restype = P
        L.wkref_graph_from_store.argtypes = [P, C.c_uint64, P, P, C.c_uint64]
        L.wkref_query_many.argtypes = [P, P, P, P, C.c_uint32, C.c_int, P, P]
        L.wkref_query_mt.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64)]
        L.wkref_pattern.argtypes = [P, P, C.c_uint64, C.c_int, C.c_int, P, C.c_int, C.c_int,
                                    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_int), P]
        L.wkref_filter_bound.argtypes = [P, C.c_uint64, C.c_int, P, C.c_int,
                                         C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class RefGraph:
    """A graph the reference engine reads: every key's list as given (get_triples / get_index),
    or, with `store` (an oracle.OracleStore, kept alive here), that GStore's arrays in place,
    probed the way the reference's store probes them."""

    def __init__(self, store=None, arrays=None):
        """store: an oracle.OracleStore; arrays: (slots pointer, slot count, edges pointer,
        segment rows uint64[k,10]) of any store in the GStore layout, whose owner the caller
        keeps alive."""
        self.store = store
        if store is not None:
            arrays = store.arrays()
        if arrays is None:
            self.h = lib().wkref_graph_new()
        else:
            sp, ns, ep, segs = arrays
            self._segs = np.ascontiguousarray(segs, dtype=np.uint64)
            self.h = lib().wkref_graph_from_store(sp, ns, ep, _p(self._segs), self._segs.shape[0])

    def run_split(self, query_flat, nvars, mt_factor):
        """One query with its index start split into mt_factor sub-queries, each on its own
        engine and host thread, merged by the first engine's reply map.  Returns (status,
        rows of the final table)."""
        q = np.ascontiguousarray(query_flat, dtype=np.int32)
        rows = C.c_uint64()
        rc = lib().wkref_query_mt(self.h, _p(q), q.size // 5, nvars, mt_factor, C.byref(rows))
        return rc, rows.value

    def run_many(self, flat_list, nvars_list, threads):
        """Queries through execute_sparql_query on `threads` threads, one engine each.  Returns
        (row counts, statuses)."""
        pats = np.ascontiguousarray(np.concatenate([np.asarray(f, np.int32).reshape(-1) for f in flat_list]),
                                    dtype=np.int32)
        offs = np.zeros(len(flat_list) + 1, np.int32)
        offs[1:] = np.cumsum([np.asarray(f).size // 5 for f in flat_list])
        nv = np.ascontiguousarray(nvars_list, dtype=np.int32)
        rows = np.zeros(len(flat_list), np.uint64)
        st = np.zeros(len(flat_list), np.int32)
        lib().wkref_query_many(self.h, _p(pats), _p(offs), _p(nv), len(flat_list), threads, _p(rows), _p(st))
        return rows, st

    def put(self, vid, pid, d, vals):
        vals = np.ascontiguousarray(vals, dtype=np.uint32)
        lib().wkref_graph_put(self.h, vid, pid, d, _p(vals), vals.size)

    def close(self):
        if self.h:
            lib().wkref_graph_free(self.h)
            self.h = None

    __del__ = close

    def pattern(self, table, nvars, pattern, mt_tid=0, mt_factor=1):
        """One pattern through the engine's dispatch over a given table (column i = variable
        -(i + 1)), as the first pattern of a group that inherited it.  Returns (status, table,
        v2c)."""
        t = np.ascontiguousarray(table, dtype=np.uint32)
        if t.ndim == 1:
            t = t.reshape(-1, 1)
        pat = np.ascontiguousarray(pattern, dtype=np.int32)
        out = C.POINTER(C.c_uint32)()
        rows = C.c_uint64()
        cols = C.c_int()
        v2c = np.zeros(max(nvars, 1), np.int32)
        rc = lib().wkref_pattern(self.h, _p(t), t.shape[0], t.shape[1], nvars, _p(pat), mt_tid,
                                 mt_factor, C.byref(out), C.byref(rows), C.byref(cols), _p(v2c))
        if rc:
            return rc, None, None
        n = rows.value * cols.value
        try:
            r = np.ctypeslib.as_array(out, shape=(max(n, 1),))[:n].copy().reshape(rows.value, cols.value)
        finally:
            lib().wkref_free(out)
        return 0, r, list(v2c[:nvars])

    def run(self, query_flat, nvars, required=None, distinct=False, limit=-1, offset=0):
        """Run one planned query through SPARQLEngine::execute_sparql_query.
        Returns (status, table, v2c)."""
        q = np.ascontiguousarray(query_flat, dtype=np.int32)
        req = np.array(required if required is not None else [-(i + 1) for i in range(nvars)], np.int32)
        tab = C.POINTER(C.c_uint32)()
        rows = C.c_uint64()
        cols = C.c_int()
        v2c = np.zeros(max(nvars, 1), np.int32)
        rc = lib().wkref_query(self.h, _p(q), q.shape[0], nvars, _p(req), req.size, int(distinct),
                               limit, offset, C.byref(tab), C.byref(rows), C.byref(cols), _p(v2c))
        if rc:
            return rc, None, None
        n = rows.value * cols.value
        try:
            t = np.ctypeslib.as_array(tab, shape=(max(n, 1),))[:n].copy().reshape(rows.value, cols.value)
        finally:
            lib().wkref_free(tab)
        return 0, t, list(v2c[:nvars])


def graph_from_store(store, triples, vocab):
    """A RefGraph holding every key of `triples` with the lists `store` (anything with
    get_triples / get_index) answers: normal keys [s|p|OUT], [o|p|IN] (type triples only OUT),
    the type index [0|t|IN] and the predicate indexes [0|p|IN], [0|p|OUT]; and, from a store
    built versatile, every vertex's predicate lists [v|PREDICATE_ID|OUT], [v|PREDICATE_ID|IN]."""
    g = RefGraph()
    seen = set()
    versatile = getattr(store, "versatile", False)
    for s, p, o in triples:
        s, p, o = int(s), int(p), int(o)
        keys = [(s, p, 1), (o, p, 0)]
        if versatile:
            keys += [(s, 0, 1), (o, 0, 0)]
        for key in keys:
            if key[2] == 0 and 1 < key[0] < (1 << 17):
                continue   # a type id object is never an IN key
            if key[2] == 0 and p == 1 and key[1] != 0:
                continue
            if key not in seen:
                seen.add(key)
                g.put(key[0], key[1], key[2], store.get_triples(*key))
    preds = sorted(set(int(x) for x in np.unique(triples[:, 1])))
    types = sorted(set(int(x) for x in np.unique(triples[triples[:, 1] == 1][:, 2])))
    for t in types:
        g.put(0, t, 0, store.get_index(t, 0))
    for p in preds:
        if p == 1:
            continue
        for d in (0, 1):
            g.put(0, p, d, store.get_index(p, d))
    return g


def bound_vars(query_flat):
    """The variables a planned pattern list binds, in the order their columns are added (the
    object of an index or constant start, the object of each known_to_unknown step, and an
    unknown predicate's variable before its object's, as the versatile operators add them).
    Asking the final stage for exactly these keeps its projection (sparql.hpp:1500-1529) the
    identity, so the reference's table is the pattern stage's table."""
    bound = []
    for s, p, o, d, t in np.asarray(query_flat).reshape(-1, 5):
        if p < 0 and p not in bound:
            bound.append(int(p))
        if o < 0 and o not in bound:
            bound.append(int(o))
    return bound


def filter_bound(table, bound_cols):
    """The reference engine's filter stage with one BOUND filter per column of bound_cols, on a
    given row-major uint32 table (execute_filter, sparql.hpp:1356-1376)."""
    t = np.ascontiguousarray(table, dtype=np.uint32)
    cols = np.array(bound_cols, np.int32)
    out = C.POINTER(C.c_uint32)()
    rows = C.c_uint64()
    rc = lib().wkref_filter_bound(_p(t), t.shape[0], t.shape[1], _p(cols), cols.size, C.byref(out),
                                  C.byref(rows))
    if rc:
        raise RuntimeError("reference filter status %d" % rc)
    n = rows.value * t.shape[1]
    try:
        return np.ctypeslib.as_array(out, shape=(max(n, 1),))[:n].copy().reshape(rows.value, t.shape[1])
    finally:
        lib().wkref_free(out)
