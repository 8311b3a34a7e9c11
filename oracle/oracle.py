"""ORACLE — test infrastructure only: ctypes wrapper of oracle/liboracle.so.

The C++ restatement of the reference CPU engine (oracle/wukong_oracle.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm import this module; the
product library never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_store_build.restype = P
        L.orc_store_build.argtypes = [P, C.c_uint64, P, C.c_uint64]
        L.orc_store_build2.restype = P
        L.orc_store_build2.argtypes = [P, C.c_uint64, P, C.c_uint64, C.c_int]
        L.orc_pattern.argtypes = [P, P, C.c_uint64, C.c_int, C.c_int, P, C.c_int, C.c_int,
                                  C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_int), P]
        L.orc_store_free.argtypes = [P]
        L.orc_get_triples.argtypes = [P, C.c_uint32, C.c_uint32, C.c_int,
                                      C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]
        L.orc_get_index.argtypes = [P, C.c_uint32, C.c_int,
                                    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]
        L.orc_store_sizes.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_uint64)]
        L.orc_store_export.argtypes = [P, P, P, P]
        L.orc_store_arrays.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.orc_query_run.argtypes = [P, P, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_int), P]
        L.orc_queries_run_parallel.argtypes = [P, P, P, P, C.c_uint32, C.c_int, P, P]
        L.orc_step.argtypes = [P, C.c_int, P, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_uint32,
                               C.c_uint32, C.c_int, C.POINTER(C.POINTER(C.c_uint32)),
                               C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
        L.orc_free.argtypes = [P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class OracleStore:
    """Store built by the reference's construction rules from (s, p, o) triples."""

    def __init__(self, pso, pos=None, versatile=False):
        """versatile: also the vertex-predicate lists [v|PREDICATE_ID|d] the unknown-predicate
        operators read (the reference's default VERSATILE build)."""
        pso = np.ascontiguousarray(pso, dtype=np.uint32)
        pos = pso if pos is None else np.ascontiguousarray(pos, dtype=np.uint32)
        self.versatile = bool(versatile)
        self.h = lib().orc_store_build2(_p(pso), pso.shape[0], _p(pos), pos.shape[0], int(versatile))
        if not self.h:
            raise RuntimeError("oracle store build failed")

    def close(self):
        if self.h:
            lib().orc_store_free(self.h)
            self.h = None

    __del__ = close

    def get_triples(self, vid, pid, d):
        p = C.POINTER(C.c_uint32)()
        n = C.c_uint64()
        rc = lib().orc_get_triples(self.h, vid, pid, d, C.byref(p), C.byref(n))
        if rc:
            raise RuntimeError("oracle lookup status %d" % rc)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)

    def get_index(self, pid, d):
        return self.get_triples(0, pid, d)

    def arrays(self):
        """The store in place, borrowed (valid while this store lives): (slots pointer, slot
        count, edges pointer, segs uint64[k,10])."""
        ns, ne, ng = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().orc_store_sizes(self.h, C.byref(ns), C.byref(ne), C.byref(ng))
        segs = np.zeros((ng.value, 10), np.uint64)
        lib().orc_store_export(self.h, None, None, _p(segs))
        sp, ep = C.c_void_p(), C.c_void_p()
        lib().orc_store_arrays(self.h, C.byref(sp), C.byref(ep))
        return sp.value, ns.value, ep.value, segs

    def export(self):
        """(slots uint64[n,2], edges uint32[m], segs uint64[k,10]) in the store's own layout."""
        ns, ne, ng = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().orc_store_sizes(self.h, C.byref(ns), C.byref(ne), C.byref(ng))
        slots = np.zeros((ns.value, 2), np.uint64)
        edges = np.zeros(max(ne.value, 1), np.uint32)
        segs = np.zeros((ng.value, 10), np.uint64)
        lib().orc_store_export(self.h, _p(slots), _p(edges), _p(segs))
        return slots, edges[:ne.value], segs

    def run(self, query_flat, nvars, mt_factor=1):
        """Run one planned query (n x 5 int32 patterns).  Returns (status, table, v2c)."""
        q = np.ascontiguousarray(query_flat, dtype=np.int32)
        tab = C.POINTER(C.c_uint32)()
        rows = C.c_uint64()
        cols = C.c_int()
        v2c = np.zeros(max(nvars, 1), np.int32)
        rc = lib().orc_query_run(self.h, _p(q), q.shape[0], nvars, mt_factor, C.byref(tab),
                                 C.byref(rows), C.byref(cols), _p(v2c))
        if rc:
            return rc, None, None
        n = rows.value * cols.value
        try:
            t = np.ctypeslib.as_array(tab, shape=(max(n, 1),))[:n].copy().reshape(rows.value, cols.value)
        finally:
            lib().orc_free(tab)
        return 0, t, list(v2c[:nvars])

    def step(self, op, table, cs, pid, d, ce=0, end_const=0):
        """One known_to_* operator over an input table; op 0 = k2u, 1 = k2k, 2 = k2c."""
        t = np.ascontiguousarray(table, dtype=np.uint32)
        out = C.POINTER(C.c_uint32)()
        rows = C.c_uint64()
        cols = C.c_int()
        rc = lib().orc_step(self.h, op, _p(t), t.shape[0], t.shape[1], cs, ce, end_const, pid, d,
                            C.byref(out), C.byref(rows), C.byref(cols))
        if rc:
            raise RuntimeError("oracle step status %d" % rc)
        n = rows.value * cols.value
        try:
            r = np.ctypeslib.as_array(out, shape=(max(n, 1),))[:n].copy().reshape(rows.value, cols.value)
        finally:
            lib().orc_free(out)
        return r

    def pattern(self, table, nvars, pattern, mt_tid=0, mt_factor=1):
        """One pattern (s, p, o, d, pred_type) through the dispatch over a given table whose
        column i holds variable -(i + 1), as the first pattern of a group that inherited the
        table.  Returns (status, table, v2c)."""
        t = np.ascontiguousarray(table, dtype=np.uint32)
        if t.ndim == 1:
            t = t.reshape(-1, 1)
        pat = np.ascontiguousarray(pattern, dtype=np.int32)
        out = C.POINTER(C.c_uint32)()
        rows = C.c_uint64()
        cols = C.c_int()
        v2c = np.zeros(max(nvars, 1), np.int32)
        rc = lib().orc_pattern(self.h, _p(t), t.shape[0], t.shape[1], nvars, _p(pat), mt_tid, mt_factor,
                               C.byref(out), C.byref(rows), C.byref(cols), _p(v2c))
        if rc:
            return rc, None, None
        n = rows.value * cols.value
        try:
            r = np.ctypeslib.as_array(out, shape=(max(n, 1),))[:n].copy().reshape(rows.value, cols.value)
        finally:
            lib().orc_free(out)
        return 0, r, list(v2c[:nvars])

    def run_many(self, flat_list, nvars_list, threads):
        """Run many queries, one per thread at a time; returns (rows, status) arrays."""
        offs = np.zeros(len(flat_list) + 1, np.int32)
        for i, f in enumerate(flat_list):
            offs[i + 1] = offs[i] + f.shape[0]
        pats = np.ascontiguousarray(np.concatenate(flat_list) if flat_list else np.zeros((0, 5)),
                                    dtype=np.int32)
        nv = np.ascontiguousarray(nvars_list, dtype=np.int32)
        rows = np.zeros(len(flat_list), np.uint64)
        status = np.zeros(len(flat_list), np.int32)
        lib().orc_queries_run_parallel(self.h, _p(pats), _p(offs), _p(nv), len(flat_list), threads,
                                       _p(rows), _p(status))
        return rows, status


def sorted_rows(t):
    """Rows of a result table in lexicographic order (the multiset used for parity)."""
    if t is None or t.size == 0:
        return np.zeros((0, 0 if t is None else t.shape[1]), np.uint32)
    idx = np.lexsort(t.T[::-1])
    return t[idx]


# ---------------------------------------------------------------- dataset and plan readers
# Plain-Python restatements of the reference's ID-format reader and .fmt plan reader, the
# checkers of wk_load_id_dir and wk_plan_apply_fmt.

def read_id_dir(path):
    """Triples of a dataset directory as the reference's POSIX loader reads them: entries whose
    name starts with "id_" (dot entries skipped; posix_loader.hpp:49-70, base_loader.hpp:548),
    in sorted path order (base_loader.hpp:236), each file read as "s p o" triples until an
    extraction fails (base_loader.hpp:242-247): a token that is not a number in [0, 2^32) ends
    the file, and an incomplete last triple is dropped.  Returns an (n, 3) uint32 array."""
    src = path if path.endswith("/") else path + "/"
    names = sorted(src + e for e in os.listdir(src) if not e.startswith(".") and e.startswith("id_"))
    out = []
    for name in names:
        with open(name, "rb") as f:
            toks = f.read().split()
        vals = []
        for t in toks:
            if not t.isdigit() or len(t) > 10 or int(t) > 0xFFFFFFFF:
                break
            vals.append(int(t))
        out.extend(vals[:len(vals) - len(vals) % 3])
    return np.array(out, dtype=np.uint32).reshape(-1, 3)


def apply_fmt(written, text, predicate_id=0, in_dir=0, out_dir=1):
    """Planned patterns [(s, p, d, o), ...] from written ones [(s, p, o), ...] and a .fmt text,
    as Planner::set_plan (planner.hpp:723-770) reads it and set_direction
    (planner.hpp:667-699) applies it.  Returns None where set_plan returns false (fewer lines
    than patterns), raises ValueError where the reference would index out of range and
    NotImplementedError for union / optional groups."""
    orders, dirs = [], []
    order, d = 0, ">"
    for raw in text.split("\n"):
        line = raw.strip()
        if not line or line.startswith("#") or line == "{":
            continue
        if line == "}":
            break
        if line.lower().startswith("union") or line.lower().startswith("optional"):
            raise NotImplementedError("nested group")
        parts = line.split()
        head = parts[0]
        i = 1 if head[:1] in "+-" else 0
        j = i
        while j < len(head) and head[j].isdigit():
            j += 1
        if j == i:
            order = 0                         # failed extraction stores 0; dir is untouched
        else:
            order = int(head[:j])
            rest = head[j:] if j < len(head) else (parts[1] if len(parts) > 1 else "")
            if rest:
                d = rest
        orders.append(order)
        dirs.append(d)
    if len(orders) < len(written):
        return None
    planned = []
    for k, dd in zip(orders, dirs):
        if k < 1 or k > len(written):
            raise ValueError("line names no pattern")
        s, p, o = written[k - 1]
        direction = out_dir
        if dd == "<":
            direction, s, o = in_dir, o, s
        elif dd == "<<":
            direction, s, p, o = in_dir, p, predicate_id, s
        elif dd == ">>":
            direction, s, p = out_dir, p, predicate_id
        planned.append((s, p, direction, o))
    return planned


def final_process(table, keep_cols, distinct=False, offset=0, limit=-1):
    """SPARQLEngine::final_process without ORDER BY (sparql.hpp:1419-1546) on a row-major
    uint32 table: an empty table is returned unchanged; with DISTINCT the rows are sorted by all
    columns as signed 32-bit values (ReduceCmp, sparql.hpp:1403-1417) and of each run of
    neighbours equal on the required columns the first is kept; then OFFSET and LIMIT; then the
    projection onto the required columns in their order."""
    t = np.asarray(table, dtype=np.uint32)
    if t.shape[0] == 0:
        return t
    rows = [tuple(int(x) for x in r) for r in t.view(np.int32)]
    if distinct:
        rows.sort()
        kept = [rows[0]]
        for r in rows[1:]:
            if any(r[c] != kept[-1][c] for c in keep_cols):
                kept.append(r)
        rows = kept
    rows = rows[offset:]
    if limit >= 0:
        rows = rows[:limit]
    out = np.array([[r[c] for c in keep_cols] for r in rows], dtype=np.int32).reshape(-1, len(keep_cols))
    return out.view(np.uint32)


BLANK_ID = 0xFFFFFFFF


def bound_filter(table, bound_cols):
    """The BOUND filters of a query: SPARQLEngine::bound_filter (sparql.hpp:1222-1234) for each
    column, ANDed as execute_filter applies them (sparql.hpp:1356-1376): a row is kept when none
    of the columns holds BLANK_ID; kept rows keep their order."""
    t = np.asarray(table, dtype=np.uint32)
    keep = np.ones(t.shape[0], bool)
    for c in bound_cols:
        keep &= t[:, c] != BLANK_ID
    return t[keep]
