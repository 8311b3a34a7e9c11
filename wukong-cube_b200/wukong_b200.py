"""ctypes binding of libwukong_b200.so (include/wukong_b200.h).

A thin host-side mirror of the reference's GPU engine interface for Python callers (tests,
bench): ``Context`` plays GPUEngine/GPUAgent (src/gpu/gpu_engine.hpp, gpu_agent.hpp), ``Query``
is a planned SPARQLQuery pattern list (src/core/sparql/query.hpp:145-170) and every call raises
``WukongError`` carrying the status code of src/core/common/errors.hpp when the library fails.
The library must be built (``python wukong-cube_b200/wk_build.py``); there is no fallback path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# WK_LIB_PATH selects another build of the library (e.g. an instrumented variant)
LIB_PATH = os.environ.get("WK_LIB_PATH") or os.path.join(HERE, "libwukong_b200.so")

IN, OUT = 0, 1
PREDICATE_ID, TYPE_ID = 0, 1
NO_RESULT = 0xFFFF
MODE_PLAIN, MODE_RESIDENT, MODE_GRAPH = 0, 1, 2
KNOB_LANES, KNOB_BATCH_LANES, KNOB_SLICE_ROWS, KNOB_BATCH_SLICE_ROWS, KNOB_FLAT_ROWS = 0, 1, 2, 3, 4
KNOB_BATCH_FLAT = 5
KNOB_SPIN_LIMIT = 6

SUCCESS = 0
UNKNOWN_PATTERN = 3
ATTR_DISABLE = 4
NO_REQUIRED_VAR = 5
OBJ_ERROR = 7
VERTEX_INVALID = 8
UNKNOWN_SUB = 9
FIRST_PATTERN_ERROR = 11
E_OOM, E_CAPACITY, E_TIMEOUT, E_BADARG, E_CUDA, E_NOSTORE, E_CORRUPT, E_UNSUPPORTED = range(100, 108)


class WukongError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("wukong status %d: %s" % (code, msg))
        self.code = code


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_cols", C.c_int32), ("rbuf_bytes", C.c_uint64),
                ("working_set_cap_bytes", C.c_uint64), ("tune", C.c_int32),
                ("reserved", C.c_int32 * 7)]


class SegMeta(C.Structure):
    _fields_ = [("index", C.c_int32), ("pid", C.c_uint32), ("dir", C.c_int32),
                ("reserved", C.c_uint32), ("num_keys", C.c_uint64), ("num_buckets", C.c_uint64),
                ("bucket_start", C.c_uint64), ("num_edges", C.c_uint64),
                ("edge_start", C.c_uint64), ("ext_start", C.c_uint64), ("ext_num", C.c_uint64)]


class Pattern(C.Structure):
    _fields_ = [("subject", C.c_int32), ("predicate", C.c_int32), ("object", C.c_int32),
                ("direction", C.c_int32), ("pred_type", C.c_int32)]


class QueryC(C.Structure):
    _fields_ = [("patterns", C.POINTER(Pattern)), ("n_patterns", C.c_int32),
                ("nvars", C.c_int32), ("mt_tid", C.c_int32), ("mt_factor", C.c_int32)]


class SynthParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_orgs", C.c_uint32), ("zipf", C.c_int32),
                ("zipf_s", C.c_double)]


class SynthVocab(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "t_org", "t_unit", "t_person_a", "t_person_b", "t_person_c", "t_course", "t_doc",
        "p_sub_org_of", "p_member_of", "p_takes", "p_degree_from", "p_author",
        "first_vid", "next_vid")]


class ServeConfig(C.Structure):
    _fields_ = [("working_set_cap_bytes", C.c_uint64), ("arena_bytes", C.c_uint64),
                ("min_proj_bytes", C.c_uint64), ("lane_table_bytes", C.c_uint64),
                ("max_inflight", C.c_uint32), ("max_heavy_inflight", C.c_uint32),
                ("light_ctas_per_sm", C.c_int32), ("blind", C.c_int32), ("reserved", C.c_int32 * 2)]


class TuneResult(C.Structure):
    _fields_ = [("batch_lanes", C.c_int32), ("batch_slice_rows", C.c_int32), ("lanes", C.c_int32),
                ("slice_rows", C.c_int32), ("batch_ms_default", C.c_double),
                ("batch_ms_tuned", C.c_double), ("single_ms_default", C.c_double),
                ("single_ms_tuned", C.c_double), ("candidates", C.c_int32),
                ("batch_flat", C.c_int32), ("reserved", C.c_int32 * 2)]


class StepProf(C.Structure):
    _fields_ = [("kind", C.c_int32), ("cols_in", C.c_int32), ("cols_out", C.c_int32),
                ("reserved", C.c_int32), ("rows_in", C.c_uint64), ("rows_out", C.c_uint64),
                ("sum_deg", C.c_uint64), ("alg_bytes", C.c_uint64), ("ms", C.c_double)]


STEP_KINDS = ["index_to_unknown", "const_to_unknown", "known_to_unknown", "known_to_known",
              "known_to_const", "batch_level", "batch_setup", "batch_result_scan", "batch_gather"]


def _prof_list(arr, n):
    return [{"kind": STEP_KINDS[arr[i].kind], "cols_in": arr[i].cols_in,
             "cols_out": arr[i].cols_out, "rows_in": arr[i].rows_in, "rows_out": arr[i].rows_out,
             "sum_deg": arr[i].sum_deg, "alg_bytes": arr[i].alg_bytes, "ms": arr[i].ms}
            for i in range(n)]


class QResult(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("elem_offset", C.c_uint64), ("cols", C.c_int32),
                ("status", C.c_int32), ("t_arrive_us", C.c_double), ("t_done_us", C.c_double)]


_lib = None

# name -> (restype, argtypes)
_P = C.c_void_p
_SIGS = {
    "wk_strerror": (C.c_char_p, [C.c_int]),
    "wk_last_error": (C.c_char_p, [_P]),
    "wk_synth_generate": (C.c_int, [C.POINTER(SynthParams), C.POINTER(C.POINTER(C.c_uint32)),
                                    C.POINTER(C.c_uint64), C.POINTER(SynthVocab)]),
    "wk_free": (None, [_P]),
    "wk_load_id_dir": (C.c_int, [C.c_char_p, C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]),
    "wk_plan_apply_fmt": (C.c_int, [C.POINTER(Pattern), C.c_int32, C.c_char_p, C.POINTER(Pattern),
                                    C.c_int32, C.POINTER(C.c_int32)]),
    "wk_gstore_build": (C.c_int, [_P, C.c_uint64, _P, C.c_uint64, C.c_double, C.POINTER(_P)]),
    "wk_gstore_build_ex": (C.c_int, [_P, C.c_uint64, _P, C.c_uint64, C.c_double, C.c_int32, C.POINTER(_P)]),
    "wk_gstore_free": (None, [_P]),
    "wk_gstore_info": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "wk_gstore_arrays": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "wk_gstore_get_triples": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int32,
                                        C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]),
    "wk_gstore_get_index": (C.c_int, [_P, C.c_uint32, C.c_int32,
                                      C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]),
    "wk_ctx_create": (C.c_int, [C.POINTER(Config), C.POINTER(_P)]),
    "wk_ctx_destroy": (C.c_int, [_P]),
    "wk_ctx_sync": (C.c_int, [_P]),
    "wk_ctx_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "wk_ctx_check": (C.c_int, [_P]),
    "wk_store_upload": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint64]),
    "wk_store_upload_gstore": (C.c_int, [_P, _P]),
    "wk_store_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "wk_store_build_device": (C.c_int, [_P, _P, C.c_uint64, C.c_double, C.c_int32]),
    "wk_store_export": (C.c_int, [_P, _P, C.c_uint64, _P, C.c_uint64, C.POINTER(SegMeta), C.c_uint32,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "wk_table_alloc": (C.c_int, [_P, C.c_uint64, C.POINTER(_P)]),
    "wk_table_free": (C.c_int, [_P, _P]),
    "wk_table_upload": (C.c_int, [_P, _P, _P, C.c_uint64, C.c_int32]),
    "wk_table_final_process": (C.c_int, [_P, _P, C.POINTER(C.c_int32), C.c_int32, C.c_int32,
                                         C.c_int64, C.c_int64, _P]),
    "wk_table_download": (C.c_int, [_P, _P, _P, C.c_uint64]),
    "wk_table_filter_bound": (C.c_int, [_P, _P, C.POINTER(C.c_int32), C.c_int32, _P]),
    "wk_table_shape": (C.c_int, [_P, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]),
    "wk_table_device_ptr": (C.c_int, [_P, _P, C.POINTER(_P)]),
    "wk_step_index_to_unknown": (C.c_int, [_P, C.c_uint32, C.c_int32, C.c_int32, C.c_int32, _P]),
    "wk_step_const_to_unknown": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int32, _P]),
    "wk_step_known_to_unknown": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_int32, _P]),
    "wk_step_known_to_known": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_uint32, C.c_int32, _P]),
    "wk_step_known_to_const": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, _P]),
    "wk_step_known_to_unknown_noalloc": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_int32, _P]),
    "wk_step_const_to_known": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, _P]),
    "wk_step_index_to_known": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_int32, C.c_int32, C.c_int32, _P]),
    "wk_step_known_unknown_unknown": (C.c_int, [_P, _P, C.c_int32, C.c_int32, _P]),
    "wk_step_known_unknown_const": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_int32, _P]),
    "wk_step_const_unknown_unknown": (C.c_int, [_P, C.c_uint32, C.c_int32, _P]),
    "wk_step_const_unknown_const": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int32, _P]),
    "wk_query_validate_ex": (C.c_int, [C.POINTER(QueryC), C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32)]),
    "wk_query_execute": (C.c_int, [_P, C.POINTER(QueryC), C.c_int32, C.POINTER(_P),
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_uint64)]),
    "wk_query_execute_host": (C.c_int, [_P, C.POINTER(QueryC), C.c_int32, _P, C.c_uint64,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_uint64)]),
    "wk_query_enqueue": (C.c_int, [_P, C.POINTER(QueryC), C.c_int32]),
    "wk_query_profile": (C.c_int, [_P, C.POINTER(QueryC), C.c_int32, C.POINTER(StepProf),
                                   C.c_int32, C.POINTER(C.c_int32)]),
    "wk_query_validate": (C.c_int, [C.POINTER(QueryC), C.c_int32, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32)]),
    "wk_batch_execute": (C.c_int, [_P, C.POINTER(QueryC), C.c_uint32, _P, C.c_uint64,
                                   C.POINTER(QResult)]),
    "wk_batch_execute_stream": (C.c_int, [_P, C.POINTER(QueryC), C.c_uint32, C.c_uint32, _P,
                                          C.c_uint64, C.POINTER(QResult)]),
    "wk_batch_execute_device": (C.c_int, [_P, C.POINTER(QueryC), C.c_uint32,
                                          C.POINTER(C.c_uint64)]),
    "wk_batch_replay": (C.c_int, [_P]),
    "wk_debug_phase_cycles": (C.c_int, [C.POINTER(C.c_ulonglong), C.c_int32, C.c_int32]),
    "wk_debug_fail_next": (C.c_int, [_P, C.c_uint32]),
    "wk_debug_device_allocs": (C.c_int, [C.POINTER(C.c_uint64)]),
    "wk_ctx_tune_set": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "wk_ctx_tune_get": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32)]),
    "wk_ctx_autotune": (C.c_int, [_P, C.POINTER(QueryC), C.c_uint32, C.c_int32, C.POINTER(TuneResult)]),
    "wk_measure_random_reads": (C.c_int, [_P, C.c_uint64, C.c_int32, C.POINTER(C.c_double)]),
    "wk_batch_profile": (C.c_int, [_P, C.POINTER(QueryC), C.c_uint32, C.c_int32,
                                   C.POINTER(StepProf), C.c_int32, C.POINTER(C.c_int32)]),
    "wk_serve_run_open_loop": (C.c_int, [_P, C.POINTER(ServeConfig), C.POINTER(QueryC),
                                         C.c_uint32, _P, _P, C.c_uint64, C.POINTER(QResult)]),
}


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libwukong_b200.so is not built: run wukong-cube_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGS)


def _check(rc, ctx=None):
    if rc != SUCCESS:
        L = lib()
        msg = L.wk_strerror(rc).decode()
        if ctx is not None:
            detail = L.wk_last_error(ctx).decode()
            if detail:
                msg += " (" + detail + ")"
        raise WukongError(rc, msg)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


# ---------------------------------------------------------------- synthetic graph + host store
SYNTH_LIB_PATH = os.path.join(HERE, "libwk_synth.so")
_synth_lib = None


def _synth_only_lib():
    """The generator's own small library (libwk_synth.so: wk_synth.cpp alone)."""
    global _synth_lib
    if _synth_lib is None:
        if not os.path.exists(SYNTH_LIB_PATH):
            raise RuntimeError("libwk_synth.so is not built: run wukong-cube_b200/wk_build.py")
        L = C.CDLL(SYNTH_LIB_PATH)
        for name in ("wk_synth_generate", "wk_free"):
            f = getattr(L, name)
            f.restype, f.argtypes = _SIGS[name]
        _synth_lib = L
    return _synth_lib


def synth_generate(n_orgs, seed=0, zipf=False, zipf_s=1.1, generator_only=False):
    """Seeded LUBM-shaped triples as an (n, 3) uint32 array and the id vocabulary.

    generator_only: use libwk_synth.so (the generator alone) instead of the product library,
    so that a process that only needs the workload does not load the product."""
    L = _synth_only_lib() if generator_only else lib()
    p = SynthParams(seed, n_orgs, 1 if zipf else 0, zipf_s)
    buf = C.POINTER(C.c_uint32)()
    n = C.c_uint64()
    v = SynthVocab()
    _check(L.wk_synth_generate(C.byref(p), C.byref(buf), C.byref(n), C.byref(v)))
    try:
        arr = np.ctypeslib.as_array(buf, shape=(n.value * 3,)).copy().reshape(-1, 3)
    finally:
        L.wk_free(buf)
    vocab = {f: getattr(v, f) for f, _ in SynthVocab._fields_}
    return arr, vocab


def load_id_dir(path):
    """The triples of an ID-format dataset directory (its id_* files) as an (n, 3) uint32
    array, read as the reference's POSIX loader reads them (wk_load_id_dir)."""
    L = lib()
    buf = C.POINTER(C.c_uint32)()
    n = C.c_uint64()
    _check(L.wk_load_id_dir(os.fsencode(path), C.byref(buf), C.byref(n)))
    try:
        arr = np.ctypeslib.as_array(buf, shape=(max(n.value, 1) * 3,))[:n.value * 3].copy()
    finally:
        L.wk_free(buf)
    return arr.reshape(-1, 3)


def plan_fmt(written, fmt_text, nvars=None):
    """A Query from a pattern group in written order [(subject, predicate, object), ...] and a
    user-defined plan (.fmt text), ordered and oriented as the reference's planner applies
    such a file (wk_plan_apply_fmt)."""
    src = (Pattern * max(len(written), 1))()
    for i, (s, p, o) in enumerate(written):
        src[i] = Pattern(int(s), int(p), int(o), OUT, 0)
    cap = max(len(fmt_text.splitlines()), 1)
    out = (Pattern * cap)()
    n = C.c_int32()
    _check(lib().wk_plan_apply_fmt(src, len(written), fmt_text.encode(), out, cap, C.byref(n)))
    return Query([(out[i].subject, out[i].predicate, out[i].direction, out[i].object)
                  for i in range(n.value)], nvars=nvars)


class GStore:
    """Host-built static segment store (SegmentRDFGraph::init_gstore layout)."""

    def __init__(self, pso, pos=None, load_factor=0.0, versatile=False):
        """versatile: also every vertex's predicate lists (wk_gstore_build_ex), which the
        unknown-predicate patterns read."""
        L = lib()
        pso = np.ascontiguousarray(pso, dtype=np.uint32)
        pos = pso if pos is None else np.ascontiguousarray(pos, dtype=np.uint32)
        h = C.c_void_p()
        _check(L.wk_gstore_build_ex(_ptr(pso), pso.shape[0], _ptr(pos), pos.shape[0],
                                    load_factor, 1 if versatile else 0, C.byref(h)))
        self.h = h
        self.versatile = bool(versatile)

    def close(self):
        if self.h:
            lib().wk_gstore_free(self.h)
            self.h = None

    __del__ = close

    def info(self):
        s, e, k = C.c_uint64(), C.c_uint64(), C.c_uint64()
        g = C.c_uint32()
        _check(lib().wk_gstore_info(self.h, C.byref(s), C.byref(e), C.byref(g), C.byref(k)))
        return {"slots": s.value, "edges": e.value, "segments": g.value, "keys": k.value}

    def arrays(self):
        """(slots uint64[n,2], edges uint32[n], segs SegMeta array) views into the store."""
        info = self.info()
        sp, ep, gp = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(lib().wk_gstore_arrays(self.h, C.byref(sp), C.byref(ep), C.byref(gp)))
        slots = np.ctypeslib.as_array(C.cast(sp, C.POINTER(C.c_uint64)),
                                      shape=(max(info["slots"], 1) * 2,))[:info["slots"] * 2]
        edges = (np.ctypeslib.as_array(C.cast(ep, C.POINTER(C.c_uint32)), shape=(info["edges"],))
                 if info["edges"] else np.zeros(0, np.uint32))
        segs = (SegMeta * info["segments"]).from_address(gp.value)
        return slots.reshape(-1, 2), edges, segs

    def get_triples(self, vid, pid, d):
        p = C.POINTER(C.c_uint32)()
        n = C.c_uint64()
        _check(lib().wk_gstore_get_triples(self.h, vid, pid, d, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)

    def get_index(self, tpid, d):
        p = C.POINTER(C.c_uint32)()
        n = C.c_uint64()
        _check(lib().wk_gstore_get_index(self.h, tpid, d, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)


# ---------------------------------------------------------------- queries
class Query:
    """A planned pattern list: [(subject, predicate, direction, object), ...] with variables
    numbered -1, -2, ... as in SPARQLQuery (query.hpp:418-440)."""

    def __init__(self, patterns, nvars=None, mt_tid=0, mt_factor=1):
        self.patterns = [tuple(int(x) for x in p) for p in patterns]
        if nvars is None:
            ids = [x for p in self.patterns for x in (p[0], p[1], p[3]) if x < 0]
            nvars = -min(ids) if ids else 0
        self.nvars = nvars
        self.mt_tid = mt_tid
        self.mt_factor = mt_factor

    def flat(self):
        """n x 5 int32 (subject, predicate, object, direction, pred_type) for the oracle."""
        return np.array([[s, p, o, d, 0] for (s, p, d, o) in self.patterns], dtype=np.int32).reshape(-1, 5)

    def as_c(self):
        arr = (Pattern * max(len(self.patterns), 1))()
        for i, (s, p, d, o) in enumerate(self.patterns):
            arr[i] = Pattern(s, p, o, d, 0)
        q = QueryC(arr, len(self.patterns), self.nvars, self.mt_tid, self.mt_factor)
        q._keep = arr
        return q


PHASES = ["claim", "stage", "probe_tail", "scan", "lookback", "ranges", "write", "drain",
          "probe_setup", "probe_walk", "membership", "spare"]


def device_allocs():
    """Device allocations the library has made in this process (wk_debug_device_allocs)."""
    n = C.c_uint64()
    _check(lib().wk_debug_device_allocs(C.byref(n)))
    return n.value


def phase_cycles(reset=True):
    """Per-phase cycle totals of the exploration launch (instrumented builds only)."""
    arr = (C.c_ulonglong * len(PHASES))()
    _check(lib().wk_debug_phase_cycles(arr, len(PHASES), 1 if reset else 0))
    return dict(zip(PHASES, list(arr)))


def validate(q, max_cols=32, versatile=False):
    """Plan check without a device: (status, v2c_map, col_num); versatile: for a store with the
    vertex-predicate lists (wk_query_validate_ex)."""
    qc = q.as_c()
    v2c = (C.c_int32 * max(q.nvars, 1))()
    cols = C.c_int32()
    rc = lib().wk_query_validate_ex(C.byref(qc), max_cols, 1 if versatile else 0, v2c, C.byref(cols))
    return rc, list(v2c)[:q.nvars], cols.value


def queries_as_c(queries):
    """A contiguous wk_query array for the batch / serving calls."""
    qs = (QueryC * max(len(queries), 1))()
    keep = []
    for i, q in enumerate(queries):
        c = q.as_c()
        keep.append(c._keep)
        qs[i] = c
    return qs, keep


class Table:
    def __init__(self, ctx, capacity_elems=1):
        self.ctx = ctx
        h = C.c_void_p()
        _check(lib().wk_table_alloc(ctx.h, capacity_elems, C.byref(h)), ctx.h)
        self.h = h

    def free(self):
        if self.h:
            lib().wk_table_free(self.ctx.h, self.h)
            self.h = None

    def upload(self, arr):
        arr = np.ascontiguousarray(arr, dtype=np.uint32)
        if arr.ndim == 1:
            arr = arr.reshape(-1, 1)
        _check(lib().wk_table_upload(self.ctx.h, self.h, _ptr(arr), arr.shape[0], arr.shape[1]),
               self.ctx.h)

    def shape(self):
        r, c = C.c_uint64(), C.c_int32()
        _check(lib().wk_table_shape(self.ctx.h, self.h, C.byref(r), C.byref(c)), self.ctx.h)
        return r.value, c.value

    def download(self):
        rows, cols = self.shape()
        out = np.zeros(max(rows * cols, 1), dtype=np.uint32)
        _check(lib().wk_table_download(self.ctx.h, self.h, _ptr(out), out.size), self.ctx.h)
        return out[:rows * cols].reshape(rows, cols)

    def final_process(self, keep_cols, distinct=False, offset=0, limit=-1, out=None):
        """The post-pattern stage on the device (wk_table_final_process) into `out` (a new Table
        when None; an existing one is reused, grown when needed)."""
        out = out if out is not None else Table(self.ctx)
        keep = (C.c_int32 * max(len(keep_cols), 1))(*[int(c) for c in keep_cols])
        _check(lib().wk_table_final_process(self.ctx.h, self.h, keep, len(keep_cols),
                                            1 if distinct else 0, offset, limit, out.h), self.ctx.h)
        return out

    def filter_bound(self, bound_cols):
        """The BOUND filters on the device (wk_table_filter_bound) into a new Table."""
        out = Table(self.ctx)
        cols = (C.c_int32 * max(len(bound_cols), 1))(*[int(c) for c in bound_cols])
        _check(lib().wk_table_filter_bound(self.ctx.h, self.h, cols, len(bound_cols), out.h),
               self.ctx.h)
        return out


class Context:
    """One device context (GPUAgent + GPUEngine for one GPU)."""

    def __init__(self, device=0, max_cols=0, rbuf_bytes=0, working_set_cap_bytes=0):
        cfg = Config(device, max_cols, rbuf_bytes, working_set_cap_bytes, 0, (C.c_int32 * 7)())
        h = C.c_void_p()
        _check(lib().wk_ctx_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().wk_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def stream(self):
        s = C.c_void_p()
        _check(lib().wk_ctx_stream(self.h, C.byref(s)), self.h)
        return s.value

    def sync(self):
        _check(lib().wk_ctx_sync(self.h), self.h)

    def check(self):
        _check(lib().wk_ctx_check(self.h), self.h)

    def tune_set(self, knob, value):
        _check(lib().wk_ctx_tune_set(self.h, knob, value), self.h)

    def tune_get(self, knob):
        v = C.c_int32()
        _check(lib().wk_ctx_tune_get(self.h, knob, C.byref(v)), self.h)
        return v.value

    def autotune(self, queries, iters=5):
        """Time every knob setting on these queries and keep the fastest; returns the choice."""
        qs, keep = queries_as_c(queries)
        r = TuneResult()
        _check(lib().wk_ctx_autotune(self.h, qs, len(queries), iters, C.byref(r)), self.h)
        return {k: getattr(r, k) for k, _ in TuneResult._fields_ if k != "reserved"}

    def measure_random_reads(self, region_bytes=8 << 30, iters=5):
        """Independent random 16-byte reads per second from a fresh device buffer of this size
        (the ceiling of probes and short list reads)."""
        v = C.c_double()
        _check(lib().wk_measure_random_reads(self.h, region_bytes, iters, C.byref(v)), self.h)
        return v.value

    def upload_gstore(self, g):
        _check(lib().wk_store_upload_gstore(self.h, g.h), self.h)

    def upload_store(self, segs, slots, edges):
        slots = np.ascontiguousarray(slots, dtype=np.uint64)
        edges = np.ascontiguousarray(edges, dtype=np.uint32)
        n_segs = len(segs)
        _check(lib().wk_store_upload(self.h, C.cast(segs, C.c_void_p), n_segs, _ptr(slots),
                                     slots.size // 2, _ptr(edges), edges.size), self.h)

    def build_store(self, triples, load_factor=0.0, versatile=False):
        """Build the store on the device from (n, 3) id triples (wk_store_build_device)."""
        t = np.ascontiguousarray(triples, dtype=np.uint32).reshape(-1, 3)
        _check(lib().wk_store_build_device(self.h, _ptr(t), t.shape[0], load_factor, 1 if versatile else 0),
               self.h)

    def export_store(self):
        """The context's store as host arrays: (slots uint64[n, 2], edges uint32[m], segs list of
        dicts), in wk_store_upload's layout (wk_store_export)."""
        ns, ne, ng = C.c_uint64(), C.c_uint64(), C.c_uint32()
        L = lib()
        _check(L.wk_store_export(self.h, None, 0, None, 0, None, 0, C.byref(ns), C.byref(ne), C.byref(ng)), self.h)
        slots = np.zeros((max(ns.value, 1), 2), np.uint64)
        edges = np.zeros(max(ne.value, 1), np.uint32)
        segs = (SegMeta * max(ng.value, 1))()
        _check(L.wk_store_export(self.h, _ptr(slots), ns.value, _ptr(edges), ne.value, segs, ng.value,
                                 C.byref(ns), C.byref(ne), C.byref(ng)), self.h)
        seg_list = [{f: getattr(segs[i], f) for f, _ in SegMeta._fields_} for i in range(ng.value)]
        return slots[:ns.value], edges[:ne.value], seg_list

    def store_bytes(self):
        b = C.c_uint64()
        _check(lib().wk_store_bytes(self.h, C.byref(b)), self.h)
        return b.value

    def table(self, arr=None, capacity=1):
        t = Table(self, capacity)
        if arr is not None:
            t.upload(arr)
        return t

    # single steps (GPUEngineCuda::known_to_* analogues)
    def index_to_unknown(self, tpid, d, out, mt_tid=0, mt_factor=1):
        _check(lib().wk_step_index_to_unknown(self.h, tpid, d, mt_tid, mt_factor, out.h), self.h)

    def const_to_unknown(self, vid, pid, d, out):
        _check(lib().wk_step_const_to_unknown(self.h, vid, pid, d, out.h), self.h)

    def known_to_unknown(self, tin, col_start, pid, d, out):
        _check(lib().wk_step_known_to_unknown(self.h, tin.h, col_start, pid, d, out.h), self.h)

    def known_to_known(self, tin, col_start, col_end, pid, d, out):
        _check(lib().wk_step_known_to_known(self.h, tin.h, col_start, col_end, pid, d, out.h), self.h)

    def known_to_const(self, tin, col_start, end_vid, pid, d, out):
        _check(lib().wk_step_known_to_const(self.h, tin.h, col_start, end_vid, pid, d, out.h), self.h)

    def const_to_known(self, tin, col_end, vid, pid, d, out):
        _check(lib().wk_step_const_to_known(self.h, tin.h, col_end, vid, pid, d, out.h), self.h)

    def index_to_known(self, tin, col_end, tpid, d, out, mt_tid=0, mt_factor=1):
        _check(lib().wk_step_index_to_known(self.h, tin.h, col_end, tpid, d, mt_tid, mt_factor, out.h),
               self.h)

    def known_unknown_unknown(self, tin, col_start, d, out):
        _check(lib().wk_step_known_unknown_unknown(self.h, tin.h, col_start, d, out.h), self.h)

    def known_unknown_const(self, tin, col_start, end_vid, d, out):
        _check(lib().wk_step_known_unknown_const(self.h, tin.h, col_start, end_vid, d, out.h), self.h)

    def const_unknown_unknown(self, vid, d, out):
        _check(lib().wk_step_const_unknown_unknown(self.h, vid, d, out.h), self.h)

    def const_unknown_const(self, vid, end_vid, d, out):
        _check(lib().wk_step_const_unknown_const(self.h, vid, end_vid, d, out.h), self.h)

    def execute(self, q, mode=MODE_RESIDENT):
        """Run a whole planned query; returns (table (rows, cols) uint32, v2c_map list)."""
        qc = q.as_c()
        v2c = (C.c_int32 * max(q.nvars, 1))()
        cols = C.c_int32()
        rows = C.c_uint64()
        t = C.c_void_p()
        _check(lib().wk_query_execute(self.h, C.byref(qc), mode, C.byref(t), v2c, C.byref(cols),
                                      C.byref(rows)), self.h)
        n = rows.value * cols.value
        out = np.zeros(max(n, 1), dtype=np.uint32)
        _check(lib().wk_table_download(self.h, t, _ptr(out), out.size), self.h)
        return out[:n].reshape(rows.value, cols.value), list(v2c)[:q.nvars]

    def execute_host(self, q, host_out, mode=MODE_RESIDENT):
        """Run a query and copy its table into host_out (uint32, pinned or not); returns rows, cols."""
        qc = q.as_c()
        v2c = (C.c_int32 * max(q.nvars, 1))()
        cols = C.c_int32()
        rows = C.c_uint64()
        _check(lib().wk_query_execute_host(self.h, C.byref(qc), mode, C.c_void_p(host_out.ctypes.data),
                                           host_out.size, v2c, C.byref(cols), C.byref(rows)), self.h)
        return rows.value, cols.value

    def enqueue(self, q, mode=MODE_GRAPH):
        qc = q.as_c()
        _check(lib().wk_query_enqueue(self.h, C.byref(qc), mode), self.h)

    def profile(self, q, iters=5):
        """Per-step kernel times (CUDA events on the context stream) and sizes."""
        qc = q.as_c()
        arr = (StepProf * 16)()
        n = C.c_int32()
        _check(lib().wk_query_profile(self.h, C.byref(qc), iters, arr, 16, C.byref(n)), self.h)
        return _prof_list(arr, n.value)

    def batch_profile(self, queries, iters=3):
        """Per-level kernel times and algorithmic bytes of a batch."""
        qs, keep = queries_as_c(queries)
        arr = (StepProf * 16)()
        n = C.c_int32()
        _check(lib().wk_batch_profile(self.h, qs, len(queries), iters, arr, 16, C.byref(n)), self.h)
        return _prof_list(arr, n.value)

    def batch(self, queries, cap_elems=None, stream_batch=None):
        """Run queries together; returns list of (table, status).  With stream_batch, the
        queries run as a pipelined stream of batches of that size (wk_batch_execute_stream)."""
        qs, keep = queries_as_c(queries)
        res = (QResult * max(len(queries), 1))()
        if cap_elems is None:
            cap_elems = 1 << 22
        while True:
            out = np.zeros(max(cap_elems, 1), dtype=np.uint32)
            if stream_batch is None:
                rc = lib().wk_batch_execute(self.h, qs, len(queries), _ptr(out), out.size, res)
            else:
                rc = lib().wk_batch_execute_stream(self.h, qs, len(queries), stream_batch, _ptr(out),
                                                   out.size, res)
            if rc == E_CAPACITY and "host buffer" in lib().wk_last_error(self.h).decode():
                cap_elems *= 4
                continue
            _check(rc, self.h)
            break
        tables = []
        for i in range(len(queries)):
            r = res[i]
            n = r.rows * r.cols
            t = out[r.elem_offset:r.elem_offset + n].reshape(r.rows, r.cols) if r.status == 0 else None
            tables.append((t, r.status))
        return tables

    def batch_device(self, queries):
        qs, keep = queries_as_c(queries)
        tot = C.c_uint64()
        _check(lib().wk_batch_execute_device(self.h, qs, len(queries), C.byref(tot)), self.h)
        return tot.value

    def batch_replay(self):
        _check(lib().wk_batch_replay(self.h), self.h)

    def serve(self, queries, arrival_us, cap_elems=1 << 24, **cfg):
        """Continuous batching over an open-loop arrival schedule (microseconds from start).
        Returns [(table or None, status, t_arrive_us, t_done_us, rows)] in query order; with
        blind=1 the tables stay on the device (None here) and only the row counts come back."""
        qs, keep = queries_as_c(queries)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        c = ServeConfig()
        for k, v in cfg.items():
            setattr(c, k, v)
        res = (QResult * max(len(queries), 1))()
        out = np.zeros(max(cap_elems, 1), dtype=np.uint32)
        _check(lib().wk_serve_run_open_loop(self.h, C.byref(c), qs, len(queries), _ptr(arr), _ptr(out),
                                            out.size, res), self.h)
        ret = []
        for i in range(len(queries)):
            r = res[i]
            t = None
            if r.status == 0 and not c.blind:
                t = out[r.elem_offset:r.elem_offset + r.rows * r.cols].reshape(r.rows, r.cols)
            ret.append((t, r.status, r.t_arrive_us, r.t_done_us, r.rows))
        return ret
