"""Generate tests/golden/ref_engine_20orgs.json: the answers of the REFERENCE's own CPU engine on
the 20-organisation graph.

The answers come from oracle/_ref/libwkref.so: the reference's src/core/engine/sparql.hpp and the
headers it includes, compiled unmodified from the reference tree (oracle/Makefile, target
"ref") against stand-ins for the Boost / TBB / network names the pattern operators do not use.
Each query runs through SPARQLEngine::execute_sparql_query, so the patterns go through the
reference's own dispatch and operators (sparql.hpp:197-552, 932-1055) and the modifiers through
its own final_process (:1419-1546); tables with planted BLANK_IDs go through its filter stage
with BOUND filters (execute_filter, :1356-1376).  The engine reads a graph that serves, for every key, the
list the oracle's store holds (the store's construction is pinned separately by the reference's
tests/test_graph.cc answers, tests/test_oracle_known_answers.py).

The CPU suite checks the oracle against these answers; the GPU suite checks the CUDA path
against the same digests.  Run from the repository root, where the reference tree is present:
    python tests/golden/make_ref_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "wukong-cube_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "oracle", "refpin")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

OUT = os.path.join(HERE, "ref_engine_20orgs.json")


def digest(rows):
    """sha256 of the rows (row-major uint32 little-endian)."""
    a = np.ascontiguousarray(np.asarray(rows).astype("<u4"))
    return hashlib.sha256(a.tobytes()).hexdigest()


def fixture_queries(v, inst):
    import workloads
    import wukong_b200 as wk
    units = inst[v["t_unit"]]
    qs = [("small_chain", workloads.small_chain(v, int(units[0]))),
          ("small_chain_last_unit", workloads.small_chain(v, int(units[-1]))),
          ("heavy_star", workloads.heavy_star(v)),
          ("heavy_star_person_b", workloads.heavy_star(v, v["t_person_b"])),
          ("heavy_star_person_c", workloads.heavy_star(v, v["t_person_c"])),
          ("heavy_triangle", workloads.heavy_triangle(v)),
          # known_to_unknown on TYPE_ID / IN reads the type index (sparql.hpp:342-345)
          ("type_of_then_instances", wk.Query([(int(units[0]), 1, wk.OUT, -1),
                                               (-1, 1, wk.IN, -2)])),
          ("unknown_subject", wk.Query([(-1, v["p_takes"], wk.OUT, -2)])),
          ("const_const", wk.Query([(int(units[0]), v["p_sub_org_of"], wk.OUT,
                                     int(inst[v["t_org"]][0]))])),
          ("missing_vertex", wk.Query([(int(units[-1]) + 7_000_000, v["p_member_of"], wk.IN, -1)]))]
    for i, q in enumerate(workloads.light_queries(v, inst, 300, seed=3)):
        qs.append(("light_%03d" % i, q))
    return qs


def final_cases(v, inst):
    """(name, query, required variables, distinct, limit, offset) for the final stage."""
    import workloads
    units = inst[v["t_unit"]]
    chain = workloads.small_chain(v, int(units[0]))
    star = workloads.heavy_star(v)
    return [("chain_distinct_course", chain, [-2], True, -1, 0),
            ("chain_distinct_both", chain, [-1, -2], True, -1, 0),
            ("chain_distinct_swapped", chain, [-2, -1], True, -1, 0),
            ("chain_limit_offset", chain, [-1, -2], False, 10, 5),
            ("chain_offset_past_end", chain, [-1], False, -1, 100000),
            ("chain_distinct_limit_offset", chain, [-1], True, 7, 3),
            ("star_distinct_unit_person", star, [-2, -1], True, -1, 0),
            ("star_distinct_course", star, [-3], True, -1, 0),
            ("star_distinct_limit_offset", star, [-3, -2], True, 25, 10)]


def bound_cases(o, v, inst):
    """(name, table, bound columns) for the BOUND filter: tables of real rows with BLANK_ID
    (an unbound variable, as OPTIONAL leaves it) planted at seeded random places."""
    import workloads
    rng = np.random.default_rng(11)
    units = inst[v["t_unit"]]
    _, chain, _ = o.run(workloads.small_chain(v, int(units[1])).flat(), 2)
    base = np.concatenate([chain[:90], chain[:90, :1]], axis=1).astype(np.uint32)   # 3 columns
    blank = 0xFFFFFFFF
    t1 = base.copy()
    t1[rng.random(t1.shape) < 0.15] = blank
    t2 = base.copy()
    t2[:, 2] = blank
    t3 = base[:0].copy()
    return [("one_column", t1, [1]),
            ("two_columns", t1, [0, 2]),
            ("every_column", t1, [0, 1, 2]),
            ("column_all_blank", t2, [2]),
            ("column_all_blank_not_asked", t2, [0]),
            ("no_filter_columns", t1, []),
            ("empty_table", t3, [0])]


def versatile_queries(v, inst):
    """Queries with an unknown predicate (the versatile operators, sparql.hpp:554-739) and with a
    constant start whose object is already known (const_to_known, :132-189)."""
    import wukong_b200 as wk
    units, persons, courses = inst[v["t_unit"]], inst[v["t_person_a"]], inst[v["t_course"]]
    u0, u1, p0, c0 = int(units[0]), int(units[1]), int(persons[3]), int(courses[2])
    m, t, s = v["p_member_of"], v["p_takes"], v["p_sub_org_of"]
    Q = wk.Query
    return [
        ("v_const_unknown_unknown_out", Q([(p0, -1, wk.OUT, -2)], nvars=2)),
        ("v_const_unknown_unknown_in", Q([(u0, -1, wk.IN, -2)], nvars=2)),
        ("v_const_unknown_const", Q([(p0, -1, wk.OUT, u0)], nvars=1)),
        ("v_const_unknown_const_none", Q([(p0, -1, wk.OUT, u1)], nvars=1)),
        ("v_known_unknown_unknown", Q([(u0, m, wk.IN, -1), (-1, -2, wk.OUT, -3)], nvars=3)),
        ("v_known_unknown_unknown_in", Q([(u0, m, wk.IN, -1), (-1, t, wk.OUT, -2), (-2, -3, wk.IN, -4)], nvars=4)),
        ("v_known_unknown_const", Q([(u0, m, wk.IN, -1), (-1, -2, wk.OUT, u0)], nvars=2)),
        ("v_chain_after_versatile", Q([(p0, -1, wk.OUT, -2), (-2, -3, wk.OUT, -4)], nvars=4)),
        ("v_known_pred_var", Q([(u0, m, wk.IN, -1), (-1, -2, wk.OUT, -3), (-3, -2, wk.OUT, -4)], nvars=4)),
        ("v_unknown_start", Q([(-1, -2, wk.OUT, -3)], nvars=3)),
        ("v_const_unknown_known", Q([(u0, m, wk.IN, -1), (u0, -2, wk.IN, -1)], nvars=2)),
        ("const_to_known", Q([(u0, m, wk.IN, -1), (-1, t, wk.OUT, -2), (c0, t, wk.IN, -1)], nvars=2)),
        ("const_to_known_index_const", Q([(u0, m, wk.IN, -1), (v["t_person_a"], 1, wk.IN, -1)], nvars=1)),
        ("const_to_known_type", Q([(u0, m, wk.IN, -1), (-1, 1, wk.OUT, -2), (p0, 1, wk.OUT, -2)], nvars=2)),
        ("const_to_known_second_pred", Q([(u1, m, wk.IN, -1), (u0, s, wk.OUT, -2), (u1, m, wk.IN, -1)], nvars=2)),
    ]


def pattern_cases(o, v, inst):
    """(name, table, nvars, pattern, mt_tid, mt_factor): one pattern over a given table, as the
    first pattern of a group that inherited it (index_to_known runs only there)."""
    import wukong_b200 as wk
    persons, courses, units = inst[v["t_person_a"]], inst[v["t_course"]], inst[v["t_unit"]]
    mixed = np.concatenate([persons[:300], courses[:80], persons[-40:]]).reshape(-1, 1).astype(np.uint32)
    two = np.stack([persons[:60], np.resize(units, 60)], axis=1).astype(np.uint32)
    cases = [("c2k", mixed, 1, [int(units[0]), v["p_member_of"], -1, wk.IN, 0], 0, 1),
             ("c2k_second_col", two, 2, [int(persons[5]), v["p_member_of"], -2, wk.OUT, 0], 0, 1),
             ("kuu_out", mixed[:50], 3, [-1, -2, -3, wk.OUT, 0], 0, 1),
             ("kuu_in", np.resize(courses, 40).reshape(-1, 1).astype(np.uint32), 3, [-1, -2, -3, wk.IN, 0], 0, 1),
             ("kuc", two, 3, [-1, -3, int(units[0]), wk.OUT, 0], 0, 1),
             ("kuc_second_col", two, 3, [-2, -3, int(inst[v["t_org"]][0]), wk.OUT, 0], 0, 1)]
    for mt in (1, 2, 3):
        for tid in range(mt):
            cases.append(("i2k_mt%d_%d" % (mt, tid), mixed, 1, [v["t_person_a"], 1, -1, wk.IN, 0], tid, mt))
    cases.append(("i2k_predicate_index", mixed, 1, [v["p_takes"], 0, -1, wk.IN, 0], 0, 1))
    return cases


def main():
    import oracle
    import refengine
    import wukong_b200 as wk
    if not refengine.available():
        raise SystemExit("oracle/_ref/libwkref.so is not built (make -C oracle ref)")
    tr, v = wk.synth_generate(20, seed=0, generator_only=True)
    o = oracle.OracleStore(tr)
    g = refengine.graph_from_store(o, tr, v)
    inst = {t: o.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    doc = {"source": "reference CPU engine (SPARQLEngine::execute_sparql_query, compiled from the "
                     "reference tree by oracle/Makefile) on the oracle store's lists",
           "graph": {"orgs": 20, "seed": 0, "triples": int(tr.shape[0]),
                     "triples_sha256": digest(tr)},
           "vocab": {k: int(x) for k, x in v.items()},
           "queries": [], "final": []}
    for name, q in fixture_queries(v, inst):
        st, rows, v2c = g.run(q.flat(), q.nvars, required=refengine.bound_vars(q.flat()) or [-1])
        s = oracle.sorted_rows(rows) if st == 0 else np.zeros((0, 0), np.uint32)
        doc["queries"].append({"name": name, "patterns": [list(map(int, p)) for p in q.patterns],
                               "nvars": q.nvars, "status": int(st),
                               "v2c": [int(x) for x in v2c] if st == 0 else None,
                               "rows": int(s.shape[0]), "cols": int(s.shape[1]) if s.ndim == 2 else 0,
                               "sorted_sha256": digest(s), "head": s[:3].tolist()})
    for name, q, req, distinct, limit, offset in final_cases(v, inst):
        st, rows, v2c = g.run(q.flat(), q.nvars, required=req, distinct=distinct, limit=limit,
                              offset=offset)
        assert st == 0, name
        doc["final"].append({"name": name, "patterns": [list(map(int, p)) for p in q.patterns],
                             "nvars": q.nvars, "required": req, "distinct": distinct,
                             "limit": limit, "offset": offset, "rows": int(rows.shape[0]),
                             "cols": int(rows.shape[1]), "table_sha256": digest(rows),
                             "head": rows[:3].tolist()})
    # the versatile store (the reference's default build): the same graph with every vertex's
    # predicate lists
    ov = oracle.OracleStore(tr, versatile=True)
    gv = refengine.graph_from_store(ov, tr, v)
    doc["versatile"] = []
    for name, q in versatile_queries(v, inst):
        st, rows, v2c = gv.run(q.flat(), q.nvars, required=refengine.bound_vars(q.flat()) or [-1])
        srt = oracle.sorted_rows(rows) if st == 0 else np.zeros((0, 0), np.uint32)
        doc["versatile"].append({"name": name, "patterns": [list(map(int, p)) for p in q.patterns],
                                 "nvars": q.nvars, "status": int(st),
                                 "v2c": [int(x) for x in v2c] if st == 0 else None,
                                 "rows": int(srt.shape[0]),
                                 "cols": int(srt.shape[1]) if srt.ndim == 2 else 0,
                                 "sorted_sha256": digest(srt), "head": srt[:3].tolist()})
    doc["patterns"] = []
    for name, table, nvars, pat, tid, mt in pattern_cases(ov, v, inst):
        st, rows, v2c = gv.pattern(table, nvars, pat, tid, mt)
        doc["patterns"].append({"name": name, "table": table.tolist(), "nvars": nvars,
                                "pattern": [int(x) for x in pat], "mt_tid": tid, "mt_factor": mt,
                                "status": int(st), "v2c": [int(x) for x in v2c] if st == 0 else None,
                                "rows": int(rows.shape[0]) if st == 0 else 0,
                                "cols": int(rows.shape[1]) if st == 0 else 0,
                                "table_sha256": digest(rows) if st == 0 else None})
    doc["bound"] = []
    for name, table, bcols in bound_cases(o, v, inst):
        got = refengine.filter_bound(table, bcols)
        doc["bound"].append({"name": name, "table": table.tolist(), "cols": int(table.shape[1]),
                             "bound_cols": bcols, "rows": int(got.shape[0]),
                             "table_sha256": digest(got)})
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT, len(doc["queries"]), "queries,", len(doc["final"]), "final-stage cases,",
          len(doc["bound"]), "BOUND cases,", len(doc["versatile"]), "versatile queries,",
          len(doc["patterns"]), "single patterns")


if __name__ == "__main__":
    main()
