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
    doc["bound"] = []
    for name, table, bcols in bound_cases(o, v, inst):
        got = refengine.filter_bound(table, bcols)
        doc["bound"].append({"name": name, "table": table.tolist(), "cols": int(table.shape[1]),
                             "bound_cols": bcols, "rows": int(got.shape[0]),
                             "table_sha256": digest(got)})
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT, len(doc["queries"]), "queries,", len(doc["final"]), "final-stage cases,",
          len(doc["bound"]), "BOUND cases")


if __name__ == "__main__":
    main()
