"""Generate tests/golden/oracle_20orgs.json: frozen oracle outputs on the 20-organisation graph.

The reference engine cannot be built in this environment (its headers need Boost, TBB and MPI),
so these fixtures are produced by the oracle (the CPU restatement of the reference engine)
and freeze its answers: the CPU suite re-runs the oracle against them, and the GPU suite checks
the CUDA path against the same digests without needing the oracle's store.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "wukong-cube_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

OUT = os.path.join(HERE, "oracle_20orgs.json")


def digest(rows):
    """sha256 of the sorted rows (row-major uint32 little-endian) and their shape."""
    a = np.ascontiguousarray(rows.astype("<u4"))
    return hashlib.sha256(a.tobytes()).hexdigest()


def fixture_queries(v, inst):
    import workloads
    import wukong_b200 as wk
    units = inst[v["t_unit"]]
    qs = [("small_chain", workloads.small_chain(v, int(units[0]))),
          ("small_chain_last_unit", workloads.small_chain(v, int(units[-1]))),
          ("heavy_star", workloads.heavy_star(v)),
          ("heavy_star_person_b", workloads.heavy_star(v, v["t_person_b"])),
          ("heavy_triangle", workloads.heavy_triangle(v)),
          ("unknown_subject", wk.Query([(-1, v["p_takes"], wk.OUT, -2)])),
          ("missing_vertex", wk.Query([(int(units[-1]) + 7_000_000, v["p_member_of"], wk.IN, -1)]))]
    for i, q in enumerate(workloads.light_queries(v, inst, 48, seed=3)):
        qs.append(("light_%02d" % i, q))
    return qs


def main():
    import oracle
    import wukong_b200 as wk
    tr, v = wk.synth_generate(20, seed=0)
    o = oracle.OracleStore(tr)
    g = wk.GStore(tr)
    inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    doc = {"graph": {"orgs": 20, "seed": 0, "triples": int(tr.shape[0]),
                     "triples_sha256": digest(tr)},
           "vocab": {k: int(x) for k, x in v.items()},
           "queries": []}
    for name, q in fixture_queries(v, inst):
        st, rows, v2c = o.run(q.flat(), q.nvars)
        s = oracle.sorted_rows(rows) if st == 0 else np.zeros((0, 0), np.uint32)
        doc["queries"].append({"name": name, "patterns": [list(map(int, p)) for p in q.patterns],
                               "nvars": q.nvars, "status": int(st),
                               "v2c": [int(x) for x in v2c] if st == 0 else None,
                               "rows": int(s.shape[0]), "cols": int(s.shape[1]) if s.ndim == 2 else 0,
                               "sorted_sha256": digest(s), "head": s[:3].tolist()})
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT, len(doc["queries"]), "queries")


if __name__ == "__main__":
    main()
