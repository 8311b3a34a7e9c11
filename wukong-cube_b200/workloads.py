"""Planned queries over the synthetic LUBM-shaped graph.

Plans are already in the form the planner hands the engine (Planner::set_direction,
src/optimizer/planner.hpp:667-699): each pattern is (subject, predicate, direction, object)
with IN patterns already swapped so the subject is the bound side, variables are -1, -2, ...,
and an index start is (type_or_predicate, TYPE_ID | PREDICATE_ID, IN, ?x).
"""
import numpy as np

from wukong_b200 import IN, OUT, PREDICATE_ID, TYPE_ID, Query


def small_chain(v, unit):
    """Single-query parity case: ?p memberOf <unit> . ?p takes ?c . ?c type Course ."""
    return Query([(unit, v["p_member_of"], IN, -1),
                  (-1, v["p_takes"], OUT, -2),
                  (-2, TYPE_ID, OUT, v["t_course"])])


def heavy_star(v, person_type=None):
    """?p type PersonX . ?p memberOf ?u . ?p takes ?c  (starts from the type index)."""
    t = v["t_person_a"] if person_type is None else person_type
    return Query([(t, TYPE_ID, IN, -1),
                  (-1, v["p_member_of"], OUT, -2),
                  (-1, v["p_takes"], OUT, -3)])


def heavy_triangle(v):
    """?p memberOf ?u . ?u subOrgOf ?o . ?p degreeFrom ?o  (starts from the predicate index)."""
    return Query([(v["p_member_of"], PREDICATE_ID, IN, -1),
                  (-1, v["p_member_of"], OUT, -2),
                  (-2, v["p_sub_org_of"], OUT, -3),
                  (-1, v["p_degree_from"], OUT, -3)])


def _templates(v):
    """Six-pattern chains per start class; a light query keeps the first L patterns."""
    m, t, s, d, a = (v["p_member_of"], v["p_takes"], v["p_sub_org_of"], v["p_degree_from"],
                     v["p_author"])
    T = TYPE_ID
    return {
        # start type, weight, patterns with the constant as None
        "doc": (v["t_doc"], 0.50, [(None, a, IN, -1), (-1, m, OUT, -2), (-2, s, OUT, -3),
                                    (-1, t, OUT, -4), (-4, T, OUT, v["t_course"]),
                                    (-1, d, OUT, -3)]),
        "person": (v["t_person_b"], 0.20, [(None, t, OUT, -1), (-1, t, IN, -2), (-2, m, OUT, -3),
                                            (-2, T, OUT, v["t_person_b"]), (-3, s, OUT, -4),
                                            (-2, d, OUT, -4)]),
        "course": (v["t_course"], 0.15, [(None, t, IN, -1), (-1, m, OUT, -2), (-2, s, OUT, -3),
                                           (-1, d, OUT, -3), (-1, T, OUT, v["t_person_c"]),
                                           (-1, a, OUT, -4)]),
        "unit": (v["t_unit"], 0.10, [(None, m, IN, -1), (-1, t, OUT, -2), (-2, T, OUT, v["t_course"]),
                                      (-1, d, OUT, -3), (-3, T, OUT, v["t_org"]),
                                      (-1, T, OUT, v["t_person_a"])]),
        "org": (v["t_org"], 0.03, [(None, s, IN, -1), (-1, m, IN, -2), (-2, t, OUT, -3),
                                    (-3, T, OUT, v["t_course"]), (-2, T, OUT, v["t_person_a"]),
                                    (-2, d, OUT, -4)]),
        "alumni": (v["t_org"], 0.02, [(None, d, IN, -1), (-1, m, OUT, -2), (-2, s, OUT, -3),
                                       (-1, T, OUT, v["t_person_c"]), (-3, T, OUT, v["t_org"]),
                                       (-1, t, OUT, -4)]),
    }


def light_queries(v, instances, n, seed=1, min_len=2, max_len=6):
    """n light queries from uniformly random constants of randomly drawn start classes.

    instances: dict type_id -> uint32 array of that type's vertices (the type index).
    Start classes are weighted roughly inversely to their typical table sizes, so intermediate
    table sizes follow a heavy-tailed (about power-law) distribution from 1 to ~1e4 rows.
    """
    rng = np.random.default_rng(seed)
    tm = _templates(v)
    names = list(tm)
    w = np.array([tm[k][1] for k in names])
    w = w / w.sum()
    kinds = rng.choice(len(names), size=n, p=w)
    lens = rng.integers(min_len, max_len + 1, size=n)
    out = []
    for i in range(n):
        ttype, _, pats = tm[names[kinds[i]]]
        pool = instances[ttype]
        c = int(pool[rng.integers(0, len(pool))])
        ps = [(c if x is None else x, p, d, o) for (x, p, d, o) in pats[:lens[i]]]
        out.append(Query(ps, nvars=4))
    return out
