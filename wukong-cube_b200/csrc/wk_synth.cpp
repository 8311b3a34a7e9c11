// Seeded LUBM-shaped synthetic RDF graph.
//
// Organisations -> units (15-25, unit subOrgOf org) -> persons (30-60 per unit, person type
// drawn uniformly from three, person memberOf unit) and courses (10-20 per unit).  Each person
// takes 2-8 distinct courses of its unit and has one degreeFrom edge to an organisation; type-A
// persons author 5-15 docs.  Every entity has one rdf:type triple.  With zipf = 1, degreeFrom
// targets and course choices follow a Zipf law of exponent zipf_s (hub organisations and
// popular courses); otherwise they are uniform.
//
// Ids follow Wukong's encoding (src/core/store/vertex.hpp:37-57,
// datagen/generate_data.cpp:356-373): 0 = __PREDICATE__, 1 = rdf:type, predicate and type ids
// in [2, 2^17), vertex ids from 2^17 upward.  Each organisation draws from its own random
// stream, so the graph does not depend on how the work is split.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "wk_format.h"
#include "wk_internal.h"

namespace wk {
namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {   // splitmix64 (Steele, Lea, Flood 2014)
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform integer in [lo, hi]
    uint32_t range(uint32_t lo, uint32_t hi) {
        uint64_t span = (uint64_t)hi - lo + 1;
        return lo + (uint32_t)(((next() >> 32) * span) >> 32);
    }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Inverse-CDF sampler over ranks 0..n-1 with P(k) proportional to (k+1)^-s.
struct Zipf {
    std::vector<double> cdf;
    Zipf(uint32_t n, double s) : cdf(n) {
        double acc = 0;
        for (uint32_t k = 0; k < n; ++k) {
            acc += std::pow((double)(k + 1), -s);
            cdf[k] = acc;
        }
        for (auto& c : cdf) c /= acc;
    }
    uint32_t draw(Rng& r) const {
        double u = r.unit();
        auto it = std::lower_bound(cdf.begin(), cdf.end(), u);
        if (it == cdf.end()) --it;
        return (uint32_t)(it - cdf.begin());
    }
};

}  // namespace

int synth_generate(const wk_synth_params& p, std::vector<uint32_t>& out, wk_synth_vocab& v) {
    if (p.n_orgs == 0) return WK_E_BADARG;
    v.t_org = 2; v.t_unit = 3; v.t_person_a = 4; v.t_person_b = 5; v.t_person_c = 6;
    v.t_course = 7; v.t_doc = 8;
    v.p_sub_org_of = 9; v.p_member_of = 10; v.p_takes = 11; v.p_degree_from = 12;
    v.p_author = 13;
    v.first_vid = kVidMin;

    const double zs = p.zipf_s > 0 ? p.zipf_s : 1.1;
    Zipf org_zipf(p.zipf ? p.n_orgs : 1, zs);

    // ~13.5k triples per organisation on average; reserve to avoid regrowth.
    out.clear();
    out.reserve((size_t)p.n_orgs * 14000 * 3);
    auto emit = [&](uint32_t s, uint32_t pr, uint32_t o) {
        out.push_back(s); out.push_back(pr); out.push_back(o);
    };

    uint64_t next = kVidMin;
    const uint32_t org0 = (uint32_t)next;
    next += p.n_orgs;
    for (uint32_t g = 0; g < p.n_orgs; ++g) emit(org0 + g, kTypeId, v.t_org);

    std::vector<uint32_t> courses, chosen;
    for (uint32_t g = 0; g < p.n_orgs; ++g) {
        Rng r(p.seed * 0x100000001B3ull + 0x51ED2701ull + (uint64_t)g * 0x9E3779B97F4A7C15ull);
        const uint32_t org = org0 + g;
        const uint32_t n_units = r.range(15, 25);
        for (uint32_t u = 0; u < n_units; ++u) {
            const uint32_t unit = (uint32_t)next++;
            emit(unit, kTypeId, v.t_unit);
            emit(unit, v.p_sub_org_of, org);
            const uint32_t n_courses = r.range(10, 20);
            courses.resize(n_courses);
            for (uint32_t c = 0; c < n_courses; ++c) {
                courses[c] = (uint32_t)next++;
                emit(courses[c], kTypeId, v.t_course);
            }
            Zipf local_zipf(p.zipf ? n_courses : 1, zs);
            const uint32_t n_persons = r.range(30, 60);
            for (uint32_t i = 0; i < n_persons; ++i) {
                const uint32_t person = (uint32_t)next++;
                const uint32_t kind = r.range(0, 2);
                emit(person, kTypeId, v.t_person_a + kind);
                emit(person, v.p_member_of, unit);
                const uint32_t n_takes = std::min(r.range(2, 8), n_courses);
                chosen.clear();
                while (chosen.size() < n_takes) {
                    uint32_t c = p.zipf ? local_zipf.draw(r) : r.range(0, n_courses - 1);
                    if (std::find(chosen.begin(), chosen.end(), c) == chosen.end())
                        chosen.push_back(c);
                }
                for (uint32_t c : chosen) emit(person, v.p_takes, courses[c]);
                const uint32_t target = p.zipf ? org_zipf.draw(r) : r.range(0, p.n_orgs - 1);
                emit(person, v.p_degree_from, org0 + target);
                if (kind == 0) {
                    const uint32_t n_docs = r.range(5, 15);
                    for (uint32_t d = 0; d < n_docs; ++d) {
                        const uint32_t doc = (uint32_t)next++;
                        emit(doc, kTypeId, v.t_doc);
                        emit(person, v.p_author, doc);
                    }
                }
            }
            if (next >= 0xFFFFFFF0ull) return WK_E_CAPACITY;
        }
    }
    v.next_vid = (uint32_t)next;
    return WK_SUCCESS;
}

}  // namespace wk

extern "C" int wk_synth_generate(const wk_synth_params* p, uint32_t** triples, uint64_t* n_triples,
                                 wk_synth_vocab* vocab) {
    if (!p || !triples || !n_triples) return WK_E_BADARG;
    std::vector<uint32_t> out;
    wk_synth_vocab v{};
    int rc;
    try {
        rc = wk::synth_generate(*p, out, v);
    } catch (const std::bad_alloc&) {
        return WK_E_OOM;
    }
    if (rc != WK_SUCCESS) return rc;
    uint32_t* buf = (uint32_t*)std::malloc(std::max<size_t>(out.size(), 1) * sizeof(uint32_t));
    if (!buf) return WK_E_OOM;
    if (!out.empty()) std::memcpy(buf, out.data(), out.size() * sizeof(uint32_t));
    *triples = buf;
    *n_triples = out.size() / 3;
    if (vocab) *vocab = v;
    return WK_SUCCESS;
}

extern "C" void wk_free(void* p) { std::free(p); }
