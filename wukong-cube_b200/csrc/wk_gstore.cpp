// Host builder of the static segment store.
//
// Produces exactly the layout SegmentRDFGraph::init_gstore writes
// (src/core/store/segment_rdf_dgraph.hpp:1182-1269) from the loader's id triples:
//   * triples are sorted and de-duplicated per direction (base_loader.hpp:481-496), so every
//     neighbour list is ascending and unique;
//   * one normal segment per (predicate, direction) holds keys [vid|pid|dir]; the IN side
//     skips triples whose object is a type/predicate id (segment_rdf_dgraph.hpp:580-584);
//   * the index segment of each direction holds [0|pid|IN] = subjects of pid,
//     [0|pid|OUT] = objects of pid, and the type index [0|type|IN] = instances
//     (collect_idx_info :951-994, insert_idx :284-347), predicate lists first, then types;
//   * keys go to bucket_start + hash(key) % num_buckets, into the first empty slot of 0..6,
//     overflowing through slot 7 into extension buckets (insert_key_to_seg :203-271);
//   * a versatile build (the reference's default, VERSATILE) adds each vertex's predicate list:
//     keys [vid|PREDICATE_ID|OUT] / [vid|PREDICATE_ID|IN] in two more normal segments, the
//     predicates ascending (insert_vp :365-455).
// How many buckets a segment gets is this builder's own choice (the reference derives it from
// the configured memory size, :117-163): enough for a mean fill of load_factor of the 7 data
// slots, so chains stay rare and most probes touch only the bucket's first sector.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include <parallel/algorithm>

#include "wk_internal.h"

namespace wk {

void SegIndex::build(const wk_seg_meta* segs, uint32_t n) {
    normal.assign((size_t)2 << kNbitsIdx, -1);
    index_seg[0] = index_seg[1] = -1;
    for (uint32_t i = 0; i < n; ++i) {
        const wk_seg_meta& m = segs[i];
        if (m.dir < 0 || m.dir > 1) continue;
        if (m.index) {
            index_seg[m.dir] = (int32_t)i;
        } else if (m.pid < (1u << kNbitsIdx)) {
            normal[(size_t)m.pid * 2 + m.dir] = (int32_t)i;
        }
    }
}

namespace {

// Keys of one direction, grouped by predicate: pairs (vid << 32 | value), sorted, unique.
struct DirLists {
    std::vector<uint64_t> pairs;          // grouped by predicate
    std::vector<uint64_t> pred_begin;     // [pid] -> first pair, size 2^17 + 1
};

// Counting-sort the triples by predicate, then sort each group's (vid, value) words.
void group_by_predicate(const uint32_t* t, uint64_t n, bool in_dir, DirLists& out) {
    const size_t np = (size_t)1 << kNbitsIdx;
    std::vector<uint64_t> cnt(np + 1, 0);
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t s = t[3 * i], p = t[3 * i + 1], o = t[3 * i + 2];
        (void)s;
        if (p == kPredicateId || p >= np) continue;
        if (in_dir && is_tpid(o)) continue;
        cnt[p + 1]++;
    }
    for (size_t p = 0; p < np; ++p) cnt[p + 1] += cnt[p];
    out.pairs.resize(cnt[np]);
    std::vector<uint64_t> pos(cnt.begin(), cnt.end() - 1);
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t s = t[3 * i], p = t[3 * i + 1], o = t[3 * i + 2];
        if (p == kPredicateId || p >= np) continue;
        if (in_dir && is_tpid(o)) continue;
        out.pairs[pos[p]++] = in_dir ? ((uint64_t)o << 32 | s) : ((uint64_t)s << 32 | o);
    }
    // sort + dedup each predicate group, then compact
    std::vector<uint64_t> new_begin(np + 1, 0);
    uint64_t w = 0;
    for (size_t p = 0; p < np; ++p) {
        uint64_t b = cnt[p], e = cnt[p + 1];
        new_begin[p] = w;
        if (b == e) continue;
        __gnu_parallel::sort(out.pairs.begin() + b, out.pairs.begin() + e);
        uint64_t last = ~0ull;
        for (uint64_t i = b; i < e; ++i) {
            if (out.pairs[i] == last) continue;
            last = out.pairs[i];
            out.pairs[w++] = last;
        }
    }
    new_begin[np] = w;
    out.pairs.resize(w);
    out.pred_begin.swap(new_begin);
}

struct KeyRec {
    uint64_t key;
    uint64_t ptr;
};

struct Builder {
    wk_gstore& g;
    uint64_t ext_used = 0;
    explicit Builder(wk_gstore& gs) : g(gs) {}

    // insert_key_to_seg: first empty of slots 0..6, else follow / create the slot-7 chain
    void insert(const wk_seg_meta& m, uint64_t key, uint64_t ptr) {
        uint64_t b = m.bucket_start + hash_u64(key) % m.num_buckets;
        for (;;) {
            Slot* bk = &g.slots[b * kAssoc];
            for (int i = 0; i < kAssoc - 1; ++i) {
                if (bk[i].key == 0) {
                    bk[i].key = key;
                    bk[i].ptr = ptr;
                    return;
                }
            }
            if (bk[kAssoc - 1].key != 0) {
                b = key_vid(bk[kAssoc - 1].key);
                continue;
            }
            uint64_t nb = g.slots.size() / kAssoc;   // append one extension bucket
            g.slots.resize(g.slots.size() + kAssoc, Slot{0, 0});
            ext_used++;
            g.slots[b * kAssoc + kAssoc - 1].key = make_key(nb, 0, 0);
            g.slots[nb * kAssoc].key = key;
            g.slots[nb * kAssoc].ptr = ptr;
            return;
        }
    }
};

uint64_t buckets_for(uint64_t keys, double load) {
    if (keys == 0) return 1;   // min_buckets_per_seg (segment_rdf_dgraph.hpp:108,140)
    double nb = std::ceil((double)keys / ((kAssoc - 1) * load));
    return std::max<uint64_t>(1, (uint64_t)nb);
}

}  // namespace

// The vertex-predicate lists of a VERSATILE build (insert_vp, segment_rdf_dgraph.hpp:365-455):
// for every key vertex of one direction, its distinct predicates in ascending order.  `L`
// holds that direction's (vid << 32 | value) pairs grouped by ascending predicate.  Returns
// (vid << 32 | pid) pairs sorted by vertex, then predicate.
std::vector<uint64_t> vertex_predicates(const DirLists& L) {
    const size_t np = (size_t)1 << kNbitsIdx;
    std::vector<uint64_t> vp;
    for (size_t p = 0; p < np; ++p) {
        uint64_t last = ~0ull;
        for (uint64_t i = L.pred_begin[p]; i < L.pred_begin[p + 1]; ++i) {
            const uint64_t v = L.pairs[i] >> 32;
            if (v != last) vp.push_back(v << 32 | p);
            last = v;
        }
    }
    __gnu_parallel::sort(vp.begin(), vp.end());
    return vp;
}

int gstore_build(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos, uint64_t n_pos,
                 double load, bool versatile, wk_gstore& g) {
    // Default: about 0.7 keys per bucket.  A key's slot is its insertion rank in the bucket, so
    // at this fill about 94% of keys sit in the first 32-byte sector (slots 0-1) and their probe
    // is one request (at 1.4 keys per bucket it was 83%); HBM is plentiful, latency is not.
    if (load <= 0) load = 0.1;
    if (load > 1) return WK_E_BADARG;
    const size_t np = (size_t)1 << kNbitsIdx;
    DirLists outl, inl;
    group_by_predicate(pso, n_pso, false, outl);
    group_by_predicate(pos, n_pos, true, inl);

    // Which predicates exist (either direction) and the key count of every segment.
    auto count_keys = [](const DirLists& d, size_t p) {
        uint64_t k = 0, last = ~0ull;
        for (uint64_t i = d.pred_begin[p]; i < d.pred_begin[p + 1]; ++i) {
            uint64_t v = d.pairs[i] >> 32;
            if (v != last) { ++k; last = v; }
        }
        return k;
    };
    std::vector<uint32_t> preds;
    for (size_t p = 0; p < np; ++p)
        if (outl.pred_begin[p + 1] > outl.pred_begin[p] || inl.pred_begin[p + 1] > inl.pred_begin[p])
            preds.push_back((uint32_t)p);

    // Index lists.  [0|p|IN] = distinct subjects of p, [0|p|OUT] = distinct objects of p
    // (one entry per normal key, in key order); [0|t|IN] = instances of type t.
    std::vector<std::pair<uint32_t, std::vector<uint32_t>>> idx_in, idx_out;
    std::vector<std::vector<uint32_t>> type_inst(np);
    for (uint32_t p : preds) {
        if (p == kTypeId) {
            for (uint64_t i = outl.pred_begin[p]; i < outl.pred_begin[p + 1]; ++i) {
                uint32_t s = (uint32_t)(outl.pairs[i] >> 32), t = (uint32_t)outl.pairs[i];
                if (is_tpid(t)) type_inst[t].push_back(s);
            }
            continue;
        }
        std::vector<uint32_t> subj, obj;
        uint64_t last = ~0ull;
        for (uint64_t i = outl.pred_begin[p]; i < outl.pred_begin[p + 1]; ++i) {
            uint64_t v = outl.pairs[i] >> 32;
            if (v != last) { subj.push_back((uint32_t)v); last = v; }
        }
        last = ~0ull;
        for (uint64_t i = inl.pred_begin[p]; i < inl.pred_begin[p + 1]; ++i) {
            uint64_t v = inl.pairs[i] >> 32;
            if (v != last) { obj.push_back((uint32_t)v); last = v; }
        }
        if (!subj.empty()) idx_in.emplace_back(p, std::move(subj));
        if (!obj.empty()) idx_out.emplace_back(p, std::move(obj));
    }
    for (size_t t = 0; t < np; ++t)
        if (!type_inst[t].empty()) idx_in.emplace_back((uint32_t)t, std::move(type_inst[t]));

    // VERSATILE: [v|PREDICATE_ID|OUT] for every subject, [v|PREDICATE_ID|IN] for every object
    // that is not a type id (the IN lists already leave those out)
    std::vector<uint64_t> vp_out, vp_in;
    if (versatile) {
        vp_out = vertex_predicates(outl);
        vp_in = vertex_predicates(inl);
    }
    auto vp_keys = [](const std::vector<uint64_t>& vp) {
        uint64_t k = 0, last = ~0ull;
        for (uint64_t x : vp) {
            if ((x >> 32) != last) ++k;
            last = x >> 32;
        }
        return k;
    };

    // Segment table: (PREDICATE_ID, OUT), (PREDICATE_ID, IN) in a versatile build, then (p, OUT),
    // (p, IN) for every predicate, then index OUT, index IN.
    g.segs.clear();
    uint64_t bucket_off = 0, edge_off = 0;
    auto add_seg = [&](int index, uint32_t pid, int dir, uint64_t keys, uint64_t edges) {
        wk_seg_meta m{};
        m.index = index;
        m.pid = pid;
        m.dir = dir;
        m.num_keys = keys;
        m.num_buckets = buckets_for(keys, load);
        m.bucket_start = bucket_off;
        m.num_edges = edges;
        m.edge_start = edge_off;
        bucket_off += m.num_buckets;
        edge_off += edges;
        g.segs.push_back(m);
    };
    if (versatile) {
        add_seg(0, kPredicateId, kOut, vp_keys(vp_out), vp_out.size());
        add_seg(0, kPredicateId, kIn, vp_keys(vp_in), vp_in.size());
    }
    for (uint32_t p : preds) {
        add_seg(0, p, kOut, count_keys(outl, p), outl.pred_begin[p + 1] - outl.pred_begin[p]);
        add_seg(0, p, kIn, count_keys(inl, p), inl.pred_begin[p + 1] - inl.pred_begin[p]);
    }
    uint64_t idx_out_edges = 0, idx_in_edges = 0;
    for (auto& e : idx_out) idx_out_edges += e.second.size();
    for (auto& e : idx_in) idx_in_edges += e.second.size();
    add_seg(1, kPredicateId, kOut, idx_out.size(), idx_out_edges);
    add_seg(1, kPredicateId, kIn, idx_in.size(), idx_in_edges);

    g.slots.assign(bucket_off * kAssoc, Slot{0, 0});
    g.edges.resize(edge_off);
    g.n_keys = 0;
    Builder b(g);

    // Normal segments: keys in (vid) order, values ascending.
    size_t si = 0;
    if (versatile) {
        for (int d = 0; d < 2; ++d, ++si) {
            const std::vector<uint64_t>& vp = d == 0 ? vp_out : vp_in;
            const int dir = d == 0 ? kOut : kIn;
            wk_seg_meta& m = g.segs[si];
            uint64_t w = m.edge_start, ext0 = b.ext_used, i = 0;
            while (i < vp.size()) {
                const uint64_t vid = vp[i] >> 32, start = w;
                uint64_t j = i;
                while (j < vp.size() && (vp[j] >> 32) == vid) g.edges[w++] = (uint32_t)vp[j++];
                b.insert(m, make_key(vid, kPredicateId, dir), make_ptr(j - i, start));
                g.n_keys++;
                i = j;
            }
            m.ext_num = b.ext_used - ext0;
        }
    }
    for (uint32_t p : preds) {
        for (int d = 0; d < 2; ++d, ++si) {
            const DirLists& L = (d == 0) ? outl : inl;
            const int dir = (d == 0) ? kOut : kIn;
            wk_seg_meta& m = g.segs[si];
            uint64_t w = m.edge_start;
            uint64_t i = L.pred_begin[p], e = L.pred_begin[p + 1];
            uint64_t ext0 = b.ext_used;
            while (i < e) {
                uint64_t vid = L.pairs[i] >> 32, j = i;
                uint64_t start = w;
                while (j < e && (L.pairs[j] >> 32) == vid) g.edges[w++] = (uint32_t)L.pairs[j++];
                b.insert(m, make_key(vid, p, dir), make_ptr(j - i, start));
                g.n_keys++;
                i = j;
            }
            m.ext_num = b.ext_used - ext0;
        }
    }
    // Index segments.
    auto fill_index = [&](wk_seg_meta& m, std::vector<std::pair<uint32_t, std::vector<uint32_t>>>& lists) {
        uint64_t w = m.edge_start, ext0 = b.ext_used;
        for (auto& e : lists) {
            uint64_t start = w;
            for (uint32_t v : e.second) g.edges[w++] = v;
            b.insert(m, make_key(0, e.first, m.dir), make_ptr(e.second.size(), start));
            g.n_keys++;
        }
        m.ext_num = b.ext_used - ext0;
    };
    fill_index(g.segs[si], idx_out);
    fill_index(g.segs[si + 1], idx_in);

    // Extension buckets were appended after the main-header region in segment order; record
    // each segment's extent.
    uint64_t ext_off = bucket_off;
    for (auto& m : g.segs) {
        m.ext_start = m.ext_num ? ext_off : 0;
        ext_off += m.ext_num;
    }
    g.index.build(g.segs.data(), (uint32_t)g.segs.size());
    return WK_SUCCESS;
}

}  // namespace wk

extern "C" int wk_gstore_build(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos,
                               uint64_t n_pos, double load_factor, wk_gstore** out) {
    return wk_gstore_build_ex(pso, n_pso, pos, n_pos, load_factor, 0, out);
}

extern "C" int wk_gstore_build_ex(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos,
                                  uint64_t n_pos, double load_factor, int32_t versatile,
                                  wk_gstore** out) {
    if (!out || (!pso && n_pso) || (!pos && n_pos)) return WK_E_BADARG;
    wk_gstore* g = nullptr;
    try {
        g = new wk_gstore();
        int rc = wk::gstore_build(pso, n_pso, pos, n_pos, load_factor, versatile != 0, *g);
        if (rc != WK_SUCCESS) {
            delete g;
            return rc;
        }
    } catch (const std::bad_alloc&) {
        delete g;
        return WK_E_OOM;
    }
    *out = g;
    return WK_SUCCESS;
}

extern "C" void wk_gstore_free(wk_gstore* g) { delete g; }

extern "C" int wk_gstore_info(const wk_gstore* g, uint64_t* n_slots, uint64_t* n_edges,
                              uint32_t* n_segs, uint64_t* n_keys) {
    if (!g) return WK_E_BADARG;
    if (n_slots) *n_slots = g->slots.size();
    if (n_edges) *n_edges = g->edges.size();
    if (n_segs) *n_segs = (uint32_t)g->segs.size();
    if (n_keys) *n_keys = g->n_keys;
    return WK_SUCCESS;
}

extern "C" int wk_gstore_arrays(const wk_gstore* g, const void** slots, const uint32_t** edges,
                                const wk_seg_meta** segs) {
    if (!g) return WK_E_BADARG;
    if (slots) *slots = g->slots.data();
    if (edges) *edges = g->edges.data();
    if (segs) *segs = g->segs.data();
    return WK_SUCCESS;
}

static int gstore_lookup(const wk_gstore* g, uint64_t vid, uint32_t pid, int32_t dir,
                         const uint32_t** edges, uint64_t* sz) {
    if (!g || !edges || !sz || dir < 0 || dir > 1) return WK_E_BADARG;
    *edges = nullptr;
    *sz = 0;
    int32_t s = g->index.find(vid, pid, dir);
    if (s < 0 || pid >= (1u << wk::kNbitsIdx)) return WK_SUCCESS;
    int corrupt = 0;
    uint64_t ptr = wk::host_probe(g->slots.data(), g->slots.size() / wk::kAssoc,
                                  wk::to_desc(g->segs[s]), wk::make_key(vid, pid, dir), &corrupt);
    if (corrupt) return WK_E_CORRUPT;
    if (ptr == 0) return WK_SUCCESS;
    uint64_t off = wk::ptr_off(ptr), n = wk::ptr_size(ptr);
    if (off + n > g->edges.size()) return WK_E_CORRUPT;
    *edges = g->edges.data() + off;
    *sz = n;
    return WK_SUCCESS;
}

extern "C" int wk_gstore_get_triples(const wk_gstore* g, uint32_t vid, uint32_t pid, int32_t dir,
                                     const uint32_t** edges, uint64_t* sz) {
    return gstore_lookup(g, vid, pid, dir, edges, sz);
}

extern "C" int wk_gstore_get_index(const wk_gstore* g, uint32_t tpid, int32_t dir,
                                   const uint32_t** edges, uint64_t* sz) {
    return gstore_lookup(g, 0, tpid, dir, edges, sz);
}
