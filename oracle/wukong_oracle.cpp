// ORACLE — test infrastructure only.
//
// A plain C++17 restatement of the reference engine's CPU path for the triple-pattern
// exploration step, used as the bit-exact checker of the CUDA path and as the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// load it; the product library never links it.
//
// What it restates (paths relative to the reference project):
//   * the static KV store: KVStore::insert_key / get_slot_local / get_values_local / bucket_local
//     (src/core/store/kvstore.hpp:151-202, 260-268, 292-314, 394-407),
//     alloc_ext_buckets (:446-457), StaticKVStore::alloc_entries (static_kvstore.hpp:52-64);
//   * SegmentRDFGraph::init_gstore and its helpers (src/core/store/segment_rdf_dgraph.hpp):
//     init_seg_metas (:655-944, non-VERSATILE branches), alloc_buckets_to_seg with
//     global_auto_bkt_alloc off (:117-163), insert_key_to_seg (:203-271), insert_normal_triples
//     (:513-547), insert_triples (:559-590), collect_idx_info (:951-994), insert_idx (:284-347),
//     get_triples / get_index (:1114-1129);
//   * the loader's per-direction sort + dedup (src/loader/base_loader.hpp:90-103, 481-496;
//     triple_sort_by_pso / _pos in src/core/common/type.hpp:181-230);
//   * SPARQLEngine's pattern operators index_to_unknown, const_to_unknown, known_to_unknown,
//     known_to_known, known_to_const (src/core/engine/sparql.hpp:197-552), BASIC pattern
//     groups only, and execute_one_pattern's dispatch (:932-1055);
//   * Result's var2col / add_var2col / var_stat / append_row_to (src/core/sparql/query.hpp:
//     409-510) and start_from_index (:816-838);
//   * the mt_factor split of an index start (sparql.hpp:213-224, dispatch :1058-1105) with the
//     sub-results concatenated in sub-query order (Result::append_result, query.hpp:676-707).
// The reference's own engine stands behind this file: oracle/Makefile (target "ref") compiles
// src/core/engine/sparql.hpp and what it includes from the reference tree against small
// stand-ins for Boost / TBB / the network (oracle/refpin), and tests/golden holds its answers,
// which this file must reproduce.  The store construction is pinned by the known-answer checks
// of tests/test_graph.cc re-derived in tests/test_oracle_known_answers.py.
//   * VERSATILE (the reference's default build, CMakeLists.txt USE_VERSATILE ON): the
//     vertex-predicate lists (insert_vp, segment_rdf_dgraph.hpp:365-455) when the store is
//     built with them, and the unknown-predicate operators (sparql.hpp:554-739) plus
//     index_to_known / const_to_known (:83-189).  The global sets [0|TYPE_ID|IN/OUT] and
//     [0|PREDICATE_ID|OUT] (:333-346) are not built: no pattern operator reads them.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- vertex.hpp:37-182
enum { NBITS_DIR = 1, NBITS_IDX = 17, NBITS_VID = 64 - NBITS_IDX - NBITS_DIR };
enum { PREDICATE_ID = 0, TYPE_ID = 1 };
enum dir_t { IN = 0, OUT = 1 };
static const uint32_t BLANK_ID = 0xFFFFFFFFu;
static inline bool is_tpid(int64_t id) { return id > 1 && id < (1 << NBITS_IDX); }

struct ikey_t {
    uint64_t dir : NBITS_DIR;
    uint64_t pid : NBITS_IDX;
    uint64_t vid : NBITS_VID;
    ikey_t() : dir(0), pid(0), vid(0) {}
    ikey_t(uint64_t v, uint64_t p, uint64_t d) : dir(d), pid(p), vid(v) {}
    bool operator==(const ikey_t& k) const { return vid == k.vid && pid == k.pid && dir == k.dir; }
    bool is_empty() const { return vid == 0 && pid == 0 && dir == 0; }
    uint64_t hash() const {   // vertex.hpp:106-116 + math.hpp:59-68
        uint64_t r = 0;
        r += vid;
        r <<= NBITS_IDX;
        r += pid;
        r <<= NBITS_DIR;
        r += dir;
        uint64_t key = r;
        key = (~key) + (key << 21);
        key = key ^ (key >> 24);
        key = (key + (key << 3)) + (key << 8);
        key = key ^ (key >> 14);
        key = (key + (key << 2)) + (key << 4);
        key = key ^ (key >> 28);
        key = key + (key << 31);
        return key;
    }
};
struct iptr_t {
    uint64_t size : 28;
    uint64_t off : 34;
    uint64_t type : 2;
    iptr_t() : size(0), off(0), type(0) {}
    iptr_t(uint64_t s, uint64_t o) : size(s), off(o), type(0) {}
};
struct slot_t {
    ikey_t key;
    iptr_t ptr;
};
static_assert(sizeof(slot_t) == 16, "vertex_t is 16 bytes");

struct triple_t {
    uint32_t s, p, o;
    bool operator==(const triple_t& t) const { return s == t.s && p == t.p && o == t.o; }
};

// ---------------------------------------------------------------- segment_meta.hpp:60-222
struct ext_bucket_extent_t {
    uint64_t num_ext_buckets = 0, off = 0, start = 0;
};
struct rdf_seg_meta_t {
    uint64_t num_keys = 0, num_buckets = 0, bucket_start = 0, num_edges = 0, edge_start = 0,
             edge_off = 0;
    std::vector<ext_bucket_extent_t> ext_bucket_list;
    uint64_t get_ext_bucket() {
        for (auto& ext : ext_bucket_list)
            if (ext.off < ext.num_ext_buckets) return ext.start + ext.off++;
        return 0;
    }
};
struct segid_t {
    int index;
    int dir;
    uint32_t pid;
    segid_t(int idx, uint32_t p, int d) : index(idx), dir(d), pid(p) {}
    explicit segid_t(const ikey_t& key) {   // segment_meta.hpp:168-178
        dir = (int)key.dir;
        if (key.vid == 0) {
            index = 1;
            pid = PREDICATE_ID;
        } else {
            index = 0;
            pid = (uint32_t)key.pid;
        }
    }
    bool operator<(const segid_t& s) const {   // :196-206
        if (pid != s.pid) return pid < s.pid;
        if (index != s.index) return index < s.index;
        return dir < s.dir;
    }
};

struct error_code : std::runtime_error {
    int code;
    explicit error_code(int c) : std::runtime_error("wukong error"), code(c) {}
};

// Sort with one thread per chunk, then merge chunk pairs; for a total order the result is the
// same sequence std::sort gives (this only shortens the oracle's build on large graphs).
template <class T, class Cmp>
static void par_sort(std::vector<T>& v, Cmp cmp) {
    const size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 64));
    if (v.size() < (1u << 20) || nt == 1) {
        std::sort(v.begin(), v.end(), cmp);
        return;
    }
    std::vector<size_t> b(nt + 1);
    for (size_t i = 0; i <= nt; ++i) b[i] = v.size() * i / nt;
    std::vector<std::thread> th;
    for (size_t i = 0; i < nt; ++i)
        th.emplace_back([&, i] { std::sort(v.begin() + b[i], v.begin() + b[i + 1], cmp); });
    for (auto& t : th) t.join();
    for (size_t step = 1; step < nt; step *= 2) {
        th.clear();
        for (size_t i = 0; i + step < nt; i += 2 * step) {
            const size_t lo = b[i], mid = b[i + step], hi = b[std::min(nt, i + 2 * step)];
            th.emplace_back([&, lo, mid, hi] {
                std::inplace_merge(v.begin() + lo, v.begin() + mid, v.begin() + hi, cmp);
            });
        }
        for (auto& t : th) t.join();
    }
}
enum { SUCCESS = 0, UNKNOWN_ERROR = 1, UNKNOWN_PATTERN = 3, OBJ_ERROR = 7, VERTEX_INVALID = 8,
       UNKNOWN_SUB = 9, FIRST_PATTERN_ERROR = 11, STORE_ERROR = 106 };
#define ORACLE_ASSERT(c, code) \
    do {                       \
        if (!(c)) throw error_code(code); \
    } while (0)

// ---------------------------------------------------------------- the store
class Store {
public:
    std::vector<slot_t> slots;
    std::vector<uint32_t> values;    // edge_t
    std::map<segid_t, rdf_seg_meta_t> seg_map;
    std::vector<uint32_t> predicates;
    std::vector<uint32_t> edge_predicates, type_predicates;
    uint64_t num_buckets = 0;        // main-header region
    uint64_t last_ext = 0;
    uint64_t last_entry = 0;
    uint64_t main_hdr_off = 0;
    static const int ASSOCIATIVITY = 8;
    static const int est_load_factor = 55;   // global.hpp:127
    std::map<uint32_t, std::vector<uint32_t>> pidx_in_map, pidx_out_map, tidx_map;
    // VERSATILE builds (segment_rdf_dgraph.hpp:365-455): every vertex's predicates, key
    // [vid|PREDICATE_ID|OUT] for the subjects of pso, [vid|PREDICATE_ID|IN] for the objects of
    // pos that are not type ids; each list ascending (the loader sorts by spo / ops there).
    bool versatile = false;
    std::map<uint32_t, std::vector<uint32_t>> vp_out, vp_in;

    // kvstore.hpp:446-457: extension buckets live after the main-header region
    uint64_t alloc_ext_buckets(uint64_t n) {
        uint64_t orig = last_ext;
        last_ext += n;
        slots.resize((num_buckets + last_ext) * ASSOCIATIVITY);
        return num_buckets + orig;
    }
    uint64_t alloc_entries(uint64_t n) {   // static_kvstore.hpp:52-64
        uint64_t orig = last_entry;
        last_entry += n;
        return orig;
    }
    uint64_t bucket_local(const ikey_t& key, const rdf_seg_meta_t* seg) const {
        return seg->bucket_start + key.hash() % seg->num_buckets;   // kvstore.hpp:260-268
    }

    // kvstore.hpp:292-314 (the loop is bounded here so a corrupt chain cannot hang the oracle)
    slot_t get_slot_local(const ikey_t& key, const rdf_seg_meta_t* seg) const {
        uint64_t bucket_id = bucket_local(key, seg);
        for (uint64_t hop = 0; hop <= slots.size() / ASSOCIATIVITY; ++hop) {
            for (int i = 0; i < ASSOCIATIVITY; i++) {
                uint64_t slot_id = bucket_id * ASSOCIATIVITY + i;
                if (slot_id >= slots.size()) throw error_code(STORE_ERROR);
                if (i < ASSOCIATIVITY - 1) {
                    if (slots[slot_id].key == key) return slots[slot_id];
                } else {
                    if (slots[slot_id].key.is_empty()) return slot_t();
                    bucket_id = slots[slot_id].key.vid;
                    break;
                }
            }
        }
        throw error_code(STORE_ERROR);
    }
    // kvstore.hpp:394-407
    const uint32_t* get_values_local(const ikey_t& key, uint64_t& sz,
                                     const rdf_seg_meta_t* seg) const {
        slot_t slot = get_slot_local(key, seg);
        if (slot.key.is_empty()) {
            sz = 0;
            return nullptr;
        }
        sz = slot.ptr.size;
        return &values[slot.ptr.off];
    }

    // segment_rdf_dgraph.hpp:1114-1129.  A segment the store never created is an empty list
    // (the reference would index a default-constructed meta with num_buckets = 0).
    const uint32_t* get_triples(uint32_t vid, uint32_t pid, int d, uint64_t& sz) const {
        ikey_t key(vid, pid, d);
        if (key.pid != pid) {   // pid wider than 17 bits cannot be a key
            sz = 0;
            return nullptr;
        }
        auto it = seg_map.find(segid_t(key));
        if (it == seg_map.end() || it->second.num_buckets == 0) {
            sz = 0;
            return nullptr;
        }
        return get_values_local(key, sz, &it->second);
    }
    const uint32_t* get_index(uint32_t pid, int d, uint64_t& sz) const {
        return get_triples(0, pid, d, sz);
    }

    // segment_rdf_dgraph.hpp:117-163, global_auto_bkt_alloc == false branch, with the
    // GPU-build extension extent EXT_BUCKET_EXTENT_LEN(n) = n * 15 / 100 + 1.
    void alloc_buckets_to_seg(rdf_seg_meta_t& seg) {
        uint64_t nbuckets;
        if (seg.num_keys == 0)
            nbuckets = 0;
        else
            nbuckets = (uint64_t)(seg.num_keys * (100.0 / (est_load_factor * ASSOCIATIVITY)));
        seg.num_buckets = std::max<uint64_t>(nbuckets, 1);
        seg.bucket_start = main_hdr_off;
        main_hdr_off += seg.num_buckets;
    }
    void alloc_ext_extent(rdf_seg_meta_t& seg) {
        if (seg.num_buckets > 0) {
            uint64_t n = seg.num_buckets * 15 / 100 + 1;
            ext_bucket_extent_t e;
            e.num_ext_buckets = n;
            e.start = alloc_ext_buckets(n);
            seg.ext_bucket_list.push_back(e);
        }
    }

    // segment_rdf_dgraph.hpp:203-271
    uint64_t insert_key_to_seg(const ikey_t& key, const iptr_t& ptr) {
        rdf_seg_meta_t& seg = seg_map[segid_t(key)];
        uint64_t bucket_id = bucket_local(key, &seg);
        uint64_t slot_id = bucket_id * ASSOCIATIVITY;
        while (slot_id < slots.size()) {
            for (int i = 0; i < ASSOCIATIVITY - 1; i++, slot_id++) {
                if (slots[slot_id].key == key) throw error_code(STORE_ERROR);   // conflict
                if (slots[slot_id].key.is_empty()) {
                    slots[slot_id].key = key;
                    slots[slot_id].ptr = ptr;
                    return slot_id;
                }
            }
            if (!slots[slot_id].key.is_empty()) {
                slot_id = slots[slot_id].key.vid * ASSOCIATIVITY;
                continue;
            }
            uint64_t ext_bucket_id = seg.get_ext_bucket();
            if (ext_bucket_id == 0) {
                uint64_t n = seg.num_buckets * 15 / 100 + 1;
                ext_bucket_extent_t e;
                e.num_ext_buckets = n;
                e.start = alloc_ext_buckets(n);
                seg.ext_bucket_list.push_back(e);
                ext_bucket_id = seg.get_ext_bucket();
            }
            slots[slot_id].key.vid = ext_bucket_id;
            slot_id = ext_bucket_id * ASSOCIATIVITY;
            slots[slot_id].key = key;
            slots[slot_id].ptr = ptr;
            return slot_id;
        }
        throw error_code(STORE_ERROR);
    }

    // segment_rdf_dgraph.hpp:951-994
    void collect_idx_info(const slot_t& slot) {
        uint32_t vid = (uint32_t)slot.key.vid, pid = (uint32_t)slot.key.pid;
        if (slot.key.dir == IN) {
            if (pid == PREDICATE_ID) {
            } else if (pid == TYPE_ID) {
                throw error_code(STORE_ERROR);
            } else {
                pidx_out_map[pid].push_back(vid);
            }
        } else {
            if (pid == PREDICATE_ID) {
            } else if (pid == TYPE_ID) {
                for (uint64_t e = 0; e < slot.ptr.size; e++)
                    tidx_map[values[slot.ptr.off + e]].push_back(vid);
            } else {
                pidx_in_map[pid].push_back(vid);
            }
        }
    }

    // segment_rdf_dgraph.hpp:513-547
    size_t insert_normal_triples(const std::vector<triple_t>& t, rdf_seg_meta_t& seg, size_t s,
                                 int dir) {
        ikey_t key;
        size_t e = s + 1;
        if (dir == OUT) {
            while (e < t.size() && t[s].s == t[e].s && t[s].p == t[e].p) e++;
            key = ikey_t(t[s].s, t[s].p, OUT);
        } else {
            while (e < t.size() && t[s].o == t[e].o && t[s].p == t[e].p) e++;
            key = ikey_t(t[s].o, t[s].p, IN);
        }
        if (seg.edge_off == 0) seg.edge_off = seg.edge_start;   // alloc_entries_in_seg :185-194
        uint64_t off = seg.edge_off;
        seg.edge_off += e - s;
        uint64_t slot_id = insert_key_to_seg(key, iptr_t(e - s, off));
        for (size_t i = s; i < e; i++) values[off++] = (dir == OUT) ? t[i].o : t[i].s;
        collect_idx_info(slots[slot_id]);
        return e;
    }

    // segment_rdf_dgraph.hpp:559-590 (one engine)
    void insert_triples(segid_t segid, const std::vector<triple_t>& vec,
                        const std::map<uint32_t, size_t>& pmap) {
        auto& segment = seg_map[segid];
        uint32_t pid = segid.pid;
        if (segment.num_edges == 0) return;
        auto it = pmap.find(pid);
        if (it == pmap.end()) return;
        size_t s = it->second;
        while (s < vec.size() && vec[s].p == pid) {
            if (segid.dir == IN)
                while (s < vec.size() && vec[s].p == pid && is_tpid(vec[s].o)) s++;
            if (s >= vec.size() || vec[s].p != pid) break;
            s = insert_normal_triples(vec, segment, s, segid.dir);
        }
    }

    // segment_rdf_dgraph.hpp:284-347 (non-VERSATILE)
    void insert_idx(const std::map<uint32_t, std::vector<uint32_t>>& pidx_map, int d) {
        rdf_seg_meta_t& segment = seg_map[segid_t(1, PREDICATE_ID, d)];
        uint64_t off = segment.edge_start;
        for (uint32_t pid : edge_predicates) {
            auto it = pidx_map.find(pid);
            if (it == pidx_map.end()) continue;
            insert_key_to_seg(ikey_t(0, pid, d), iptr_t(it->second.size(), off));
            for (uint32_t v : it->second) values[off++] = v;
        }
        if (d == IN) {
            for (auto& e : tidx_map) {
                insert_key_to_seg(ikey_t(0, e.first, IN), iptr_t(e.second.size(), off));
                for (uint32_t v : e.second) values[off++] = v;
            }
        }
    }

    // segment_rdf_dgraph.hpp:655-944, one engine, no attributes, no VERSATILE.
    void init_seg_metas(const std::vector<triple_t>& pso, const std::vector<triple_t>& pos) {
        std::map<uint32_t, uint64_t> n_out, n_in, i_in, i_out;
        for (uint32_t pred : predicates) {
            seg_map[segid_t(0, pred, IN)];
            seg_map[segid_t(0, pred, OUT)];
        }
        seg_map[segid_t(1, PREDICATE_ID, IN)];
        seg_map[segid_t(1, PREDICATE_ID, OUT)];

        uint64_t s = 0;
        while (s < pso.size()) {
            uint64_t e = s + 1;
            while (e < pso.size() && pso[s].s == pso[e].s && pso[s].p == pso[e].p) {
                if (pso[e].p == TYPE_ID && is_tpid(pso[e].o)) i_in[pso[e].o]++;
                e++;
            }
            n_out[pso[s].p] += e - s;
            i_in[pso[s].p]++;
            if (pso[s].p == TYPE_ID && is_tpid(pso[s].o)) i_in[pso[s].o]++;
            s = e;
        }
        uint64_t type_triples = 0;
        while (type_triples < pos.size() && is_tpid(pos[type_triples].o)) type_triples++;
        s = type_triples;
        while (s < pos.size()) {
            uint64_t e = s + 1;
            while (e < pos.size() && pos[s].o == pos[e].o && pos[s].p == pos[e].p) e++;
            if (!is_tpid(pos[s].o)) {   // a type triple of a later predicate is never a key
                n_in[pos[s].p] += e - s;
                i_out[pos[s].p]++;
            }
            s = e;
        }

        for (uint32_t pred : predicates) {
            if (pred == PREDICATE_ID) continue;
            if (n_in[pred] + n_out[pred] > 0)
                edge_predicates.push_back(pred);
            else if (i_in[pred] > 0)
                type_predicates.push_back(pred);
        }

        rdf_seg_meta_t& idx_out_seg = seg_map[segid_t(1, PREDICATE_ID, OUT)];
        rdf_seg_meta_t& idx_in_seg = seg_map[segid_t(1, PREDICATE_ID, IN)];
        std::vector<rdf_seg_meta_t*> order;
        for (uint32_t pred : predicates) {
            if (pred == PREDICATE_ID) continue;
            rdf_seg_meta_t& out_seg = seg_map[segid_t(0, pred, OUT)];
            rdf_seg_meta_t& in_seg = seg_map[segid_t(0, pred, IN)];
            out_seg.num_edges = n_out[pred];
            in_seg.num_edges = n_in[pred];
            idx_out_seg.num_edges += i_out[pred];
            idx_in_seg.num_edges += i_in[pred];
            // normal_nkeys[OUT] is the index IN count (one per subject key) and vice versa
            out_seg.num_keys = out_seg.num_edges == 0 ? 0 : i_in[pred];
            in_seg.num_keys = in_seg.num_edges == 0 ? 0 : i_out[pred];
            out_seg.edge_start = alloc_entries(out_seg.num_edges);
            in_seg.edge_start = alloc_entries(in_seg.num_edges);
            alloc_buckets_to_seg(out_seg);
            alloc_buckets_to_seg(in_seg);
            order.push_back(&out_seg);
            order.push_back(&in_seg);
        }
        if (versatile) {   // :837-851: the vid-predicate segments
            rdf_seg_meta_t& pout = seg_map[segid_t(0, PREDICATE_ID, OUT)];
            rdf_seg_meta_t& pin = seg_map[segid_t(0, PREDICATE_ID, IN)];
            for (auto& e : vp_out) pout.num_edges += e.second.size();
            for (auto& e : vp_in) pin.num_edges += e.second.size();
            pout.num_keys = vp_out.size();
            pin.num_keys = vp_in.size();
            pout.edge_start = alloc_entries(pout.num_edges);
            pin.edge_start = alloc_entries(pin.num_edges);
            alloc_buckets_to_seg(pout);
            alloc_buckets_to_seg(pin);
            order.push_back(&pout);
            order.push_back(&pin);
        }
        idx_out_seg.edge_start = alloc_entries(idx_out_seg.num_edges);
        idx_out_seg.num_keys += edge_predicates.empty() ? 0 : edge_predicates.size() - 1;
        alloc_buckets_to_seg(idx_out_seg);
        idx_in_seg.edge_start = alloc_entries(idx_in_seg.num_edges);
        uint64_t nin = edge_predicates.size() + type_predicates.size();
        idx_in_seg.num_keys += nin ? nin - 1 : 0;
        alloc_buckets_to_seg(idx_in_seg);
        order.push_back(&idx_out_seg);
        order.push_back(&idx_in_seg);

        num_buckets = main_hdr_off;
        slots.assign(num_buckets * ASSOCIATIVITY, slot_t());
        for (rdf_seg_meta_t* m : order) alloc_ext_extent(*m);
        values.assign(last_entry, 0);
    }

    // segment_rdf_dgraph.hpp:1182-1269 with the loader's sort + dedup in front
    void init_gstore(std::vector<triple_t> pso, std::vector<triple_t> pos) {
        auto by_pso = [](const triple_t& a, const triple_t& b) {
            if (a.p != b.p) return a.p < b.p;
            if (a.s != b.s) return a.s < b.s;
            return a.o < b.o;
        };
        auto by_pos = [](const triple_t& a, const triple_t& b) {
            if (a.p != b.p) return a.p < b.p;
            if (a.o != b.o) return a.o < b.o;
            return a.s < b.s;
        };
        // the orders are total, so a parallel sort gives the loader's sequence exactly
        par_sort(pso, by_pso);
        par_sort(pos, by_pos);
        pso.erase(std::unique(pso.begin(), pso.end()), pso.end());
        pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
        // predicates known to the string server: every predicate id used, plus the type ids
        std::vector<uint32_t> ids;
        for (auto& t : pso) {
            ids.push_back(t.p);
            if (t.p == TYPE_ID && is_tpid(t.o)) ids.push_back(t.o);
        }
        for (auto& t : pos) ids.push_back(t.p);
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        predicates = ids;

        if (versatile) {
            // distinct (s, p) of pso in (p, s) order: appending p per s gives each s's
            // predicates ascending; likewise (o, p) of pos, type-id objects skipped (:404-411)
            for (size_t i = 0; i < pso.size(); ++i)
                if (i == 0 || pso[i].p != pso[i - 1].p || pso[i].s != pso[i - 1].s)
                    vp_out[pso[i].s].push_back(pso[i].p);
            for (size_t i = 0; i < pos.size(); ++i)
                if (!is_tpid(pos[i].o) && (i == 0 || pos[i].p != pos[i - 1].p || pos[i].o != pos[i - 1].o))
                    vp_in[pos[i].o].push_back(pos[i].p);
        }
        init_seg_metas(pso, pos);

        std::map<uint32_t, size_t> out_map, in_map;   // init_triple_map: first row of each pid
        for (size_t i = 0; i < pso.size(); ++i)
            if (!out_map.count(pso[i].p)) out_map[pso[i].p] = i;
        for (size_t i = 0; i < pos.size(); ++i)
            if (!in_map.count(pos[i].p)) in_map[pos[i].p] = i;
        for (uint32_t pid : edge_predicates) {
            insert_triples(segid_t(0, pid, OUT), pso, out_map);
            insert_triples(segid_t(0, pid, IN), pos, in_map);
        }
        insert_idx(pidx_in_map, IN);
        insert_idx(pidx_out_map, OUT);
        if (versatile) {   // insert_vp (:371-455)
            for (int d = 0; d < 2; ++d) {
                auto& vp = d == OUT ? vp_out : vp_in;
                rdf_seg_meta_t& seg = seg_map[segid_t(0, PREDICATE_ID, d)];
                uint64_t off = seg.edge_start;
                for (auto& e : vp) {
                    insert_key_to_seg(ikey_t(e.first, PREDICATE_ID, d), iptr_t(e.second.size(), off));
                    for (uint32_t v : e.second) values[off++] = v;
                }
            }
        }
    }
};

// ---------------------------------------------------------------- query.hpp (subset)
enum vstat { KNOWN_VAR = 0, UNKNOWN_VAR, CONST_VAR };
static const int NO_RESULT = (1 << 16) - 1;
constexpr int const_pair(int t1, int t2) { return (t1 << 4) | t2; }

struct Pattern {
    int32_t subject, predicate, object, direction, pred_type;
};

struct Result {
    int col_num = 0;
    int nvars = 0;
    std::vector<int> v2c_map;
    std::vector<uint32_t> result_table;

    vstat var_stat(int32_t vid) {   // query.hpp:409-416
        if (vid >= 0) return CONST_VAR;
        if (var2col(vid) == NO_RESULT) return UNKNOWN_VAR;
        return KNOWN_VAR;
    }
    int var2col(int32_t vid) {   // :425-440
        ORACLE_ASSERT(vid < 0, VERTEX_INVALID);
        ORACLE_ASSERT(nvars > 0, VERTEX_INVALID);
        if (v2c_map.empty()) v2c_map.assign(nvars, NO_RESULT);
        int idx = -(vid + 1);
        ORACLE_ASSERT(idx < nvars && idx >= 0, VERTEX_INVALID);
        return v2c_map[idx] & 0xFFFF;
    }
    void add_var2col(int32_t vid, int col) {   // :443-459 (plain ASSERTs: UNKNOWN_ERROR)
        ORACLE_ASSERT(vid < 0 && col >= 0, UNKNOWN_ERROR);
        if (v2c_map.empty()) v2c_map.assign(nvars, NO_RESULT);
        int idx = -(vid + 1);
        ORACLE_ASSERT(idx < nvars && idx >= 0, UNKNOWN_ERROR);
        ORACLE_ASSERT(v2c_map[idx] == NO_RESULT, UNKNOWN_ERROR);   // a variable is set once
        v2c_map[idx] = col;   // col2ext(col, SID_t)
    }
    uint64_t get_row_num() const { return col_num == 0 ? 0 : result_table.size() / col_num; }
    uint32_t get_row_col(uint64_t r, int c) const { return result_table[col_num * r + c]; }
    void append_row_to(uint64_t r, std::vector<uint32_t>& u) const {
        for (int c = 0; c < col_num; c++) u.push_back(get_row_col(r, c));
    }
};

struct Query {
    std::vector<Pattern> patterns;
    int pattern_step = 0;
    int mt_factor = 1, mt_tid = 0;
    Result result;
    bool start_from_index() const {   // query.hpp:816-838
        if (patterns.empty()) return false;
        if (is_tpid(patterns[0].subject)) {
            ORACLE_ASSERT(patterns[0].predicate == PREDICATE_ID || patterns[0].predicate == TYPE_ID,
                          OBJ_ERROR);
            return true;
        }
        return false;
    }
};

// ---------------------------------------------------------------- sparql.hpp:197-552, 932-1055
class Engine {
public:
    const Store* graph;
    explicit Engine(const Store* g) : graph(g) {}

    void index_to_unknown(Query& req) {   // :197-234
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t tpid = pattern.subject, id01 = pattern.predicate, end = pattern.object;
        int d = pattern.direction;
        Result& res = req.result;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        ORACLE_ASSERT(id01 == PREDICATE_ID || id01 == TYPE_ID, OBJ_ERROR);
        ORACLE_ASSERT(res.col_num == 0, FIRST_PATTERN_ERROR);
        std::vector<uint32_t> updated;
        uint64_t sz = 0;
        const uint32_t* edges = graph->get_index((uint32_t)tpid, d, sz);
        int start = req.mt_tid % req.mt_factor;
        uint64_t length = sz / req.mt_factor;
        for (uint64_t k = start * length; k < (start + 1) * length; k++) updated.push_back(edges[k]);
        if (start == req.mt_factor - 1)
            for (uint64_t k = (start + 1) * length; k < sz; k++) updated.push_back(edges[k]);
        res.result_table.swap(updated);
        res.col_num = 1;
        res.add_var2col(end, 0);
        req.pattern_step++;
    }

    void const_to_unknown(Query& req) {   // :241-288 (SID_t branch)
        Pattern& pattern = req.patterns[req.pattern_step];
        Result& res = req.result;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        ORACLE_ASSERT(res.col_num == 0, FIRST_PATTERN_ERROR);
        uint64_t sz = 0;
        const uint32_t* vids = graph->get_triples((uint32_t)pattern.subject,
                                                  (uint32_t)pattern.predicate, pattern.direction, sz);
        std::vector<uint32_t> updated(vids, vids + sz);
        res.result_table.swap(updated);
        res.add_var2col(pattern.object, res.col_num);
        res.col_num = res.col_num + 1;
        req.pattern_step++;
    }

    void known_to_unknown(Query& req) {   // :298-410 (SID_t, BASIC)
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t start = pattern.subject, pid = pattern.predicate, end = pattern.object;
        int d = pattern.direction;
        Result& res = req.result;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        std::vector<uint32_t> updated;
        updated.reserve(res.result_table.size());
        uint32_t cached = BLANK_ID;
        const uint32_t* vids = nullptr;
        uint64_t sz = 0;
        uint64_t nrows = res.get_row_num();
        int cs = res.var2col(start);
        for (uint64_t i = 0; i < nrows; i++) {
            uint32_t cur = res.get_row_col(i, cs);
            if (cur != cached) {
                cached = cur;
                if (pid == TYPE_ID && d == IN) {
                    // get_index(cur, IN): ikey_t(0, cur, IN) keeps 17 bits of cur; a wider
                    // value is not an index id and has no list.
                    if (cur < (1u << NBITS_IDX))
                        vids = graph->get_index(cur, d, sz);
                    else {
                        vids = nullptr;
                        sz = 0;
                    }
                } else {
                    vids = graph->get_triples(cur, (uint32_t)pid, d, sz);
                }
            }
            for (uint64_t k = 0; k < sz; k++) {
                res.append_row_to(i, updated);
                updated.push_back(vids[k]);
            }
        }
        res.result_table.swap(updated);
        res.add_var2col(end, res.col_num);
        res.col_num = res.col_num + 1;
        req.pattern_step++;
    }

    void known_to_known(Query& req) {   // :419-479 (BASIC)
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t start = pattern.subject, pid = pattern.predicate, end = pattern.object;
        int d = pattern.direction;
        Result& res = req.result;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        std::vector<uint32_t> updated;
        uint32_t cached = BLANK_ID;
        const uint32_t* vids = nullptr;
        uint64_t sz = 0;
        uint64_t nrows = res.get_row_num();
        int cs = res.var2col(start), ce = res.var2col(end);
        for (uint64_t i = 0; i < nrows; i++) {
            uint32_t cur = res.get_row_col(i, cs);
            if (cur != cached) {
                cached = cur;
                vids = graph->get_triples(cur, (uint32_t)pid, d, sz);
            }
            uint32_t known = res.get_row_col(i, ce);
            for (uint64_t k = 0; k < sz; k++) {
                if (vids[k] == known) {
                    res.append_row_to(i, updated);
                    break;
                }
            }
        }
        res.result_table.swap(updated);
        req.pattern_step++;
    }

    void known_to_const(Query& req) {   // :487-552 (BASIC)
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t start = pattern.subject, pid = pattern.predicate, end = pattern.object;
        int d = pattern.direction;
        Result& res = req.result;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        std::vector<uint32_t> updated;
        uint32_t cached = BLANK_ID;
        const uint32_t* vids = nullptr;
        uint64_t sz = 0;
        bool exist = false;
        uint64_t nrows = res.get_row_num();
        int cs = res.var2col(start);
        for (uint64_t i = 0; i < nrows; i++) {
            uint32_t cur = res.get_row_col(i, cs);
            if (cur != cached) {
                exist = false;
                cached = cur;
                vids = graph->get_triples(cur, (uint32_t)pid, d, sz);
                for (uint64_t k = 0; k < sz; k++) {
                    if (vids[k] == (uint32_t)end) {
                        exist = true;
                        res.append_row_to(i, updated);
                        break;
                    }
                }
            } else if (exist) {
                res.append_row_to(i, updated);
            }
        }
        res.result_table.swap(updated);
        req.pattern_step++;
    }

    // :83-130 (BASIC): keep the rows whose `end` value is in the index list (its mt slice)
    void index_to_known(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t tpid = pattern.subject, id01 = pattern.predicate, end = pattern.object;
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        int col = res.var2col(end);
        ORACLE_ASSERT(col != NO_RESULT, VERTEX_INVALID);
        ORACLE_ASSERT(id01 == PREDICATE_ID || id01 == TYPE_ID, OBJ_ERROR);
        uint64_t sz = 0;
        const uint32_t* edges = graph->get_index((uint32_t)tpid, pattern.direction, sz);
        int start = req.mt_tid % req.mt_factor;
        uint64_t length = sz / req.mt_factor;
        std::vector<uint32_t> set;
        for (uint64_t k = start * length; k < (start + 1) * length; k++) set.push_back(edges[k]);
        if (start == req.mt_factor - 1)
            for (uint64_t k = (start + 1) * length; k < sz; k++) set.push_back(edges[k]);
        std::sort(set.begin(), set.end());
        std::vector<uint32_t> updated;
        uint64_t nrows = res.get_row_num();
        for (uint64_t i = 0; i < nrows; i++)
            if (std::binary_search(set.begin(), set.end(), res.get_row_col(i, col)))
                res.append_row_to(i, updated);
        res.result_table.swap(updated);
        req.pattern_step++;
    }

    // :132-189 (BASIC): keep the rows whose `end` value is a neighbour of the constant
    void const_to_known(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        int col = res.var2col(pattern.object);
        ORACLE_ASSERT(col != NO_RESULT, VERTEX_INVALID);
        uint64_t sz = 0;
        const uint32_t* vids = graph->get_triples((uint32_t)pattern.subject, (uint32_t)pattern.predicate,
                                                  pattern.direction, sz);
        std::vector<uint32_t> set(vids, vids + sz);
        std::sort(set.begin(), set.end());
        std::vector<uint32_t> updated;
        uint64_t nrows = res.get_row_num();
        for (uint64_t i = 0; i < nrows; i++)
            if (std::binary_search(set.begin(), set.end(), res.get_row_col(i, col)))
                res.append_row_to(i, updated);
        res.result_table.swap(updated);
        req.pattern_step++;
    }

    // The versatile operators (:554-739) read the vertex's predicate list [v|PREDICATE_ID|d]
    // and then the vertex's list for each of those predicates.
    // C ?P ?X (:559-592): a (p, x) row for every predicate p of C and neighbour x over p.
    void const_unknown_unknown(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        const uint32_t start = (uint32_t)pattern.subject;
        const int d = pattern.direction;
        uint64_t npids = 0;
        const uint32_t* pids = graph->get_triples(start, PREDICATE_ID, d, npids);
        std::vector<uint32_t> tpids(pids, pids + npids), updated;
        for (uint32_t p : tpids) {
            uint64_t sz = 0;
            const uint32_t* vids = graph->get_triples(start, p, d, sz);
            for (uint64_t k = 0; k < sz; k++) {
                updated.push_back(p);
                updated.push_back(vids[k]);
            }
        }
        res.result_table.swap(updated);
        res.col_num = 2;
        res.add_var2col(pattern.predicate, 0);
        res.add_var2col(pattern.object, 1);
        req.pattern_step++;
    }

    // ?X ?P ?Y (:600-640): every known row times its start's (p, y) pairs.
    void known_unknown_unknown(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        const int d = pattern.direction;
        std::vector<uint32_t> updated;
        uint64_t nrows = res.get_row_num();
        int cs = res.var2col(pattern.subject);
        for (uint64_t i = 0; i < nrows; i++) {
            uint32_t cur = res.get_row_col(i, cs);
            uint64_t npids = 0;
            const uint32_t* pids = graph->get_triples(cur, PREDICATE_ID, d, npids);
            std::vector<uint32_t> tpids(pids, pids + npids);
            for (uint32_t p : tpids) {
                uint64_t sz = 0;
                const uint32_t* vids = graph->get_triples(cur, p, d, sz);
                for (uint64_t k = 0; k < sz; k++) {
                    res.append_row_to(i, updated);
                    updated.push_back(p);
                    updated.push_back(vids[k]);
                }
            }
        }
        res.result_table.swap(updated);
        res.add_var2col(pattern.predicate, res.col_num);
        res.add_var2col(pattern.object, res.col_num + 1);
        res.col_num += 2;
        req.pattern_step++;
    }

    // ?X ?P C (:649-689): a row times every predicate of its start that reaches C.
    void known_unknown_const(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        const int d = pattern.direction;
        const uint32_t end = (uint32_t)pattern.object;
        std::vector<uint32_t> updated;
        uint64_t nrows = res.get_row_num();
        int cs = res.var2col(pattern.subject);
        for (uint64_t i = 0; i < nrows; i++) {
            uint32_t prev = res.get_row_col(i, cs);
            uint64_t npids = 0;
            const uint32_t* pids = graph->get_triples(prev, PREDICATE_ID, d, npids);
            std::vector<uint32_t> tpids(pids, pids + npids);
            for (uint32_t p : tpids) {
                uint64_t sz = 0;
                const uint32_t* vids = graph->get_triples(prev, p, d, sz);
                for (uint64_t k = 0; k < sz; k++)
                    if (vids[k] == end) {
                        res.append_row_to(i, updated);
                        updated.push_back(p);
                        break;
                    }
            }
        }
        res.result_table.swap(updated);
        res.add_var2col(pattern.predicate, res.col_num);
        res.col_num += 1;
        req.pattern_step++;
    }

    // C1 ?P C2 (:697-739): every predicate of C1 that reaches C2; first pattern only.
    void const_unknown_const(Query& req) {
        Pattern& pattern = req.patterns[req.pattern_step];
        ORACLE_ASSERT(pattern.pred_type == 0, UNKNOWN_PATTERN);
        Result& res = req.result;
        ORACLE_ASSERT(res.col_num == 0, FIRST_PATTERN_ERROR);
        const uint32_t start = (uint32_t)pattern.subject, end = (uint32_t)pattern.object;
        const int d = pattern.direction;
        uint64_t npids = 0;
        const uint32_t* pids = graph->get_triples(start, PREDICATE_ID, d, npids);
        std::vector<uint32_t> tpids(pids, pids + npids), updated;
        for (uint32_t p : tpids) {
            uint64_t sz = 0;
            const uint32_t* vids = graph->get_triples(start, p, d, sz);
            for (uint64_t k = 0; k < sz; k++)
                if (vids[k] == end) {
                    updated.push_back(p);
                    break;
                }
        }
        res.result_table.swap(updated);
        res.col_num = 1;
        res.add_var2col(pattern.predicate, 0);
        req.pattern_step++;
    }

    void execute_one_pattern(Query& req) {   // :932-1055
        Pattern& pattern = req.patterns[req.pattern_step];
        int32_t start = pattern.subject, predicate = pattern.predicate, end = pattern.object;
        if (req.pattern_step == 0 && req.start_from_index()) {
            if (req.result.var2col(end) != NO_RESULT)
                index_to_known(req);
            else
                index_to_unknown(req);
            return;
        }
        if (req.result.var_stat(predicate) != CONST_VAR) {
            // an unknown (or earlier bound) predicate: the VERSATILE operators, on a store that
            // holds the vertex-predicate lists; without them the pattern is unsupported
            ORACLE_ASSERT(graph->versatile, UNKNOWN_PATTERN);
            switch (const_pair(req.result.var_stat(start), req.result.var_stat(end))) {
            case const_pair(CONST_VAR, UNKNOWN_VAR): const_unknown_unknown(req); break;
            case const_pair(CONST_VAR, CONST_VAR): const_unknown_const(req); break;
            case const_pair(KNOWN_VAR, UNKNOWN_VAR): known_unknown_unknown(req); break;
            case const_pair(KNOWN_VAR, CONST_VAR): known_unknown_const(req); break;
            default: throw error_code(UNKNOWN_PATTERN);   // [C|?|K], [K|?|K], [U|?|*]
            }
            return;
        }
        switch (const_pair(req.result.var_stat(start), req.result.var_stat(end))) {
        case const_pair(CONST_VAR, KNOWN_VAR): const_to_known(req); break;
        case const_pair(CONST_VAR, UNKNOWN_VAR): const_to_unknown(req); break;
        case const_pair(KNOWN_VAR, CONST_VAR): known_to_const(req); break;
        case const_pair(KNOWN_VAR, KNOWN_VAR): known_to_known(req); break;
        case const_pair(KNOWN_VAR, UNKNOWN_VAR): known_to_unknown(req); break;
        case const_pair(UNKNOWN_VAR, CONST_VAR):
        case const_pair(UNKNOWN_VAR, KNOWN_VAR):
        case const_pair(UNKNOWN_VAR, UNKNOWN_VAR): throw error_code(UNKNOWN_SUB);
        default: throw error_code(UNKNOWN_PATTERN);   // CONST|CONST
        }
    }

    int run(Query& req) {
        try {
            while (req.pattern_step < (int)req.patterns.size()) execute_one_pattern(req);
        } catch (const error_code& e) {
            return e.code;
        }
        return SUCCESS;
    }
};

}  // namespace oracle

// ---------------------------------------------------------------- C entry points (ctypes)
using namespace oracle;

struct OracleStore {
    Store store;
};

extern "C" {

// Build the store from n x 3 (s, p, o) triples for each direction; versatile adds the
// vertex-predicate lists the unknown-predicate operators read.
void* orc_store_build2(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos, uint64_t n_pos,
                       int versatile) {
    auto* h = new OracleStore();
    h->store.versatile = versatile != 0;
    std::vector<triple_t> a(n_pso), b(n_pos);
    for (uint64_t i = 0; i < n_pso; ++i) a[i] = {pso[3 * i], pso[3 * i + 1], pso[3 * i + 2]};
    for (uint64_t i = 0; i < n_pos; ++i) b[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    try {
        h->store.init_gstore(std::move(a), std::move(b));
    } catch (const error_code&) {
        delete h;
        return nullptr;
    }
    return h;
}

void* orc_store_build(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos, uint64_t n_pos) {
    return orc_store_build2(pso, n_pso, pos, n_pos, 0);
}

void orc_store_free(void* h) { delete (OracleStore*)h; }

int orc_get_triples(void* h, uint32_t vid, uint32_t pid, int dir, const uint32_t** out, uint64_t* sz) {
    try {
        *out = ((OracleStore*)h)->store.get_triples(vid, pid, dir, *sz);
    } catch (const error_code& e) {
        return e.code;
    }
    return 0;
}

int orc_get_index(void* h, uint32_t pid, int dir, const uint32_t** out, uint64_t* sz) {
    return orc_get_triples(h, 0, pid, dir, out, sz);
}

// Export the store in the layout of wk_seg_meta (see include/wukong_b200.h) so that the GPU
// path can be fed a store built by the reference's own construction rules.
// seg_out rows: index, pid, dir, num_keys, num_buckets, bucket_start, num_edges, edge_start,
// ext_start, ext_num (10 x uint64 each).
void orc_store_sizes(void* h, uint64_t* n_slots, uint64_t* n_edges, uint64_t* n_segs) {
    Store& s = ((OracleStore*)h)->store;
    *n_slots = s.slots.size();
    *n_edges = s.values.size();
    *n_segs = s.seg_map.size();
}

// The store's slot and value arrays in place (borrowed: valid until orc_store_free).
void orc_store_arrays(void* h, const void** slots, const uint32_t** edges) {
    Store& s = ((OracleStore*)h)->store;
    *slots = s.slots.data();
    *edges = s.values.data();
}

// slots / edges may be null: only the segment rows are written.
void orc_store_export(void* h, void* slots, uint32_t* edges, uint64_t* seg_out) {
    Store& s = ((OracleStore*)h)->store;
    if (slots) std::memcpy(slots, s.slots.data(), s.slots.size() * sizeof(slot_t));
    if (edges && !s.values.empty()) std::memcpy(edges, s.values.data(), s.values.size() * 4);
    uint64_t i = 0;
    for (auto& kv : s.seg_map) {
        const segid_t& id = kv.first;
        const rdf_seg_meta_t& m = kv.second;
        uint64_t* r = seg_out + 10 * i++;
        r[0] = id.index;
        r[1] = id.pid;
        r[2] = id.dir;
        r[3] = m.num_keys;
        r[4] = m.num_buckets;
        r[5] = m.bucket_start;
        r[6] = m.num_edges;
        r[7] = m.edge_start;
        r[8] = m.ext_bucket_list.empty() ? 0 : m.ext_bucket_list[0].start;
        r[9] = m.ext_bucket_list.empty() ? 0 : m.ext_bucket_list[0].num_ext_buckets;
    }
}

// Run one planned query.  patterns: n x 5 int32 (subject, predicate, object, direction,
// pred_type).  mt_factor > 1 splits an index start into that many slices run on as many
// threads and concatenated in slice order.  On success *table is malloc'd (free with
// orc_free), v2c_map receives nvars entries.
int orc_query_run(void* h, const int32_t* patterns, int n, int nvars, int mt_factor,
                  uint32_t** table, uint64_t* rows, int* cols, int32_t* v2c_map) {
    const Store* st = &((OracleStore*)h)->store;
    Query base;
    for (int i = 0; i < n; ++i)
        base.patterns.push_back({patterns[5 * i], patterns[5 * i + 1], patterns[5 * i + 2],
                                 patterns[5 * i + 3], patterns[5 * i + 4]});
    base.result.nvars = nvars;
    if (mt_factor < 1) mt_factor = 1;
    bool split = false;
    try {
        split = mt_factor > 1 && base.start_from_index();
    } catch (const error_code& e) {
        return e.code;
    }
    std::vector<Query> subs(split ? mt_factor : 1, base);
    std::vector<int> rc(subs.size(), 0);
    if (split) {
        std::vector<std::thread> th;
        for (int t = 0; t < mt_factor; ++t) {
            subs[t].mt_factor = mt_factor;
            subs[t].mt_tid = t;
            th.emplace_back([&, t] { rc[t] = Engine(st).run(subs[t]); });
        }
        for (auto& x : th) x.join();
    } else {
        rc[0] = Engine(st).run(subs[0]);
    }
    for (int r : rc)
        if (r) return r;
    uint64_t total = 0;
    for (auto& q : subs) total += q.result.result_table.size();
    uint32_t* buf = (uint32_t*)std::malloc(std::max<uint64_t>(total, 1) * 4);
    uint64_t w = 0;
    for (auto& q : subs) {
        if (!q.result.result_table.empty())
            std::memcpy(buf + w, q.result.result_table.data(), q.result.result_table.size() * 4);
        w += q.result.result_table.size();
    }
    Result& r0 = subs[0].result;
    *table = buf;
    *cols = r0.col_num;
    *rows = r0.col_num ? total / r0.col_num : 0;
    if (r0.v2c_map.empty()) r0.v2c_map.assign(nvars, NO_RESULT);
    for (int i = 0; i < nvars; ++i) v2c_map[i] = r0.v2c_map[i];
    return 0;
}

// Run many light queries, one query per thread at a time over `threads` threads (the CPU
// engines each take whole queries).  offsets: n + 1 int32 into patterns (in patterns), nvars
// per query.  Returns per-query row counts and statuses; tables are discarded.
int orc_queries_run_parallel(void* h, const int32_t* patterns, const int32_t* offsets,
                             const int32_t* nvars, uint32_t n, int threads, uint64_t* rows,
                             int32_t* status) {
    const Store* st = &((OracleStore*)h)->store;
    std::atomic<uint32_t> next{0};
    if (threads < 1) threads = 1;
    auto worker = [&] {
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= n) break;
            Query q;
            for (int k = offsets[i]; k < offsets[i + 1]; ++k)
                q.patterns.push_back({patterns[5 * k], patterns[5 * k + 1], patterns[5 * k + 2],
                                      patterns[5 * k + 3], patterns[5 * k + 4]});
            q.result.nvars = nvars[i];
            status[i] = Engine(st).run(q);
            rows[i] = q.result.get_row_num();
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(worker);
    for (auto& x : th) x.join();
    return 0;
}

// Run one known_to_* operator over an arbitrary input table (rows x cols, row-major).
// op: 0 = known_to_unknown, 1 = known_to_known, 2 = known_to_const.  Column i of the input
// is variable -(i + 1); the unknown end of known_to_unknown is variable -(cols + 1).
int orc_step(void* h, int op, const uint32_t* table, uint64_t rows, int cols, int cs, int ce,
             uint32_t end_const, uint32_t pid, int dir, uint32_t** out, uint64_t* out_rows,
             int* out_cols) {
    const Store* st = &((OracleStore*)h)->store;
    Query q;
    Pattern p;
    p.subject = -(cs + 1);
    p.predicate = (int32_t)pid;
    p.direction = dir;
    p.pred_type = 0;
    p.object = op == 0 ? -(cols + 1) : (op == 1 ? -(ce + 1) : (int32_t)end_const);
    q.patterns.push_back(p);
    q.result.nvars = cols + 1;
    q.result.col_num = cols;
    q.result.v2c_map.assign(cols + 1, NO_RESULT);
    for (int i = 0; i < cols; ++i) q.result.v2c_map[i] = i;
    q.result.result_table.assign(table, table + rows * (uint64_t)cols);
    Engine e(st);
    try {
        if (op == 0) e.known_to_unknown(q);
        else if (op == 1) e.known_to_known(q);
        else e.known_to_const(q);
    } catch (const error_code& ex) {
        return ex.code;
    }
    auto& t = q.result.result_table;
    uint32_t* buf = (uint32_t*)std::malloc(std::max<size_t>(t.size(), 1) * 4);
    if (!t.empty()) std::memcpy(buf, t.data(), t.size() * 4);
    *out = buf;
    *out_cols = q.result.col_num;
    *out_rows = q.result.col_num ? t.size() / q.result.col_num : 0;
    return 0;
}

// Run one pattern through the dispatch (execute_one_pattern) on a given table: rows x cols,
// column i holding variable -(i + 1), nvars >= cols variables in all.  pattern: 5 int32 as in
// orc_query_run.  The table plays the result a pattern group starts with (as a union or
// optional sub-query inherits one), so the pattern runs as pattern 0: an index pattern whose
// object is known runs index_to_known, with the given mt slice.  On success *out (malloc'd)
// is the new table and v2c receives nvars entries.
int orc_pattern(void* h, const uint32_t* table, uint64_t rows, int cols, int nvars,
                const int32_t* pattern, int mt_tid, int mt_factor, uint32_t** out, uint64_t* out_rows,
                int* out_cols, int32_t* v2c) {
    const Store* st = &((OracleStore*)h)->store;
    Query q;
    q.patterns.push_back({pattern[0], pattern[1], pattern[2], pattern[3], pattern[4]});
    q.mt_tid = mt_tid;
    q.mt_factor = mt_factor < 1 ? 1 : mt_factor;
    q.result.nvars = nvars;
    q.result.col_num = cols;
    q.result.v2c_map.assign(nvars, NO_RESULT);
    for (int i = 0; i < cols && i < nvars; ++i) q.result.v2c_map[i] = i;
    q.result.result_table.assign(table, table + rows * (uint64_t)cols);
    int rc = Engine(st).run(q);
    if (rc) return rc;
    auto& t = q.result.result_table;
    uint32_t* buf = (uint32_t*)std::malloc(std::max<size_t>(t.size(), 1) * 4);
    if (!t.empty()) std::memcpy(buf, t.data(), t.size() * 4);
    *out = buf;
    *out_cols = q.result.col_num;
    *out_rows = q.result.col_num ? t.size() / q.result.col_num : 0;
    for (int i = 0; i < nvars; ++i) v2c[i] = q.result.v2c_map[i];
    return 0;
}

void orc_free(void* p) { std::free(p); }

}  // extern "C"
