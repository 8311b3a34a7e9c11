// The REFERENCE CPU engine, compiled from the reference's own headers (src/core/engine/
// sparql.hpp, src/core/sparql/query.hpp, src/core/store/vertex.hpp, src/utils/*, ...) as they
// lie in the reference tree, unmodified, against the stand-ins under oracle/refpin/stubs for
// what this path does not use (Boost and TBB names mapped onto the standard library; the
// messenger, the string server, core binding and the store base class reduced to what the
// engine calls).  Test infrastructure only: it is the checker's checker.  It pins the oracle's
// restatement of the pattern operators (sparql.hpp:197-552), their dispatch (:932-1055) and
// final_process (:1419-1546) to the reference's own code.
//
// A query runs through the engine's public entry point, SPARQLEngine::execute_sparql_query
// (sparql.hpp:1559-1664), as one server with one engine thread runs it: patterns, then the
// final stage (DISTINCT / OFFSET / LIMIT / projection), and the reply the messenger keeps.
// The graph it reads serves the lists it was given (get_triples / get_index, dgraph.hpp:225-232).
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <thread>
#include <unordered_map>
#include <vector>

#include "core/engine/sparql.hpp"
#include "core/store/segment_meta.hpp"

using namespace wukong;

namespace {

struct KeyHash {
    size_t operator()(uint64_t k) const { return std::hash<uint64_t>()(k * 0x9e3779b97f4a7c15ull); }
};

uint64_t pack(sid_t vid, sid_t pid, int dir) {
    return ((uint64_t)vid << 18) | ((uint64_t)pid << 1) | (uint64_t)(dir & 1);
}

class ListGraph : public DGraph {
public:
    std::unordered_map<uint64_t, std::vector<edge_t>, KeyHash> lists;
    edge_t* get_triples(int tid, sid_t vid, sid_t pid, dir_t d, uint64_t& sz) override {
        auto it = lists.find(pack(vid, pid, d));
        if (it == lists.end() || it->second.empty()) {
            sz = 0;
            return nullptr;
        }
        sz = it->second.size();
        return it->second.data();
    }
    edge_t* get_index(int tid, sid_t pid, dir_t d, uint64_t& sz) override {
        return get_triples(tid, 0, pid, d, sz);
    }
};

// A GStore built elsewhere (the slot array, the value array and the segment table, borrowed),
// served the way SegmentRDFGraph::get_triples / get_index (segment_rdf_dgraph.hpp:1114-1129)
// serve the local store: the key's segment from an ordered map of segid_t, then
// KVStore::get_values_local (kvstore.hpp:292-409) over the reference's own vertex_t / ikey_t /
// iptr_t and ikey_t::hash().  kvstore.hpp itself needs the RDMA, MPI and TBB headers, so its
// bucket walk is restated: slots 0-6 compared with the key, slot 7 empty ends the search, else
// its vid names the next bucket.  The walk is bounded by the bucket count, which the reference's
// is not (a store without a cycle never reaches the bound).
class SlotGraph : public DGraph {
public:
    const vertex_t* slots = nullptr;
    uint64_t num_buckets = 0;
    edge_t* values = nullptr;
    std::map<segid_t, rdf_seg_meta_t> segs;

    edge_t* lookup(const ikey_t& key, uint64_t& sz) {
        sz = 0;
        auto it = segs.find(segid_t(key));
        if (it == segs.end() || it->second.num_buckets == 0) return nullptr;
        const rdf_seg_meta_t& m = it->second;
        uint64_t b = m.bucket_start + key.hash() % m.num_buckets;
        for (uint64_t hop = 0; hop <= num_buckets && b < num_buckets; ++hop) {
            const vertex_t* bk = slots + b * 8;
            for (int i = 0; i < 7; ++i)
                if (bk[i].key == key) {
                    sz = bk[i].ptr.size;
                    return values + bk[i].ptr.off;
                }
            ikey_t link = bk[7].key;
            if (link.is_empty()) return nullptr;
            b = link.vid;
        }
        return nullptr;
    }
    edge_t* get_triples(int tid, sid_t vid, sid_t pid, dir_t d, uint64_t& sz) override {
        return lookup(ikey_t(vid, pid, d), sz);
    }
    edge_t* get_index(int tid, sid_t pid, dir_t d, uint64_t& sz) override {
        return lookup(ikey_t(0, pid, d), sz);
    }
};

void engine_globals() {
    static bool once = [] {
        Global::num_servers = 1;
        Global::num_threads = 2;
        Global::num_proxies = 1;
        Global::num_engines = 1;
        Global::silent = true;
        Global::enable_vattr = false;
        return true;
    }();
    (void)once;
}

}  // namespace

extern "C" {

void* wkref_graph_new() { return static_cast<DGraph*>(new ListGraph()); }
void wkref_graph_free(void* g) { delete static_cast<DGraph*>(g); }

// The list of key [vid | pid | dir] (vid 0: an index key), in list order (a graph made by
// wkref_graph_new only).
void wkref_graph_put(void* g, uint32_t vid, uint32_t pid, int dir, const uint32_t* vals, uint64_t n) {
    ListGraph* lg = dynamic_cast<ListGraph*>(static_cast<DGraph*>(g));
    if (!lg) return;
    auto& v = lg->lists[pack(vid, pid, dir)];
    v.resize(n);
    for (uint64_t i = 0; i < n; ++i) v[i].val = vals[i];
}

// A graph over a GStore's arrays, borrowed (they must outlive it): n_slots 16-byte slots,
// the value array, and n_segs segment rows of 10 uint64 (index, pid, dir, num_keys,
// num_buckets, bucket_start, num_edges, edge_start, ext_start, ext_num).
void* wkref_graph_from_store(const void* slots, uint64_t n_slots, const uint32_t* values,
                             const uint64_t* seg_rows, uint64_t n_segs) {
    static_assert(sizeof(vertex_t) == 16 && sizeof(edge_t) == 4, "GStore layout");
    SlotGraph* g = new SlotGraph();
    g->slots = static_cast<const vertex_t*>(slots);
    g->num_buckets = n_slots / 8;
    g->values = reinterpret_cast<edge_t*>(const_cast<uint32_t*>(values));
    for (uint64_t i = 0; i < n_segs; ++i) {
        const uint64_t* r = seg_rows + 10 * i;
        rdf_seg_meta_t m;
        m.num_keys = r[3];
        m.num_buckets = r[4];
        m.bucket_start = r[5];
        m.num_edges = r[6];
        m.edge_start = r[7];
        g->segs[segid_t((int)r[0], (sid_t)r[1], (dir_t)r[2])] = m;
    }
    return static_cast<DGraph*>(g);
}

// Run one planned query (n x 5 int32: subject, predicate, object, direction, pred_type) with
// `nvars` variables.  required (n_req variable ids) are the selected variables; distinct,
// limit (< 0: none) and offset are the query's modifiers.  On success *table (rows x cols,
// malloc'd) is the final table, v2c[nvars] its column map; the return is the engine's status
// code (errors.hpp), 0 on success.
int wkref_query(void* g, const int32_t* pats, int n, int nvars, const int32_t* required, int n_req,
                int distinct, int limit, uint32_t offset, uint32_t** table, uint64_t* rows, int* cols,
                int32_t* v2c) {
    engine_globals();
    SPARQLQuery::PatternGroup group;
    for (int i = 0; i < n; ++i) {
        SPARQLQuery::Pattern p(pats[5 * i], pats[5 * i + 1], (ssid_t)pats[5 * i + 3], pats[5 * i + 2]);
        p.pred_type = (char)pats[5 * i + 4];
        group.patterns.push_back(p);
    }
    std::vector<ssid_t> req(required, required + n_req);
    SPARQLQuery q(group, nvars, req);
    q.distinct = distinct != 0;
    q.limit = limit;
    q.offset = offset;
    q.pqid = 0;   // the reply goes to a proxy (thread 0), so the final stage runs
    Coder coder(0, 1);
    Messenger msgr;
    StringMapping str;
    SPARQLEngine engine(0, 1, &str, static_cast<DGraph*>(g), &coder, &msgr);
    engine.execute_sparql_query(q);
    if (msgr.replies.size() != 1) return UNKNOWN_ERROR;
    SPARQLQuery& r = msgr.replies[0];
    const int status = r.result.get_status_code();
    if (status != SUCCESS) return status;
    const uint64_t nr = r.result.get_row_num();
    const int nc = r.result.get_col_num();
    uint32_t* out = (uint32_t*)std::malloc(std::max<uint64_t>(nr * nc, 1) * sizeof(uint32_t));
    if (!out) return UNKNOWN_ERROR;
    for (uint64_t i = 0; i < nr * (uint64_t)nc; ++i) out[i] = r.result.result_table[i];
    *table = out;
    *rows = nr;
    *cols = nc;
    for (int i = 0; i < nvars; ++i) v2c[i] = r.result.var2col(-(i + 1));
    return SUCCESS;
}

// The engine's filter stage on a given table (rows x cols, variable -(c+1) in column c): one
// BOUND(?x) filter per column in bound_cols (Filter::Builtin_bound over a Variable argument),
// run through execute_sparql_query with no patterns, so execute_filter and then final_process
// (identity projection) apply.  *out (malloc'd) receives the kept rows.
int wkref_filter_bound(const uint32_t* table, uint64_t rows, int cols, const int32_t* bound_cols, int nb,
                       uint32_t** out, uint64_t* out_rows) {
    SPARQLQuery::PatternGroup group;
    for (int k = 0; k < nb; ++k) {
        SPARQLQuery::Filter f;
        f.type = SPARQLQuery::Filter::Type::Builtin_bound;
        f.arg1 = new SPARQLQuery::Filter();
        f.arg1->type = SPARQLQuery::Filter::Type::Variable;
        f.arg1->valueArg = -(bound_cols[k] + 1);
        group.filters.push_back(f);
    }
    std::vector<ssid_t> req;
    for (int c = 0; c < cols; ++c) req.push_back(-(c + 1));
    SPARQLQuery q(group, cols, req);
    for (int c = 0; c < cols; ++c) q.result.add_var2col(-(c + 1), c);
    q.result.set_col_num(cols);
    q.result.result_table.assign(table, table + rows * (uint64_t)cols);
    q.result.update_nrows();
    q.pqid = 0;
    Coder coder(0, 1);
    Messenger msgr;
    StringMapping str;
    SPARQLEngine engine(0, 1, &str, nullptr, &coder, &msgr);
    engine.execute_sparql_query(q);
    if (msgr.replies.size() != 1) return UNKNOWN_ERROR;
    SPARQLQuery& r = msgr.replies[0];
    if (r.result.get_status_code() != SUCCESS) return r.result.get_status_code();
    const uint64_t nr = r.result.get_row_num();
    uint32_t* o = (uint32_t*)std::malloc(std::max<uint64_t>(nr * cols, 1) * sizeof(uint32_t));
    if (!o) return UNKNOWN_ERROR;
    for (uint64_t i = 0; i < nr * (uint64_t)cols; ++i) o[i] = r.result.result_table[i];
    *out = o;
    *out_rows = nr;
    return SUCCESS;
}

// One pattern through the engine's dispatch over a given table (rows x cols, variable -(c+1) in
// column c, nvars variables), as the first pattern of a group that inherited that table (a
// union / optional sub-query does), so an index pattern with a known object runs
// index_to_known.  mt_factor > 1 runs slice mt_tid as the engine runs a forked sub-query: it
// reports to a parent, so the final stage does not run.  *out (malloc'd), *out_rows, *out_cols
// and v2c[nvars] receive the result; the return is the engine's status.
int wkref_pattern(void* g, const uint32_t* table, uint64_t rows, int cols, int nvars, const int32_t* pat,
                  int mt_tid, int mt_factor, uint32_t** out, uint64_t* out_rows, int* out_cols,
                  int32_t* v2c) {
    SPARQLQuery::PatternGroup group;
    SPARQLQuery::Pattern p(pat[0], pat[1], (ssid_t)pat[3], pat[2]);
    p.pred_type = (char)pat[4];
    group.patterns.push_back(p);
    std::vector<ssid_t> req;
    SPARQLQuery q(group, nvars, req);
    for (int c = 0; c < cols; ++c) q.result.add_var2col(-(c + 1), c);
    q.result.set_col_num(cols);
    q.result.result_table.assign(table, table + rows * (uint64_t)cols);
    q.result.update_nrows();
    q.mt_factor = mt_factor < 1 ? 1 : mt_factor;
    q.mt_tid = mt_tid;
    q.pqid = 1;   // a sub-query's reply (thread 1 is an engine): no dispatch, no final stage
    Coder coder(0, 1);
    Messenger msgr;
    StringMapping str;
    SPARQLEngine engine(0, 1, &str, static_cast<DGraph*>(g), &coder, &msgr);
    engine.execute_sparql_query(q);
    if (msgr.replies.size() != 1) return UNKNOWN_ERROR;
    SPARQLQuery& r = msgr.replies[0];
    if (r.result.get_status_code() != SUCCESS) return r.result.get_status_code();
    const uint64_t nr = r.result.get_row_num();
    const int nc = r.result.get_col_num();
    uint32_t* o = (uint32_t*)std::malloc(std::max<uint64_t>(nr * nc, 1) * sizeof(uint32_t));
    if (!o) return UNKNOWN_ERROR;
    for (uint64_t i = 0; i < nr * (uint64_t)nc; ++i) o[i] = r.result.result_table[i];
    *out = o;
    *out_rows = nr;
    *out_cols = nc;
    for (int i = 0; i < nvars; ++i) v2c[i] = r.result.var2col(-(i + 1));
    return SUCCESS;
}

// Many planned queries through execute_sparql_query on `threads` host threads, each with its own
// engine (as each engine thread of a server has one), whole queries per thread.  offsets:
// n + 1 int32 into patterns (5 int32 each); nvars per query.  The selected variables are the
// ones the patterns bind (each unknown predicate, then each unknown object, in pattern order),
// so the final stage's projection keeps the pattern stage's table; a variable that nothing
// binds must not be selected (the projection would read column -1).  The tables are dropped
// and only row counts and statuses come back.
int wkref_query_many(void* g, const int32_t* patterns, const int32_t* offsets, const int32_t* nvars,
                     uint32_t n, int threads, uint64_t* rows, int32_t* status) {
    engine_globals();
    std::atomic<uint32_t> next{0};
    if (threads < 1) threads = 1;
    auto worker = [&] {
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= n) break;
            SPARQLQuery::PatternGroup group;
            for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
                const int32_t* p = patterns + 5 * k;
                SPARQLQuery::Pattern pt(p[0], p[1], (ssid_t)p[3], p[2]);
                pt.pred_type = (char)p[4];
                group.patterns.push_back(pt);
            }
            std::vector<ssid_t> req;
            for (auto& pt : group.patterns)
                for (ssid_t x : {pt.predicate, pt.object})
                    if (x < 0 && std::find(req.begin(), req.end(), x) == req.end()) req.push_back(x);
            SPARQLQuery q(group, nvars[i], req);
            q.pqid = 0;
            Coder coder(0, 1);
            Messenger msgr;
            StringMapping str;
            SPARQLEngine engine(0, 1, &str, static_cast<DGraph*>(g), &coder, &msgr);
            engine.execute_sparql_query(q);
            if (msgr.replies.size() != 1) {
                status[i] = UNKNOWN_ERROR;
                rows[i] = 0;
                continue;
            }
            status[i] = msgr.replies[0].result.get_status_code();
            rows[i] = status[i] == SUCCESS ? msgr.replies[0].result.get_row_num() : 0;
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(worker);
    for (auto& x : th) x.join();
    return SUCCESS;
}

// One planned query split as the reference splits an index start over a server's engine threads
// (SPARQLEngine::dispatch, sparql.hpp:1057-1083): the proxy's query (mt_factor slices, every
// variable the patterns bind selected) goes to one engine, which sends mt_factor sub-queries
// (mt_tid 0 .. mt_factor - 1); each runs on its own engine on its own host thread and replies;
// the replies go back to the first engine, whose reply map merges them (rmap.hpp:56-110) and
// which then runs the final stage and replies to the proxy.  Returns the status; *rows the
// final table's rows.
int wkref_query_mt(void* g, const int32_t* pats, int n, int nvars, int mt_factor, uint64_t* rows) {
    engine_globals();
    *rows = 0;
    SPARQLQuery::PatternGroup group;
    for (int i = 0; i < n; ++i) {
        SPARQLQuery::Pattern p(pats[5 * i], pats[5 * i + 1], (ssid_t)pats[5 * i + 3], pats[5 * i + 2]);
        p.pred_type = (char)pats[5 * i + 4];
        group.patterns.push_back(p);
    }
    std::vector<ssid_t> req;
    for (auto& pt : group.patterns)
        for (ssid_t x : {pt.predicate, pt.object})
            if (x < 0 && std::find(req.begin(), req.end(), x) == req.end()) req.push_back(x);
    SPARQLQuery q(group, nvars, req);
    q.mt_factor = mt_factor < 1 ? 1 : mt_factor;
    q.pqid = 0;
    DGraph* graph = static_cast<DGraph*>(g);
    Coder coder(0, 1);
    Messenger msgr;
    StringMapping str;
    SPARQLEngine engine(0, 1, &str, graph, &coder, &msgr);
    engine.execute_sparql_query(q);
    // with one slice the query ran whole; otherwise msgr holds the sub-queries it sent
    std::vector<SPARQLQuery> subs;
    subs.swap(msgr.replies);
    if (q.mt_factor > 1) {
        std::vector<SPARQLQuery> replies(subs.size());
        std::vector<std::thread> th;
        for (size_t j = 0; j < subs.size(); ++j)
            th.emplace_back([&, j] {
                Coder c(0, 1);
                Messenger m;
                StringMapping st;
                SPARQLEngine e(0, 1, &st, graph, &c, &m);
                e.execute_sparql_query(subs[j]);
                if (m.replies.size() == 1) replies[j] = m.replies[0];
                else replies[j].result.set_status_code(UNKNOWN_ERROR);
            });
        for (auto& t : th) t.join();
        for (auto& r : replies) engine.execute_sparql_query(r);
        subs.swap(msgr.replies);
    }
    if (subs.size() != 1) return UNKNOWN_ERROR;
    const int status = subs[0].result.get_status_code();
    if (status == SUCCESS) *rows = subs[0].result.get_row_num();
    return status;
}

void wkref_free(void* p) { std::free(p); }

}  // extern "C"
