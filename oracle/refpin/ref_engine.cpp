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
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "core/engine/sparql.hpp"

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

}  // namespace

extern "C" {

void* wkref_graph_new() { return new ListGraph(); }
void wkref_graph_free(void* g) { delete static_cast<ListGraph*>(g); }

// The list of key [vid | pid | dir] (vid 0: an index key), in list order.
void wkref_graph_put(void* g, uint32_t vid, uint32_t pid, int dir, const uint32_t* vals, uint64_t n) {
    auto& v = static_cast<ListGraph*>(g)->lists[pack(vid, pid, dir)];
    v.resize(n);
    for (uint64_t i = 0; i < n; ++i) v[i].val = vals[i];
}

// Run one planned query (n x 5 int32: subject, predicate, object, direction, pred_type) with
// `nvars` variables.  required (n_req variable ids) are the selected variables; distinct,
// limit (< 0: none) and offset are the query's modifiers.  On success *table (rows x cols,
// malloc'd) is the final table, v2c[nvars] its column map; the return is the engine's status
// code (errors.hpp), 0 on success.
int wkref_query(void* g, const int32_t* pats, int n, int nvars, const int32_t* required, int n_req,
                int distinct, int limit, uint32_t offset, uint32_t** table, uint64_t* rows, int* cols,
                int32_t* v2c) {
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
    SPARQLEngine engine(0, 1, &str, static_cast<ListGraph*>(g), &coder, &msgr);
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
    SPARQLEngine engine(0, 1, &str, static_cast<ListGraph*>(g), &coder, &msgr);
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

void wkref_free(void* p) { std::free(p); }

}  // extern "C"
