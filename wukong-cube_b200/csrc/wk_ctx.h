// Device context, tables and plan resolution shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "wk_internal.h"
#include "wk_explore.h"
#include "wk_flat.h"
#include "wk_kernels.h"
#include "wk_versatile.h"

// A device result table (the reference's rbuf + GPUResult, query.hpp:311-362).
struct wk_table {
    uint32_t* d = nullptr;     // row-major elements
    uint64_t cap = 0;          // elements held
    uint64_t* d_rows = nullptr;// row count, written by the kernels
    int32_t cols = 0;
};

namespace wk {

// Host mirror of SPARQLQuery::Result's column bookkeeping (query.hpp:409-459).
struct ColMap {
    int nvars = 0;
    int col_num = 0;
    std::vector<int32_t> v2c;   // NO_RESULT (0xFFFF) when unbound
    explicit ColMap(int n) : nvars(n), v2c(n > 0 ? n : 0, WK_NO_RESULT) {}
    // 0 = KNOWN, 1 = UNKNOWN, 2 = CONST; -1 = invalid variable id (VERTEX_INVALID)
    int var_stat(int32_t id) const {
        if (id >= 0) return 2;
        int idx = -(id + 1);
        if (idx >= nvars) return -1;
        return v2c[idx] == WK_NO_RESULT ? 1 : 0;
    }
    int col(int32_t id) const { return v2c[-(id + 1)]; }
    void bind(int32_t id, int c) { v2c[-(id + 1)] = c; }
    // bind an unbound variable; false if it is bound already (add_var2col's assertion)
    bool bind_new(int32_t id, int c) {
        if (v2c[-(id + 1)] != WK_NO_RESULT) return false;
        v2c[-(id + 1)] = c;
        return true;
    }
};

// One resolved exploration step of a plan.
//   kIndex index_to_unknown, kConst const_to_unknown, kK2U / kK2K / kK2C known_to_*,
//   kC2K const_to_known, kI2K index_to_known (single steps only: a query starts unbound),
//   kCUU / kCUC / kKUU / kKUC the unknown-predicate (versatile) operators.
struct PlanStep {
    enum Kind { kIndex, kConst, kK2U, kK2K, kK2C, kC2K, kI2K, kCUU, kCUC, kKUU, kKUC } kind;
    uint32_t pid = 0;
    int32_t dir = 0;
    uint32_t start_const = 0;   // kIndex: tpid; kConst: start vertex
    int32_t cs = 0, ce = 0;     // input columns
    uint32_t end_const = 0;     // kK2C, kKUC, kCUC
    int32_t in_cols = 0, out_cols = 0;
    int32_t mt_tid = 0, mt_factor = 1;   // kI2K: the slice of the index list
};

// Resolve a planned pattern list into steps, as SPARQLEngine::execute_one_pattern dispatches
// (sparql.hpp:932-1055; the GPU engine's gpu_engine.hpp:265-338 is its subset).  With
// `versatile` (the store holds the vertex-predicate lists) an unknown predicate goes to the
// versatile operators, else it is WK_UNKNOWN_PATTERN.  Returns a WK_* status; fills v2c_map /
// col_num of the result.
int resolve_plan(const wk_query& q, int max_cols, std::vector<PlanStep>& steps, ColMap& cm,
                 bool versatile = false);
inline bool is_versatile_step(int kind) {
    return kind == PlanStep::kCUU || kind == PlanStep::kCUC || kind == PlanStep::kKUU || kind == PlanStep::kKUC;
}

}  // namespace wk

struct wk_ctx {
    std::mutex mu;
    wk_config cfg{};
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;

    // resident store
    wk::Slot* d_slots = nullptr;
    uint64_t n_slots = 0;
    uint32_t* d_edges = nullptr;
    uint64_t n_edges = 0;
    std::vector<wk_seg_meta> segs;
    wk::SegIndex index;
    bool has_store = false;
    bool versatile = false;           // the store holds the vertex-predicate lists
    wk::PredSeg* d_pseg = nullptr;    // predicate segments by pid * 2 + dir (versatile steps)
    uint32_t n_pseg = 0;
    std::map<uint32_t, uint64_t> index_len;   // tpid * 2 + dir -> length of its index list
    uint64_t* d_inline_orig = nullptr;   // (slot index, original pointer word) of every slot
    uint64_t n_inline = 0;               // whose one-entry list is kept in the slot itself
    bool borrowed_store = false;   // a serving lane: the store belongs to its parent context
    wk::CtaUse beside_use{0, 0, 0};   // a serving lane leaves room on every SM for this many
    int beside_ctas = 0;              // resident CTAs of this size (the iteration launches)
    int sorted_lists = 0;
    int default_lanes = 2;
    int batch_lanes = 4;
    std::map<int, int> tuned_lanes;
    uint64_t spin_limit = 0;         // polls of a bounded wait on another CTA (0: the default)
    uint32_t slice_rows = 0;         // list length above which rows go to the slice queue
    uint32_t batch_slice_rows = 0;   // (0: the kernel's default, kHeavyRows)
    int32_t batch_flat = 0;          // bit k: batch level k runs as the flat passes, not tiles
    // single-query steps with at least this many input rows run the flat pipeline (0: never)
    uint64_t flat_min_rows = 65536;
    void* d_flat = nullptr;          // its scratch (wk_flat.h)
    uint64_t flat_cap_rows = 0;
    void* d_final_scratch = nullptr;   // scratch of the post-pattern stage and the BOUND filter
    size_t final_scratch_bytes = 0;

    // scan control of the context stream
    wk::StepCtl* d_ctl = nullptr;
    wk::HeavyItem* d_heavy = nullptr;    // long-list slices of the context stream
    uint64_t heavy_cap = 0;
    unsigned long long* d_status = nullptr;
    uint64_t status_cap = 0;
    wk::StepCtl* h_ctl = nullptr;     // pinned
    uint64_t* h_rows = nullptr;       // pinned
    uint32_t inject_err = 0;          // error bits the next control-block read reports (tests)

    // ping-pong result buffers for whole queries (GPUMem rbuf pair, gpu_mem.hpp:53-60)
    wk_table rbuf[2];

    // CUDA graphs of resident query plans
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        const wk_table* final_table = nullptr;
        uint64_t cap0 = 0, cap1 = 0;
    };
    std::map<std::string, GraphEntry> graphs;

    std::map<long long, int> bps_cache;   // (op, cols) -> blocks per SM
    std::string last_error;

    // batch / serving state (wk_batch.cu); batch2 is the second state of the pipelined path
    void* batch = nullptr;
    void* batch2 = nullptr;
    void* batch_host = nullptr;   // plans, streams and events reused by every batch call
    // serving lanes, kept between serving runs so their tables stay grown (wk_serve.cu)
    std::vector<wk_ctx*> lanes;
    wk::CtaUse lanes_use{0, 0, 0};
    int lanes_ctas = 0;

    wk::DevStore dev_store() const {
        wk::DevStore s;
        s.slots = d_slots;
        s.n_buckets = n_slots / wk::kAssoc;
        s.edges = d_edges;
        s.n_edges = n_edges;
        return s;
    }
    wk::SegDesc seg_of(uint64_t vid, uint32_t pid, int dir) const {
        int32_t i = index.find(vid, pid, dir);
        wk::SegDesc d{0, 0, 0, 0};
        if (i >= 0 && pid < (1u << wk::kNbitsIdx)) d = wk::to_desc(segs[i]);
        return d;
    }
    int fail(int code, const std::string& msg) {
        last_error = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        last_error = std::string(what) + ": " + cudaGetErrorString(e);
        return WK_E_CUDA;
    }
    int blocks_per_sm(int op, int cols, int lanes);
    // lanes per probe group for (op, cols): the tuned choice, else 2 (one 32-byte sector)
    int lanes_for(int op, int cols) const {
        auto it = tuned_lanes.find(op * 1000 + cols);
        return it != tuned_lanes.end() ? it->second : default_lanes;
    }
    void drop_graphs();
    int ensure_status(uint64_t tiles);
    int ensure_heavy(uint64_t out_rows_cap);
    int ensure_flat(uint64_t in_rows_cap);
    int final_scratch_reserve(size_t bytes);
    int table_reserve(wk_table* t, uint64_t elems);
    int read_ctl(uint32_t* err, uint64_t* need);
    int clear_ctl_err();
};

namespace wk {
// How a known_to_* step of a single query is launched.
enum FlatMode {
    kTileOnly = 0,   // the tile launch (wk_explore.cu)
    kFlatAuto = 1,   // both, each guarded on the device by flat_min_rows: one of them runs
    kFlatOnly = 2,   // the flat pipeline (wk_flat.cu); needs ensure_flat for the input
};
// Enqueue one resolved step reading `in` (may be null for index/const starts) into `out`.
int enqueue_step(wk_ctx* ctx, const PlanStep& st, const wk_table* in, wk_table* out,
                 int32_t mt_tid, int32_t mt_factor, cudaStream_t s, int grid_override,
                 int flat_mode = kTileOnly);
// The device descriptor of a resolved step.
StepDesc make_step_desc(const wk_ctx* ctx, const PlanStep& s);

// A context on its own (lowest-priority) stream with its own control block, status array,
// slice queue and tables, reading the parent's resident store; its exploration launches
// leave room on every SM for `beside_ctas` CTAs of size `beside_use`.  Released with
// wk_ctx_destroy, before the parent.
int ctx_make_child(wk_ctx* parent, const CtaUse& beside_use, int beside_ctas, wk_ctx** out);
// Run a whole query (mode: WK_MODE_RESIDENT or WK_MODE_GRAPH) and report its final table and row
// count (host sync).
int query_run_rows(wk_ctx* ctx, const wk_query* q, int32_t mode, const wk_table** t, uint64_t* rows);
// Copy `elems` elements of a device table to host memory (host sync).
int table_copy_out(wk_ctx* ctx, const wk_table* t, uint64_t elems, uint32_t* host);
// Size a serving lane's tables and scan scratch for `elems`-element tables up front.
int lane_prepare(wk_ctx* lane, uint64_t elems);
// Make device arrays (dev_malloc'd) the context's store; the context owns them from here on.
int store_adopt(wk_ctx* ctx, Slot* d_slots, uint64_t n_slots, uint32_t* d_edges, uint64_t n_edges,
                const std::vector<wk_seg_meta>& segs);
cudaError_t gbuild_kernel_attrs();   // wk_gbuild.cu
// Lanes for one (explore op, input columns) step of single queries (the autotuner's choice).
int tune_step_lanes(wk_ctx* ctx, int op, int cols, int lanes);
}  // namespace wk
