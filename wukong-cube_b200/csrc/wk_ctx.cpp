// C ABI: context, resident store, result tables, single steps and whole queries.
//
// Stands in for the reference's GPUEngine / GPUEngineCuda / GPUMem / GPUCache
// (src/gpu/gpu_engine.hpp, gpu_engine_cuda.hpp, gpu_mem.hpp, gpu_cache.hpp).  The whole store
// is uploaded once and stays resident, so there is no segment paging, no per-step mapping
// upload and no per-step host sync unless the caller asks for the plain mode.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "wk_batch.h"
#include "wk_ctx.h"

#define WK_CUDA(ctx, call)                                   \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call); \
    } while (0)

namespace {

const char* kMessages[] = {
    "Everything is ok",
    "Something wrong happened",
    "Something wrong in the query syntax, fail to parse!",
    "Unsupported triple pattern.",
    "MUST enable attribute support!",
    "NO required variables!",
    "Unsupport UNION on attribute results",
    "Object should not be an index",
    "Subject or object is not valid",
    "Tripple pattern should not start from unknown subject.",
    "You may change SETTING files to avoid this error. (e.g. global.hpp/config/...)",
    "Const_X_X or index_X_X must be the first pattern.",
    "Unsupported filter type.",
    "Query file not found.",
};

constexpr uint64_t kPadWords = 16;

std::atomic<uint64_t> g_device_allocs{0};

}  // namespace

void wk::note_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
uint64_t wk::device_alloc_count() { return g_device_allocs.load(std::memory_order_relaxed); }

extern "C" int wk_debug_device_allocs(uint64_t* count) {
    if (!count) return WK_E_BADARG;
    *count = wk::device_alloc_count();
    return WK_SUCCESS;
}

extern "C" const char* wk_strerror(int code) {
    if (code >= 0 && code < (int)(sizeof(kMessages) / sizeof(kMessages[0]))) return kMessages[code];
    switch (code) {
    case WK_E_OOM: return "device allocation failed";
    case WK_E_CAPACITY: return "result or working set exceeds a configured capacity";
    case WK_E_TIMEOUT: return "a bounded device-side wait gave up";
    case WK_E_BADARG: return "invalid argument";
    case WK_E_CUDA: return "CUDA runtime error";
    case WK_E_NOSTORE: return "no GStore uploaded";
    case WK_E_CORRUPT: return "key table chain out of range";
    case WK_E_UNSUPPORTED: return "unsupported on this path";
    default: return "unknown status";
    }
}

extern "C" const char* wk_last_error(const wk_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : "null context";
}

// ---------------------------------------------------------------- context helpers
int wk_ctx::blocks_per_sm(int op, int cols, int lanes) {
    long long k = ((long long)op * 1000 + cols) * 16 + lanes;
    auto it = bps_cache.find(k);
    if (it != bps_cache.end()) return it->second;
    const int w_out = (op == wk::kXK2U || op == wk::kXStart) ? cols + 1 : cols;
    int nb = beside_ctas > 0 ? wk::explore_blocks_beside(cols, w_out, lanes, beside_use, beside_ctas)
                             : wk::explore_blocks_per_sm(cols, w_out, lanes);
    bps_cache[k] = nb;
    return nb;
}

int wk_ctx::ensure_heavy(uint64_t out_rows_cap) {
    const uint64_t need = out_rows_cap / wk::kMinSliceRows + 64;
    if (need <= heavy_cap) return WK_SUCCESS;
    const uint64_t cap = need + need / 2;
    WK_CUDA(this, cudaStreamSynchronize(stream));
    if (d_heavy) cudaFree(d_heavy);
    d_heavy = nullptr;
    heavy_cap = 0;
    if (wk::dev_malloc(&d_heavy, cap * sizeof(wk::HeavyItem)) != cudaSuccess) {
        cudaGetLastError();
        return fail(WK_E_OOM, "long-list slice queue");
    }
    heavy_cap = cap;
    drop_graphs();
    return WK_SUCCESS;
}

int wk_ctx::ensure_flat(uint64_t in_rows_cap) {
    if (in_rows_cap <= flat_cap_rows && d_flat) return WK_SUCCESS;
    const uint64_t rows = std::max<uint64_t>(in_rows_cap + in_rows_cap / 4, 1 << 16);
    WK_CUDA(this, cudaStreamSynchronize(stream));
    if (d_flat) cudaFree(d_flat);
    d_flat = nullptr;
    flat_cap_rows = 0;
    if (wk::dev_malloc(&d_flat, wk::flat_scratch_bytes(rows, wk::flat_grid(sm_count))) != cudaSuccess) {
        cudaGetLastError();
        return fail(WK_E_OOM, "flat pipeline scratch");
    }
    flat_cap_rows = rows;
    drop_graphs();   // captured launches hold the old scratch pointers
    return WK_SUCCESS;
}

int wk_ctx::final_scratch_reserve(size_t bytes) {
    if (bytes <= final_scratch_bytes) return WK_SUCCESS;
    WK_CUDA(this, cudaStreamSynchronize(stream));
    if (d_final_scratch) cudaFree(d_final_scratch);
    d_final_scratch = nullptr;
    final_scratch_bytes = 0;
    const size_t cap = bytes + bytes / 4;
    if (wk::dev_malloc(&d_final_scratch, cap) != cudaSuccess) {
        cudaGetLastError();
        return fail(WK_E_OOM, "post-pattern scratch");
    }
    final_scratch_bytes = cap;
    return WK_SUCCESS;
}

int wk_ctx::ensure_status(uint64_t tiles) {
    if (tiles <= status_cap) return WK_SUCCESS;
    uint64_t cap = std::max<uint64_t>(tiles + tiles / 2, 1 << 14);
    WK_CUDA(this, cudaStreamSynchronize(stream));
    if (d_status) WK_CUDA(this, cudaFree(d_status));
    d_status = nullptr;
    if (wk::dev_malloc(&d_status, cap * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        status_cap = 0;
        return fail(WK_E_OOM, "status array");
    }
    WK_CUDA(this, cudaMemsetAsync(d_status, 0, cap * sizeof(unsigned long long), stream));
    unsigned long long c = cap;
    WK_CUDA(this, cudaMemcpyAsync(&d_ctl->status_cap, &c, sizeof(c), cudaMemcpyHostToDevice, stream));
    WK_CUDA(this, cudaStreamSynchronize(stream));
    status_cap = cap;
    drop_graphs();   // captured launches hold the old status pointer
    return WK_SUCCESS;
}

void wk_ctx::drop_graphs() {
    for (auto& g : graphs)
        if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    graphs.clear();
}

int wk_ctx::table_reserve(wk_table* t, uint64_t elems) {
    if (t->cap >= elems && t->d) return WK_SUCCESS;
    if (t == &rbuf[0] || t == &rbuf[1]) drop_graphs();
    WK_CUDA(this, cudaStreamSynchronize(stream));
    if (t->d) cudaFree(t->d);
    t->d = nullptr;
    t->cap = 0;
    if (wk::dev_malloc(&t->d, (elems + kPadWords) * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(WK_E_OOM, "result table of " + std::to_string(elems) + " elements");
    }
    t->cap = elems;
    if (!t->d_rows) {
        if (wk::dev_malloc(&t->d_rows, sizeof(uint64_t)) != cudaSuccess) {
            cudaGetLastError();
            return fail(WK_E_OOM, "row counter");
        }
        WK_CUDA(this, cudaMemsetAsync(t->d_rows, 0, sizeof(uint64_t), stream));
    }
    return WK_SUCCESS;
}

int wk_ctx::read_ctl(uint32_t* err, uint64_t* need) {
    WK_CUDA(this, cudaMemcpyAsync(h_ctl, d_ctl, sizeof(wk::StepCtl), cudaMemcpyDeviceToHost, stream));
    WK_CUDA(this, cudaStreamSynchronize(stream));
    *err = h_ctl->err | inject_err;   // a failure staged by wk_debug_fail_next counts once
    *need = h_ctl->need;
    inject_err = 0;
    return WK_SUCCESS;
}

extern "C" int wk_debug_fail_next(wk_ctx* ctx, uint32_t err_bits) {
    if (!ctx || (err_bits & ~(uint32_t)(wk::kErrOverflow | wk::kErrTimeout | wk::kErrCorrupt))) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->inject_err = err_bits;
    return WK_SUCCESS;
}

int wk_ctx::clear_ctl_err() {
    WK_CUDA(this, cudaMemsetAsync(&d_ctl->err, 0, sizeof(unsigned), stream));
    WK_CUDA(this, cudaMemsetAsync(&d_ctl->need, 0, sizeof(unsigned long long), stream));
    return WK_SUCCESS;
}

// ---------------------------------------------------------------- plan resolution
namespace wk {

int resolve_plan(const wk_query& q, int max_cols, std::vector<PlanStep>& steps, ColMap& cm,
                 bool versatile) {
    steps.clear();
    if (q.n_patterns < 0 || q.nvars < 0 || (q.n_patterns > 0 && !q.patterns)) return WK_E_BADARG;
    for (int i = 0; i < q.n_patterns; ++i) {
        const wk_pattern& p = q.patterns[i];
        if (p.direction != WK_IN && p.direction != WK_OUT) return WK_E_BADARG;
        PlanStep st{};
        st.dir = p.direction;
        if (i == 0 && is_tpid(p.subject)) {
            // start_from_index (query.hpp:816-838) -> index_to_unknown (sparql.hpp:197-234)
            if (p.predicate != WK_PREDICATE_ID && p.predicate != WK_TYPE_ID) return WK_OBJ_ERROR;
            int vs = cm.var_stat(p.object);
            if (vs < 0 || vs == 2) return WK_VERTEX_INVALID;
            // index_to_known needs a known object, and nothing is bound before the first
            // pattern; the single step wk_step_index_to_known runs it over a given table
            if (vs == 0) return WK_UNKNOWN_PATTERN;
            if (p.pred_type != 0) return WK_UNKNOWN_PATTERN;
            st.kind = PlanStep::kIndex;
            st.start_const = (uint32_t)p.subject;
            st.in_cols = 0;
            st.out_cols = 1;
            cm.col_num = 1;
            cm.bind(p.object, 0);
            steps.push_back(st);
            continue;
        }
        const int vs = cm.var_stat(p.subject), ve = cm.var_stat(p.object);
        if (p.predicate < 0) {
            // an unknown (or earlier bound) predicate: the versatile operators (sparql.hpp:
            // 554-739, dispatch :954-1012); they read the vertex-predicate lists
            const int vp = cm.var_stat(p.predicate);
            if (vp < 0) return WK_VERTEX_INVALID;
            if (!versatile) return WK_UNKNOWN_PATTERN;
            if (vs < 0 || ve < 0) return WK_VERTEX_INVALID;
            if (p.pred_type != 0) return WK_UNKNOWN_PATTERN;
            if (vs == 2 && ve == 1) {            // C ?P ?X: the table becomes (p, x) rows
                st.kind = PlanStep::kCUU;
                st.start_const = (uint32_t)p.subject;
                st.in_cols = 0;
                st.out_cols = 2;
                cm.col_num = 2;
                // add_var2col asserts (UNKNOWN_ERROR) on a variable already bound, the
                // predicate's first, then the object's (which may be the same variable)
                if (!cm.bind_new(p.predicate, 0) || !cm.bind_new(p.object, 1)) return WK_UNKNOWN_ERROR;
            } else if (vs == 2 && ve == 2) {     // C1 ?P C2
                if (cm.col_num != 0) return WK_FIRST_PATTERN_ERROR;
                st.kind = PlanStep::kCUC;
                st.start_const = (uint32_t)p.subject;
                st.end_const = (uint32_t)p.object;
                st.in_cols = 0;
                st.out_cols = 1;
                cm.col_num = 1;
                if (!cm.bind_new(p.predicate, 0)) return WK_UNKNOWN_ERROR;
            } else if (vs == 0 && ve == 1) {     // ?X ?P ?Y
                st.kind = PlanStep::kKUU;
                st.cs = cm.col(p.subject);
                st.in_cols = cm.col_num;
                st.out_cols = cm.col_num + 2;
                if (st.out_cols > max_cols) return WK_E_CAPACITY;
                if (!cm.bind_new(p.predicate, cm.col_num) || !cm.bind_new(p.object, cm.col_num + 1))
                    return WK_UNKNOWN_ERROR;
                cm.col_num += 2;
            } else if (vs == 0 && ve == 2) {     // ?X ?P C
                st.kind = PlanStep::kKUC;
                st.cs = cm.col(p.subject);
                st.end_const = (uint32_t)p.object;
                st.in_cols = cm.col_num;
                st.out_cols = cm.col_num + 1;
                if (st.out_cols > max_cols) return WK_E_CAPACITY;
                if (!cm.bind_new(p.predicate, cm.col_num)) return WK_UNKNOWN_ERROR;
                cm.col_num += 1;
            } else {
                return WK_UNKNOWN_PATTERN;   // [C|?|K], [K|?|K], [U|?|*]
            }
            steps.push_back(st);
            continue;
        }
        if (p.pred_type != 0) return WK_ATTR_DISABLE;
        st.pid = (uint32_t)p.predicate;
        if (vs < 0 || ve < 0) return WK_VERTEX_INVALID;
        if (vs == 2 && ve == 1) {
            if (cm.col_num != 0) return WK_FIRST_PATTERN_ERROR;
            st.kind = PlanStep::kConst;
            st.start_const = (uint32_t)p.subject;
            st.in_cols = 0;
            st.out_cols = 1;
            cm.bind(p.object, 0);
            cm.col_num = 1;
        } else if (vs == 2 && ve == 0) {
            // C P ?X with ?X known: const_to_known (sparql.hpp:132-189)
            st.kind = PlanStep::kC2K;
            st.start_const = (uint32_t)p.subject;
            st.ce = cm.col(p.object);
            st.in_cols = st.out_cols = cm.col_num;
        } else if (vs == 0 && ve == 2) {
            st.kind = PlanStep::kK2C;
            st.cs = cm.col(p.subject);
            st.end_const = (uint32_t)p.object;
            st.in_cols = st.out_cols = cm.col_num;
        } else if (vs == 0 && ve == 0) {
            st.kind = PlanStep::kK2K;
            st.cs = cm.col(p.subject);
            st.ce = cm.col(p.object);
            st.in_cols = st.out_cols = cm.col_num;
        } else if (vs == 0 && ve == 1) {
            st.kind = PlanStep::kK2U;
            st.cs = cm.col(p.subject);
            st.in_cols = cm.col_num;
            st.out_cols = cm.col_num + 1;
            if (st.out_cols > max_cols) return WK_E_CAPACITY;
            cm.bind(p.object, cm.col_num);
            cm.col_num += 1;
        } else if (vs == 1) {
            return WK_UNKNOWN_SUB;
        } else {
            return WK_UNKNOWN_PATTERN;   // CONST|CONST
        }
        steps.push_back(st);
    }
    return WK_SUCCESS;
}

int enqueue_step(wk_ctx* ctx, const PlanStep& st, const wk_table* in, wk_table* out,
                 int32_t mt_tid, int32_t mt_factor, cudaStream_t s, int grid_override, int flat_mode) {
    out->cols = st.out_cols;
    if (st.kind == PlanStep::kIndex || st.kind == PlanStep::kConst) {
        ListArgs a{};
        a.store = ctx->dev_store();
        if (st.kind == PlanStep::kIndex) {
            a.key = make_key(0, st.start_const, st.dir);
            a.seg = ctx->seg_of(0, st.start_const, st.dir);
            a.mt_tid = mt_tid;
            a.mt_factor = mt_factor > 0 ? mt_factor : 1;
        } else {
            a.key = make_key(st.start_const, st.pid, st.dir);
            a.seg = ctx->seg_of(st.start_const, st.pid, st.dir);
            a.mt_tid = 0;
            a.mt_factor = 1;
        }
        a.out = out->d;
        a.out_rows = out->d_rows;
        a.out_cap = out->cap;
        a.ctl = ctx->d_ctl;
        // index lists are long (every instance of a type, every subject of a predicate): a
        // full-occupancy grid; a constant's list is usually short
        int grid = st.kind == PlanStep::kIndex ? ctx->sm_count * 8 : std::min(ctx->sm_count * 2, 512);
        if (grid_override > 0) grid = grid_override;
        cudaError_t e = launch_list(a, grid, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "list kernel launch");
        return WK_SUCCESS;
    }
    if (is_versatile_step(st.kind)) {
        // one virtual row for the constant forms; the flat scratch holds the per-row counts
        const bool virt = st.kind == PlanStep::kCUU || st.kind == PlanStep::kCUC;
        if (!virt && (!in || st.in_cols <= 0)) return WK_E_BADARG;
        if (!ctx->d_flat) return ctx->fail(WK_E_BADARG, "versatile step without its scratch");
        VersArgs v{};
        v.store = ctx->dev_store();
        v.vp_seg = ctx->seg_of(1, kPredicateId, st.dir);
        v.pseg = ctx->d_pseg;
        v.n_pseg = ctx->n_pseg;
        v.op = st.kind == PlanStep::kKUU ? kVKUU : st.kind == PlanStep::kKUC ? kVKUC
             : st.kind == PlanStep::kCUU ? kVCUU : kVCUC;
        v.dir = st.dir;
        v.virtual_row = virt ? 1 : 0;
        v.start_const = st.start_const;
        v.end_const = st.end_const;
        v.cs = st.cs;
        v.cin = virt ? 0 : st.in_cols;
        v.in_rows = in ? in->d_rows : nullptr;
        v.in = in ? in->d : nullptr;
        v.w_in = virt ? 0 : st.in_cols;
        v.in_cap_rows = virt ? 1 : in->cap / st.in_cols;
        if (!virt && v.in_cap_rows > ctx->flat_cap_rows)
            return ctx->fail(WK_E_BADARG, "versatile step scratch smaller than its input");
        v.out = out->d;
        v.w_out = st.out_cols;
        v.out_cap_rows = out->cap / st.out_cols;
        v.out_rows = out->d_rows;
        v.pos = reinterpret_cast<uint64_t*>(ctx->d_flat);
        v.part = v.pos + 2 * ctx->flat_cap_rows + 1;
        v.ctl = ctx->d_ctl;
        v.sorted_lists = ctx->sorted_lists;
        cudaError_t e = launch_versatile(v, vers_grid(virt ? 1 : v.in_cap_rows, ctx->sm_count), s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "versatile step launch");
        return WK_SUCCESS;
    }
    if (!in || st.in_cols <= 0) return WK_E_BADARG;
    ExploreArgs a{};
    a.store = ctx->dev_store();
    a.seg_index[0] = ctx->seg_of(0, 0, kIn);
    a.seg_index[1] = ctx->seg_of(0, 0, kOut);
    a.one = make_step_desc(ctx, st);
    a.desc = nullptr;
    a.n_queries = 1;
    a.virtual_rows = 0;
    a.in_rows = in->d_rows;
    a.owner_in = nullptr;
    a.in = in->d;
    a.w_in = st.in_cols;
    a.in_cap_rows = in->cap / st.in_cols;
    a.out = out->d;
    a.w_out = st.out_cols;
    a.out_cap_rows = out->cap / st.out_cols;
    a.owner_out = nullptr;
    a.out_rows = out->d_rows;
    a.qfirst = a.qcount = nullptr;
    a.heavy = ctx->d_heavy;
    a.heavy_cap = ctx->heavy_cap;
    a.ctl = ctx->d_ctl;
    a.status = ctx->d_status;
    a.sorted_lists = ctx->sorted_lists;
    a.lanes = ctx->lanes_for(a.one.op, st.in_cols);
    a.slice_rows = ctx->slice_rows;
    a.spin_limit = ctx->spin_limit;
    // The flat pipeline needs its scratch sized for this input; without it the tile launch runs.
    if (!ctx->flat_min_rows || !ctx->d_flat || a.in_cap_rows > ctx->flat_cap_rows ||
        a.in_cap_rows < ctx->flat_min_rows || grid_override > 0)
        flat_mode = kTileOnly;
    if (flat_mode != kFlatOnly) {
        if (flat_mode == kFlatAuto) a.max_rows = ctx->flat_min_rows;
        int grid = grid_override > 0 ? grid_override
                                     : ctx->blocks_per_sm(a.one.op, st.in_cols, a.lanes) * ctx->sm_count;
        cudaError_t e = launch_explore(a, grid, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "exploration launch");
    }
    if (flat_mode != kTileOnly) {
        FlatArgs f{};
        f.store = a.store;
        f.seg_index[0] = a.seg_index[0];
        f.seg_index[1] = a.seg_index[1];
        f.step = a.one;
        f.in_rows = a.in_rows;
        f.in = a.in;
        f.w_in = a.w_in;
        f.in_cap_rows = a.in_cap_rows;
        f.out = a.out;
        f.w_out = a.w_out;
        f.out_cap_rows = a.out_cap_rows;
        f.out_rows = a.out_rows;
        f.min_rows = flat_mode == kFlatAuto ? ctx->flat_min_rows : 0;
        // a serving lane leaves room on every SM for the iteration launches' CTAs beside it
        const int grid = ctx->beside_ctas > 0 ? flat_grid_beside(ctx->sm_count, ctx->beside_use, ctx->beside_ctas)
                                              : flat_grid(ctx->sm_count);
        f.pos = reinterpret_cast<uint64_t*>(ctx->d_flat);
        f.off = f.pos + ctx->flat_cap_rows + 1;
        f.part = f.off + ctx->flat_cap_rows;
        f.ctl = ctx->d_ctl;
        f.sorted_lists = ctx->sorted_lists;
        cudaError_t e = launch_flat(f, grid, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "flat pipeline launch");
    }
    return WK_SUCCESS;
}

StepDesc make_step_desc(const wk_ctx* ctx, const PlanStep& s) {
    StepDesc d;
    std::memset(&d, 0, sizeof(d));
    d.dir = (uint8_t)s.dir;
    d.cin = (uint8_t)s.in_cols;
    d.cout = (uint8_t)s.out_cols;
    d.cs = (uint8_t)s.cs;
    d.ce = (uint8_t)s.ce;
    d.pid = s.pid;
    d.end_const = s.end_const;
    switch (s.kind) {
    case PlanStep::kIndex:
        d.op = kXStart;
        d.start_key = make_key(0, s.start_const, s.dir);
        d.seg = ctx->seg_of(0, s.start_const, s.dir);
        break;
    case PlanStep::kConst:
        d.op = kXStart;
        d.start_key = make_key(s.start_const, s.pid, s.dir);
        d.seg = ctx->seg_of(s.start_const, s.pid, s.dir);
        break;
    case PlanStep::kK2U:
        d.op = kXK2U;
        d.type_index = (s.pid == kTypeId && s.dir == kIn) ? 1 : 0;
        d.seg = ctx->seg_of(1, s.pid, s.dir);   // any nonzero vid: the normal segment
        break;
    case PlanStep::kK2K:
        d.op = kXK2K;
        d.seg = ctx->seg_of(1, s.pid, s.dir);
        break;
    case PlanStep::kC2K:
        d.op = kXC2K;
        d.start_key = make_key(s.start_const, s.pid, s.dir);
        d.seg = ctx->seg_of(s.start_const, s.pid, s.dir);
        break;
    case PlanStep::kI2K:
        d.op = kXI2K;
        d.start_key = make_key(0, s.start_const, s.dir);
        d.seg = ctx->seg_of(0, s.start_const, s.dir);
        d.mt = (uint32_t)(s.mt_tid & 0xFFFF) | ((uint32_t)(s.mt_factor & 0xFFFF) << 16);
        break;
    default:
        d.op = kXK2C;
        d.seg = ctx->seg_of(1, s.pid, s.dir);
        break;
    }
    return d;
}

}  // namespace wk

// ---------------------------------------------------------------- context
static int ctx_init_device(wk_ctx* ctx, bool low_priority);

extern "C" int wk_ctx_create(const wk_config* cfg, wk_ctx** out) {
    if (!out) return WK_E_BADARG;
    wk_ctx* ctx = nullptr;
    try {
        ctx = new wk_ctx();
    } catch (const std::bad_alloc&) {
        return WK_E_OOM;
    }
    if (cfg) ctx->cfg = *cfg;
    if (ctx->cfg.max_cols <= 0) ctx->cfg.max_cols = 32;
    if (ctx->cfg.max_cols > 32) {
        delete ctx;
        return WK_E_BADARG;   // shared-memory staging holds at most 32 columns per row
    }
    if (ctx->cfg.rbuf_bytes == 0) ctx->cfg.rbuf_bytes = 64ull << 20;
    if (ctx->cfg.working_set_cap_bytes == 0) ctx->cfg.working_set_cap_bytes = 40ull << 30;
    ctx->device = ctx->cfg.device;
    int rc = ctx_init_device(ctx, false);
    if (rc) {
        wk_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return WK_SUCCESS;
}

int wk::ctx_make_child(wk_ctx* parent, const CtaUse& beside_use, int beside_ctas, wk_ctx** out) {
    wk_ctx* ctx = nullptr;
    try {
        ctx = new wk_ctx();
    } catch (const std::bad_alloc&) {
        return parent->fail(WK_E_OOM, "serving lane");
    }
    ctx->cfg = parent->cfg;
    ctx->device = parent->device;
    ctx->beside_use = beside_use;
    ctx->beside_ctas = std::max(0, beside_ctas);
    int rc = ctx_init_device(ctx, true);
    if (rc) {
        parent->last_error = "serving lane: " + ctx->last_error;
        wk_ctx_destroy(ctx);
        return rc;
    }
    ctx->d_slots = parent->d_slots;
    ctx->n_slots = parent->n_slots;
    ctx->d_edges = parent->d_edges;
    ctx->n_edges = parent->n_edges;
    ctx->segs = parent->segs;
    ctx->index = parent->index;
    ctx->has_store = parent->has_store;
    ctx->versatile = parent->versatile;
    ctx->d_pseg = parent->d_pseg;
    ctx->n_pseg = parent->n_pseg;
    ctx->borrowed_store = true;
    ctx->sorted_lists = parent->sorted_lists;
    ctx->default_lanes = parent->default_lanes;
    ctx->batch_lanes = parent->batch_lanes;
    ctx->tuned_lanes = parent->tuned_lanes;
    *out = ctx;
    return WK_SUCCESS;
}

// Stream, control block and status array of a new context on its device.  Lanes (children)
// get the lowest stream priority so that pending CTAs of the parent's launches go first.
static int ctx_init_device(wk_ctx* ctx, bool low_priority) {
    auto bail = [&](cudaError_t e, const char* what) {
        cudaGetLastError();
        ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
        return WK_E_CUDA;
    };
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return bail(e, "cudaSetDevice");
    e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e != cudaSuccess) return bail(e, "sm count");
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e != cudaSuccess) return bail(e, "stream priorities");
    e = cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, low_priority ? least : greatest);
    if (e != cudaSuccess) return bail(e, "stream");
    e = wk::explore_kernel_attrs();
    if (e == cudaSuccess) e = wk::small_kernel_attrs();
    if (e == cudaSuccess) e = wk::batch_kernel_attrs();
    if (e == cudaSuccess) e = wk::serve_kernel_attrs();
    if (e == cudaSuccess) e = wk::flat_kernel_attrs();
    if (e == cudaSuccess) e = wk::final_kernel_attrs();
    if (e == cudaSuccess) e = wk::versatile_kernel_attrs();
    if (e == cudaSuccess) e = wk::gbuild_kernel_attrs();
    if (e != cudaSuccess) return bail(e, "kernel attributes");
    e = wk::dev_malloc(&ctx->d_ctl, sizeof(wk::StepCtl));
    if (e != cudaSuccess) return bail(e, "control block");
    e = cudaMallocHost(&ctx->h_ctl, sizeof(wk::StepCtl));
    if (e != cudaSuccess) return bail(e, "pinned control block");
    e = cudaMallocHost(&ctx->h_rows, sizeof(uint64_t) * 4);
    if (e != cudaSuccess) return bail(e, "pinned rows");
    wk::StepCtl init{};
    init.epoch = 1;
    e = cudaMemcpy(ctx->d_ctl, &init, sizeof(init), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(e, "control init");
    return ctx->ensure_status(1 << 14);
}

void wk_batch_release(wk_ctx* ctx);   // wk_batch.cu

extern "C" int wk_ctx_destroy(wk_ctx* ctx) {
    if (!ctx) return WK_E_BADARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (wk_ctx* lane : ctx->lanes) wk_ctx_destroy(lane);   // they read this context's store
    ctx->lanes.clear();
    wk_batch_release(ctx);
    ctx->drop_graphs();
    for (auto& t : ctx->rbuf) {
        if (t.d) cudaFree(t.d);
        if (t.d_rows) cudaFree(t.d_rows);
    }
    if (ctx->d_slots && !ctx->borrowed_store) cudaFree(ctx->d_slots);
    if (ctx->d_edges && !ctx->borrowed_store) cudaFree(ctx->d_edges);
    if (ctx->d_pseg && !ctx->borrowed_store) cudaFree(ctx->d_pseg);
    if (ctx->d_inline_orig && !ctx->borrowed_store) cudaFree(ctx->d_inline_orig);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->d_heavy) cudaFree(ctx->d_heavy);
    if (ctx->d_flat) cudaFree(ctx->d_flat);
    if (ctx->d_final_scratch) cudaFree(ctx->d_final_scratch);
    if (ctx->d_ctl) cudaFree(ctx->d_ctl);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->h_rows) cudaFreeHost(ctx->h_rows);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return WK_SUCCESS;
}

extern "C" int wk_ctx_sync(wk_ctx* ctx) {
    if (!ctx) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return WK_SUCCESS;
}

extern "C" int wk_ctx_stream(wk_ctx* ctx, void** stream) {
    if (!ctx || !stream) return WK_E_BADARG;
    *stream = (void*)ctx->stream;
    return WK_SUCCESS;
}

// ---------------------------------------------------------------- store
extern "C" int wk_store_upload(wk_ctx* ctx, const wk_seg_meta* segs, uint32_t n_segs,
                               const void* slots, uint64_t n_slots, const uint32_t* edges,
                               uint64_t n_edges) {
    if (!ctx || (!segs && n_segs) || (!slots && n_slots) || (!edges && n_edges)) return WK_E_BADARG;
    if (n_slots % wk::kAssoc) return ctx->fail(WK_E_BADARG, "slot count is not a multiple of 8");
    // the exploration probe holds bucket ids in 32 bits (2^32 buckets would be 512 GiB)
    if (n_slots / wk::kAssoc >= (1ull << 32)) return ctx->fail(WK_E_CAPACITY, "2^32 buckets or more");
    std::lock_guard<std::mutex> lk(ctx->mu);
    const uint64_t nb = n_slots / wk::kAssoc;
    for (uint32_t i = 0; i < n_segs; ++i) {
        const wk_seg_meta& m = segs[i];
        if (m.dir != WK_IN && m.dir != WK_OUT)
            return ctx->fail(WK_E_BADARG, "segment direction");
        if (m.bucket_start > nb || m.num_buckets > nb - m.bucket_start)
            return ctx->fail(WK_E_CORRUPT, "segment buckets outside the slot array");
        if (m.edge_start + m.num_edges > n_edges)
            return ctx->fail(WK_E_CORRUPT, "segment edges outside the edge array");
    }
    WK_CUDA(ctx, cudaSetDevice(ctx->device));
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_slots) cudaFree(ctx->d_slots);
    if (ctx->d_edges) cudaFree(ctx->d_edges);
    ctx->d_slots = nullptr;
    ctx->d_edges = nullptr;
    ctx->has_store = false;
    if (wk::dev_malloc(&ctx->d_slots, std::max<uint64_t>(n_slots, wk::kAssoc) * sizeof(wk::Slot)) != cudaSuccess ||
        wk::dev_malloc(&ctx->d_edges, (n_edges + kPadWords) * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return ctx->fail(WK_E_OOM, "store upload");
    }
    if (n_slots)
        WK_CUDA(ctx, cudaMemcpy(ctx->d_slots, slots, n_slots * sizeof(wk::Slot), cudaMemcpyHostToDevice));
    if (n_edges)
        WK_CUDA(ctx, cudaMemcpy(ctx->d_edges, edges, n_edges * sizeof(uint32_t), cudaMemcpyHostToDevice));
    std::vector<wk_seg_meta> sv(segs, segs + n_segs);
    wk::Slot* ds = ctx->d_slots;
    uint32_t* de = ctx->d_edges;
    return wk::store_adopt(ctx, ds, n_slots, de, n_edges, sv);
}

// Make device arrays the context's store: segment lookup, predicate segment table, the
// sorted-list check.  The context owns the arrays from here on, on failure too.
int wk::store_adopt(wk_ctx* ctx, Slot* d_slots, uint64_t n_slots, uint32_t* d_edges, uint64_t n_edges,
                    const std::vector<wk_seg_meta>& segs) {
    ctx->d_slots = d_slots;
    ctx->d_edges = d_edges;
    ctx->n_slots = n_slots;
    ctx->n_edges = n_edges;
    ctx->has_store = false;
    const uint32_t n_segs = (uint32_t)segs.size();
    ctx->segs = segs;
    ctx->index.build(ctx->segs.data(), n_segs);
    {
        // the predicate segments by pid * 2 + dir, for the versatile steps' list walks; a
        // vertex-predicate segment (pid PREDICATE_ID) makes the store versatile
        std::vector<wk::PredSeg> ps;
        ctx->versatile = false;
        for (uint32_t i = 0; i < n_segs; ++i) {
            const wk_seg_meta& m = segs[i];
            if (m.index || m.pid >= (1u << wk::kNbitsIdx)) continue;
            if (m.pid == wk::kPredicateId) ctx->versatile = true;
            ps.push_back(wk::PredSeg{m.pid * 2 + (uint32_t)m.dir, 0, wk::to_desc(m)});
        }
        std::sort(ps.begin(), ps.end(), [](const wk::PredSeg& a, const wk::PredSeg& b) { return a.key < b.key; });
        if (ctx->d_pseg) cudaFree(ctx->d_pseg);
        ctx->d_pseg = nullptr;
        ctx->n_pseg = 0;
        if (wk::dev_malloc(&ctx->d_pseg, std::max<size_t>(ps.size(), 1) * sizeof(wk::PredSeg)) != cudaSuccess) {
            cudaGetLastError();
            return ctx->fail(WK_E_OOM, "predicate segment table");
        }
        if (!ps.empty())
            WK_CUDA(ctx, cudaMemcpy(ctx->d_pseg, ps.data(), ps.size() * sizeof(wk::PredSeg), cudaMemcpyHostToDevice));
        ctx->n_pseg = (uint32_t)ps.size();
    }
    {
        // the index lists' lengths (the keys [0|tpid|dir] of the two index segments: a few
        // buckets per predicate and type), which the serving admission projects from
        ctx->index_len.clear();
        const uint64_t nb = n_slots / wk::kAssoc;
        std::vector<wk::Slot> bk;
        for (int d = 0; d < 2; ++d) {
            const int32_t i = ctx->index.index_seg[d];
            if (i < 0) continue;
            const wk_seg_meta& m = segs[i];
            const uint64_t ranges[2][2] = {{m.bucket_start, m.num_buckets}, {m.ext_start, m.ext_num}};
            for (auto& r : ranges) {
                if (!r[1] || r[0] >= nb || r[1] > nb - r[0]) continue;
                bk.resize(r[1] * wk::kAssoc);
                WK_CUDA(ctx, cudaMemcpy(bk.data(), d_slots + r[0] * wk::kAssoc, bk.size() * sizeof(wk::Slot),
                                        cudaMemcpyDeviceToHost));
                for (size_t k = 0; k < bk.size(); ++k) {
                    const uint64_t key = bk[k].key;
                    if (k % wk::kAssoc == wk::kAssoc - 1 || key == 0 || wk::key_vid(key) != 0) continue;
                    ctx->index_len[wk::key_pid(key) * 2 + wk::key_dir(key)] = wk::ptr_size(bk[k].ptr);
                }
            }
        }
    }
    ctx->has_store = true;
    {
        // are all lists ascending + unique?  (lets the filters binary-search long lists)
        unsigned* d_flag = nullptr;
        WK_CUDA(ctx, wk::dev_malloc(&d_flag, sizeof(unsigned)));
        WK_CUDA(ctx, cudaMemsetAsync(d_flag, 0, sizeof(unsigned), ctx->stream));
        cudaError_t e = wk::launch_sorted_check(ctx->dev_store(), d_flag, ctx->stream);
        unsigned flag = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, d_flag, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(d_flag);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "sorted-list check");
        if (flag & 2u) {
            ctx->has_store = false;
            return ctx->fail(WK_E_CORRUPT, "a key's list lies outside the edge array");
        }
        ctx->sorted_lists = (flag & 1u) ? 0 : 1;
    }
    {
        // one-entry lists into their keys' pointer words, the original words kept aside: count,
        // then convert
        if (ctx->d_inline_orig) cudaFree(ctx->d_inline_orig);
        ctx->d_inline_orig = nullptr;
        ctx->n_inline = 0;
        struct Counts {
            unsigned long long n;
            unsigned clash, pad;
        };
        Counts* d_c = nullptr;
        Counts h_c{};
        WK_CUDA(ctx, wk::dev_malloc(&d_c, sizeof(Counts)));
        cudaError_t e = cudaMemsetAsync(d_c, 0, sizeof(Counts), ctx->stream);
        if (e == cudaSuccess) e = wk::launch_inline(ctx->dev_store(), &d_c->n, &d_c->clash, nullptr, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_c, d_c, sizeof(Counts), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e == cudaSuccess && !h_c.clash && h_c.n) {
            if (wk::dev_malloc(&ctx->d_inline_orig, h_c.n * 16) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(d_c);
                ctx->has_store = false;
                return ctx->fail(WK_E_OOM, "one-entry list table");
            }
            e = cudaMemsetAsync(d_c, 0, sizeof(Counts), ctx->stream);
            if (e == cudaSuccess)
                e = wk::launch_inline(ctx->dev_store(), &d_c->n, &d_c->clash, ctx->d_inline_orig, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            ctx->n_inline = h_c.n;
        }
        cudaFree(d_c);
        if (e != cudaSuccess) {
            ctx->has_store = false;
            return ctx->cuda_fail(e, "one-entry lists");
        }
        if (h_c.clash) {
            ctx->has_store = false;
            return ctx->fail(WK_E_UNSUPPORTED, "a pointer word of type 3 (attribute values are not served)");
        }
    }
    ctx->drop_graphs();
    return WK_SUCCESS;
}

// A copy of the context's store in host memory, in the layout wk_store_upload takes.
extern "C" int wk_store_export(wk_ctx* ctx, void* slots, uint64_t slots_cap, uint32_t* edges, uint64_t edges_cap,
                               wk_seg_meta* segs, uint32_t segs_cap, uint64_t* n_slots, uint64_t* n_edges,
                               uint32_t* n_segs) {
    if (!ctx) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n_slots) *n_slots = ctx->n_slots;
    if (n_edges) *n_edges = ctx->n_edges;
    if (n_segs) *n_segs = (uint32_t)ctx->segs.size();
    if (!slots && !edges && !segs) return WK_SUCCESS;   // sizes only
    if ((slots && slots_cap < ctx->n_slots) || (edges && edges_cap < ctx->n_edges) ||
        (segs && segs_cap < ctx->segs.size()))
        return ctx->fail(WK_E_CAPACITY, "export buffers too small");
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (slots && ctx->n_slots) {
        WK_CUDA(ctx, cudaMemcpy(slots, ctx->d_slots, ctx->n_slots * sizeof(wk::Slot), cudaMemcpyDeviceToHost));
        // the device copy keeps one-entry lists in their keys' pointer words; put the original
        // words back
        if (ctx->n_inline) {
            std::vector<uint64_t> orig(ctx->n_inline * 2);
            WK_CUDA(ctx, cudaMemcpy(orig.data(), ctx->d_inline_orig, orig.size() * 8, cudaMemcpyDeviceToHost));
            wk::Slot* h = static_cast<wk::Slot*>(slots);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)ctx->n_inline; ++i) h[orig[2 * i]].ptr = orig[2 * i + 1];
        }
    }
    if (edges && ctx->n_edges)
        WK_CUDA(ctx, cudaMemcpy(edges, ctx->d_edges, ctx->n_edges * 4, cudaMemcpyDeviceToHost));
    if (segs && !ctx->segs.empty()) std::memcpy(segs, ctx->segs.data(), ctx->segs.size() * sizeof(wk_seg_meta));
    return WK_SUCCESS;
}

extern "C" int wk_store_upload_gstore(wk_ctx* ctx, const wk_gstore* g) {
    if (!ctx || !g) return WK_E_BADARG;
    return wk_store_upload(ctx, g->segs.data(), (uint32_t)g->segs.size(), g->slots.data(),
                           g->slots.size(), g->edges.data(), g->edges.size());
}

extern "C" int wk_store_bytes(const wk_ctx* ctx, uint64_t* bytes) {
    if (!ctx || !bytes) return WK_E_BADARG;
    *bytes = ctx->n_slots * sizeof(wk::Slot) + ctx->n_edges * sizeof(uint32_t) +
             ctx->segs.size() * sizeof(wk_seg_meta);
    return WK_SUCCESS;
}

// ---------------------------------------------------------------- tables
extern "C" int wk_table_alloc(wk_ctx* ctx, uint64_t capacity_elems, wk_table** out) {
    if (!ctx || !out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    wk_table* t = new (std::nothrow) wk_table();
    if (!t) return WK_E_OOM;
    int rc = ctx->table_reserve(t, std::max<uint64_t>(capacity_elems, 1));
    if (rc) {
        delete t;
        return rc;
    }
    *out = t;
    return WK_SUCCESS;
}

extern "C" int wk_table_free(wk_ctx* ctx, wk_table* t) {
    if (!ctx || !t) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStreamSynchronize(ctx->stream);
    if (t->d) cudaFree(t->d);
    if (t->d_rows) cudaFree(t->d_rows);
    delete t;
    return WK_SUCCESS;
}

extern "C" int wk_table_upload(wk_ctx* ctx, wk_table* t, const uint32_t* host, uint64_t rows,
                               int32_t cols) {
    if (!ctx || !t || (!host && rows && cols) || cols < 0) return WK_E_BADARG;
    if (cols > ctx->cfg.max_cols) return ctx->fail(WK_E_CAPACITY, "too many columns");
    std::lock_guard<std::mutex> lk(ctx->mu);
    const uint64_t n = rows * (uint64_t)cols;
    int rc = ctx->table_reserve(t, std::max<uint64_t>(n, 1));
    if (rc) return rc;
    if (n) WK_CUDA(ctx, cudaMemcpyAsync(t->d, host, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h_rows[0] = cols ? rows : 0;
    WK_CUDA(ctx, cudaMemcpyAsync(t->d_rows, ctx->h_rows, 8, cudaMemcpyHostToDevice, ctx->stream));
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    t->cols = cols;
    return WK_SUCCESS;
}

static int table_rows(wk_ctx* ctx, const wk_table* t, uint64_t* rows) {
    WK_CUDA(ctx, cudaMemcpyAsync(ctx->h_rows, t->d_rows, 8, cudaMemcpyDeviceToHost, ctx->stream));
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *rows = ctx->h_rows[0];
    return WK_SUCCESS;
}

extern "C" int wk_table_shape(wk_ctx* ctx, const wk_table* t, uint64_t* rows, int32_t* cols) {
    if (!ctx || !t) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    uint64_t r = 0;
    int rc = table_rows(ctx, t, &r);
    if (rc) return rc;
    if (rows) *rows = r;
    if (cols) *cols = t->cols;
    return WK_SUCCESS;
}

static int table_download(wk_ctx* ctx, const wk_table* t, uint32_t* host, uint64_t cap_elems,
                          uint64_t* rows_out) {
    uint64_t r = 0;
    int rc = table_rows(ctx, t, &r);
    if (rc) return rc;
    if (rows_out) *rows_out = r;
    const uint64_t n = r * (uint64_t)t->cols;
    if (n > cap_elems) return ctx->fail(WK_E_CAPACITY, "host buffer too small");
    if (n > t->cap) return ctx->fail(WK_E_CORRUPT, "row count beyond table capacity");
    if (n) WK_CUDA(ctx, cudaMemcpyAsync(host, t->d, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return WK_SUCCESS;
}

extern "C" int wk_table_download(wk_ctx* ctx, const wk_table* t, uint32_t* host, uint64_t cap_elems) {
    if (!ctx || !t || (!host && cap_elems)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    return table_download(ctx, t, host, cap_elems, nullptr);
}

extern "C" int wk_table_device_ptr(wk_ctx* ctx, const wk_table* t, uint32_t** dptr) {
    if (!ctx || !t || !dptr) return WK_E_BADARG;
    *dptr = t->d;
    return WK_SUCCESS;
}

// ---------------------------------------------------------------- single steps (plain)
// Run one step with a host sync; grow the output and rerun if it did not fit.
static int run_step_sync(wk_ctx* ctx, const wk::PlanStep& st, const wk_table* in, wk_table* out,
                         int32_t mt_tid, int32_t mt_factor) {
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (wk::is_versatile_step(st.kind)) {
        if (!ctx->versatile)
            return ctx->fail(WK_UNKNOWN_PATTERN, "the store holds no vertex-predicate lists (build it versatile)");
        int rc = ctx->ensure_flat(in && in->cols > 0 ? in->cap / in->cols : 1);
        if (rc) return rc;
    }
    int flat = wk::kTileOnly;
    if (in && in->cols > 0 && !wk::is_versatile_step(st.kind)) {
        int rc = ctx->ensure_status(in->cap / in->cols / wk::kTileRows + 2);
        if (rc) return rc;
        // the host syncs after every step here anyway, so it picks the launch by the row count
        uint64_t rows = 0;
        rc = table_rows(ctx, in, &rows);
        if (rc) return rc;
        // a row count past the capacity marks a table whose writing step overflowed
        if (rows * (uint64_t)in->cols > in->cap)
            return ctx->fail(WK_E_CORRUPT, "input row count beyond table capacity");
        if (ctx->flat_min_rows && rows >= ctx->flat_min_rows) {
            rc = ctx->ensure_flat(in->cap / in->cols);
            if (rc) return rc;
            flat = wk::kFlatOnly;
        }
    }
    for (int attempt = 0; attempt < 8; ++attempt) {
        int rc = ctx->ensure_heavy(out->cap);
        if (rc) return rc;
        rc = wk::enqueue_step(ctx, st, in, out, mt_tid, mt_factor, ctx->stream, 0, flat);
        if (rc) return rc;
        uint32_t err = 0;
        uint64_t need = 0;
        rc = ctx->read_ctl(&err, &need);
        if (rc) return rc;
        if (!err) return WK_SUCCESS;
        rc = ctx->clear_ctl_err();
        if (rc) return rc;
        if (err & wk::kErrCorrupt) return ctx->fail(WK_E_CORRUPT, "key table chain out of range");
        if (err & wk::kErrTimeout) return ctx->fail(WK_E_TIMEOUT, "tile look-back timed out");
        if (err & wk::kErrStatus) return ctx->fail(WK_E_CAPACITY, "status array too small");
        if (err & wk::kErrOverflow) {
            // `need` counts rows (the list copy of a start step has one column)
            const uint64_t elems = need * (uint64_t)std::max(st.out_cols, 1);
            rc = ctx->table_reserve(out, elems + elems / 8 + 1024);
            if (rc) return rc;
        }
    }
    return ctx->fail(WK_E_CAPACITY, "output kept overflowing");
}

static int check_in(wk_ctx* ctx, const wk_table* in, int32_t cs, int32_t ce) {
    if (!in || in->cols <= 0) return ctx->fail(WK_E_BADARG, "input table has no columns");
    if (cs < 0 || cs >= in->cols || ce < 0 || ce >= in->cols)
        return ctx->fail(WK_E_BADARG, "column out of range");
    return WK_SUCCESS;
}

extern "C" int wk_step_index_to_unknown(wk_ctx* ctx, uint32_t tpid, int32_t dir, int32_t mt_tid,
                                        int32_t mt_factor, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || mt_factor < 1 || mt_tid < 0)
        return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kIndex;
    st.start_const = tpid;
    st.dir = dir;
    st.out_cols = 1;
    return run_step_sync(ctx, st, nullptr, out, mt_tid, mt_factor);
}

extern "C" int wk_step_const_to_unknown(wk_ctx* ctx, uint32_t vid, uint32_t pid, int32_t dir,
                                        wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kConst;
    st.start_const = vid;
    st.pid = pid;
    st.dir = dir;
    st.out_cols = 1;
    return run_step_sync(ctx, st, nullptr, out, 0, 1);
}

extern "C" int wk_step_known_to_unknown(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                        uint32_t pid, int32_t dir, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || in == out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    int rc = check_in(ctx, in, col_start, col_start);
    if (rc) return rc;
    if (in->cols + 1 > ctx->cfg.max_cols) return ctx->fail(WK_E_CAPACITY, "too many columns");
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kK2U;
    st.pid = pid;
    st.dir = dir;
    st.cs = col_start;
    st.in_cols = in->cols;
    st.out_cols = in->cols + 1;
    return run_step_sync(ctx, st, in, out, 0, 1);
}

extern "C" int wk_step_known_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                      int32_t col_end, uint32_t pid, int32_t dir, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || in == out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    int rc = check_in(ctx, in, col_start, col_end);
    if (rc) return rc;
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kK2K;
    st.pid = pid;
    st.dir = dir;
    st.cs = col_start;
    st.ce = col_end;
    st.in_cols = st.out_cols = in->cols;
    return run_step_sync(ctx, st, in, out, 0, 1);
}

extern "C" int wk_step_known_to_const(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                      uint32_t end_vid, uint32_t pid, int32_t dir, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || in == out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    int rc = check_in(ctx, in, col_start, col_start);
    if (rc) return rc;
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kK2C;
    st.pid = pid;
    st.dir = dir;
    st.cs = col_start;
    st.end_const = end_vid;
    st.in_cols = st.out_cols = in->cols;
    return run_step_sync(ctx, st, in, out, 0, 1);
}

// C P ?X with ?X known: const_to_known (sparql.hpp:132-189).
extern "C" int wk_step_const_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_end, uint32_t vid,
                                      uint32_t pid, int32_t dir, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || in == out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    int rc = check_in(ctx, in, col_end, col_end);
    if (rc) return rc;
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kC2K;
    st.start_const = vid;
    st.pid = pid;
    st.dir = dir;
    st.ce = col_end;
    st.in_cols = st.out_cols = in->cols;
    return run_step_sync(ctx, st, in, out, 0, 1);
}

// IDX P ?X with ?X known: index_to_known (sparql.hpp:83-130), slice mt_tid of mt_factor.
extern "C" int wk_step_index_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_end, uint32_t tpid,
                                      int32_t dir, int32_t mt_tid, int32_t mt_factor, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || in == out || mt_factor < 1 || mt_tid < 0 ||
        mt_factor > 0xFFFF)
        return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    int rc = check_in(ctx, in, col_end, col_end);
    if (rc) return rc;
    wk::PlanStep st{};
    st.kind = wk::PlanStep::kI2K;
    st.start_const = tpid;
    st.dir = dir;
    st.ce = col_end;
    st.mt_tid = mt_tid % mt_factor;
    st.mt_factor = mt_factor;
    st.in_cols = st.out_cols = in->cols;
    return run_step_sync(ctx, st, in, out, 0, 1);
}

// The unknown-predicate steps (sparql.hpp:554-739) on a versatile store.
static int versatile_step(wk_ctx* ctx, wk::PlanStep::Kind kind, const wk_table* in, int32_t col_start,
                          uint32_t start_vid, uint32_t end_vid, int32_t dir, wk_table* out) {
    if (!ctx || !out || (dir != WK_IN && dir != WK_OUT) || (in && in == out)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    wk::PlanStep st{};
    st.kind = kind;
    st.dir = dir;
    st.start_const = start_vid;
    st.end_const = end_vid;
    if (kind == wk::PlanStep::kKUU || kind == wk::PlanStep::kKUC) {
        int rc = check_in(ctx, in, col_start, col_start);
        if (rc) return rc;
        st.cs = col_start;
        st.in_cols = in->cols;
        st.out_cols = in->cols + (kind == wk::PlanStep::kKUU ? 2 : 1);
        if (st.out_cols > ctx->cfg.max_cols) return ctx->fail(WK_E_CAPACITY, "too many columns");
    } else {
        in = nullptr;
        st.out_cols = kind == wk::PlanStep::kCUU ? 2 : 1;
    }
    return run_step_sync(ctx, st, in, out, 0, 1);
}

extern "C" int wk_step_known_unknown_unknown(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                             int32_t dir, wk_table* out) {
    if (!in) return WK_E_BADARG;
    return versatile_step(ctx, wk::PlanStep::kKUU, in, col_start, 0, 0, dir, out);
}

extern "C" int wk_step_known_unknown_const(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                           uint32_t end_vid, int32_t dir, wk_table* out) {
    if (!in) return WK_E_BADARG;
    return versatile_step(ctx, wk::PlanStep::kKUC, in, col_start, 0, end_vid, dir, out);
}

extern "C" int wk_step_const_unknown_unknown(wk_ctx* ctx, uint32_t vid, int32_t dir, wk_table* out) {
    return versatile_step(ctx, wk::PlanStep::kCUU, nullptr, 0, vid, 0, dir, out);
}

extern "C" int wk_step_const_unknown_const(wk_ctx* ctx, uint32_t vid, uint32_t end_vid, int32_t dir,
                                           wk_table* out) {
    return versatile_step(ctx, wk::PlanStep::kCUC, nullptr, 0, vid, end_vid, dir, out);
}

// ---------------------------------------------------------------- whole queries
static std::string plan_key(const std::vector<wk::PlanStep>& steps, const wk_query& q,
                            const wk_ctx* ctx) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append((const char*)p, n); };
    for (auto& s : steps) put(&s, sizeof(s));
    put(&q.mt_tid, 4);
    put(&q.mt_factor, 4);
    for (auto& t : ctx->rbuf) {
        put(&t.d, sizeof(t.d));
        put(&t.cap, sizeof(t.cap));
    }
    put(&ctx->d_status, sizeof(ctx->d_status));
    put(&ctx->d_flat, sizeof(ctx->d_flat));
    put(&ctx->flat_cap_rows, sizeof(ctx->flat_cap_rows));
    put(&ctx->flat_min_rows, sizeof(ctx->flat_min_rows));
    return k;
}

// Plans that start from an index build large tables: their steps launch both the tile launch
// and the flat pipeline, and the device picks by the row count.
static int plan_flat_mode(const std::vector<wk::PlanStep>& steps) {
    return (!steps.empty() && steps[0].kind == wk::PlanStep::kIndex) ? wk::kFlatAuto : wk::kTileOnly;
}

// Flat scratch for every step input of a plan (the rbuf capacities bound the row counts).
static int plan_ensure_flat(wk_ctx* ctx, const std::vector<wk::PlanStep>& steps) {
    bool vers = false;
    for (auto& s : steps) vers |= wk::is_versatile_step(s.kind);
    if (!vers && (plan_flat_mode(steps) == wk::kTileOnly || !ctx->flat_min_rows)) return WK_SUCCESS;
    uint64_t rows = 1;
    for (size_t i = 1; i < steps.size(); ++i)
        if (steps[i].in_cols > 0) rows = std::max<uint64_t>(rows, ctx->rbuf[(i - 1) & 1].cap / steps[i].in_cols);
    // the versatile steps always use the scratch; the flat passes only from their threshold on
    return (vers || rows >= ctx->flat_min_rows) ? ctx->ensure_flat(rows) : WK_SUCCESS;
}

static int enqueue_plan(wk_ctx* ctx, const std::vector<wk::PlanStep>& steps, const wk_query& q) {
    const int fm = plan_flat_mode(steps);
    for (size_t i = 0; i < steps.size(); ++i) {
        const wk_table* in = i ? &ctx->rbuf[(i - 1) & 1] : nullptr;
        wk_table* out = &ctx->rbuf[i & 1];
        int rc = wk::enqueue_step(ctx, steps[i], in, out, q.mt_tid, q.mt_factor, ctx->stream, 0, fm);
        if (rc) return rc;
    }
    return WK_SUCCESS;
}

static int query_run(wk_ctx* ctx, const wk_query* q, int32_t mode, const wk_table** out_table,
                     int32_t* v2c_map, int32_t* col_num) {
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    std::vector<wk::PlanStep> steps;
    wk::ColMap cm(q->nvars);
    int rc = wk::resolve_plan(*q, ctx->cfg.max_cols, steps, cm, ctx->versatile);
    if (rc) return ctx->fail(rc, wk_strerror(rc));
    if (q->mt_factor < 1 || q->mt_tid < 0) return ctx->fail(WK_E_BADARG, "mt_factor");
    for (auto& t : ctx->rbuf) {
        rc = ctx->table_reserve(&t, std::max<uint64_t>(t.cap, ctx->cfg.rbuf_bytes / 4));
        if (rc) return rc;
    }
    if (steps.empty()) {
        WK_CUDA(ctx, cudaMemsetAsync(ctx->rbuf[0].d_rows, 0, 8, ctx->stream));
        ctx->rbuf[0].cols = 0;
        *out_table = &ctx->rbuf[0];
    } else if (mode == WK_MODE_PLAIN) {
        // one launch per pattern, host sync + size read-back after each (the reference's shape)
        for (size_t i = 0; i < steps.size(); ++i) {
            const wk_table* in = i ? &ctx->rbuf[(i - 1) & 1] : nullptr;
            rc = run_step_sync(ctx, steps[i], in, &ctx->rbuf[i & 1], q->mt_tid, q->mt_factor);
            if (rc) return rc;
        }
        *out_table = &ctx->rbuf[(steps.size() - 1) & 1];
    } else {
        for (int attempt = 0;; ++attempt) {
            if (attempt >= 8) return ctx->fail(WK_E_CAPACITY, "results kept overflowing");
            uint64_t mx = std::max(ctx->rbuf[0].cap, ctx->rbuf[1].cap);
            rc = ctx->ensure_status(mx / wk::kTileRows + 2);
            if (rc) return rc;
            rc = ctx->ensure_heavy(mx);
            if (rc) return rc;
            rc = plan_ensure_flat(ctx, steps);
            if (rc) return rc;
            if (mode == WK_MODE_GRAPH) {
                std::string key = plan_key(steps, *q, ctx);
                auto it = ctx->graphs.find(key);
                if (it == ctx->graphs.end()) {
                    if (ctx->graphs.size() > 256) ctx->drop_graphs();
                    cudaGraph_t graph;
                    WK_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                    int erc = enqueue_plan(ctx, steps, *q);
                    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
                    if (erc) return erc;
                    if (ce != cudaSuccess) return ctx->cuda_fail(ce, "end capture");
                    wk_ctx::GraphEntry ge;
                    ce = cudaGraphInstantiate(&ge.exec, graph, 0);
                    cudaGraphDestroy(graph);
                    if (ce != cudaSuccess) return ctx->cuda_fail(ce, "graph instantiate");
                    it = ctx->graphs.emplace(key, ge).first;
                }
                WK_CUDA(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
            } else {
                rc = enqueue_plan(ctx, steps, *q);
                if (rc) return rc;
            }
            uint32_t err = 0;
            uint64_t need = 0;
            rc = ctx->read_ctl(&err, &need);
            if (rc) return rc;
            if (!err) break;
            rc = ctx->clear_ctl_err();
            if (rc) return rc;
            if (err & wk::kErrCorrupt) return ctx->fail(WK_E_CORRUPT, "key table chain out of range");
            if (err & wk::kErrTimeout) return ctx->fail(WK_E_TIMEOUT, "tile look-back timed out");
            if (err & (wk::kErrOverflow | wk::kErrStatus)) {
                int wmax = 1;
                for (auto& s : steps) wmax = std::max(wmax, s.out_cols);
                const uint64_t elems = need * (uint64_t)wmax;   // `need` counts rows
                uint64_t want = std::max<uint64_t>(elems + elems / 4, mx * 2);
                for (auto& t : ctx->rbuf) {
                    rc = ctx->table_reserve(&t, want);
                    if (rc) return rc;
                }
            }
        }
        *out_table = &ctx->rbuf[(steps.size() - 1) & 1];
    }
    // a replayed graph does not run enqueue_step, so set the final table's width here
    if (!steps.empty()) ctx->rbuf[(steps.size() - 1) & 1].cols = steps.back().out_cols;
    if (col_num) *col_num = cm.col_num;
    if (v2c_map)
        for (int i = 0; i < q->nvars; ++i) v2c_map[i] = cm.v2c[i];
    return WK_SUCCESS;
}

extern "C" int wk_query_execute(wk_ctx* ctx, const wk_query* q, int32_t mode,
                                const wk_table** out_table, int32_t* v2c_map, int32_t* col_num,
                                uint64_t* rows) {
    if (!ctx || !q || mode < 0 || mode > 2) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const wk_table* t = nullptr;
    int rc = query_run(ctx, q, mode, &t, v2c_map, col_num);
    if (rc) return rc;
    if (out_table) *out_table = t;
    if (rows) {
        rc = table_rows(ctx, t, rows);
        if (rc) return rc;
    }
    return WK_SUCCESS;
}

extern "C" int wk_query_execute_host(wk_ctx* ctx, const wk_query* q, int32_t mode, uint32_t* host_out,
                                     uint64_t cap_elems, int32_t* v2c_map, int32_t* col_num,
                                     uint64_t* rows) {
    if (!ctx || !q || mode < 0 || mode > 2 || (!host_out && cap_elems)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const wk_table* t = nullptr;
    int rc = query_run(ctx, q, mode, &t, v2c_map, col_num);
    if (rc) return rc;
    return table_download(ctx, t, host_out, cap_elems, rows);
}

int wk::query_run_rows(wk_ctx* ctx, const wk_query* q, int32_t mode, const wk_table** t, uint64_t* rows) {
    int rc = query_run(ctx, q, mode, t, nullptr, nullptr);
    if (rc) return rc;
    rc = table_rows(ctx, *t, rows);
    if (rc) return rc;
    if (*rows * (uint64_t)(*t)->cols > (*t)->cap)
        return ctx->fail(WK_E_CORRUPT, "row count beyond table capacity");
    return WK_SUCCESS;
}

int wk::lane_prepare(wk_ctx* lane, uint64_t elems) {
    elems = std::max<uint64_t>(elems, lane->cfg.rbuf_bytes / 4);
    for (auto& t : lane->rbuf) {
        int rc = lane->table_reserve(&t, std::max(t.cap, elems));
        if (rc) return rc;
    }
    const uint64_t mx = std::max(lane->rbuf[0].cap, lane->rbuf[1].cap);
    int rc = lane->ensure_status(mx / kTileRows + 2);
    if (!rc) rc = lane->ensure_heavy(mx);
    if (!rc && lane->flat_min_rows) rc = lane->ensure_flat(mx);
    return rc;
}

int wk::table_copy_out(wk_ctx* ctx, const wk_table* t, uint64_t elems, uint32_t* host) {
    if (elems > t->cap) return ctx->fail(WK_E_BADARG, "copy beyond table capacity");
    if (elems) WK_CUDA(ctx, cudaMemcpyAsync(host, t->d, elems * 4, cudaMemcpyDeviceToHost, ctx->stream));
    WK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return WK_SUCCESS;
}

// Enqueue a query on the context stream without waiting (for device-side timing).  Buffers
// must already be large enough: run wk_query_execute on the same plan first.
extern "C" int wk_query_enqueue(wk_ctx* ctx, const wk_query* q, int32_t mode) {
    if (!ctx || !q || (mode != WK_MODE_RESIDENT && mode != WK_MODE_GRAPH)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    std::vector<wk::PlanStep> steps;
    wk::ColMap cm(q->nvars);
    int rc = wk::resolve_plan(*q, ctx->cfg.max_cols, steps, cm, ctx->versatile);
    if (rc) return rc;
    if (mode == WK_MODE_GRAPH) {
        auto it = ctx->graphs.find(plan_key(steps, *q, ctx));
        if (it == ctx->graphs.end()) return ctx->fail(WK_E_BADARG, "plan not captured yet");
        WK_CUDA(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
        if (!steps.empty()) ctx->rbuf[(steps.size() - 1) & 1].cols = steps.back().out_cols;
        return WK_SUCCESS;
    }
    return enqueue_plan(ctx, steps, *q);
}

// Sticky device-side error bits of the context stream (0 = none); clears them.
extern "C" int wk_ctx_check(wk_ctx* ctx) {
    if (!ctx) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    uint32_t err = 0;
    uint64_t need = 0;
    int rc = ctx->read_ctl(&err, &need);
    if (rc) return rc;
    if (!err) return WK_SUCCESS;
    ctx->clear_ctl_err();
    if (err & wk::kErrCorrupt) return WK_E_CORRUPT;
    if (err & wk::kErrTimeout) return WK_E_TIMEOUT;
    return WK_E_CAPACITY;
}

extern "C" int wk_query_validate(const wk_query* q, int32_t max_cols, int32_t* v2c_map,
                                 int32_t* col_num) {
    return wk_query_validate_ex(q, max_cols, 0, v2c_map, col_num);
}

extern "C" int wk_query_validate_ex(const wk_query* q, int32_t max_cols, int32_t versatile,
                                    int32_t* v2c_map, int32_t* col_num) {
    if (!q) return WK_E_BADARG;
    if (max_cols <= 0) max_cols = 32;
    std::vector<wk::PlanStep> steps;
    wk::ColMap cm(q->nvars);
    int rc = wk::resolve_plan(*q, max_cols, steps, cm, versatile != 0);
    if (rc) return rc;
    if (col_num) *col_num = cm.col_num;
    if (v2c_map)
        for (int i = 0; i < q->nvars; ++i) v2c_map[i] = cm.v2c[i];
    return WK_SUCCESS;
}

extern "C" int wk_query_profile(wk_ctx* ctx, const wk_query* q, int32_t iters, wk_step_prof* out,
                                int32_t max_steps, int32_t* n_steps) {
    if (!ctx || !q || iters < 1 || (!out && max_steps)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    std::vector<wk::PlanStep> steps;
    wk::ColMap cm(q->nvars);
    int rc = wk::resolve_plan(*q, ctx->cfg.max_cols, steps, cm, ctx->versatile);
    if (rc) return ctx->fail(rc, wk_strerror(rc));
    if ((int)steps.size() > max_steps) return ctx->fail(WK_E_CAPACITY, "profile array too small");
    const wk_table* t = nullptr;
    rc = query_run(ctx, q, WK_MODE_PLAIN, &t, nullptr, nullptr);   // sizes the buffers
    if (rc) return rc;
    rc = plan_ensure_flat(ctx, steps);
    if (rc) return rc;
    const int fm = plan_flat_mode(steps);
    cudaEvent_t e0, e1;
    WK_CUDA(ctx, cudaEventCreate(&e0));
    WK_CUDA(ctx, cudaEventCreate(&e1));
    std::vector<double> acc(steps.size(), 0.0);
    for (int it = 0; it <= iters; ++it) {
        for (size_t i = 0; i < steps.size(); ++i) {
            const wk_table* in = i ? &ctx->rbuf[(i - 1) & 1] : nullptr;
            wk_table* o = &ctx->rbuf[i & 1];
            WK_CUDA(ctx, cudaMemsetAsync(&ctx->d_ctl->sum_deg, 0, 16, ctx->stream));
            WK_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
            rc = wk::enqueue_step(ctx, steps[i], in, o, q->mt_tid, q->mt_factor, ctx->stream, 0, fm);
            if (rc) return rc;
            WK_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
            WK_CUDA(ctx, cudaEventSynchronize(e1));
            float ms = 0;
            WK_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
            if (it > 0) acc[i] += ms;
            if (it == 0) {
                wk_step_prof& p = out[i];
                std::memset(&p, 0, sizeof(p));
                p.kind = (int)steps[i].kind;
                p.cols_in = steps[i].in_cols;
                p.cols_out = steps[i].out_cols;
                uint64_t r = 0;
                if (in) {
                    rc = table_rows(ctx, in, &r);
                    if (rc) return rc;
                }
                p.rows_in = r;
                rc = table_rows(ctx, o, &r);
                if (rc) return rc;
                p.rows_out = r;
                WK_CUDA(ctx, cudaMemcpy(&p.sum_deg, &ctx->d_ctl->sum_deg, 16, cudaMemcpyDeviceToHost));
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t i = 0; i < steps.size(); ++i) out[i].ms = acc[i] / iters;
    if (n_steps) *n_steps = (int32_t)steps.size();
    uint32_t err = 0;
    uint64_t need = 0;
    rc = ctx->read_ctl(&err, &need);
    if (rc) return rc;
    if (err) {
        ctx->clear_ctl_err();
        return ctx->fail(WK_E_CAPACITY, "profile run reported device errors");
    }
    return WK_SUCCESS;
}

extern "C" int wk_ctx_tune_set(wk_ctx* ctx, int32_t knob, int32_t value) {
    if (!ctx) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (knob == WK_KNOB_LANES || knob == WK_KNOB_BATCH_LANES) {
        if (value != 1 && value != 2 && value != 4 && value != 8)
            return ctx->fail(WK_E_BADARG, "lanes must be 1, 2, 4 or 8");
        if (knob == WK_KNOB_LANES) {
            ctx->default_lanes = value;
            ctx->tuned_lanes.clear();
        } else {
            ctx->batch_lanes = value;
        }
    } else if (knob == WK_KNOB_SLICE_ROWS || knob == WK_KNOB_BATCH_SLICE_ROWS) {
        if (value < wk::kMinSliceRows || value > (1 << 23))
            return ctx->fail(WK_E_BADARG, "slice threshold must be in [8, 2^23]");
        (knob == WK_KNOB_SLICE_ROWS ? ctx->slice_rows : ctx->batch_slice_rows) = (uint32_t)value;
    } else if (knob == WK_KNOB_FLAT_ROWS) {
        if (value < 0) return ctx->fail(WK_E_BADARG, "flat threshold must be >= 0");
        ctx->flat_min_rows = (uint64_t)value;
    } else if (knob == WK_KNOB_SPIN_LIMIT) {
        if (value < 0) return ctx->fail(WK_E_BADARG, "spin limit must be >= 0");
        ctx->spin_limit = (uint64_t)value;
    } else if (knob == WK_KNOB_BATCH_FLAT) {
        if (value < 0 || value >= (1 << wk::kMaxBatchLevels))
            return ctx->fail(WK_E_BADARG, "batch level mask out of range");
        ctx->batch_flat = value;
    } else {
        return ctx->fail(WK_E_BADARG, "unknown knob");
    }
    ctx->drop_graphs();
    return WK_SUCCESS;
}

// Lanes of one (op, input columns) step of single queries (an autotuner's per-step choice).
int wk::tune_step_lanes(wk_ctx* ctx, int op, int cols, int lanes) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) return ctx->fail(WK_E_BADARG, "lanes must be 1, 2, 4 or 8");
    ctx->tuned_lanes[op * 1000 + cols] = lanes;
    ctx->drop_graphs();
    return WK_SUCCESS;
}

extern "C" int wk_ctx_tune_get(wk_ctx* ctx, int32_t knob, int32_t* value) {
    if (!ctx || !value) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (knob == WK_KNOB_LANES) *value = ctx->default_lanes;
    else if (knob == WK_KNOB_BATCH_LANES) *value = ctx->batch_lanes;
    else if (knob == WK_KNOB_SLICE_ROWS) *value = (int32_t)(ctx->slice_rows ? ctx->slice_rows : wk::kHeavyRows);
    else if (knob == WK_KNOB_BATCH_SLICE_ROWS)
        *value = (int32_t)(ctx->batch_slice_rows ? ctx->batch_slice_rows : wk::kHeavyRows);
    else if (knob == WK_KNOB_FLAT_ROWS) *value = (int32_t)std::min<uint64_t>(ctx->flat_min_rows, INT32_MAX);
    else if (knob == WK_KNOB_BATCH_FLAT) *value = ctx->batch_flat;
    else if (knob == WK_KNOB_SPIN_LIMIT)
        *value = (int32_t)std::min<uint64_t>(ctx->spin_limit ? ctx->spin_limit : wk::kDefaultSpinLimit, INT32_MAX);
    else return ctx->fail(WK_E_BADARG, "unknown knob");
    return WK_SUCCESS;
}
