// Serving: continuous batching of an open-loop arrival stream.
//
// No counterpart in the reference beyond the emulator's in-flight window
// (ConsoleProxy::run_query_emu, console_proxy.hpp:287-439) and its latency CDF
// (monitor.hpp:141-220).  Queries are admitted while their projected table bytes fit under the
// working-set cap.  Constant-start (light) queries advance in iterations, one pattern each:
//   * arrivals since the last iteration get a slot and have their planned steps installed on
//     the device;
//   * one exploration launch runs every continuing query's current step over its rows (taken
//     from the previous iteration's arena, tagged with their slot), and a second one starts the
//     newly admitted queries from their start keys, appending to the same arena;
//   * queries whose last step ran have their tables gathered and copied to the host.
// A query's step is iteration - admission iteration, so no per-step host upload is needed, and
// its tables stay on the device between steps.  Index-start (heavy) queries run whole on lanes
// (child contexts on low-priority streams, one host thread each) beside the iterations; the
// iteration launches and the lanes split each SM's CTA slots, so both run on the device at
// once and a light query never waits for a heavy step.  The integer work is the same
// exploration launch as the single-query and batch paths, so a query's result does not depend
// on what it was mixed with.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wk_batch.h"
#include "wk_ctx.h"
#include "wk_device.cuh"

namespace wk {
namespace {

constexpr int kMaxSteps = kMaxBatchLevels;

// Small CTAs: every kernel of an iteration must fit in the room the lanes leave on an SM.
constexpr int kFinishThreads = 256;

// Start of an iteration: reset the slots' output ranges and this iteration's row total, and
// install the newly admitted queries' plans in their slots with the admission iteration.
__global__ void __launch_bounds__(256)
prep_kernel(unsigned long long* qfirst, unsigned long long* qcount, uint32_t n_slots, uint64_t* total,
            StepDesc* plans, uint32_t* admit, const StepDesc* stage, const uint32_t* new_slots,
            uint32_t n_new, uint32_t iter) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < n_slots; i += nt) {
        qfirst[i] = ~0ull;
        qcount[i] = 0;
    }
    for (uint32_t e = tid; e < n_new * (uint32_t)kMaxSteps; e += nt) {
        const uint32_t i = e / kMaxSteps, k = e - i * kMaxSteps;
        const uint32_t s = new_slots[i];
        plans[(size_t)s * kMaxSteps + k] = stage[e];
        if (k == 0) admit[s] = iter;
    }
    if (tid == 0) *total = 0;
}

// Result offsets of the queries finishing this iteration (one CTA).
__global__ void __launch_bounds__(kFinishThreads)
finish_scan_kernel(const uint32_t* fin_slots, const uint32_t* fin_cols, uint32_t n_fin,
                   const unsigned long long* qcount, uint64_t* fin_off) {
    __shared__ uint64_t s_warp[kFinishThreads / 32];
    __shared__ uint64_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    for (uint32_t r0 = 0; r0 < n_fin; r0 += kFinishThreads) {
        const uint32_t i = r0 + threadIdx.x;
        uint64_t sum = 0;
        if (i < n_fin) sum = qcount[fin_slots[i]] * fin_cols[i];
        const uint64_t ex = dev::block_exclusive_sum<kFinishThreads>(sum, s_warp);
        const uint64_t carry = s_carry;
        if (i < n_fin) fin_off[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == kFinishThreads - 1) s_carry = carry + ex + sum;
        __syncthreads();
    }
    if (threadIdx.x == 0) fin_off[n_fin] = s_carry;
}

// Copy the finishing queries' tables (stride w in the arena) to the result buffer.
__global__ void __launch_bounds__(256)
finish_gather_kernel(const uint32_t* fin_slots, const uint32_t* fin_cols, uint32_t n_fin,
                     const unsigned long long* qfirst, const uint64_t* fin_off,
                     const uint32_t* arena, int w, uint32_t* out, uint64_t out_cap, StepCtl* ctl) {
    if (n_fin == 0) return;
    if (fin_off[n_fin] > out_cap) {   // the host grows the buffer and reruns the iteration
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->err, kErrResult);
        return;
    }
    dev::segmented_gather(n_fin, fin_off,
                          [&](uint32_t i, const uint32_t*& row0, uint32_t& stride, uint32_t& cols) {
                              stride = (uint32_t)w;
                              row0 = arena + qfirst[fin_slots[i]] * (uint64_t)w;
                              cols = fin_cols[i];
                          },
                          out);
}

// End of an iteration: the error word and the size request go into the packet the host reads
// back (after every other kernel of the iteration, so a result-buffer overflow is included).
__global__ void pack_kernel(const StepCtl* ctl, uint64_t* pkt) {
    pkt[0] = ctl->err;
    pkt[1] = ctl->need;
}

// Projected table bytes of a plan: the input + output table bytes of its widest step, with the
// rows each step is expected to produce taken from the store's metadata.  An index start has
// its list's exact length (the index keys read at upload); a constant start and every
// known_to_unknown step multiply by their segment's mean degree (edges / keys); a filter step
// keeps its input rows, an upper bound.
uint64_t plan_projection(const wk_ctx* ctx, const std::vector<PlanStep>& plan) {
    auto mean_deg = [&](uint32_t pid, int dir) {
        const int32_t i = ctx->index.find(1, pid, dir);
        if (i < 0 || ctx->segs[i].num_keys == 0) return 0.0;
        return (double)ctx->segs[i].num_edges / (double)ctx->segs[i].num_keys;
    };
    double rows = 1, peak = 0;
    int cols = 0;
    for (const PlanStep& s : plan) {
        const double in_bytes = rows * cols * 4.0;
        switch (s.kind) {
            case PlanStep::kIndex: {
                auto it = ctx->index_len.find(s.start_const * 2 + (uint32_t)s.dir);
                rows = it == ctx->index_len.end() ? 0.0 : (double)it->second;
                break;
            }
            case PlanStep::kConst: rows = mean_deg(s.pid, s.dir); break;
            case PlanStep::kK2U: rows *= mean_deg(s.pid, s.dir); break;
            default: break;   // filters keep at most their input rows
        }
        cols = s.out_cols;
        peak = std::max(peak, in_bytes + rows * cols * 4.0);
    }
    return peak >= 1e18 ? (uint64_t)1e18 : (uint64_t)peak;
}

struct QSlot {
    uint32_t query;       // index into the caller's query array
    uint32_t admit_iter;
    uint32_t nsteps;
    uint32_t cols;        // final column count
};

#define WKS_CUDA(ctx, call)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call); \
    } while (0)

struct Serve {
    wk_ctx* ctx;
    wk_serve_config cfg;
    uint32_t slots_n = 0;
    int w = 1;
    uint64_t rows_cap[2] = {0, 0};
    StepDesc* d_plans = nullptr;
    uint32_t* d_admit = nullptr;
    uint32_t* d_arena[2] = {nullptr, nullptr};
    uint32_t* d_owner[2] = {nullptr, nullptr};
    uint64_t* d_total = nullptr;              // [2]
    unsigned long long* d_qfirst = nullptr;   // [slots]
    unsigned long long* d_qcount = nullptr;   // [slots]
    uint32_t* d_result = nullptr;
    uint64_t result_cap = 0;
    // What an iteration sends up, in one copy: the new queries' plans (n_new x kMaxSteps
    // descriptors), then their slots, the finishing slots and their widths (u32 each).
    unsigned char* d_in = nullptr;
    unsigned char* h_in = nullptr;   // pinned
    // What it reads back, in one copy: the error word, the size request, and the finishing
    // queries' result offsets (n_fin + 1).
    uint64_t* d_pkt = nullptr;
    uint64_t* h_pkt = nullptr;       // pinned
    uint32_t* h_result = nullptr;
    // this iteration's lists (host)
    std::vector<uint32_t> new_slots, fin_slots, fin_cols;

    StepDesc* h_stage() const { return reinterpret_cast<StepDesc*>(h_in); }
    size_t in_bytes(uint32_t n_new, uint32_t n_fin) const {
        return sizeof(StepDesc) * kMaxSteps * (size_t)n_new + 4ull * (n_new + 2ull * n_fin);
    }

    ~Serve() {
        auto f = [](void* p) { if (p) cudaFree(p); };
        auto fh = [](void* p) { if (p) cudaFreeHost(p); };
        f(d_plans); f(d_admit); f(d_arena[0]); f(d_arena[1]); f(d_owner[0]); f(d_owner[1]);
        f(d_total); f(d_qfirst); f(d_qcount); f(d_in); f(d_pkt); f(d_result);
        fh(h_in); fh(h_pkt); fh(h_result);
    }

    int alloc_arena(int k, uint64_t rows) {
        if (d_arena[k]) cudaFree(d_arena[k]);
        if (d_owner[k]) cudaFree(d_owner[k]);
        d_arena[k] = nullptr;
        d_owner[k] = nullptr;
        rows = (rows + 15) & ~15ull;
        if (wk::dev_malloc(&d_arena[k], rows * w * 4 + 256) != cudaSuccess ||
            wk::dev_malloc(&d_owner[k], rows * 4 + 64) != cudaSuccess) {
            cudaGetLastError();
            return ctx->fail(WK_E_OOM, "serving arena");
        }
        rows_cap[k] = rows;
        return WK_SUCCESS;
    }

    int alloc_result(uint64_t elems) {
        if (d_result) cudaFree(d_result);
        if (h_result) cudaFreeHost(h_result);
        d_result = nullptr;
        h_result = nullptr;
        if (wk::dev_malloc(&d_result, elems * 4 + 64) != cudaSuccess ||
            cudaMallocHost(&h_result, elems * 4 + 64) != cudaSuccess) {
            cudaGetLastError();
            return ctx->fail(WK_E_OOM, "serving result buffer");
        }
        result_cap = elems;
        return WK_SUCCESS;
    }

    int init(uint32_t slots, int width) {
        slots_n = slots;
        w = std::max(width, 1);
        auto dm = [&](void** p, size_t bytes) {
            if (wk::dev_malloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            return true;
        };
        auto hm = [&](void** p, size_t bytes) { return cudaMallocHost(p, std::max<size_t>(bytes, 16)) == cudaSuccess; };
        const size_t in_cap = in_bytes(slots, slots) + 64;
        bool ok = dm((void**)&d_plans, sizeof(StepDesc) * kMaxSteps * (size_t)slots) &&
                  dm((void**)&d_admit, 4ull * slots) && dm((void**)&d_total, 16) &&
                  dm((void**)&d_qfirst, 8ull * slots) && dm((void**)&d_qcount, 8ull * slots) &&
                  dm((void**)&d_in, in_cap) && dm((void**)&d_pkt, 8ull * (slots + 3)) &&
                  hm((void**)&h_in, in_cap) && hm((void**)&h_pkt, 8ull * (slots + 3));
        if (!ok) return ctx->fail(WK_E_OOM, "serving buffers");
        new_slots.reserve(slots);
        fin_slots.reserve(slots);
        fin_cols.reserve(slots);
        const uint64_t rows = std::max<uint64_t>(cfg.arena_bytes / (4ull * w), 1 << 16);
        int rc = alloc_arena(0, rows);
        if (!rc) rc = alloc_arena(1, rows);
        if (!rc) rc = alloc_result(1 << 22);
        if (rc) return rc;
        WKS_CUDA(ctx, cudaMemset(d_total, 0, 16));
        return WK_SUCCESS;
    }

    int light_ctas() const { return std::max(1, cfg.light_ctas_per_sm); }

    ExploreArgs explore_args(uint32_t iter, int cur) const {
        ExploreArgs a{};
        a.store = ctx->dev_store();
        a.seg_index[0] = ctx->seg_of(0, 0, kIn);
        a.seg_index[1] = ctx->seg_of(0, 0, kOut);
        a.desc = d_plans;
        a.desc_stride = kMaxSteps;
        a.iter = iter;
        a.q_admit = d_admit;
        a.out = d_arena[cur];
        a.w_out = w;
        a.out_cap_rows = rows_cap[cur];
        a.owner_out = d_owner[cur];
        a.out_rows = d_total + cur;
        a.qfirst = d_qfirst;
        a.qcount = d_qcount;
        a.heavy = ctx->d_heavy;
        a.heavy_cap = ctx->heavy_cap;
        a.ctl = ctx->d_ctl;
        a.status = ctx->d_status;
        a.sorted_lists = ctx->sorted_lists;
        a.lanes = ctx->batch_lanes;
        a.slice_rows = ctx->batch_slice_rows;
        a.spin_limit = ctx->spin_limit;
        return a;
    }

    // Enqueue one iteration (no host sync): one copy up, the launches, one copy back.  The
    // plans of the n_new admitted queries are already in h_stage(); new_slots, fin_slots and
    // fin_cols hold this iteration's lists.
    int enqueue_iteration(uint32_t iter, bool has_cont) {
        const int cur = iter & 1, prev = cur ^ 1;
        const uint32_t n_new = (uint32_t)new_slots.size(), n_fin = (uint32_t)fin_slots.size();
        cudaStream_t s = ctx->stream;
        const size_t stage_bytes = sizeof(StepDesc) * kMaxSteps * (size_t)n_new;
        uint32_t* hl = reinterpret_cast<uint32_t*>(h_in + stage_bytes);
        std::memcpy(hl, new_slots.data(), 4ull * n_new);
        std::memcpy(hl + n_new, fin_slots.data(), 4ull * n_fin);
        std::memcpy(hl + n_new + n_fin, fin_cols.data(), 4ull * n_fin);
        const StepDesc* d_stage = reinterpret_cast<const StepDesc*>(d_in);
        const uint32_t* d_new = reinterpret_cast<const uint32_t*>(d_in + stage_bytes);
        const uint32_t* d_fin_slots = d_new + n_new;
        const uint32_t* d_fin_cols = d_fin_slots + n_fin;
        if (n_new || n_fin)
            WKS_CUDA(ctx, cudaMemcpyAsync(d_in, h_in, in_bytes(n_new, n_fin), cudaMemcpyHostToDevice, s));
        const uint32_t work = std::max<uint32_t>(slots_n, n_new * (uint32_t)kMaxSteps);
        prep_kernel<<<std::min<uint32_t>((work + 255) / 256, 1024), 256, 0, s>>>(
            d_qfirst, d_qcount, slots_n, d_total + cur, d_plans, d_admit, d_stage, d_new, n_new, iter);
        WKS_CUDA(ctx, cudaGetLastError());
        const int light = light_ctas();
        const int grid = std::min(explore_blocks_per_sm(w, w, ctx->batch_lanes), light) * ctx->sm_count;
        if (has_cont) {
            ExploreArgs a = explore_args(iter, cur);
            a.n_queries = slots_n;
            a.virtual_rows = 0;
            a.in_rows = d_total + prev;
            a.owner_in = d_owner[prev];
            a.in = d_arena[prev];
            a.w_in = w;
            a.in_cap_rows = rows_cap[prev];
            cudaError_t e = launch_explore(a, grid, s);
            if (e != cudaSuccess) return ctx->cuda_fail(e, "serving launch");
        }
        if (n_new) {
            ExploreArgs a = explore_args(iter, cur);
            a.n_queries = n_new;
            a.virtual_rows = 1;
            a.virt_owner = d_new;
            a.out_base_rows = d_total + cur;
            const int g0 = std::min(explore_blocks_per_sm(0, w, ctx->batch_lanes), light) * ctx->sm_count;
            cudaError_t e = launch_explore(a, g0, s);
            if (e != cudaSuccess) return ctx->cuda_fail(e, "serving start launch");
        }
        uint64_t* d_fin_off = d_pkt + 2;
        if (n_fin) {
            finish_scan_kernel<<<1, kFinishThreads, 0, s>>>(d_fin_slots, d_fin_cols, n_fin, d_qcount, d_fin_off);
            if (!cfg.blind)
                finish_gather_kernel<<<ctx->sm_count * 4, 256, 0, s>>>(
                    d_fin_slots, d_fin_cols, n_fin, d_qfirst, d_fin_off, d_arena[cur], w, d_result,
                    result_cap, ctx->d_ctl);
        }
        pack_kernel<<<1, 1, 0, s>>>(ctx->d_ctl, d_pkt);
        WKS_CUDA(ctx, cudaGetLastError());
        WKS_CUDA(ctx, cudaMemcpyAsync(h_pkt, d_pkt, 8ull * (2 + (n_fin ? n_fin + 1 : 0)),
                                      cudaMemcpyDeviceToHost, s));
        return WK_SUCCESS;
    }

    // Wait for the iteration; the error word and the size request it ended with.
    int finish_iteration(uint32_t* err, uint64_t* need) {
        WKS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *err = (uint32_t)h_pkt[0] | ctx->inject_err;   // a staged test failure counts once
        ctx->inject_err = 0;
        *need = h_pkt[1];
        return WK_SUCCESS;
    }
    const uint64_t* fin_off() const { return h_pkt + 2; }
};

// Index-start queries run whole, one at a time per lane: a child context (its own stream of
// the lowest priority, control block, tables) driven by its own host thread, so the iteration
// loop never waits for one of their steps.
struct HeavyLanes {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint32_t> work;
    std::vector<uint32_t> completed;   // finished since the iteration loop last looked
    int fatal = 0;                     // a lane's CUDA / device error ends the run
    std::string fatal_msg;
    bool stop = false;
    std::vector<std::thread> threads;

    ~HeavyLanes() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        for (auto& t : threads) t.join();
    }

    // Lanes are child contexts cached in the parent (their tables keep their grown size from
    // one serving run to the next); they are rebuilt when the room they must leave changes.
    template <class Body>
    int start(wk_ctx* parent, int n, const CtaUse& beside_use, int beside_ctas, uint64_t table_elems,
              Body body) {
        const bool same = parent->lanes_ctas == beside_ctas && parent->lanes_use.smem == beside_use.smem &&
                          parent->lanes_use.regs == beside_use.regs &&
                          parent->lanes_use.threads == beside_use.threads;
        if (!same) {
            for (wk_ctx* c : parent->lanes) wk_ctx_destroy(c);
            parent->lanes.clear();
            parent->lanes_use = beside_use;
            parent->lanes_ctas = beside_ctas;
        }
        while ((int)parent->lanes.size() < n) {
            wk_ctx* c = nullptr;
            int rc = ctx_make_child(parent, beside_use, beside_ctas, &c);
            if (rc) return rc;
            parent->lanes.push_back(c);
        }
        // Size each lane for a projected index-start query before the run starts: growing a
        // table later means a cudaFree, which waits for the whole device.
        for (int i = 0; i < n; ++i) {
            int rc = lane_prepare(parent->lanes[i], table_elems);
            if (rc) {
                parent->last_error = "serving lane: " + parent->lanes[i]->last_error;
                return rc;
            }
        }
        for (int i = 0; i < n; ++i) {
            wk_ctx* c = parent->lanes[i];
            threads.emplace_back([this, c, body] {
                cudaSetDevice(c->device);
                for (;;) {
                    uint32_t q;
                    {
                        std::unique_lock<std::mutex> lk(mu);
                        cv_work.wait(lk, [&] { return stop || !work.empty(); });
                        if (stop) return;
                        q = work.front();
                        work.pop_front();
                    }
                    const int rc = body(c, q);
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        completed.push_back(q);
                        if ((rc == WK_E_CUDA || rc == WK_E_TIMEOUT || rc == WK_E_CORRUPT) && !fatal) {
                            fatal = rc;
                            fatal_msg = c->last_error;
                        }
                    }
                    cv_done.notify_one();
                }
            });
        }
        return WK_SUCCESS;
    }

    void submit(uint32_t q) {
        {
            std::lock_guard<std::mutex> lk(mu);
            work.push_back(q);
        }
        cv_work.notify_one();
    }
};

}  // namespace

cudaError_t serve_kernel_attrs() {
    cudaError_t e;
    if ((e = use_max_shared_carveout(prep_kernel)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(pack_kernel)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(finish_scan_kernel)) != cudaSuccess) return e;
    return use_max_shared_carveout(finish_gather_kernel);
}

}  // namespace wk

using Clock = std::chrono::steady_clock;

extern "C" int wk_serve_run_open_loop(wk_ctx* ctx, const wk_serve_config* cfg_in, const wk_query* queries,
                                      uint32_t n, const double* arrival_us, uint32_t* host_out,
                                      uint64_t cap_elems, wk_qresult* results) {
    if (!ctx || (!queries && n) || (!arrival_us && n) || (!results && n) || (!host_out && cap_elems))
        return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n == 0) return WK_SUCCESS;
    wk::Serve S;
    S.ctx = ctx;
    S.cfg = cfg_in ? *cfg_in : wk_serve_config{};
    if (!S.cfg.working_set_cap_bytes) S.cfg.working_set_cap_bytes = 40ull << 30;
    if (!S.cfg.arena_bytes) S.cfg.arena_bytes = 1ull << 30;
    if (!S.cfg.min_proj_bytes) S.cfg.min_proj_bytes = 64ull << 10;
    if (!S.cfg.max_inflight) S.cfg.max_inflight = 65536;
    if (!S.cfg.max_heavy_inflight) S.cfg.max_heavy_inflight = 1;
    if (S.cfg.light_ctas_per_sm <= 0) S.cfg.light_ctas_per_sm = 2;

    // Resolve every plan once (the same dispatch as a single query).
    std::vector<std::vector<wk::PlanStep>> plans(n);
    std::vector<int32_t> status(n, 0);
    std::vector<uint64_t> proj(n, 0);   // projected bytes of each query
    int width = 1;
    bool any_heavy = false;
    uint64_t heavy_proj_max = 0;
    for (uint32_t i = 0; i < n; ++i) {
        wk::ColMap cm(queries[i].nvars);
        int rc = wk::resolve_plan(queries[i], ctx->cfg.max_cols, plans[i], cm, ctx->versatile);
        if (rc == WK_SUCCESS && (int)plans[i].size() > wk::kMaxSteps) rc = WK_E_CAPACITY;
        // the unknown-predicate operators walk several lists per row: single queries only
        for (auto& x : plans[i])
            if (rc == WK_SUCCESS && wk::is_versatile_step(x.kind)) rc = WK_E_UNSUPPORTED;
        if (rc == WK_SUCCESS && queries[i].mt_factor != 1) rc = WK_E_UNSUPPORTED;
        if (rc) {
            status[i] = rc;
            plans[i].clear();
        }
        proj[i] = std::max<uint64_t>(S.cfg.min_proj_bytes, wk::plan_projection(ctx, plans[i]));
        if (!plans[i].empty() && plans[i][0].kind == wk::PlanStep::kIndex) {
            any_heavy = true;   // runs on a lane, not in the iterations
            heavy_proj_max = std::max(heavy_proj_max, proj[i]);
            continue;
        }
        for (auto& s : plans[i]) width = std::max(width, s.out_cols);
    }
    const uint32_t slots = std::min<uint32_t>(S.cfg.max_inflight, std::max<uint32_t>(n, 1));
    int rc = S.init(slots, width);
    if (rc) return rc;
    rc = ctx->ensure_status(std::max(S.rows_cap[0], S.rows_cap[1]) / wk::kTileRows + 2);
    if (!rc) rc = ctx->ensure_heavy(std::max(S.rows_cap[0], S.rows_cap[1]));
    if (rc) return rc;

    std::vector<wk::QSlot> slot(slots);
    std::vector<uint32_t> free_slots;
    for (uint32_t s = slots; s-- > 0;) free_slots.push_back(s);
    std::vector<uint32_t> active;   // slots in use
    std::vector<uint32_t> finished, cooling;
    uint32_t heavy_inflight = 0;
    uint64_t proj_bytes = 0;
    std::atomic<uint64_t> out_used{0};
    uint32_t next = 0, done = 0;
    for (uint32_t i = 0; i < n; ++i) {
        std::memset(&results[i], 0, sizeof(results[i]));
        results[i].t_arrive_us = arrival_us[i];
    }
    // Claim `elems` elements of the caller's buffer (lanes and the iteration loop share it).
    auto reserve_out = [&](uint64_t elems, uint64_t* off) {
        uint64_t cur = out_used.load();
        do {
            if (cur + elems > cap_elems) return false;
        } while (!out_used.compare_exchange_weak(cur, cur + elems));
        *off = cur;
        return true;
    };
    auto t0 = Clock::now();   // restarted once the lanes are ready
    auto now_us = [&] { return std::chrono::duration<double, std::micro>(Clock::now() - t0).count(); };

    wk::HeavyLanes H;
    if (any_heavy) {
        // Lanes leave room on every SM for the iteration launches' CTAs (the larger of the two
        // launch shapes, one CTA of margin), so both persistent launches stay resident at once
        // and neither waits for the other to finish.
        const wk::CtaUse a = wk::explore_cta_use(S.w, S.w, ctx->batch_lanes);
        const wk::CtaUse b = wk::explore_cta_use(0, S.w, ctx->batch_lanes);
        const wk::CtaUse light{std::max(a.smem, b.smem), std::max(a.regs, b.regs),
                               std::max(a.threads, b.threads)};
        const uint64_t lane_bytes =
            S.cfg.lane_table_bytes ? S.cfg.lane_table_bytes : std::min<uint64_t>(heavy_proj_max, 1ull << 30);
        rc = H.start(ctx, (int)S.cfg.max_heavy_inflight, light, S.light_ctas() + 1, lane_bytes / 4,
                     [&](wk_ctx* lane, uint32_t q) {
                         const wk_table* t = nullptr;
                         uint64_t rows = 0, off = 0;
                         wk_qresult& r = results[q];
                         // a graph per plan, captured by the lane's first query of that plan:
                         // one launch instead of one per step pass
                         int qrc = wk::query_run_rows(lane, &queries[q], WK_MODE_GRAPH, &t, &rows);
                         if (qrc == WK_SUCCESS && S.cfg.blind) {
                             r.rows = rows;
                             r.cols = t->cols;
                         } else if (qrc == WK_SUCCESS) {
                             const uint64_t elems = rows * (uint64_t)t->cols;
                             if (reserve_out(elems, &off)) {
                                 qrc = wk::table_copy_out(lane, t, elems, host_out + off);
                                 r.elem_offset = off;
                                 r.rows = rows;
                                 r.cols = t->cols;
                             } else {
                                 qrc = WK_E_CAPACITY;   // the caller's buffer is full
                             }
                         }
                         r.status = qrc;
                         r.t_done_us = now_us();
                         return qrc;
                     });
        if (rc) return rc;
    }
    t0 = Clock::now();   // arrival times count from here

    uint32_t iter = 1;   // admission iterations start at 1 so a zeroed admit[] never matches
    std::deque<uint32_t> wait_heavy, wait_light;   // arrived, not yet admitted
    // Give constant-start query q a slot and stage its plan (Done-padded) for installation
    // this iteration.
    auto admit = [&](uint32_t q) {
        const uint32_t s = free_slots.back();
        free_slots.pop_back();
        slot[s] = {q, iter, (uint32_t)plans[q].size(), (uint32_t)plans[q].back().out_cols};
        const size_t j = S.new_slots.size();
        for (int k = 0; k < wk::kMaxSteps; ++k) {
            wk::StepDesc& d = S.h_stage()[j * wk::kMaxSteps + k];
            if (k < (int)plans[q].size()) {
                d = wk::make_step_desc(ctx, plans[q][k]);
            } else {
                std::memset(&d, 0, sizeof(d));
                d.op = wk::kXDone;
            }
        }
        S.new_slots.push_back(s);
        proj_bytes += proj[q];
    };
    std::vector<uint32_t> lane_done;
    while (done < n) {
        // 0. index-start queries the lanes finished
        {
            std::lock_guard<std::mutex> lk(H.mu);
            lane_done.swap(H.completed);
            if (H.fatal) return ctx->fail(H.fatal, "serving lane: " + H.fatal_msg);
        }
        for (uint32_t q : lane_done) {
            --heavy_inflight;
            proj_bytes -= proj[q];
            ++done;
        }
        lane_done.clear();
        // 1. arrivals join their class's queue
        const double t = now_us();
        while (next < n && arrival_us[next] <= t) {
            const uint32_t q = next++;
            if (status[q] || plans[q].empty()) {   // fails at dispatch, or nothing to run
                results[q].status = status[q];
                results[q].cols = 0;
                results[q].t_done_us = now_us();
                ++done;
                continue;
            }
            (plans[q][0].kind == wk::PlanStep::kIndex ? wait_heavy : wait_light).push_back(q);
        }
        // 2. admission, FIFO within each class; a class stops at the first query that does not
        // fit under the working-set cap (unless nothing at all is resident)
        while (!wait_heavy.empty() && heavy_inflight < S.cfg.max_heavy_inflight &&
               (proj_bytes + proj[wait_heavy.front()] <= S.cfg.working_set_cap_bytes ||
                (active.empty() && !heavy_inflight))) {
            const uint32_t q = wait_heavy.front();
            wait_heavy.pop_front();
            ++heavy_inflight;
            proj_bytes += proj[q];
            H.submit(q);
        }
        S.new_slots.clear();
        while (!wait_light.empty() && !free_slots.empty() &&
               (proj_bytes + proj[wait_light.front()] <= S.cfg.working_set_cap_bytes ||
                (active.empty() && !heavy_inflight && S.new_slots.empty()))) {
            admit(wait_light.front());
            wait_light.pop_front();
        }
        const bool has_cont = !active.empty();
        if (!has_cont) {   // nothing continues, so no launch will read the cooling slots' rows
            for (uint32_t s : cooling) free_slots.push_back(s);
            cooling.clear();
        }
        for (uint32_t s : S.new_slots) active.push_back(s);
        if (active.empty()) {
            // idle until the next arrival or a lane finishing, whichever comes first
            double wait = next < n ? arrival_us[next] - now_us() : 1e6;
            if (!wait_light.empty() && !free_slots.empty()) wait = 0;
            if (wait > 50) {
                std::unique_lock<std::mutex> lk(H.mu);
                if (H.completed.empty() && !H.fatal)
                    H.cv_done.wait_for(lk, std::chrono::microseconds((long)std::min(wait - 20, 1e6)));
            }
            continue;
        }
        // 3. which queries run their last step in this iteration
        S.fin_slots.clear();
        S.fin_cols.clear();
        for (uint32_t s : active) {
            const wk::QSlot& sl = slot[s];
            if (iter - sl.admit_iter == sl.nsteps - 1) {
                S.fin_slots.push_back(s);
                S.fin_cols.push_back(sl.cols);
            }
        }
        const uint32_t n_fin = (uint32_t)S.fin_slots.size();
        // 4. run it; grow the output arena and rerun if a table did not fit
        for (int attempt = 0;; ++attempt) {
            if (attempt >= 6) return ctx->fail(WK_E_CAPACITY, "serving arena kept overflowing");
            rc = S.enqueue_iteration(iter, has_cont);
            if (rc) return rc;
            uint32_t err = 0;
            uint64_t need = 0;
            rc = S.finish_iteration(&err, &need);   // synchronises the stream
            if (rc) return rc;
            if (!err) break;
            ctx->clear_ctl_err();
            if (err & wk::kErrCorrupt) return ctx->fail(WK_E_CORRUPT, "key table chain out of range");
            if (err & wk::kErrTimeout) return ctx->fail(WK_E_TIMEOUT, "serving launch timed out");
            if (err & wk::kErrResult) {
                const uint64_t total = S.fin_off()[n_fin];
                rc = S.alloc_result(total + total / 2 + 1024);
                if (rc) return rc;
            }
            if (err & (wk::kErrOverflow | wk::kErrStatus)) {
                const int cur = iter & 1;
                uint64_t rows = std::max<uint64_t>(S.rows_cap[cur] * 2, need + need / 4);
                if (rows * 4ull * S.w > S.cfg.working_set_cap_bytes)
                    return ctx->fail(WK_E_CAPACITY, "a step exceeds the working-set cap");
                rc = S.alloc_arena(cur, rows);
                if (!rc) rc = ctx->ensure_status(S.rows_cap[cur] / wk::kTileRows + 2);
                if (!rc) rc = ctx->ensure_heavy(S.rows_cap[cur]);
                if (rc) return rc;
            }
        }
        // 5. completions
        if (n_fin) {
            const uint64_t* fo = S.fin_off();
            const uint64_t total = S.cfg.blind ? 0 : fo[n_fin];
            if (total) {
                WKS_CUDA(ctx, cudaMemcpyAsync(S.h_result, S.d_result, total * 4, cudaMemcpyDeviceToHost, ctx->stream));
                WKS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            }
            const double td = now_us();
            for (uint32_t i = 0; i < n_fin; ++i) {
                const uint32_t s = S.fin_slots[i];
                const uint32_t q = slot[s].query;
                wk_qresult& r = results[q];
                r.rows = (fo[i + 1] - fo[i]) / slot[s].cols;   // every plan ends with >= 1 column
                r.cols = (int32_t)slot[s].cols;
                r.status = WK_SUCCESS;
                r.t_done_us = td;
                const uint64_t elems = r.rows * (uint64_t)r.cols;
                uint64_t off = 0;
                if (S.cfg.blind) {
                    // row count only
                } else if (reserve_out(elems, &off)) {
                    r.elem_offset = off;
                    if (elems) std::memcpy(host_out + off, S.h_result + fo[i], elems * 4);
                } else {
                    r.status = WK_E_CAPACITY;   // the caller's buffer is full
                }
                proj_bytes -= proj[q];
                finished.push_back(s);
                ++done;
            }
            active.erase(std::remove_if(active.begin(), active.end(),
                                        [&](uint32_t s) { return iter - slot[s].admit_iter == slot[s].nsteps - 1; }),
                         active.end());
        }
        // A finished query's rows are still in this iteration's arena and are dropped by the
        // next iteration; its slot is reused only after that.
        for (uint32_t s : cooling) free_slots.push_back(s);
        cooling.swap(finished);
        finished.clear();
        ++iter;
    }
    return WK_SUCCESS;
}
