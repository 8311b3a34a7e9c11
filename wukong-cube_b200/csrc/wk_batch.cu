// Batched light queries: all queries of a batch advance one pattern per level.
//
// No counterpart in the reference, which serves one query per GPU agent at a time
// (gpu_agent.hpp:173-246) and leaves light queries to the CPU engines
// (console_proxy.hpp:387-392).  Level k's input is level k-1's output: every query's rows,
// contiguous and in query order, each tagged with its owner query.  One exploration launch per
// level (wk_explore.cu: a persistent launch whose CTAs claim tiles from a device counter) runs
// each row's own query step, and records each query's output range (qfirst, qcount); rows of
// queries that have no step at a level simply produce nothing.  Level 0's input is one virtual
// row per query, its start key.  After the last level a one-CTA scan lays the final tables out
// back to back and a gather copies them.  The whole sequence is replayed from a CUDA graph
// cached per batch shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "wk_batch.h"
#include "wk_ctx.h"
#include "wk_device.cuh"

namespace wk {
namespace {

constexpr int kScanThreads = 1024;

// Final table of each query: its rows at its last level, laid out back to back.  CTA t owns
// queries [t * 1024, (t + 1) * 1024): it first adds up the element counts of every query
// before its own (a strided read of at most a few thousand words per thread block, from L2),
// then scans its own queries.  No CTA waits for another.
__device__ __forceinline__ uint64_t final_elems(const ResultScanArgs& a, uint32_t q, int* lev,
                                                uint64_t* rows, uint64_t* base) {
    *lev = (int)a.nsteps[q] - 1;
    *rows = 0;
    *base = 0;
    if (*lev >= 0) {
        *rows = a.qcount[(size_t)*lev * a.n + q];
        *base = a.qfirst[(size_t)*lev * a.n + q];
    }
    return *rows * a.final_cols[q];
}

__global__ void __launch_bounds__(kScanThreads) result_scan_kernel(const ResultScanArgs a) {
    __shared__ uint64_t s_warp[kScanThreads / 32];
    const uint32_t n = a.n;
    const uint32_t t0 = blockIdx.x * kScanThreads;
    // eight queries per thread at a time: their step counts, then their row counts and widths,
    // are loaded together (one dependent round trip per eight queries, not per query)
    uint64_t before = 0;
    constexpr int kU = 8;
    for (uint32_t q0 = threadIdx.x; q0 < t0; q0 += kU * kScanThreads) {
        int lev[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t q = q0 + u * kScanThreads;
            lev[u] = q < t0 ? (int)a.nsteps[q] - 1 : -1;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t q = q0 + u * kScanThreads;
            if (lev[u] >= 0) before += a.qcount[(size_t)lev[u] * a.n + q] * a.final_cols[q];
        }
    }
    // block total of `before` (the inclusive sum of the last thread)
    const uint64_t bex = dev::block_exclusive_sum<kScanThreads>(before, s_warp);
    __shared__ uint64_t s_base;
    if (threadIdx.x == kScanThreads - 1) s_base = bex + before;
    __syncthreads();
    const uint32_t q = t0 + threadIdx.x;
    int lev = -1;
    uint64_t rows = 0, base = 0, elems = 0;
    if (q < n) {
        elems = final_elems(a, q, &lev, &rows, &base);
        a.final_level[q] = rows ? lev : -1;
        a.final_base[q] = rows ? base : 0;
        a.final_rows[q] = rows;
    }
    const uint64_t ex = dev::block_exclusive_sum<kScanThreads>(elems, s_warp);
    if (q < n) a.res_off[q] = s_base + ex;
    if (n > 0 ? q == n - 1 : q == 0) a.res_off[n] = s_base + ex + elems;
}

// Copy each query's final table (stride of its level) into the compact result buffer.
__global__ void __launch_bounds__(256) gather_kernel(const GatherArgs a) {
    if (a.n == 0) return;
    if (a.res_off[a.n] > a.out_cap) {   // the host grows the buffer and reruns
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctl->err, kErrOverflow);
        return;
    }
    // a table with rows has a valid final level (result_scan_kernel), so only those are read
    dev::segmented_gather(a.n, a.res_off,
                          [&](uint32_t q, const uint32_t*& row0, uint32_t& stride, uint32_t& cols) {
                              const int lev = a.final_level[q];
                              stride = (uint32_t)a.width[lev];
                              row0 = a.region[lev] + a.final_base[q] * (uint64_t)stride;
                              cols = a.final_cols[q];
                          },
                          a.out);
}

}  // namespace

cudaError_t launch_result_scan(const ResultScanArgs& a, cudaStream_t s) {
    result_scan_kernel<<<std::max<uint32_t>(1, (a.n + kScanThreads - 1) / kScanThreads), kScanThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs& a, int grid, cudaStream_t s) {
    if (grid < 1) grid = 1;
    gather_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t batch_kernel_attrs() {
    cudaError_t e = use_max_shared_carveout(result_scan_kernel);
    return e != cudaSuccess ? e : use_max_shared_carveout(gather_kernel);
}

}  // namespace wk

// ---------------------------------------------------------------- host side of the batch
namespace {

using wk::kMaxBatchLevels;

struct BatchState {
    uint32_t n_cap = 0;
    int l_cap = 0;
    uint64_t rows_cap = 0;     // rows per level region
    int w_cap = 0;             // widest row the regions were sized for
    wk::StepDesc* d_desc = nullptr;       // [l_cap][n_cap]
    uint32_t* d_owner = nullptr;          // [l_cap][rows_cap]
    uint64_t* d_total_out = nullptr;      // [l_cap]
    unsigned long long* d_qfirst = nullptr;   // [l_cap][n_cap]
    unsigned long long* d_qcount = nullptr;   // [l_cap][n_cap]
    uint32_t* d_nsteps = nullptr;         // [n_cap]
    uint32_t* d_final_cols = nullptr;     // [n_cap]
    int32_t* d_final_level = nullptr;     // [n_cap]
    uint64_t* d_final_base = nullptr;     // [n_cap]
    uint64_t* d_final_rows = nullptr;     // [n_cap]
    uint64_t* d_res_off = nullptr;        // [n_cap + 1]
    uint32_t* d_arena = nullptr;          // [l_cap][rows_cap * w_cap] (+ padding)
    uint32_t* d_result = nullptr;         // compact results
    uint64_t result_cap = 0;
    uint64_t* d_flat = nullptr;           // flat-level scratch: pos, off, part (wk_flat.h)
    uint64_t flat_rows = 0;               // rows it is sized for: max(rows_cap, n_cap)
    // pinned host staging
    wk::StepDesc* h_desc = nullptr;
    uint32_t* h_nsteps = nullptr;
    uint32_t* h_final_cols = nullptr;
    uint64_t* h_final_rows = nullptr;
    uint64_t* h_res_off = nullptr;
    wk::StepCtl* h_ctl = nullptr;         // control block snapshot after this state's batch
    // graph of the launch sequence for one batch shape
    cudaGraphExec_t exec = nullptr;
    std::string shape;
};

void free_state(BatchState* b) {
    auto f = [](void* p) { if (p) cudaFree(p); };
    f(b->d_desc); f(b->d_owner); f(b->d_total_out); f(b->d_qfirst); f(b->d_qcount);
    f(b->d_nsteps); f(b->d_final_cols); f(b->d_final_level); f(b->d_final_base);
    f(b->d_final_rows); f(b->d_res_off); f(b->d_arena); f(b->d_result); f(b->d_flat);
    auto fh = [](void* p) { if (p) cudaFreeHost(p); };
    fh(b->h_desc); fh(b->h_nsteps); fh(b->h_final_cols); fh(b->h_final_rows); fh(b->h_res_off);
    fh(b->h_ctl);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    *b = BatchState();
}

#define WKB_CUDA(ctx, call)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call); \
    } while (0)

int ensure_state(wk_ctx* ctx, BatchState* b, uint32_t n, int levels, uint64_t rows_cap, int w,
                 uint64_t result_cap) {
    rows_cap = (rows_cap + 15) & ~15ull;   // keeps every level region 16-byte aligned
    if (n <= b->n_cap && levels <= b->l_cap && rows_cap <= b->rows_cap && w <= b->w_cap &&
        result_cap <= b->result_cap)
        return WK_SUCCESS;
    n = std::max(n, b->n_cap);
    levels = std::max(levels, b->l_cap);
    rows_cap = std::max(rows_cap, b->rows_cap);
    w = std::max(w, b->w_cap);
    result_cap = std::max(result_cap, b->result_cap);
    // every stream, the pipelined path's copy stream too, may still read the old buffers
    WKB_CUDA(ctx, cudaDeviceSynchronize());
    free_state(b);
    auto dm = [&](void** p, size_t bytes) {
        if (wk::dev_malloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    auto hm = [&](void** p, size_t bytes) {
        return cudaMallocHost(p, std::max<size_t>(bytes, 16)) == cudaSuccess;
    };
    bool ok = dm((void**)&b->d_desc, sizeof(wk::StepDesc) * levels * (size_t)n) &&
              dm((void**)&b->d_owner, 4ull * levels * rows_cap) &&
              dm((void**)&b->d_total_out, 8ull * levels) &&
              dm((void**)&b->d_qfirst, 8ull * levels * n) && dm((void**)&b->d_qcount, 8ull * levels * n) &&
              dm((void**)&b->d_nsteps, 4ull * n) && dm((void**)&b->d_final_cols, 4ull * n) &&
              dm((void**)&b->d_final_level, 4ull * n) && dm((void**)&b->d_final_base, 8ull * n) &&
              dm((void**)&b->d_final_rows, 8ull * n) && dm((void**)&b->d_res_off, 8ull * (n + 1)) &&
              dm((void**)&b->d_arena, 4ull * levels * rows_cap * w + 256) &&
              dm((void**)&b->d_result, 4ull * result_cap + 64) &&
              hm((void**)&b->h_desc, sizeof(wk::StepDesc) * levels * (size_t)n) &&
              hm((void**)&b->h_nsteps, 4ull * n) && hm((void**)&b->h_final_cols, 4ull * n) &&
              hm((void**)&b->h_final_rows, 8ull * n) && hm((void**)&b->h_res_off, 8ull * (n + 1)) &&
              hm((void**)&b->h_ctl, sizeof(wk::StepCtl));
    const uint64_t frows = std::max<uint64_t>(rows_cap, n);
    ok = ok && dm((void**)&b->d_flat, wk::flat_scratch_bytes(frows, wk::flat_grid(ctx->sm_count)));
    if (!ok) {
        free_state(b);
        return ctx->fail(WK_E_OOM, "batch buffers");
    }
    b->flat_rows = frows;
    b->n_cap = n;
    b->l_cap = levels;
    b->rows_cap = rows_cap;
    b->w_cap = w;
    b->result_cap = result_cap;
    return WK_SUCCESS;
}

struct Plan {
    uint32_t n = 0;
    int levels = 0;
    int width[kMaxBatchLevels] = {0};
    std::vector<int32_t> status;
    std::vector<wk::PlanStep> steps;    // [n][kMaxBatchLevels]
    std::vector<uint8_t> nsteps;        // [n]
};

// Host-side state kept between batch calls of a context: the plans (their arrays are large,
// and touching fresh pages for them cost 0.4 ms per 16,384-query batch) and the pipelined
// path's streams and events (creating them cost 0.17 ms per call).  Calls on one context are
// serialised by its mutex, so one set serves every call.
struct BatchHost {
    Plan plan[2];
    cudaStream_t copy_stream = nullptr, upload_stream = nullptr;
    cudaEvent_t ready[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    cudaEvent_t uploaded[2] = {nullptr, nullptr};
    ~BatchHost() {
        for (int k = 0; k < 2; ++k)
            for (cudaEvent_t e : {ready[k], copied[k], uploaded[k]})
                if (e) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (upload_stream) cudaStreamDestroy(upload_stream);
    }
};

BatchHost* batch_host(wk_ctx* ctx) {
    if (!ctx->batch_host) ctx->batch_host = new BatchHost();
    return (BatchHost*)ctx->batch_host;
}

// Resolve every query (host threads, no allocation per query) and fill the pinned descriptor
// staging.
int build_plan(wk_ctx* ctx, BatchState* b, const wk_query* queries, uint32_t n, Plan& P) {
    P.n = n;
    P.levels = 0;
    std::fill(P.width, P.width + kMaxBatchLevels, 0);
    P.status.assign(n, 0);
    P.steps.resize((size_t)n * kMaxBatchLevels);
    P.nsteps.assign(n, 0);
    const int max_cols = ctx->cfg.max_cols;
    const bool versatile = ctx->versatile;
#pragma omp parallel if (n >= 2048)
    {
        std::vector<wk::PlanStep> st;
        st.reserve(kMaxBatchLevels + 4);
        int levels = 0, width[kMaxBatchLevels] = {0};
#pragma omp for schedule(static) nowait
        for (int64_t qi = 0; qi < (int64_t)n; ++qi) {
            const uint32_t q = (uint32_t)qi;
            wk::ColMap cm(queries[q].nvars);
            int rc = wk::resolve_plan(queries[q], max_cols, st, cm, versatile);
            if (rc == WK_SUCCESS && (int)st.size() > kMaxBatchLevels) rc = WK_E_CAPACITY;
            // the unknown-predicate operators walk several lists per row: single queries only
            for (auto& x : st)
                if (rc == WK_SUCCESS && wk::is_versatile_step(x.kind)) rc = WK_E_UNSUPPORTED;
            if (rc == WK_SUCCESS && queries[q].mt_factor != 1) rc = WK_E_UNSUPPORTED;
            if (rc) {
                P.status[q] = rc;
                st.clear();
            }
            P.nsteps[q] = (uint8_t)st.size();
            std::copy(st.begin(), st.end(), P.steps.begin() + (size_t)q * kMaxBatchLevels);
            levels = std::max<int>(levels, (int)st.size());
            for (size_t k = 0; k < st.size(); ++k) width[k] = std::max(width[k], st[k].out_cols);
        }
#pragma omp critical
        {
            P.levels = std::max(P.levels, levels);
            for (int k = 0; k < kMaxBatchLevels; ++k) P.width[k] = std::max(P.width[k], width[k]);
        }
    }
    int w = 1;
    for (int k = 0; k < P.levels; ++k) w = std::max(w, P.width[k]);
    int rc = ensure_state(ctx, b, n, std::max(P.levels, 1), std::max<uint64_t>(b->rows_cap, 1 << 20),
                          std::max(b->w_cap, std::max(w, 8)), std::max<uint64_t>(b->result_cap, 1 << 22));
    if (rc) return rc;
    const int L = P.levels;
#pragma omp parallel for schedule(static) if (n >= 2048)
    for (int64_t qi = 0; qi < (int64_t)n; ++qi) {
        const uint32_t q = (uint32_t)qi;
        const int ns = P.nsteps[q];
        const wk::PlanStep* st = P.steps.data() + (size_t)q * kMaxBatchLevels;
        b->h_nsteps[q] = (uint32_t)ns;
        b->h_final_cols[q] = ns ? (uint32_t)st[ns - 1].out_cols : 0;
        for (int k = 0; k < L; ++k) {
            wk::StepDesc& d = b->h_desc[(size_t)k * n + q];
            if (k >= ns) {
                std::memset(&d, 0, sizeof(d));
                d.op = wk::kXDone;
            } else {
                d = wk::make_step_desc(ctx, st[k]);
            }
        }
    }
    return WK_SUCCESS;
}

// Copy the batch's descriptors from the pinned staging to the device.
int upload_plan(wk_ctx* ctx, BatchState* b, const Plan& P, cudaStream_t s = nullptr) {
    const uint32_t n = P.n;
    if (!s) s = ctx->stream;
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_desc, b->h_desc, sizeof(wk::StepDesc) * (size_t)P.levels * n,
                                  cudaMemcpyHostToDevice, s));
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_nsteps, b->h_nsteps, 4ull * n, cudaMemcpyHostToDevice, s));
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_final_cols, b->h_final_cols, 4ull * n, cudaMemcpyHostToDevice, s));
    return WK_SUCCESS;
}

// Events and counter read-backs around each level launch (profiling runs only).
struct ProfHooks {
    cudaEvent_t ev[2 * kMaxBatchLevels];
    cudaEvent_t extra[6];        // around the setup memsets, the result scan, the gather
    unsigned long long* h_cnt;   // pinned [kMaxBatchLevels][2]: sum_deg, alg_bytes
};

// Enqueue the device work of a batch whose descriptors are resident.
int enqueue_batch(wk_ctx* ctx, BatchState* b, const Plan& P, ProfHooks* ph = nullptr) {
    const uint32_t n = P.n;
    const int L = P.levels;
    cudaStream_t s = ctx->stream;
    uint64_t region_off[kMaxBatchLevels + 1] = {0};
    for (int k = 0; k < L; ++k) region_off[k + 1] = region_off[k] + b->rows_cap * (uint64_t)P.width[k];
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[0], s));
    WKB_CUDA(ctx, cudaMemsetAsync(b->d_qfirst, 0xFF, 8ull * L * n, s));
    WKB_CUDA(ctx, cudaMemsetAsync(b->d_qcount, 0, 8ull * L * n, s));
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[1], s));
    const int lanes = ctx->batch_lanes;
    for (int k = 0; k < L; ++k) {
        wk::ExploreArgs a{};
        a.store = ctx->dev_store();
        a.seg_index[0] = ctx->seg_of(0, 0, wk::kIn);
        a.seg_index[1] = ctx->seg_of(0, 0, wk::kOut);
        a.desc = b->d_desc + (size_t)k * n;
        a.n_queries = n;
        a.virtual_rows = k == 0;
        a.in_rows = k > 0 ? b->d_total_out + (k - 1) : nullptr;
        a.owner_in = k > 0 ? b->d_owner + (size_t)(k - 1) * b->rows_cap : nullptr;
        a.in = k > 0 ? b->d_arena + region_off[k - 1] : nullptr;
        a.w_in = k > 0 ? P.width[k - 1] : 0;
        a.in_cap_rows = b->rows_cap;
        a.out = b->d_arena + region_off[k];
        a.w_out = P.width[k];
        a.out_cap_rows = b->rows_cap;
        a.owner_out = b->d_owner + (size_t)k * b->rows_cap;
        a.out_rows = b->d_total_out + k;
        a.qfirst = b->d_qfirst + (size_t)k * n;
        a.qcount = b->d_qcount + (size_t)k * n;
        a.heavy = ctx->d_heavy;
        a.heavy_cap = ctx->heavy_cap;
        a.ctl = ctx->d_ctl;
        a.status = ctx->d_status;
        a.sorted_lists = ctx->sorted_lists;
        a.lanes = lanes;
        a.slice_rows = ctx->batch_slice_rows;
        a.spin_limit = ctx->spin_limit;
        const int grid = wk::explore_blocks_per_sm(a.virtual_rows ? 0 : a.w_in, a.w_out, lanes) * ctx->sm_count;
        if (ph) {
            WKB_CUDA(ctx, cudaMemsetAsync(&ctx->d_ctl->sum_deg, 0, 16, s));
            WKB_CUDA(ctx, cudaEventRecord(ph->ev[2 * k], s));
        }
        cudaError_t e;
        if ((ctx->batch_flat >> k) & 1) {   // the four flat passes (wk_flat.cu), not the tile launch
            wk::FlatLevelArgs f{};
            f.store = a.store;
            f.seg_index[0] = a.seg_index[0];
            f.seg_index[1] = a.seg_index[1];
            f.desc = a.desc;
            f.n_queries = n;
            f.virtual_rows = a.virtual_rows;
            f.in_rows = a.in_rows;
            f.owner_in = a.owner_in;
            f.in = a.in;
            f.w_in = a.w_in;
            f.in_cap_rows = a.in_cap_rows;
            f.out = a.out;
            f.w_out = a.w_out;
            f.out_cap_rows = a.out_cap_rows;
            f.out_rows = a.out_rows;
            f.owner_out = a.owner_out;
            f.qfirst = a.qfirst;
            f.qcount = a.qcount;
            f.pos = b->d_flat;
            f.off = b->d_flat + b->flat_rows + 1;
            f.part = f.off + b->flat_rows;
            f.ctl = a.ctl;
            f.sorted_lists = a.sorted_lists;
            e = wk::launch_flat_level(f, wk::flat_grid(ctx->sm_count), s);
        } else {
            e = wk::launch_explore(a, grid, s);
        }
        if (e != cudaSuccess) return ctx->cuda_fail(e, "level launch");
        if (ph) {
            WKB_CUDA(ctx, cudaEventRecord(ph->ev[2 * k + 1], s));
            WKB_CUDA(ctx, cudaMemcpyAsync(ph->h_cnt + 2 * k, &ctx->d_ctl->sum_deg, 16,
                                          cudaMemcpyDeviceToHost, s));
        }
    }
    wk::ResultScanArgs ra{};
    ra.n = n;
    ra.nsteps = b->d_nsteps;
    ra.qfirst = b->d_qfirst;
    ra.qcount = b->d_qcount;
    ra.final_cols = b->d_final_cols;
    ra.final_level = b->d_final_level;
    ra.final_base = b->d_final_base;
    ra.final_rows = b->d_final_rows;
    ra.res_off = b->d_res_off;
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[2], s));
    cudaError_t e = wk::launch_result_scan(ra, s);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "result scan launch");
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[3], s));
    wk::GatherArgs ga{};
    ga.n = n;
    ga.final_level = b->d_final_level;
    ga.final_base = b->d_final_base;
    ga.final_rows = b->d_final_rows;
    ga.final_cols = b->d_final_cols;
    ga.res_off = b->d_res_off;
    for (int k = 0; k < L; ++k) {
        ga.region[k] = b->d_arena + region_off[k];
        ga.width[k] = P.width[k];
    }
    ga.out = b->d_result;
    ga.out_cap = b->result_cap;
    ga.ctl = ctx->d_ctl;
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[4], s));
    e = wk::launch_gather(ga, ctx->sm_count * 8, s);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "gather launch");
    if (ph) WKB_CUDA(ctx, cudaEventRecord(ph->extra[5], s));
    return WK_SUCCESS;
}

// Launch the batch (from a cached graph when the shape repeats); no host sync.
int launch_batch(wk_ctx* ctx, BatchState* b, const Plan& P) {
    std::string shape;
    auto put = [&](const void* p, size_t k) { shape.append((const char*)p, k); };
    put(&P.n, 4);
    put(&P.levels, 4);
    put(P.width, sizeof(P.width));
    put(&b->d_arena, sizeof(void*));
    put(&b->d_result, sizeof(void*));
    put(&b->rows_cap, 8);
    put(&b->result_cap, 8);
    put(&ctx->d_status, sizeof(void*));
    put(&ctx->d_heavy, sizeof(void*));
    put(&ctx->heavy_cap, 8);
    put(&ctx->batch_lanes, 4);
    put(&ctx->batch_slice_rows, 4);
    put(&ctx->batch_flat, 4);
    put(&b->d_flat, sizeof(void*));
    put(&ctx->d_slots, sizeof(void*));
    if (shape != b->shape || !b->exec) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        cudaGraph_t g;
        WKB_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_batch(ctx, b, P);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return ctx->cuda_fail(e, "batch capture");
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "batch instantiate");
        b->shape = shape;
    }
    WKB_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
    return WK_SUCCESS;
}

// Run a batch to completion, growing buffers on overflow.  On success the compact results are
// on the device and h_final_rows / h_res_off hold the per-query layout.
int run_batch(wk_ctx* ctx, BatchState* b, const wk_query* queries, uint32_t n, Plan& P) {
    int rc = build_plan(ctx, b, queries, n, P);
    if (rc) return rc;
    if (P.levels == 0) {
        std::fill(b->h_final_rows, b->h_final_rows + n, 0);
        std::fill(b->h_res_off, b->h_res_off + n + 1, 0);
        return WK_SUCCESS;
    }
    for (int attempt = 0; attempt < 8; ++attempt) {
        rc = ctx->ensure_status(b->rows_cap / wk::kTileRows + 2);
        if (rc) return rc;
        rc = ctx->ensure_heavy(b->rows_cap);
        if (rc) return rc;
        rc = upload_plan(ctx, b, P);
        if (rc) return rc;
        rc = launch_batch(ctx, b, P);
        if (rc) return rc;
        uint32_t err = 0;
        uint64_t need = 0;
        rc = ctx->read_ctl(&err, &need);
        if (rc) return rc;
        WKB_CUDA(ctx, cudaMemcpyAsync(b->h_final_rows, b->d_final_rows, 8ull * n, cudaMemcpyDeviceToHost, ctx->stream));
        WKB_CUDA(ctx, cudaMemcpyAsync(b->h_res_off, b->d_res_off, 8ull * (n + 1), cudaMemcpyDeviceToHost, ctx->stream));
        WKB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        const uint64_t total_elems = b->h_res_off[n];
        if (!err && total_elems <= b->result_cap) return WK_SUCCESS;
        ctx->clear_ctl_err();
        if (err & wk::kErrCorrupt) return ctx->fail(WK_E_CORRUPT, "key table chain out of range");
        if (err & wk::kErrTimeout) return ctx->fail(WK_E_TIMEOUT, "batch look-back timed out");
        uint64_t rows = b->rows_cap, res = b->result_cap;
        if (err & (wk::kErrOverflow | wk::kErrStatus)) rows = std::max<uint64_t>(rows * 2, need + need / 4);
        if (total_elems > res) res = total_elems + total_elems / 4 + 1024;
        rc = ensure_state(ctx, b, n, P.levels, rows, b->w_cap, res);
        if (rc) return rc;
        rc = build_plan(ctx, b, queries, n, P);   // staging was reallocated
        if (rc) return rc;
    }
    return ctx->fail(WK_E_CAPACITY, "batch kept overflowing");
}

BatchState* batch_state(wk_ctx* ctx) {
    if (!ctx->batch) ctx->batch = new BatchState();
    return (BatchState*)ctx->batch;
}

// The second state of the pipelined path (wk_batch_execute_stream): two batches in flight.
BatchState* batch_state2(wk_ctx* ctx) {
    if (!ctx->batch2) ctx->batch2 = new BatchState();
    return (BatchState*)ctx->batch2;
}

}  // namespace

void wk_batch_release(wk_ctx* ctx) {
    if (!ctx) return;
    for (void** p : {&ctx->batch, &ctx->batch2}) {
        if (!*p) continue;
        BatchState* b = (BatchState*)*p;
        free_state(b);
        delete b;
        *p = nullptr;
    }
    delete (BatchHost*)ctx->batch_host;
    ctx->batch_host = nullptr;
}

// Pipelined batches.  Per batch, in stream order on the context stream: the descriptor upload,
// the captured launch sequence, a snapshot of the control block (then its error word is
// cleared), and the per-query row counts and offsets; an event marks the batch ready.  While
// the device runs batch i, the host resolves batch i+1's plans into the other state and, once
// batch i-1 is ready, copies its tables to the host on a second stream.  A batch whose snapshot
// shows an overflow is rerun on its own (growing its buffers) before the pipeline goes on.
extern "C" int wk_batch_execute_stream(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t batch,
                                       uint32_t* host_out, uint64_t cap_elems, wk_qresult* results) {
    if (!ctx || (!queries && n) || (!host_out && cap_elems) || (!results && n)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n == 0) return WK_SUCCESS;
    if (batch == 0) batch = 16384;
    BatchState* B[2] = {batch_state(ctx), batch_state2(ctx)};
    BatchHost* H = batch_host(ctx);
    Plan* P = H->plan;
    uint32_t off[2] = {0, 0}, cnt[2] = {0, 0};
    bool pend[2] = {false, false};
    uint64_t out_used = 0;
    cudaStream_t& cs = H->copy_stream;     // copies to the host
    cudaStream_t& us = H->upload_stream;   // descriptor uploads
    cudaEvent_t* ready = H->ready;
    cudaEvent_t* copied = H->copied;
    cudaEvent_t* uploaded = H->uploaded;
    int rc = WK_SUCCESS;
    auto cu = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && !rc) rc = ctx->cuda_fail(e, what);
        return rc;
    };
    // Wait for the batch in state `k`, rerun it alone if it overflowed, then start its copy out.
    auto finish = [&](int k) -> int {
        if (cu(cudaEventSynchronize(ready[k]), "batch ready")) return rc;
        pend[k] = false;
        BatchState* b = B[k];
        uint64_t total = b->h_res_off[cnt[k]];
        if (b->h_ctl->err || total > b->result_cap) {
            if (b->h_ctl->err & wk::kErrCorrupt) return rc = ctx->fail(WK_E_CORRUPT, "key table chain out of range");
            if (b->h_ctl->err & wk::kErrTimeout) return rc = ctx->fail(WK_E_TIMEOUT, "batch look-back timed out");
            if (cu(cudaStreamSynchronize(cs), "copy stream")) return rc;
            if ((rc = run_batch(ctx, b, queries + off[k], cnt[k], P[k]))) return rc;
            total = b->h_res_off[cnt[k]];
        }
        if (out_used + total > cap_elems) return rc = ctx->fail(WK_E_CAPACITY, "host buffer too small");
        for (uint32_t i = 0; i < cnt[k]; ++i) {
            wk_qresult& r = results[off[k] + i];
            std::memset(&r, 0, sizeof(r));
            r.status = P[k].status[i];
            r.rows = r.status ? 0 : b->h_final_rows[i];
            r.cols = (int32_t)b->h_final_cols[i];
            r.elem_offset = out_used + b->h_res_off[i];
        }
        if (cu(cudaStreamWaitEvent(cs, ready[k], 0), "copy wait")) return rc;
        if (total && cu(cudaMemcpyAsync(host_out + out_used, b->d_result, total * 4, cudaMemcpyDeviceToHost, cs),
                        "result copy"))
            return rc;
        if (cu(cudaEventRecord(copied[k], cs), "copy event")) return rc;
        out_used += total;
        return rc;
    };
    if (!cs) cu(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "copy stream");
    if (!us) cu(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking), "upload stream");
    for (int k = 0; k < 2 && !rc; ++k) {
        if (!ready[k]) cu(cudaEventCreateWithFlags(&ready[k], cudaEventDisableTiming), "event");
        if (!copied[k]) cu(cudaEventCreateWithFlags(&copied[k], cudaEventDisableTiming), "event");
        if (!uploaded[k]) cu(cudaEventCreateWithFlags(&uploaded[k], cudaEventDisableTiming), "event");
        if (!rc) cu(cudaEventRecord(copied[k], cs), "event");
    }
    for (uint32_t i = 0, start = 0; !rc && start < n; ++i, start += batch) {
        const int k = i & 1;
        const uint32_t m = std::min(batch, n - start);
        if (pend[k] && finish(k)) break;
        // resolve this batch while the device runs the previous one and copies out the one
        // before it: the host staging of this state was last read by that earlier batch's
        // upload, which its launch waited for; its device buffers are guarded on the device
        // (the launch below waits for the copy), and a buffer that has to grow waits for the
        // whole device first (ensure_state)
        if ((rc = build_plan(ctx, B[k], queries + start, m, P[k]))) break;
        off[k] = start;
        cnt[k] = m;
        if (P[k].levels == 0) {   // nothing reaches the device: every plan failed or is empty
            if (pend[k ^ 1] && finish(k ^ 1)) break;
            for (uint32_t q = 0; q < m; ++q) {
                wk_qresult& r = results[start + q];
                std::memset(&r, 0, sizeof(r));
                r.status = P[k].status[q];
                r.elem_offset = out_used;
            }
            continue;
        }
        if ((rc = ctx->ensure_status(B[k]->rows_cap / wk::kTileRows + 2))) break;
        if ((rc = ctx->ensure_heavy(B[k]->rows_cap))) break;
        // descriptors go up on their own stream while the previous batch still computes
        if ((rc = upload_plan(ctx, B[k], P[k], us))) break;
        if (cu(cudaEventRecord(uploaded[k], us), "upload event")) break;
        if (cu(cudaStreamWaitEvent(ctx->stream, uploaded[k], 0), "upload wait")) break;
        if (cu(cudaStreamWaitEvent(ctx->stream, copied[k], 0), "state free")) break;
        if ((rc = launch_batch(ctx, B[k], P[k]))) break;
        cudaStream_t s = ctx->stream;
        cu(cudaMemcpyAsync(B[k]->h_ctl, ctx->d_ctl, sizeof(wk::StepCtl), cudaMemcpyDeviceToHost, s), "ctl");
        cu(cudaMemsetAsync(&ctx->d_ctl->err, 0, sizeof(unsigned), s), "ctl");
        cu(cudaMemsetAsync(&ctx->d_ctl->need, 0, sizeof(unsigned long long), s), "ctl");
        cu(cudaMemcpyAsync(B[k]->h_final_rows, B[k]->d_final_rows, 8ull * m, cudaMemcpyDeviceToHost, s), "rows");
        cu(cudaMemcpyAsync(B[k]->h_res_off, B[k]->d_res_off, 8ull * (m + 1), cudaMemcpyDeviceToHost, s), "offsets");
        cu(cudaEventRecord(ready[k], s), "ready");
        if (rc) break;
        pend[k] = true;
        // the previous batch: its tables go to the host while this one runs
        if (pend[k ^ 1] && finish(k ^ 1)) break;
    }
    for (int k = 0; k < 2 && !rc; ++k)   // the last batch is the only one still pending
        if (pend[k]) finish(k);
    if (cs) cudaStreamSynchronize(cs);
    if (us) cudaStreamSynchronize(us);
    cudaStreamSynchronize(ctx->stream);
    return rc;
}

extern "C" int wk_batch_execute(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t* host_out,
                                uint64_t cap_elems, wk_qresult* results) {
    if (!ctx || (!queries && n) || (!host_out && cap_elems) || (!results && n)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n == 0) return WK_SUCCESS;
    BatchState* b = batch_state(ctx);
    Plan& P = batch_host(ctx)->plan[0];
    int rc = run_batch(ctx, b, queries, n, P);
    if (rc) return rc;
    const uint64_t total = b->h_res_off[n];
    for (uint32_t q = 0; q < n; ++q) {
        wk_qresult& r = results[q];
        std::memset(&r, 0, sizeof(r));
        r.status = P.status[q];
        r.rows = P.status[q] ? 0 : b->h_final_rows[q];
        r.cols = (int32_t)b->h_final_cols[q];
        r.elem_offset = b->h_res_off[q];
    }
    if (total > cap_elems) return ctx->fail(WK_E_CAPACITY, "host buffer too small");
    if (total)
        WKB_CUDA(ctx, cudaMemcpyAsync(host_out, b->d_result, total * 4, cudaMemcpyDeviceToHost, ctx->stream));
    WKB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return WK_SUCCESS;
}

extern "C" int wk_batch_execute_device(wk_ctx* ctx, const wk_query* queries, uint32_t n,
                                       uint64_t* total_rows) {
    if (!ctx || (!queries && n)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n == 0) {
        if (total_rows) *total_rows = 0;
        return WK_SUCCESS;
    }
    BatchState* b = batch_state(ctx);
    Plan& P = batch_host(ctx)->plan[0];
    int rc = run_batch(ctx, b, queries, n, P);
    if (rc) return rc;
    uint64_t t = 0;
    for (uint32_t q = 0; q < n; ++q) t += P.status[q] ? 0 : b->h_final_rows[q];
    if (total_rows) *total_rows = t;
    return WK_SUCCESS;
}

// Replay the last batch's graph on the context stream without waiting (for device timing).
extern "C" int wk_batch_replay(wk_ctx* ctx) {
    if (!ctx) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    BatchState* b = (BatchState*)ctx->batch;
    if (!b || !b->exec) return ctx->fail(WK_E_BADARG, "no batch has run on this context");
    WKB_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
    return WK_SUCCESS;
}

extern "C" int wk_batch_profile(wk_ctx* ctx, const wk_query* queries, uint32_t n, int32_t iters,
                                wk_step_prof* out, int32_t max_levels, int32_t* n_levels) {
    if (!ctx || (!queries && n) || iters < 1 || (!out && max_levels)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    BatchState* b = batch_state(ctx);
    Plan& P = batch_host(ctx)->plan[0];
    int rc = run_batch(ctx, b, queries, n, P);   // sizes the buffers
    if (rc) return rc;
    if (P.levels + 3 > max_levels) return ctx->fail(WK_E_CAPACITY, "profile array too small");
    ProfHooks ph;
    for (auto& e : ph.ev) WKB_CUDA(ctx, cudaEventCreate(&e));
    for (auto& e : ph.extra) WKB_CUDA(ctx, cudaEventCreate(&e));
    WKB_CUDA(ctx, cudaMallocHost(&ph.h_cnt, sizeof(unsigned long long) * 2 * kMaxBatchLevels));
    std::vector<double> acc(P.levels + 3, 0.0);
    for (int it = 0; it <= iters && rc == WK_SUCCESS; ++it) {
        rc = enqueue_batch(ctx, b, P, &ph);
        if (rc) break;
        WKB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < P.levels + 3; ++k) {
            float ms = 0;
            if (k < P.levels)
                WKB_CUDA(ctx, cudaEventElapsedTime(&ms, ph.ev[2 * k], ph.ev[2 * k + 1]));
            else
                WKB_CUDA(ctx, cudaEventElapsedTime(&ms, ph.extra[2 * (k - P.levels)],
                                                   ph.extra[2 * (k - P.levels) + 1]));
            if (it > 0) acc[k] += ms;
        }
    }
    if (rc == WK_SUCCESS) {
        std::vector<uint64_t> tot(P.levels, 0);
        WKB_CUDA(ctx, cudaMemcpy(tot.data(), b->d_total_out, 8ull * P.levels, cudaMemcpyDeviceToHost));
        for (int k = 0; k < P.levels; ++k) {
            wk_step_prof& p = out[k];
            std::memset(&p, 0, sizeof(p));
            p.kind = 5;
            p.cols_in = k ? P.width[k - 1] : 0;
            p.cols_out = P.width[k];
            p.rows_in = k ? tot[k - 1] : n;
            p.rows_out = tot[k];
            p.sum_deg = ph.h_cnt[2 * k];
            p.alg_bytes = ph.h_cnt[2 * k + 1];
            p.ms = acc[k] / iters;
        }
        for (int k = 0; k < 3; ++k) {   // setup memsets, result scan, gather
            wk_step_prof& p = out[P.levels + k];
            std::memset(&p, 0, sizeof(p));
            p.kind = 6 + k;
            p.ms = acc[P.levels + k] / iters;
        }
        if (n_levels) *n_levels = P.levels + 3;
    }
    for (auto& e : ph.extra) cudaEventDestroy(e);
    for (auto& e : ph.ev) cudaEventDestroy(e);
    cudaFreeHost(ph.h_cnt);
    return rc;
}

