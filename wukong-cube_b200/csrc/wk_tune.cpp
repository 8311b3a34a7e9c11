// The autotuner: picks the exploration launch's tile-schedule knobs by timing the caller's own
// workload.  No counterpart in the reference (its kernels have one fixed launch shape,
// gpu_hash.cu:96-326).
//
// Knobs (wk_ctx_tune_set): lanes per probe group (1 / 2 / 4 / 8 lanes: one thread per row
// reading the home sector, or a group reading 32 / 64 / 128 bytes of a bucket per request) and the slice threshold (lists longer than it are written
// block-per-row as slices by every CTA, shorter ones group-per-row by the CTA that probed them),
// and for batches the mask of levels that run as the flat passes instead of the tile launch
// (chosen greedily level by level after the tile settings).
// Constant-start queries are timed as one batch replayed from its CUDA graph (CUDA events on
// the context stream); index-start queries step by step through wk_query_profile, so lanes are
// chosen per (step kind, input columns).  Everything goes through the public entry points, so
// the tuner holds no lock of its own between them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "wk_batch.h"
#include "wk_ctx.h"

namespace {

constexpr int kLanes[] = {1, 2, 4, 8};
constexpr int kSlices[] = {8, 16, 32, 128, 512};

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// Mean device ms of one batch replay (the batch is captured by the first call).
int time_batch(wk_ctx* ctx, const std::vector<wk_query>& qs, int iters, cudaStream_t s, Events& ev,
               double* ms) {
    uint64_t total = 0;
    int rc = wk_batch_execute_device(ctx, qs.data(), (uint32_t)qs.size(), &total);
    if (rc) return rc;
    if ((rc = wk_batch_replay(ctx))) return rc;   // warm
    if (cudaEventRecord(ev.a, s) != cudaSuccess) return WK_E_CUDA;
    for (int i = 0; i < iters; ++i)
        if ((rc = wk_batch_replay(ctx))) return rc;
    if (cudaEventRecord(ev.b, s) != cudaSuccess || cudaEventSynchronize(ev.b) != cudaSuccess) return WK_E_CUDA;
    float t = 0;
    cudaEventElapsedTime(&t, ev.a, ev.b);
    *ms = t / iters;
    return wk_ctx_check(ctx);
}

// Per-step device ms of every index-start query, added up per (explore op, input columns).
int time_singles(wk_ctx* ctx, const std::vector<wk_query>& qs, int iters,
                 std::map<int, double>* per_step, double* total) {
    *total = 0;
    wk_step_prof prof[32];
    for (const wk_query& q : qs) {
        int32_t ns = 0;
        int rc = wk_query_profile(ctx, &q, iters, prof, 32, &ns);
        if (rc) return rc;
        for (int i = 0; i < ns; ++i) {
            *total += prof[i].ms;
            int op = -1;   // wk_step_prof kinds 2..4 are the exploration ops K2U, K2K, K2C
            if (prof[i].kind == 2) op = wk::kXK2U;
            if (prof[i].kind == 3) op = wk::kXK2K;
            if (prof[i].kind == 4) op = wk::kXK2C;
            if (op >= 0 && per_step) (*per_step)[op * 1000 + prof[i].cols_in] += prof[i].ms;
        }
    }
    return WK_SUCCESS;
}

}  // namespace

extern "C" int wk_measure_random_reads(wk_ctx* ctx, uint64_t region_bytes, int32_t iters,
                                       double* reads_per_s) {
    if (!ctx || !reads_per_s || iters < 1 || region_bytes < (1ull << 20)) return WK_E_BADARG;
    constexpr int kPer = 32;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const int grid = ctx->sm_count * 8;
    void* buf = nullptr;
    uint32_t* sink = nullptr;
    Events ev;
    auto done = [&](int rc) {
        if (buf) cudaFree(buf);
        if (sink) cudaFree(sink);
        return rc;
    };
    if (wk::dev_malloc(&buf, region_bytes) != cudaSuccess || wk::dev_malloc(&sink, 4) != cudaSuccess) {
        cudaGetLastError();
        return done(ctx->fail(WK_E_OOM, "random-read calibration buffer"));
    }
    cudaError_t e = cudaMemsetAsync(buf, 1, region_bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaEventCreate(&ev.a);
    if (e == cudaSuccess) e = cudaEventCreate(&ev.b);
    if (e == cudaSuccess) e = wk::launch_random_reads(buf, region_bytes, kPer, 0, sink, grid, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev.a, ctx->stream);
    for (int i = 0; i < iters && e == cudaSuccess; ++i)
        e = wk::launch_random_reads(buf, region_bytes, kPer, 1 + (uint64_t)i, sink, grid, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev.b, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev.b);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (e != cudaSuccess) return done(ctx->cuda_fail(e, "random-read calibration"));
    *reads_per_s = (double)grid * 256 * kPer * iters / (ms * 1e-3);
    return done(WK_SUCCESS);
}

extern "C" int wk_ctx_autotune(wk_ctx* ctx, const wk_query* queries, uint32_t n, int32_t iters,
                               wk_tune_result* out) {
    if (!ctx || (!queries && n) || iters < 1 || !out) return WK_E_BADARG;
    std::memset(out, 0, sizeof(*out));
    std::vector<wk_query> light, heavy;
    int light_levels = 0;   // levels of the light batch
    for (uint32_t i = 0; i < n; ++i) {
        std::vector<wk::PlanStep> steps;
        wk::ColMap cm(queries[i].nvars);
        if (wk::resolve_plan(queries[i], ctx->cfg.max_cols, steps, cm, ctx->versatile) || steps.empty()) continue;
        bool vers = false;
        for (auto& x : steps) vers |= wk::is_versatile_step(x.kind);
        if (vers) continue;   // not a tile-schedule workload
        const bool is_heavy = steps[0].kind == wk::PlanStep::kIndex;
        (is_heavy ? heavy : light).push_back(queries[i]);
        if (!is_heavy) light_levels = std::max(light_levels, std::min((int)steps.size(), wk::kMaxBatchLevels));
    }
    void* sp = nullptr;
    int rc = wk_ctx_stream(ctx, &sp);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)sp;
    Events ev;
    if (cudaEventCreate(&ev.a) != cudaSuccess || cudaEventCreate(&ev.b) != cudaSuccess)
        return ctx->fail(WK_E_CUDA, "autotune events");
    auto get = [&](int knob) {
        int32_t v = 0;
        wk_ctx_tune_get(ctx, knob, &v);
        return v;
    };
    out->batch_lanes = get(WK_KNOB_BATCH_LANES);
    out->batch_slice_rows = get(WK_KNOB_BATCH_SLICE_ROWS);
    out->lanes = get(WK_KNOB_LANES);
    out->slice_rows = get(WK_KNOB_SLICE_ROWS);

    if (!light.empty()) {
        double best = 0;
        if ((rc = time_batch(ctx, light, iters, s, ev, &best))) return rc;
        out->batch_ms_default = best;
        int bl = out->batch_lanes, bs = out->batch_slice_rows, bf = 0;
        // every tile setting (all levels on the tile launch) ...
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_FLAT, 0))) return rc;
        best = 1e30;
        for (int l : kLanes)
            for (int sl : kSlices) {
                if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_LANES, l))) return rc;
                if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_SLICE_ROWS, sl))) return rc;
                double ms = 0;
                if ((rc = time_batch(ctx, light, iters, s, ev, &ms))) return rc;
                ++out->candidates;
                if (ms < best) {
                    best = ms;
                    bl = l;
                    bs = sl;
                }
            }
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_LANES, bl))) return rc;
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_SLICE_ROWS, bs))) return rc;
        // ... then, level by level, the flat passes where they are faster (greedy)
        for (int k = 0; k < light_levels; ++k) {
            if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_FLAT, bf | (1 << k)))) return rc;
            double ms = 0;
            if ((rc = time_batch(ctx, light, iters, s, ev, &ms))) return rc;
            ++out->candidates;
            if (ms < best) {
                best = ms;
                bf |= 1 << k;
            }
        }
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_BATCH_FLAT, bf))) return rc;
        out->batch_lanes = bl;
        out->batch_slice_rows = bs;
        out->batch_flat = bf;
        out->batch_ms_tuned = best;
    }

    if (!heavy.empty()) {
        double total = 0;
        if ((rc = time_singles(ctx, heavy, iters, nullptr, &total))) return rc;
        out->single_ms_default = total;
        // lanes: per (op, columns) step, the fastest of the four
        std::map<int, std::map<int, double>> by_lanes;   // step key -> lanes -> ms
        std::map<int, double> sum_by_lanes;
        for (int l : kLanes) {
            if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_LANES, l))) return rc;
            std::map<int, double> per;
            double t = 0;
            if ((rc = time_singles(ctx, heavy, iters, &per, &t))) return rc;
            ++out->candidates;
            sum_by_lanes[l] = t;
            for (auto& kv : per) by_lanes[kv.first][l] = kv.second;
        }
        int best_l = kLanes[0];
        for (int l : kLanes)
            if (sum_by_lanes[l] < sum_by_lanes[best_l]) best_l = l;
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_LANES, best_l))) return rc;   // clears per-step choices
        for (auto& kv : by_lanes) {
            int bl = best_l;
            for (auto& lm : kv.second)
                if (lm.second < kv.second[bl]) bl = lm.first;
            if ((rc = wk::tune_step_lanes(ctx, kv.first / 1000, kv.first % 1000, bl))) return rc;
        }
        out->lanes = best_l;
        // slice threshold
        double best = 0;
        int bs = out->slice_rows;
        for (int sl : kSlices) {
            if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_SLICE_ROWS, sl))) return rc;
            double t = 0;
            if ((rc = time_singles(ctx, heavy, iters, nullptr, &t))) return rc;
            ++out->candidates;
            if (sl == kSlices[0] || t < best) {
                best = t;
                bs = sl;
            }
        }
        if ((rc = wk_ctx_tune_set(ctx, WK_KNOB_SLICE_ROWS, bs))) return rc;
        out->slice_rows = bs;
        out->single_ms_tuned = best;
    }
    return WK_SUCCESS;
}
