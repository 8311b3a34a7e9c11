// known_to_unknown without any allocation: wk_step_known_to_unknown_noalloc.
//
// wk_step_known_to_unknown grows the context's scan scratch (status array, long-list slice
// queue) and the output table when a step needs more, and every growth is a cudaMalloc /
// cudaFree.  Some callers cannot allow that: code that runs while another stream of the same
// device must not be stalled (cudaFree waits for the whole device), callers that account for
// every device byte up front, and callers that must not enter the allocator at all.  This
// variant runs the same exploration launch with its scan scratch in one fixed device array of
// this file, and fails with WK_E_CAPACITY where the other entry point would allocate.
//
// Limits: inputs up to (kNoAllocTiles - 2) * kTileRows rows (16,382 tiles of 256 rows =
// 4,193,792 rows; the status array keeps the two spare words the allocating path keeps) and up
// to kNoAllocSlices long-list slices.  Every row whose list is longer than the context's slice
// threshold (128 rows unless tuned) takes ceil(length / 2,048) slices, so 8,192 slices hold
// between 8,192 such rows (about 1 M output rows at 129 rows each) and 16.7 M output rows of
// long lists.  The output table must already hold the step's result.  The scratch is one array
// per device, shared by every context and stream of that device, so calls that overlap in time
// on one device race and the caller must serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "wk_ctx.h"

namespace {

constexpr uint64_t kNoAllocTiles = 16384;    // status words: one per 256-row input tile
constexpr uint64_t kNoAllocSlices = 8192;    // long-list slices of the queue
constexpr size_t kCtlBytes = 256;            // control block, padded
constexpr size_t kScratchBytes =
    kCtlBytes + kNoAllocTiles * sizeof(unsigned long long) + kNoAllocSlices * sizeof(wk::HeavyItem);
static_assert(sizeof(wk::StepCtl) <= kCtlBytes, "control block fits its slot");
static_assert(kScratchBytes % 8 == 0, "scratch is whole words");

constexpr int kMaxDevices = 64;

}  // namespace

// The scratch: control block, status words, slice queue (448 KiB per device).
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchBytes / 8];

namespace {

std::mutex g_setup_mu;
char* g_scratch[kMaxDevices] = {};   // device address of g_noalloc_scratch, per device

// Zero what the scan expects zeroed (status words, slice tags, counters) and start the epoch.
__global__ void noalloc_init_kernel(unsigned long long* base) {
    const size_t n = kScratchBytes / 8;
    for (size_t i = kCtlBytes / 8 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        base[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        wk::StepCtl c{};
        c.epoch = 1;
        c.status_cap = kNoAllocTiles;
        *reinterpret_cast<wk::StepCtl*>(base) = c;
    }
}

// The set-up of one device, with that device current: the scratch's address and its first
// clearing.
int scratch_setup(wk_ctx* ctx, char** out) {
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaSetDevice");
    void* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    e = wk::use_max_shared_carveout(noalloc_init_kernel);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "no-alloc kernel attribute");
    noalloc_init_kernel<<<64, 256, 0, ctx->stream>>>((unsigned long long*)p);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "no-alloc scratch set-up");
    *out = (char*)p;
    return WK_SUCCESS;
}

// Once per device: the set-up above, after which the calling thread's current device is what
// it was before the call, on success and on failure alike.
int scratch_for(wk_ctx* ctx, char** out) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return ctx->fail(WK_E_BADARG, "device id");
    if (!g_scratch[ctx->device]) {
        int prev = 0;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGetDevice");
        char* p = nullptr;
        const int rc = scratch_setup(ctx, &p);
        e = cudaSetDevice(prev);
        if (rc) return rc;
        if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaSetDevice (restoring the caller's device)");
        g_scratch[ctx->device] = p;
    }
    *out = g_scratch[ctx->device];
    return WK_SUCCESS;
}

}  // namespace

extern "C" int wk_step_known_to_unknown_noalloc(wk_ctx* ctx, const wk_table* in, int32_t col_start,
                                                uint32_t pid, int32_t dir, wk_table* out) {
    if (!ctx || !in || !out || (dir != WK_IN && dir != WK_OUT) || in == out) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (in->cols <= 0 || !in->d || !in->d_rows) return ctx->fail(WK_E_BADARG, "input table has no columns");
    if (col_start < 0 || col_start >= in->cols) return ctx->fail(WK_E_BADARG, "column out of range");
    if (in->cols + 1 > ctx->cfg.max_cols) return ctx->fail(WK_E_CAPACITY, "too many columns");
    if (!out->d || !out->d_rows) return ctx->fail(WK_E_BADARG, "output table not allocated");
    char* base = nullptr;
    int rc = scratch_for(ctx, &base);
    if (rc) return rc;
    auto* ctl = reinterpret_cast<wk::StepCtl*>(base);
    auto* status = reinterpret_cast<unsigned long long*>(base + kCtlBytes);
    auto* slices = reinterpret_cast<wk::HeavyItem*>(base + kCtlBytes + kNoAllocTiles * 8);

    uint64_t rows = 0;
    cudaError_t e = cudaMemcpyAsync(&rows, in->d_rows, sizeof(rows), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "input row count");
    // a row count past the table's capacity marks a table whose writing step overflowed
    if (rows * (uint64_t)in->cols > in->cap)
        return ctx->fail(WK_E_CORRUPT, "input row count " + std::to_string(rows) +
                                           " beyond the table's capacity (the step that wrote it overflowed)");
    if ((rows + wk::kTileRows - 1) / wk::kTileRows + 2 > kNoAllocTiles)
        return ctx->fail(WK_E_CAPACITY, "input has " + std::to_string(rows) + " rows; the no-alloc step takes at most " +
                                            std::to_string((kNoAllocTiles - 2) * wk::kTileRows));

    wk::PlanStep st{};
    st.kind = wk::PlanStep::kK2U;
    st.pid = pid;
    st.dir = dir;
    st.cs = col_start;
    st.in_cols = in->cols;
    st.out_cols = in->cols + 1;
    wk::ExploreArgs a{};
    a.store = ctx->dev_store();
    a.seg_index[0] = ctx->seg_of(0, 0, wk::kIn);
    a.seg_index[1] = ctx->seg_of(0, 0, wk::kOut);
    a.one = wk::make_step_desc(ctx, st);
    a.n_queries = 1;
    a.in_rows = in->d_rows;
    a.in = in->d;
    a.w_in = st.in_cols;
    a.in_cap_rows = in->cap / st.in_cols;
    a.out = out->d;
    a.w_out = st.out_cols;
    a.out_cap_rows = out->cap / st.out_cols;
    a.out_rows = out->d_rows;
    a.heavy = slices;
    a.heavy_cap = kNoAllocSlices;
    a.ctl = ctl;
    a.status = status;
    a.sorted_lists = ctx->sorted_lists;
    a.lanes = ctx->lanes_for(a.one.op, st.in_cols);
    a.slice_rows = ctx->slice_rows;
    a.spin_limit = ctx->spin_limit;
    out->cols = st.out_cols;
    // the same launch shape as wk_step_known_to_unknown's tile launch (a serving lane's context
    // leaves room on every SM for the iteration launches)
    const int grid = ctx->blocks_per_sm(a.one.op, st.in_cols, a.lanes) * ctx->sm_count;
    e = wk::launch_explore(a, grid, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "no-alloc exploration launch");

    wk::StepCtl h{};
    e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "no-alloc step");
    if (!h.err) return WK_SUCCESS;
    // the error word and the size request are sticky: clear them for the next call
    e = cudaMemsetAsync(&ctl->err, 0, sizeof(ctl->err), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&ctl->need, 0, sizeof(ctl->need), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "no-alloc error reset");
    if (h.err & wk::kErrCorrupt) return ctx->fail(WK_E_CORRUPT, "key table chain out of range");
    if (h.err & wk::kErrTimeout) return ctx->fail(WK_E_TIMEOUT, "tile look-back timed out");
    if (h.err & wk::kErrStatus) return ctx->fail(WK_E_CAPACITY, "input exceeds the no-alloc tile limit");
    if (h.err & wk::kErrOverflow) {
        if (h.need > a.out_cap_rows)
            return ctx->fail(WK_E_CAPACITY, "output table holds " + std::to_string(a.out_cap_rows) +
                                                " rows; the step needs " + std::to_string(h.need));
        return ctx->fail(WK_E_CAPACITY, "long lists exceed the no-alloc slice limit of " +
                                            std::to_string(kNoAllocSlices) + " slices");
    }
    return ctx->fail(WK_E_CUDA, "unexpected device error word");
}
