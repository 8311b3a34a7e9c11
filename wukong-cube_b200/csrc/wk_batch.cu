// Batched light queries: one persistent launch per level over all queries of a batch.
//
// No counterpart in the reference, which serves one query per GPU agent at a time
// (gpu_agent.hpp:173-246) and leaves light queries to the CPU engines
// (console_proxy.hpp:387-392).  Each level launch is a device work queue: CTAs claim 512-row
// tiles of the level's flattened input (all active queries' tables in query order) from an
// atomic counter, look up each row's query and step, and run the same probe / count / scan /
// write pipeline as the single-query step kernel, so the integer results are the same.  Levels
// and their prep launches are replayed from a CUDA graph cached per batch shape.
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
using namespace dev;

constexpr int kPrepThreads = 1024;

// Query owning flattened row r: the last q with row_start[q] <= r.
__device__ __forceinline__ uint32_t find_query(const uint64_t* row_start, uint32_t n, uint64_t r) {
    uint32_t lo = 0, hi = n;   // row_start[lo] <= r < row_start[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(row_start + mid) <= r) lo = mid; else hi = mid;
    }
    return lo;
}

template <int L>
__global__ void __launch_bounds__(kStepThreads, 3) level_kernel(const LevelArgs a, int chunk_rows) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long s_tile, s_excl, s_alg, s_sd;
    __shared__ uint64_t s_warp[kStepThreads / 32];
    constexpr int kGroups = kStepThreads / L;
    constexpr int kBatches = kTileRows / (kGroups * kUnroll);
    static_assert(kBatches * kGroups * kUnroll == kTileRows, "tile shape");

    const int wi = a.w_in, wo = a.w_out;
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_pre = reinterpret_cast<uint64_t*>(s_in + ((kTileRows * wi + 3) & ~3));
    uint64_t* s_off = s_pre + kTileRows + 2;
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_off + kTileRows);
    uint32_t* s_q = s_cnt + kTileRows;
    uint32_t* s_meta = s_q + kTileRows;        // op | cin << 8 | cout << 16
    uint32_t* s_out = s_meta + kTileRows;

    const unsigned epoch = *(volatile unsigned*)&a.ctl->epoch;
    uint64_t R = a.row_start[a.n];
    uint64_t ntiles = (R + kTileRows - 1) / kTileRows;
    if (R + 1 > a.pref_cap) {
        if (threadIdx.x == 0 && blockIdx.x == 0) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)(R + 1));
        }
        ntiles = 0;
        R = 0;
    }
    if (ntiles > a.ctl->status_cap) {
        if (threadIdx.x == 0) atomicOr(&a.ctl->err, kErrStatus);
        ntiles = 0;
        R = 0;
    }
    if (ntiles == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        *a.total_out = 0;
        a.pref[0] = 0;
    }
    const int grp = threadIdx.x / L;
    const int h = threadIdx.x & (L - 1);

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl->tile_counter, 1ull);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r0 = tile * kTileRows;
        const int n = (int)min((uint64_t)kTileRows, R - r0);

        // 1. owner query of every row, and the rows themselves
        for (int i = threadIdx.x; i < n; i += kStepThreads) {
            const uint32_t q = find_query(a.row_start, a.n, r0 + i);
            s_q[i] = q;
            s_cnt[i] = 0;
        }
        if (threadIdx.x == 0) {
            s_alg = 0;
            s_sd = 0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < n * wi; e += kStepThreads) {
            const int i = e / wi, c = e - i * wi;
            const uint32_t q = s_q[i];
            const uint64_t phys = __ldg(a.src_base + q) + (r0 + i - __ldg(a.row_start + q));
            s_in[e] = __ldg(a.in + phys * wi + c);
        }
        __syncthreads();

        // 2-3. probe and count
#pragma unroll 1
        for (int b = 0; b < kBatches; ++b) {
            uint64_t key[kUnroll], bucket[kUnroll], ptr[kUnroll];
            bool valid[kUnroll], pending[kUnroll];
            int row[kUnroll];
            uint32_t target[kUnroll], op[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                row[u] = (b * kUnroll + u) * kGroups + grp;
                valid[u] = row[u] < n;
                const BatchDesc* d = a.desc + (valid[u] ? s_q[row[u]] : 0);
                op[u] = valid[u] ? d->op : kBDone;
                if (op[u] == kBDone) valid[u] = false;
                const SegDesc* sg = &d->seg;
                target[u] = d->end_const;
                if (op[u] == kBStart) {
                    key[u] = d->start_key;
                } else {
                    const uint32_t* rin = s_in + row[u] * wi;
                    const uint32_t cur = valid[u] ? rin[d->cs] : kBlankId;
                    if (op[u] == kBK2K) target[u] = rin[d->ce];
                    if (op[u] == kBK2U && d->type_index) {
                        key[u] = make_key(0, cur, kIn);
                        sg = &a.seg_index[kIn];
                        if (cur >= (1u << kNbitsIdx)) valid[u] = false;
                    } else {
                        key[u] = make_key(cur, d->pid, d->dir);
                        if (cur == 0) sg = &a.seg_index[d->dir & 1];
                    }
                    if (cur == kBlankId) valid[u] = false;
                }
                pending[u] = valid[u] && sg->num_buckets != 0 && key[u] != 0;
                bucket[u] = pending[u] ? bucket_of(key[u], *sg) : 0;
                if (h == 0 && row[u] < n)
                    s_meta[row[u]] = op[u] | ((uint32_t)d->cin << 8) | ((uint32_t)d->cout << 16);
            }
            group_probe<L>(a.store, key, bucket, pending, ptr, &a.ctl->err);
            uint64_t off[kUnroll], deg[kUnroll];
            bool has[kUnroll], found[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                off[u] = ptr_off(ptr[u]);
                deg[u] = ptr_size(ptr[u]);
                if (off[u] + deg[u] > a.store.n_edges) {
                    if (h == 0 && deg[u]) atomicOr(&a.ctl->err, kErrCorrupt);
                    deg[u] = 0;
                }
                has[u] = valid[u] && deg[u] > 0 && (op[u] == kBK2K || op[u] == kBK2C);
            }
            group_member<L>(a.store.edges, off, deg, target, has, a.sorted_lists != 0, found);
            if (h == 0) {
                unsigned long long alg = 0, sd = 0;
#pragma unroll
                for (int u = 0; u < kUnroll; ++u)
                    if (valid[u]) {
                        const bool filt = op[u] == kBK2K || op[u] == kBK2C;
                        const uint32_t cnt = filt ? (found[u] ? 1u : 0u) : (uint32_t)deg[u];
                        const uint32_t meta = s_meta[row[u]];
                        s_off[row[u]] = off[u];
                        s_cnt[row[u]] = cnt;
                        sd += deg[u];
                        alg += ((meta >> 8) & 0xFF) * 4ull + 16 + deg[u] * 4 +
                               (unsigned long long)cnt * ((meta >> 16) & 0xFF) * 4;
                    }
                if (alg) {
                    atomicAdd(&s_alg, alg);
                    atomicAdd(&s_sd, sd);
                }
            }
        }
        __syncthreads();

        // 4. positions (pref[] keeps each input row's output position for the prep launch)
        const uint64_t total = block_scan(s_cnt, s_pre, n, s_warp);
        if (threadIdx.x < 32) {
            const uint64_t ex = lookback_warp(a.status, a.ctl, tile, total, epoch);
            if (threadIdx.x == 0) {
                s_excl = ex;
                atomicAdd(&a.ctl->alg_bytes, s_alg);
                atomicAdd(&a.ctl->sum_deg, s_sd);
            }
        }
        __syncthreads();
        const uint64_t excl = s_excl;
        for (int i = threadIdx.x; i < n; i += kStepThreads) a.pref[r0 + i] = excl + s_pre[i];
        if (tile == ntiles - 1 && threadIdx.x == 0) {
            a.pref[R] = excl + total;
            *a.total_out = excl + total;
        }

        // 5. write rows of stride w_out (columns past a query's width are zero)
        if (excl + total > a.out_cap_rows) {
            if (threadIdx.x == 0) {
                atomicOr(&a.ctl->err, kErrOverflow);
                atomicMax(&a.ctl->need, (unsigned long long)(excl + total));
            }
        } else if (total) {
            for (uint64_t c0 = 0; c0 < total; c0 += chunk_rows) {
                const int m = (int)min((uint64_t)chunk_rows, total - c0);
                for (int j = threadIdx.x; j < m; j += kStepThreads) {
                    const uint64_t o = c0 + j;
                    int lo = 0, hi = n;
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (s_pre[mid] <= o) lo = mid; else hi = mid;
                    }
                    const uint32_t meta = s_meta[lo];
                    const int opv = meta & 0xFF, cin = (meta >> 8) & 0xFF, cout = (meta >> 16) & 0xFF;
                    uint32_t* dst = s_out + (size_t)j * wo;
                    const uint32_t* sr = s_in + lo * wi;
                    int c = 0;
                    if (opv != kBStart)
                        for (; c < cin; ++c) dst[c] = sr[c];
                    if (opv == kBStart || opv == kBK2U) dst[c++] = __ldg(a.store.edges + s_off[lo] + (o - s_pre[lo]));
                    (void)cout;
                    for (; c < wo; ++c) dst[c] = 0;
                }
                __syncthreads();
                store_words(a.out + (excl + c0) * wo, s_out, (uint64_t)m * wo);
                __syncthreads();
            }
        }
        __syncthreads();
    }
    exit_protocol(a.ctl, a.status, epoch);
}

// Single-CTA prep between levels: each query's rows produced by the previous level become its
// input (or its final table), and the active queries' row counts are scanned into row_start.
__global__ void __launch_bounds__(kPrepThreads) prep_kernel(const PrepArgs a) {
    __shared__ uint64_t s_warp[kPrepThreads / 32];
    const uint32_t n = a.n;
    const int k = a.level;
    const uint32_t per = (n + kPrepThreads - 1) / kPrepThreads;
    const uint32_t q0 = min(n, threadIdx.x * per), q1 = min(n, q0 + per);
    const uint64_t prev_total = k > 0 ? a.prev_row_start[n] : 0;
    uint64_t sum = 0;
    for (uint32_t q = q0; q < q1; ++q) {
        uint64_t R = 0, src = 0;
        const uint32_t ns = a.nsteps[q];
        if (k == 0) {
            R = ns > 0 ? 1 : 0;   // one virtual row: the start key
            if (ns == 0) {
                a.final_level[q] = -1;
                a.final_base[q] = 0;
                a.final_rows[q] = 0;
            }
        } else {
            uint64_t rs = a.prev_row_start[q], re = a.prev_row_start[q + 1];
            const uint64_t lim = prev_total < a.prev_pref_cap ? prev_total : a.prev_pref_cap - 1;
            if (rs > lim) rs = lim;
            if (re > lim) re = lim;
            const uint64_t p0 = a.prev_pref[rs], p1 = a.prev_pref[re];
            R = p1 >= p0 ? p1 - p0 : 0;
            src = p0;
            if (ns == (uint32_t)k) {
                a.final_level[q] = k - 1;
                a.final_base[q] = p0;
                a.final_rows[q] = R;
            }
            if (ns <= (uint32_t)k) R = 0;
        }
        if (a.src_base) a.src_base[q] = src;
        a.row_start[q] = R;   // count for now, prefix below
        sum += R;
    }
    // block-wide exclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = s_warp[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    uint64_t run = (warp ? s_warp[warp - 1] : 0) + x - sum;
    for (uint32_t q = q0; q < q1; ++q) {
        const uint64_t c = a.row_start[q];
        a.row_start[q] = run;
        run += c;
    }
    if (threadIdx.x == kPrepThreads - 1) a.row_start[n] = run;
    if (!a.res_off) return;
    // final pass: element offsets of the compact results
    __syncthreads();
    uint64_t es = 0;
    for (uint32_t q = q0; q < q1; ++q) es += a.final_rows[q] * a.final_cols[q];
    x = es;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = s_warp[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    run = (warp ? s_warp[warp - 1] : 0) + x - es;
    for (uint32_t q = q0; q < q1; ++q) {
        a.res_off[q] = run;
        run += a.final_rows[q] * a.final_cols[q];
    }
    if (threadIdx.x == kPrepThreads - 1) a.res_off[n] = run;
}

// Copy each query's final table (stride of its level) into the compact result buffer.
__global__ void gather_kernel(const GatherArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x / 32;
    for (uint32_t q = blockIdx.x * wpb + threadIdx.x / 32; q < a.n; q += gridDim.x * wpb) {
        const int lev = a.final_level[q];
        const uint64_t rows = a.final_rows[q];
        const uint32_t cols = a.final_cols[q];
        if (lev < 0 || lev >= 16 || rows == 0 || cols == 0) continue;
        const uint64_t off = a.res_off[q];
        if (off + rows * cols > a.out_cap) {
            if (lane == 0) atomicOr(&a.ctl->err, kErrOverflow);
            continue;
        }
        const uint32_t* src = a.region[lev] + a.final_base[q] * (uint64_t)a.width[lev];
        const int w = a.width[lev];
        for (uint64_t e = lane; e < rows * cols; e += 32) {
            const uint64_t r = e / cols, c = e - r * cols;
            a.out[off + e] = src[r * w + c];
        }
    }
}

template <int L>
cudaError_t set_level_attr(int bytes) {
    return cudaFuncSetAttribute(level_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace

size_t level_smem_bytes(int w_in, int w_out, int* chunk_rows) {
    size_t in_words = ((size_t)kTileRows * w_in + 3) & ~(size_t)3;
    size_t bytes = in_words * 4 + (kTileRows + 2) * 8 + kTileRows * 8 + 3 * kTileRows * 4;
    int chunk = 16 * 1024 / (w_out > 0 ? w_out * 4 : 4);
    if (chunk > 1024) chunk = 1024;
    if (chunk < 32) chunk = 32;
    bytes += (size_t)chunk * w_out * 4;
    if (chunk_rows) *chunk_rows = chunk;
    return bytes;
}

cudaError_t level_kernel_attrs() {
    const int bytes = (int)level_smem_bytes(32, 32, nullptr);
    cudaError_t e;
    if ((e = set_level_attr<2>(bytes)) != cudaSuccess) return e;
    if ((e = set_level_attr<4>(bytes)) != cudaSuccess) return e;
    return set_level_attr<8>(bytes);
}

int level_blocks_per_sm(int w_in, int w_out, int lanes) {
    size_t smem = level_smem_bytes(w_in, w_out, nullptr);
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    if (lanes == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, level_kernel<2>, kStepThreads, smem);
    if (lanes == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, level_kernel<4>, kStepThreads, smem);
    if (lanes == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, level_kernel<8>, kStepThreads, smem);
    return (e == cudaSuccess && nb > 0) ? nb : 1;
}

cudaError_t launch_level(const LevelArgs& a, int grid, cudaStream_t s) {
    int chunk = 0;
    size_t smem = level_smem_bytes(a.w_in, a.w_out, &chunk);
    if (grid < 1) grid = 1;
    switch (a.lanes) {
    case 2: level_kernel<2><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case 8: level_kernel<8><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    default: level_kernel<4><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_prep(const PrepArgs& a, cudaStream_t s) {
    prep_kernel<<<1, kPrepThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs& a, int grid, cudaStream_t s) {
    if (grid < 1) grid = 1;
    gather_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace wk

// ---------------------------------------------------------------- host side of the batch
namespace {

constexpr int kMaxLevels = 16;

struct BatchState {
    uint32_t n_cap = 0;
    int l_cap = 0;
    uint64_t rows_cap = 0;     // rows per level region / pref entries
    int w_cap = 0;             // widest row the regions were sized for
    wk::BatchDesc* d_desc = nullptr;      // [l_cap][n_cap]
    uint64_t* d_row_start = nullptr;      // [l_cap + 1][n_cap + 1]
    uint64_t* d_src_base = nullptr;       // [l_cap][n_cap]
    uint64_t* d_pref = nullptr;           // [l_cap][rows_cap + 1]
    uint64_t* d_total_out = nullptr;      // [l_cap]
    uint32_t* d_nsteps = nullptr;         // [n_cap]
    uint32_t* d_final_cols = nullptr;     // [n_cap]
    int32_t* d_final_level = nullptr;     // [n_cap]
    uint64_t* d_final_base = nullptr;     // [n_cap]
    uint64_t* d_final_rows = nullptr;     // [n_cap]
    uint64_t* d_res_off = nullptr;        // [n_cap + 1]
    uint32_t* d_arena = nullptr;          // [l_cap][rows_cap * w_cap]
    uint32_t* d_result = nullptr;         // compact results
    uint64_t result_cap = 0;
    // pinned host staging
    wk::BatchDesc* h_desc = nullptr;
    uint32_t* h_nsteps = nullptr;
    uint32_t* h_final_cols = nullptr;
    uint64_t* h_final_rows = nullptr;
    uint64_t* h_res_off = nullptr;
    // graph of the launch sequence for one batch shape
    cudaGraphExec_t exec = nullptr;
    std::string shape;
};

void free_state(BatchState* b) {
    auto f = [](void* p) { if (p) cudaFree(p); };
    f(b->d_desc); f(b->d_row_start); f(b->d_src_base); f(b->d_pref); f(b->d_total_out);
    f(b->d_nsteps); f(b->d_final_cols); f(b->d_final_level); f(b->d_final_base);
    f(b->d_final_rows); f(b->d_res_off); f(b->d_arena); f(b->d_result);
    auto fh = [](void* p) { if (p) cudaFreeHost(p); };
    fh(b->h_desc); fh(b->h_nsteps); fh(b->h_final_cols); fh(b->h_final_rows); fh(b->h_res_off);
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
    if (n <= b->n_cap && levels <= b->l_cap && rows_cap <= b->rows_cap && w <= b->w_cap &&
        result_cap <= b->result_cap)
        return WK_SUCCESS;
    n = std::max(n, b->n_cap);
    levels = std::max(levels, b->l_cap);
    rows_cap = std::max(rows_cap, b->rows_cap);
    w = std::max(w, b->w_cap);
    result_cap = std::max(result_cap, b->result_cap);
    WKB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    free_state(b);
    auto dm = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    auto hm = [&](void** p, size_t bytes) {
        return cudaMallocHost(p, std::max<size_t>(bytes, 16)) == cudaSuccess;
    };
    bool ok = dm((void**)&b->d_desc, sizeof(wk::BatchDesc) * levels * (size_t)n) &&
              dm((void**)&b->d_row_start, 8ull * (levels + 1) * (n + 1)) &&
              dm((void**)&b->d_src_base, 8ull * (levels + 1) * n) &&
              dm((void**)&b->d_pref, 8ull * levels * (rows_cap + 1)) &&
              dm((void**)&b->d_total_out, 8ull * levels) &&
              dm((void**)&b->d_nsteps, 4ull * n) && dm((void**)&b->d_final_cols, 4ull * n) &&
              dm((void**)&b->d_final_level, 4ull * n) && dm((void**)&b->d_final_base, 8ull * n) &&
              dm((void**)&b->d_final_rows, 8ull * n) && dm((void**)&b->d_res_off, 8ull * (n + 1)) &&
              dm((void**)&b->d_arena, 4ull * levels * rows_cap * w + 64) &&
              dm((void**)&b->d_result, 4ull * result_cap + 64) &&
              hm((void**)&b->h_desc, sizeof(wk::BatchDesc) * levels * (size_t)n) &&
              hm((void**)&b->h_nsteps, 4ull * n) && hm((void**)&b->h_final_cols, 4ull * n) &&
              hm((void**)&b->h_final_rows, 8ull * n) && hm((void**)&b->h_res_off, 8ull * (n + 1));
    if (!ok) {
        free_state(b);
        return ctx->fail(WK_E_OOM, "batch buffers");
    }
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
    int width[kMaxLevels] = {0};
    std::vector<int32_t> status;
};

// Resolve every query and fill the pinned descriptor staging.
int build_plan(wk_ctx* ctx, BatchState* b, const wk_query* queries, uint32_t n, Plan& P) {
    P.n = n;
    P.levels = 0;
    std::fill(P.width, P.width + kMaxLevels, 0);
    P.status.assign(n, 0);
    std::vector<std::vector<wk::PlanStep>> all(n);
    for (uint32_t q = 0; q < n; ++q) {
        wk::ColMap cm(queries[q].nvars);
        int rc = wk::resolve_plan(queries[q], ctx->cfg.max_cols, all[q], cm);
        if (rc == WK_SUCCESS && (int)all[q].size() > kMaxLevels) rc = WK_E_CAPACITY;
        if (rc == WK_SUCCESS && queries[q].mt_factor != 1) rc = WK_E_UNSUPPORTED;
        if (rc) {
            P.status[q] = rc;
            all[q].clear();
        }
        P.levels = std::max<int>(P.levels, (int)all[q].size());
        for (size_t k = 0; k < all[q].size(); ++k) P.width[k] = std::max(P.width[k], all[q][k].out_cols);
    }
    int rc = ensure_state(ctx, b, n, std::max(P.levels, 1), std::max<uint64_t>(b->rows_cap, 1 << 20),
                          std::max(b->w_cap, 8), std::max<uint64_t>(b->result_cap, 1 << 22));
    if (rc) return rc;
    for (uint32_t q = 0; q < n; ++q) {
        const auto& st = all[q];
        b->h_nsteps[q] = (uint32_t)st.size();
        b->h_final_cols[q] = st.empty() ? 0 : (uint32_t)st.back().out_cols;
        for (int k = 0; k < P.levels; ++k) {
            wk::BatchDesc& d = b->h_desc[(size_t)k * n + q];
            std::memset(&d, 0, sizeof(d));
            if (k >= (int)st.size()) {
                d.op = wk::kBDone;
                continue;
            }
            const wk::PlanStep& s = st[k];
            d.dir = (uint8_t)s.dir;
            d.cin = (uint8_t)s.in_cols;
            d.cout = (uint8_t)s.out_cols;
            d.cs = (uint8_t)s.cs;
            d.ce = (uint8_t)s.ce;
            d.pid = s.pid;
            d.end_const = s.end_const;
            switch (s.kind) {
            case wk::PlanStep::kIndex:
                d.op = wk::kBStart;
                d.start_key = wk::make_key(0, s.start_const, s.dir);
                d.seg = ctx->seg_of(0, s.start_const, s.dir);
                break;
            case wk::PlanStep::kConst:
                d.op = wk::kBStart;
                d.start_key = wk::make_key(s.start_const, s.pid, s.dir);
                d.seg = ctx->seg_of(s.start_const, s.pid, s.dir);
                break;
            case wk::PlanStep::kK2U:
                d.op = wk::kBK2U;
                d.type_index = (s.pid == wk::kTypeId && s.dir == wk::kIn) ? 1 : 0;
                d.seg = ctx->seg_of(1, s.pid, s.dir);
                break;
            case wk::PlanStep::kK2K:
                d.op = wk::kBK2K;
                d.seg = ctx->seg_of(1, s.pid, s.dir);
                break;
            default:
                d.op = wk::kBK2C;
                d.seg = ctx->seg_of(1, s.pid, s.dir);
                break;
            }
        }
    }
    return WK_SUCCESS;
}

// Events and counter read-backs around each level launch (profiling runs only).
struct ProfHooks {
    cudaEvent_t ev[2 * kMaxLevels];
    unsigned long long* h_cnt;   // pinned [kMaxLevels][2]: sum_deg, alg_bytes
};

// Copy the batch's descriptors from the pinned staging to the device.
int upload_plan(wk_ctx* ctx, BatchState* b, const Plan& P) {
    const uint32_t n = P.n;
    cudaStream_t s = ctx->stream;
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_desc, b->h_desc, sizeof(wk::BatchDesc) * (size_t)P.levels * n,
                                  cudaMemcpyHostToDevice, s));
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_nsteps, b->h_nsteps, 4ull * n, cudaMemcpyHostToDevice, s));
    WKB_CUDA(ctx, cudaMemcpyAsync(b->d_final_cols, b->h_final_cols, 4ull * n, cudaMemcpyHostToDevice, s));
    return WK_SUCCESS;
}

// Enqueue the device work of a batch whose descriptors are resident: L x (prep, level), final
// prep, gather.
int enqueue_batch(wk_ctx* ctx, BatchState* b, const Plan& P, ProfHooks* ph = nullptr) {
    const uint32_t n = P.n;
    const int L = P.levels;
    cudaStream_t s = ctx->stream;
    uint64_t region_off[kMaxLevels + 1] = {0};
    for (int k = 0; k < L; ++k) region_off[k + 1] = region_off[k] + b->rows_cap * (uint64_t)P.width[k];
    const int lanes = ctx->batch_lanes;
    for (int k = 0; k <= L; ++k) {
        wk::PrepArgs pa{};
        pa.level = k;
        pa.n = n;
        pa.nsteps = b->d_nsteps;
        if (k > 0) {
            pa.prev_row_start = b->d_row_start + (size_t)(k - 1) * (n + 1);
            pa.prev_pref = b->d_pref + (size_t)(k - 1) * (b->rows_cap + 1);
            pa.prev_total_out = b->d_total_out + (k - 1);
            pa.prev_pref_cap = b->rows_cap + 1;
        }
        pa.row_start = b->d_row_start + (size_t)k * (n + 1);
        pa.src_base = b->d_src_base + (size_t)k * n;
        pa.final_level = b->d_final_level;
        pa.final_base = b->d_final_base;
        pa.final_rows = b->d_final_rows;
        pa.final_cols = b->d_final_cols;
        pa.res_off = k == L ? b->d_res_off : nullptr;
        cudaError_t e = wk::launch_prep(pa, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "prep launch");
        if (k == L) break;
        wk::LevelArgs la{};
        la.store = ctx->dev_store();
        la.seg_index[0] = ctx->seg_of(0, 0, wk::kIn);
        la.seg_index[1] = ctx->seg_of(0, 0, wk::kOut);
        la.desc = b->d_desc + (size_t)k * n;
        la.row_start = pa.row_start;
        la.src_base = pa.src_base;
        la.n = n;
        la.in = k > 0 ? b->d_arena + region_off[k - 1] : nullptr;
        la.w_in = k > 0 ? P.width[k - 1] : 0;
        la.out = b->d_arena + region_off[k];
        la.w_out = P.width[k];
        la.out_cap_rows = b->rows_cap;
        la.pref = b->d_pref + (size_t)k * (b->rows_cap + 1);
        la.pref_cap = b->rows_cap + 1;
        la.total_out = b->d_total_out + k;
        la.ctl = ctx->d_ctl;
        la.status = ctx->d_status;
        la.sorted_lists = ctx->sorted_lists;
        la.lanes = lanes;
        const int grid = wk::level_blocks_per_sm(la.w_in, la.w_out, lanes) * ctx->sm_count;
        if (ph) {
            WKB_CUDA(ctx, cudaMemsetAsync(&ctx->d_ctl->sum_deg, 0, 16, s));
            WKB_CUDA(ctx, cudaEventRecord(ph->ev[2 * k], s));
        }
        e = wk::launch_level(la, grid, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "level launch");
        if (ph) {
            WKB_CUDA(ctx, cudaEventRecord(ph->ev[2 * k + 1], s));
            WKB_CUDA(ctx, cudaMemcpyAsync(ph->h_cnt + 2 * k, &ctx->d_ctl->sum_deg, 16,
                                          cudaMemcpyDeviceToHost, s));
        }
    }
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
    cudaError_t e = wk::launch_gather(ga, std::min<uint32_t>((n + 7) / 8, 4096), s);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "gather launch");
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
    put(&ctx->batch_lanes, 4);
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
        rc = ensure_state(ctx, b, n, P.levels, rows, std::max(b->w_cap, 8), res);
        if (rc) return rc;
        rc = build_plan(ctx, b, queries, n, P);   // staging was reallocated
        if (rc) return rc;
    }
    return ctx->fail(WK_E_CAPACITY, "batch kept overflowing");
}

}  // namespace

void wk_batch_release(wk_ctx* ctx) {
    if (!ctx || !ctx->batch) return;
    BatchState* b = (BatchState*)ctx->batch;
    free_state(b);
    delete b;
    ctx->batch = nullptr;
}

static BatchState* batch_state(wk_ctx* ctx) {
    if (!ctx->batch) {
        ctx->batch = new BatchState();
        static bool attrs = false;
        if (!attrs) {
            wk::level_kernel_attrs();
            attrs = true;
        }
    }
    return (BatchState*)ctx->batch;
}

extern "C" int wk_batch_execute(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t* host_out,
                                uint64_t cap_elems, wk_qresult* results) {
    if (!ctx || (!queries && n) || (!host_out && cap_elems) || (!results && n)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->has_store) return ctx->fail(WK_E_NOSTORE, "no store uploaded");
    if (n == 0) return WK_SUCCESS;
    BatchState* b = batch_state(ctx);
    Plan P;
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
    Plan P;
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
    Plan P;
    int rc = run_batch(ctx, b, queries, n, P);   // sizes the buffers
    if (rc) return rc;
    if (P.levels > max_levels) return ctx->fail(WK_E_CAPACITY, "profile array too small");
    ProfHooks ph;
    for (auto& e : ph.ev) WKB_CUDA(ctx, cudaEventCreate(&e));
    WKB_CUDA(ctx, cudaMallocHost(&ph.h_cnt, sizeof(unsigned long long) * 2 * kMaxLevels));
    std::vector<double> acc(P.levels, 0.0);
    std::vector<uint64_t> rows_in(P.levels + 1, 0), rows_out(P.levels, 0);
    for (int it = 0; it <= iters && rc == WK_SUCCESS; ++it) {
        rc = enqueue_batch(ctx, b, P, &ph);
        if (rc) break;
        WKB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < P.levels; ++k) {
            float ms = 0;
            WKB_CUDA(ctx, cudaEventElapsedTime(&ms, ph.ev[2 * k], ph.ev[2 * k + 1]));
            if (it > 0) acc[k] += ms;
        }
    }
    if (rc == WK_SUCCESS) {
        for (int k = 0; k < P.levels; ++k) {
            WKB_CUDA(ctx, cudaMemcpy(&rows_in[k], b->d_row_start + (size_t)k * (n + 1) + n, 8,
                                     cudaMemcpyDeviceToHost));
            WKB_CUDA(ctx, cudaMemcpy(&rows_out[k], b->d_total_out + k, 8, cudaMemcpyDeviceToHost));
            wk_step_prof& p = out[k];
            std::memset(&p, 0, sizeof(p));
            p.kind = 5;
            p.cols_in = k ? P.width[k - 1] : 0;
            p.cols_out = P.width[k];
            p.rows_in = rows_in[k];
            p.rows_out = rows_out[k];
            p.sum_deg = ph.h_cnt[2 * k];
            p.alg_bytes = ph.h_cnt[2 * k + 1];
            p.ms = acc[k] / iters;
        }
        if (n_levels) *n_levels = P.levels;
    }
    for (auto& e : ph.ev) cudaEventDestroy(e);
    cudaFreeHost(ph.h_cnt);
    return rc;
}

extern "C" int wk_serve_run_open_loop(wk_ctx* ctx, const wk_serve_config* cfg, const wk_query* queries,
                                      uint32_t n, const double* arrival_us, uint32_t* host_out,
                                      uint64_t cap_elems, wk_qresult* results) {
    (void)ctx; (void)cfg; (void)queries; (void)n; (void)arrival_us; (void)host_out; (void)cap_elems;
    (void)results;
    return WK_E_UNSUPPORTED;
}
