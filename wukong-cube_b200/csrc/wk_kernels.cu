// Exploration-step kernels for sm_100a.
//
// One launch runs one planned pattern over a whole result table (the reference chains five
// kernels, a Thrust scan and two host syncs per pattern: gpu_engine_cuda.hpp:169-177,
// gpu_hash.cu:96-836).  CTAs claim 512-row tiles from a device counter and, per tile:
//   1. start a TMA bulk copy (cp.async.bulk + mbarrier) of the tile's rows into shared memory
//      and, while it is in flight, read each row's start column straight from global memory;
//   2. probe the key table with groups of LANES lanes: each lane loads one 16-byte slot, so a
//      group reads a 32/64/128-byte slice of a bucket in one coalesced request, four rows per
//      group in flight.  Because the static store only ever inserts into the first empty slot
//      (kvstore.hpp:163-180, segment_rdf_dgraph.hpp:216-233), an empty slot before a hit ends
//      the search, so most probes read only the bucket's first 32-byte sector;
//   3. count its output rows: the neighbour count for known_to_unknown, a 0/1 membership flag
//      for known_to_known / known_to_const (a group-wide ballot over the first 8 entries, then a
//      binary search of the rest when lists are sorted, as the loader leaves them);
//   4. turn the counts into output positions with a block scan plus a decoupled look-back
//      across tiles (single pass, 64-bit offsets);
//   5. write its output rows through shared memory with 16-byte stores: known_to_unknown
//      expands each row once per neighbour in row-major, edge order (what the CPU engine
//      appends, sparql.hpp:328-370); the filters compact the surviving rows in order.
// Sizes are read from device memory, so steps chain without a host round trip; an output that
// would not fit sets kErrOverflow and records the size needed instead of writing.
#include <cuda_runtime.h>

#include "wk_device.cuh"
#include "wk_kernels.h"

namespace wk {
namespace {
using namespace dev;

template <int OP, int L>
__global__ void __launch_bounds__(kStepThreads, 4) step_kernel(const StepArgs a, int chunk_rows) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ unsigned long long s_tile, s_excl, s_deg;
    __shared__ uint64_t s_warp[kStepThreads / 32];
    constexpr int kGroups = kStepThreads / L;            // rows per pass
    constexpr int kBatches = kTileRows / (kGroups * kUnroll);
    static_assert(kBatches * kGroups * kUnroll == kTileRows, "tile shape");

    const int C = a.cols;
    const int outc = (OP == kOpK2U) ? C + 1 : C;
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_pre = reinterpret_cast<uint64_t*>(s_in + ((kTileRows * C + 3) & ~3));
    uint64_t* s_off = s_pre + kTileRows + 2;
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_off + kTileRows);
    uint32_t* s_out = s_cnt + kTileRows;

    const unsigned epoch = *(volatile unsigned*)&a.ctl->epoch;
    uint64_t R = *(volatile const uint64_t*)a.in_rows;
    if (C > 0 && R > a.in_cap / C) R = a.in_cap / C;
    uint64_t ntiles = (R + kTileRows - 1) / kTileRows;
    if (ntiles > a.ctl->status_cap) {
        if (threadIdx.x == 0) atomicOr(&a.ctl->err, kErrStatus);
        ntiles = 0;
    }
    if (ntiles == 0 && blockIdx.x == 0 && threadIdx.x == 0) *a.out_rows = 0;
    if (threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();

    const int grp = threadIdx.x / L;
    const int h = threadIdx.x & (L - 1);
    unsigned phase = 0;

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl->tile_counter, 1ull);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r0 = tile * kTileRows;
        const int n = (int)min((uint64_t)kTileRows, R - r0);
        const uint32_t* src = a.in + r0 * C;

        // 1. rows -> shared memory, asynchronously (tables carry >= 64 bytes of tail padding)
        if (threadIdx.x == 0) {
            const unsigned bytes = (unsigned)(((uint64_t)n * C * 4 + 15) & ~15ull);
            mbar_expect_tx(&s_bar, bytes);
            tma_load_1d(s_in, src, bytes, &s_bar);
            s_deg = 0;
        }
        for (int r = threadIdx.x; r < n; r += kStepThreads) s_cnt[r] = 0;
        __syncthreads();

        // 2-3. probe and count, start columns read from global memory
#pragma unroll 1
        for (int b = 0; b < kBatches; ++b) {
            uint64_t key[kUnroll], bucket[kUnroll], ptr[kUnroll];
            bool valid[kUnroll], pending[kUnroll];
            int row[kUnroll];
            uint32_t target[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                row[u] = (b * kUnroll + u) * kGroups + grp;
                valid[u] = row[u] < n;
                const uint32_t cur = valid[u] ? __ldg(src + (uint64_t)row[u] * C + a.col_start) : kBlankId;
                target[u] = (OP == kOpK2K) ? (valid[u] ? __ldg(src + (uint64_t)row[u] * C + a.col_end) : 0)
                                           : a.end_const;
                const SegDesc* sg = &a.seg;
                if (OP == kOpK2U && a.type_index) {
                    // get_index(cur, IN) (sparql.hpp:342-345); only 17-bit ids can be keys
                    key[u] = make_key(0, cur, kIn);
                    sg = &a.seg_index;
                    if (cur >= (1u << kNbitsIdx)) valid[u] = false;
                } else {
                    key[u] = make_key(cur, a.pid, a.dir);
                    if (cur == 0) sg = &a.seg_index;   // vid 0 names the index segment
                }
                if (cur == kBlankId) valid[u] = false;
                pending[u] = valid[u] && sg->num_buckets != 0 && key[u] != 0;
                bucket[u] = pending[u] ? bucket_of(key[u], *sg) : 0;
            }
            group_probe<L>(a.store, key, bucket, pending, ptr, &a.ctl->err);
            uint64_t off[kUnroll], deg[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                off[u] = ptr_off(ptr[u]);
                deg[u] = ptr_size(ptr[u]);
                if (off[u] + deg[u] > a.store.n_edges) {
                    if (h == 0 && deg[u]) atomicOr(&a.ctl->err, kErrCorrupt);
                    deg[u] = 0;
                }
            }
            if (OP == kOpK2U) {
                if (h == 0) {
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u)
                        if (valid[u]) {
                            s_off[row[u]] = off[u];
                            s_cnt[row[u]] = (uint32_t)deg[u];
                        }
                }
            } else {
                bool has[kUnroll], found[kUnroll];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) has[u] = valid[u] && deg[u] > 0;
                group_member<L>(a.store.edges, off, deg, target, has, a.sorted_lists != 0, found);
                if (h == 0) {
                    unsigned long long d = 0;
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u)
                        if (valid[u]) {
                            s_cnt[row[u]] = found[u] ? 1u : 0u;
                            d += deg[u];
                        }
                    if (d) atomicAdd(&s_deg, d);
                }
            }
        }
        __syncthreads();

        // 4. positions
        const uint64_t total = block_scan(s_cnt, s_pre, n, s_warp);
        if (threadIdx.x < 32) {
            const uint64_t ex = lookback_warp(a.status, a.ctl, tile, total, epoch);
            if (threadIdx.x == 0) {
                s_excl = ex;
                const unsigned long long d = OP == kOpK2U ? total : s_deg;
                atomicAdd(&a.ctl->sum_deg, d);
                atomicAdd(&a.ctl->alg_bytes, (unsigned long long)n * C * 4 + (unsigned long long)n * 16 +
                                                 d * 4 + (unsigned long long)total * outc * 4);
            }
        }
        mbar_wait(&s_bar, phase, &a.ctl->err);   // the tile's rows are in shared memory
        phase ^= 1;
        __syncthreads();
        const uint64_t excl = s_excl;
        if (tile == ntiles - 1 && threadIdx.x == 0) *a.out_rows = excl + total;

        // 5. write
        const uint64_t end_elems = (excl + total) * (uint64_t)outc;
        if (end_elems > a.out_cap) {
            if (threadIdx.x == 0) {
                atomicOr(&a.ctl->err, kErrOverflow);
                atomicMax(&a.ctl->need, (unsigned long long)end_elems);
            }
        } else if (total) {
            if (OP == kOpK2U) {
                for (uint64_t c0 = 0; c0 < total; c0 += chunk_rows) {
                    const int m = (int)min((uint64_t)chunk_rows, total - c0);
                    for (int j = threadIdx.x; j < m; j += kStepThreads) {
                        const uint64_t o = c0 + j;
                        int lo = 0, hi = n;   // s_pre[lo] <= o < s_pre[hi]
                        while (hi - lo > 1) {
                            const int mid = (lo + hi) >> 1;
                            if (s_pre[mid] <= o) lo = mid; else hi = mid;
                        }
                        const uint64_t k = o - s_pre[lo];
                        const uint32_t e = __ldg(a.store.edges + s_off[lo] + k);
                        uint32_t* dst = s_out + (size_t)j * outc;
                        const uint32_t* sr = s_in + lo * C;
                        for (int c = 0; c < C; ++c) dst[c] = sr[c];
                        dst[C] = e;
                    }
                    __syncthreads();
                    store_words(a.out + (excl + c0) * outc, s_out, (uint64_t)m * outc);
                    __syncthreads();
                }
            } else {
                for (int r = threadIdx.x; r < n; r += kStepThreads) {
                    if (s_cnt[r]) {
                        uint32_t* dst = s_out + s_pre[r] * C;
                        const uint32_t* sr = s_in + r * C;
                        for (int c = 0; c < C; ++c) dst[c] = sr[c];
                    }
                }
                __syncthreads();
                store_words(a.out + excl * C, s_out, total * C);
            }
        }
        __syncthreads();
    }
    exit_protocol(a.ctl, a.status, epoch);
}

__global__ void list_kernel(const ListArgs a) {
    __shared__ uint64_t s_ptr;
    if (threadIdx.x < 32) {
        uint64_t key[kUnroll] = {a.key, 0, 0, 0};
        bool pending[kUnroll] = {threadIdx.x < 8 && a.seg.num_buckets != 0 && a.key != 0, false, false,
                                 false};
        uint64_t bucket[kUnroll] = {pending[0] ? bucket_of(a.key, a.seg) : 0, 0, 0, 0};
        uint64_t ptr[kUnroll];
        group_probe<8>(a.store, key, bucket, pending, ptr, &a.ctl->err);
        if (threadIdx.x == 0) s_ptr = ptr[0];
    }
    __syncthreads();
    const uint64_t off = ptr_off(s_ptr);
    uint64_t sz = ptr_size(s_ptr);
    if (off + sz > a.store.n_edges) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && sz) atomicOr(&a.ctl->err, kErrCorrupt);
        sz = 0;
    }
    // mt_factor slice (sparql.hpp:213-224)
    const uint64_t f = a.mt_factor > 0 ? (uint64_t)a.mt_factor : 1;
    const uint64_t start = (uint64_t)a.mt_tid % f, len = sz / f;
    const uint64_t b = start * len;
    const uint64_t e = (start == f - 1) ? sz : (start + 1) * len;
    const uint64_t n = e - b;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.out_rows = n;
        atomicAdd(&a.ctl->sum_deg, (unsigned long long)sz);
        atomicAdd(&a.ctl->alg_bytes, 16ull + (unsigned long long)n * 8);
        if (n > a.out_cap) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)n);
        }
    }
    if (n > a.out_cap) return;
    const uint32_t* srcp = a.store.edges + off + b;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        a.out[i] = __ldg(srcp + i);
}

// Checks that every key's list is strictly ascending (the loader's sort + dedup), which lets
// the filters binary-search long lists.
__global__ void sorted_check_kernel(const Slot* slots, uint64_t n_slots, const uint32_t* edges,
                                    uint64_t n_edges, unsigned* unsorted) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_slots;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if ((i & (kAssoc - 1)) == kAssoc - 1) continue;   // chain link
        const Slot s = slots[i];
        if (s.key == 0) continue;
        const uint64_t off = ptr_off(s.ptr), sz = ptr_size(s.ptr);
        if (off + sz > n_edges) {
            atomicOr(unsorted, 2u);
            continue;
        }
        for (uint64_t k = 1; k < sz; ++k)
            if (edges[off + k - 1] >= edges[off + k]) {
                atomicOr(unsorted, 1u);
                break;
            }
    }
}

template <int OP>
cudaError_t launch_op(const StepArgs& a, int grid, int lanes, size_t smem, int chunk, cudaStream_t s) {
    switch (lanes) {
    case 2: step_kernel<OP, 2><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case 4: step_kernel<OP, 4><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case 8: step_kernel<OP, 8><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int OP, int L>
cudaError_t set_attr(int bytes) {
    return cudaFuncSetAttribute(step_kernel<OP, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <int OP>
int occupancy(int lanes, size_t smem) {
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    if (lanes == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<OP, 2>, kStepThreads, smem);
    if (lanes == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<OP, 4>, kStepThreads, smem);
    if (lanes == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<OP, 8>, kStepThreads, smem);
    return (e == cudaSuccess && nb > 0) ? nb : 1;
}

}  // namespace

size_t step_smem_bytes(int cols, int op, int* out_chunk_rows) {
    size_t in_words = ((size_t)kTileRows * cols + 3) & ~(size_t)3;
    size_t bytes = in_words * 4 + (kTileRows + 2) * 8 + kTileRows * 8 + kTileRows * 4;
    int chunk = 0;
    if (op == kOpK2U) {
        chunk = kChunkBytes / ((cols + 1) * 4);
        if (chunk > 1024) chunk = 1024;
        if (chunk < 32) chunk = 32;
        bytes += (size_t)chunk * (cols + 1) * 4;
    } else {
        bytes += (size_t)kTileRows * cols * 4;
    }
    if (out_chunk_rows) *out_chunk_rows = chunk;
    return bytes;
}

cudaError_t step_kernel_attrs(int max_cols) {
    size_t mx = 0;
    for (int op = 0; op < 3; ++op) {
        size_t b = step_smem_bytes(max_cols, op, nullptr);
        if (b > mx) mx = b;
    }
    const int bytes = (int)mx;
    cudaError_t e;
#define WK_ATTR(OPV, LV) \
    if ((e = set_attr<OPV, LV>(bytes)) != cudaSuccess) return e;
    WK_ATTR(kOpK2U, 2) WK_ATTR(kOpK2U, 4) WK_ATTR(kOpK2U, 8)
    WK_ATTR(kOpK2K, 2) WK_ATTR(kOpK2K, 4) WK_ATTR(kOpK2K, 8)
    WK_ATTR(kOpK2C, 2) WK_ATTR(kOpK2C, 4) WK_ATTR(kOpK2C, 8)
#undef WK_ATTR
    return cudaSuccess;
}

int step_blocks_per_sm(int cols, int op, int lanes) {
    size_t smem = step_smem_bytes(cols, op, nullptr);
    if (op == kOpK2U) return occupancy<kOpK2U>(lanes, smem);
    if (op == kOpK2K) return occupancy<kOpK2K>(lanes, smem);
    return occupancy<kOpK2C>(lanes, smem);
}

cudaError_t launch_step(const StepArgs& a, int grid, cudaStream_t s) {
    int chunk = 0;
    size_t smem = step_smem_bytes(a.cols, a.op, &chunk);
    if (grid < 1) grid = 1;
    const int lanes = a.lanes ? a.lanes : 2;
    switch (a.op) {
    case kOpK2U: return launch_op<kOpK2U>(a, grid, lanes, smem, chunk, s);
    case kOpK2K: return launch_op<kOpK2K>(a, grid, lanes, smem, chunk, s);
    case kOpK2C: return launch_op<kOpK2C>(a, grid, lanes, smem, chunk, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_list(const ListArgs& a, int grid, cudaStream_t s) {
    if (grid < 1) grid = 1;
    list_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sorted_check(const DevStore& st, unsigned* d_flag, cudaStream_t s) {
    sorted_check_kernel<<<1024, 256, 0, s>>>(st.slots, st.n_buckets * kAssoc, st.edges, st.n_edges, d_flag);
    return cudaGetLastError();
}

}  // namespace wk
