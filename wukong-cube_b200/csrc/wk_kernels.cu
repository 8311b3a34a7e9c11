// Exploration-step kernels for sm_100a.
//
// One launch runs one planned pattern over a whole result table (the reference chains five
// kernels, a Thrust scan and two host syncs per pattern: gpu_engine_cuda.hpp:169-177,
// gpu_hash.cu:96-836).  Each CTA claims 512-row tiles from a device counter and, per tile:
//   1. stages the tile's rows in shared memory with coalesced loads;
//   2. probes the key table with 8-lane groups: one 16-byte slot per lane, so a group reads
//      one 128-byte bucket in a single coalesced request, four keys per group in flight;
//      chains through slot 7 are followed until a hit or an empty link;
//   3. counts its output rows (neighbour count for known_to_unknown, a 0/1 membership flag
//      for known_to_known / known_to_const, found by a group-wide ballot over the list);
//   4. turns the counts into output positions with a block scan plus a decoupled look-back
//      across tiles (single pass, 64-bit offsets);
//   5. writes its output rows through shared memory with 16-byte stores: known_to_unknown
//      expands each row once per neighbour in row-major, edge order (what the CPU engine
//      appends, sparql.hpp:328-370); the filters compact the surviving rows in order.
// Sizes are read from device memory, so steps chain without a host round trip; an output that
// would not fit sets kErrOverflow and records the size needed instead of writing.
#include <cuda_runtime.h>

#include "wk_kernels.h"

namespace wk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kGroup = 8;                                 // lanes per bucket probe
constexpr int kGroups = kStepThreads / kGroup;            // groups per CTA
constexpr int kUnroll = 4;                                // keys per group in flight
constexpr int kRowsPerGroup = kTileRows / kGroups;        // 16
constexpr int kMaxHops = 1 << 16;                         // chain walk limit
constexpr unsigned long long kFlagAgg = 1, kFlagPrefix = 2;
constexpr unsigned long long kValMask = (1ull << 46) - 1;
constexpr unsigned long long kSpinLimit = 1ull << 24;     // look-back polls before giving up
constexpr int kChunkBytes = 32 * 1024;                    // staging of one output chunk

static_assert(kTileRows % kStepThreads == 0, "rows per thread");
static_assert(kRowsPerGroup % kUnroll == 0, "unroll");

__device__ __forceinline__ unsigned long long pack_status(unsigned epoch, unsigned long long flag,
                                                          unsigned long long v) {
    return ((unsigned long long)epoch << 48) | (flag << 46) | (v & kValMask);
}

__device__ __forceinline__ ulonglong2 load_slot(const Slot* p) {
    return __ldg(reinterpret_cast<const ulonglong2*>(p));
}

// Probe kUnroll keys per 8-lane group.  Every lane of the warp must call this (the ballots and
// shuffles are warp-wide).  On return ptr[u] is the slot's pointer word in every lane of the
// group, or 0 when the key is absent.
__device__ __forceinline__ void group_probe(const DevStore& st, const uint64_t (&bstart)[kUnroll],
                                            const uint64_t (&nbk)[kUnroll],
                                            const uint64_t (&key)[kUnroll],
                                            const bool (&valid)[kUnroll],
                                            uint64_t (&ptr)[kUnroll], unsigned* err) {
    const int lane = threadIdx.x & 31;
    const int gl = lane & (kGroup - 1);
    const int gbase = lane & ~(kGroup - 1);
    uint64_t bucket[kUnroll];
    bool pending[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        ptr[u] = 0;
        pending[u] = valid[u] && nbk[u] != 0 && key[u] != 0;
        bucket[u] = pending[u] ? bstart[u] + hash_u64(key[u]) % nbk[u] : 0;
    }
    for (int hop = 0;; ++hop) {
        bool any = false;
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) any |= pending[u];
        if (!__any_sync(kFull, any)) break;
        if (hop >= kMaxHops) {
            if (any && gl == 0) atomicOr(err, kErrCorrupt);
            break;
        }
        ulonglong2 s[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            s[u] = make_ulonglong2(0, 0);
            if (pending[u]) {
                if (bucket[u] >= st.n_buckets) {
                    pending[u] = false;
                    if (gl == 0) atomicOr(err, kErrCorrupt);
                } else {
                    s[u] = load_slot(st.slots + bucket[u] * kAssoc + gl);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const bool hit = pending[u] && gl < kAssoc - 1 && s[u].x == key[u];
            const unsigned m = (__ballot_sync(kFull, hit) >> gbase) & 0x7Fu;
            const int src = m ? gbase + __ffs(m) - 1 : gbase + kAssoc - 1;
            const uint64_t kx = __shfl_sync(kFull, s[u].x, src);
            const uint64_t py = __shfl_sync(kFull, s[u].y, src);
            if (pending[u]) {
                if (m) {
                    ptr[u] = py;
                    pending[u] = false;
                } else if (kx == 0) {
                    pending[u] = false;   // empty chain link: key absent
                } else {
                    bucket[u] = key_vid(kx);
                }
            }
        }
    }
}

// Exclusive block scan of s_cnt[0..n) into s_pre[0..n]; returns the tile total.
__device__ __forceinline__ uint64_t block_scan(const uint32_t* s_cnt, uint64_t* s_pre, int n,
                                               uint64_t* s_warp) {
    constexpr int per = kTileRows / kStepThreads;
    constexpr int nwarps = kStepThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = threadIdx.x * per;
    uint64_t v[per];
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        v[i] = (base + i < n) ? s_cnt[base + i] : 0;
        sum += v[i];
    }
    uint64_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < nwarps ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < nwarps; o <<= 1) {
            uint64_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nwarps) s_warp[lane] = w;
    }
    __syncthreads();
    uint64_t run = (warp ? s_warp[warp - 1] : 0) + x - sum;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        if (base + i < n) s_pre[base + i] = run;
        run += v[i];
    }
    const uint64_t total = s_warp[nwarps - 1];
    if (threadIdx.x == 0) s_pre[n] = total;
    __syncthreads();
    return total;
}

// Decoupled look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", 2016) by one thread.  Tiles are claimed in order from the tile counter, so every
// predecessor is held by a running CTA and the wait ends; it is still bounded.
__device__ uint64_t lookback(unsigned long long* status, StepCtl* ctl, uint64_t tile, uint64_t agg,
                             unsigned epoch) {
    volatile unsigned long long* st = status;
    if (tile == 0) {
        st[0] = pack_status(epoch, kFlagPrefix, agg);
        return 0;
    }
    st[tile] = pack_status(epoch, kFlagAgg, agg);
    uint64_t excl = 0;
    int64_t p = (int64_t)tile - 1;
    unsigned long long spins = 0;
    while (p >= 0) {
        const unsigned long long s = st[p];
        const unsigned se = (unsigned)(s >> 48);
        const unsigned long long flag = (s >> 46) & 3ull;
        if (se != epoch || flag == 0) {
            if (++spins > kSpinLimit) {
                atomicOr(&ctl->err, kErrTimeout);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        excl += s & kValMask;
        if (flag == kFlagPrefix) break;
        --p;
    }
    st[tile] = pack_status(epoch, kFlagPrefix, excl + agg);
    return excl;
}

// Copy `count` words from shared memory to global memory with 16-byte stores where aligned.
__device__ __forceinline__ void store_words(uint32_t* dst, const uint32_t* src, uint64_t count) {
    const uintptr_t addr = reinterpret_cast<uintptr_t>(dst);
    uint64_t head = ((16 - (addr & 15)) & 15) >> 2;
    if (head > count) head = count;
    if (threadIdx.x < head) dst[threadIdx.x] = src[threadIdx.x];
    const uint64_t nvec = (count - head) >> 2;
    uint4* dv = reinterpret_cast<uint4*>(dst + head);
    const uint32_t* sv = src + head;
    for (uint64_t v = threadIdx.x; v < nvec; v += blockDim.x) {
        uint4 x;
        x.x = sv[4 * v];
        x.y = sv[4 * v + 1];
        x.z = sv[4 * v + 2];
        x.w = sv[4 * v + 3];
        dv[v] = x;
    }
    const uint64_t done = head + (nvec << 2);
    if (threadIdx.x < count - done) dst[done + threadIdx.x] = src[done + threadIdx.x];
}

// The last CTA to leave resets the tile/exit counters and advances the epoch; when the 16-bit
// epoch wraps it clears the status array first so no stale word can match the next epoch.
__device__ void exit_protocol(StepCtl* ctl, unsigned long long* status, unsigned epoch) {
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->exit_counter, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    unsigned next = epoch + 1;
    if (next > 0xFFFFu) {
        for (unsigned long long i = threadIdx.x; i < ctl->status_cap; i += blockDim.x) status[i] = 0;
        next = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->tile_counter = 0;
        ctl->exit_counter = 0;
        __threadfence();
        *(volatile unsigned*)&ctl->epoch = next;
        __threadfence();
    }
}

template <int OP>
__global__ void __launch_bounds__(kStepThreads) step_kernel(const StepArgs a, int chunk_rows) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long s_tile, s_excl, s_deg;
    __shared__ uint64_t s_warp[kStepThreads / 32];

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

    const int gid = threadIdx.x / kGroup;
    const int gl = threadIdx.x & (kGroup - 1);
    const int gbase = (threadIdx.x & 31) & ~(kGroup - 1);

    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&a.ctl->tile_counter, 1ull);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r0 = tile * kTileRows;
        const int n = (int)min((uint64_t)kTileRows, R - r0);

        // 1. stage the tile's rows
        const uint32_t* src = a.in + r0 * C;
        for (int e = threadIdx.x; e < n * C; e += kStepThreads) s_in[e] = __ldg(src + e);
        for (int r = threadIdx.x; r < n; r += kStepThreads) s_cnt[r] = 0;
        if (threadIdx.x == 0) s_deg = 0;
        __syncthreads();

        // 2-3. probe and count
#pragma unroll 1
        for (int b = 0; b < kRowsPerGroup; b += kUnroll) {
            uint64_t bstart[kUnroll], nbk[kUnroll], key[kUnroll], ptr[kUnroll];
            bool valid[kUnroll];
            int row[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                row[u] = gid + kGroups * (b + u);
                valid[u] = row[u] < n;
                const uint32_t cur = valid[u] ? s_in[row[u] * C + a.col_start] : kBlankId;
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
                bstart[u] = sg->bucket_start;
                nbk[u] = sg->num_buckets;
            }
            group_probe(a.store, bstart, nbk, key, valid, ptr, &a.ctl->err);
            uint64_t off[kUnroll], deg[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                off[u] = ptr_off(ptr[u]);
                deg[u] = ptr_size(ptr[u]);
                if (off[u] + deg[u] > a.store.n_edges) {
                    if (gl == 0 && deg[u]) atomicOr(&a.ctl->err, kErrCorrupt);
                    deg[u] = 0;
                }
                if (OP != kOpK2U && gl == 0 && valid[u] && deg[u])
                    atomicAdd(&s_deg, (unsigned long long)deg[u]);
            }
            if (OP == kOpK2U) {
                if (gl == 0) {
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u)
                        if (valid[u]) {
                            s_off[row[u]] = off[u];
                            s_cnt[row[u]] = (uint32_t)deg[u];
                        }
                }
            } else {
                // membership of the target in the neighbour list, 8 elements per round
                uint32_t target[kUnroll];
                bool active[kUnroll], found[kUnroll];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    target[u] = (OP == kOpK2K) ? (valid[u] ? s_in[row[u] * C + a.col_end] : 0)
                                               : a.end_const;
                    active[u] = valid[u] && deg[u] > 0;
                    found[u] = false;
                }
                for (uint64_t k = 0;; k += kGroup) {
                    bool any = false;
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) any |= active[u];
                    if (!__any_sync(kFull, any)) break;
                    uint32_t v[kUnroll];
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u)
                        v[u] = (active[u] && k + gl < deg[u]) ? __ldg(a.store.edges + off[u] + k + gl)
                                                              : 0;
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) {
                        const bool hit = active[u] && k + gl < deg[u] && v[u] == target[u];
                        const unsigned m = (__ballot_sync(kFull, hit) >> gbase) & 0xFFu;
                        if (active[u]) {
                            if (m) {
                                found[u] = true;
                                active[u] = false;
                            } else if (k + kGroup >= deg[u]) {
                                active[u] = false;
                            }
                        }
                    }
                }
                if (gl == 0) {
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u)
                        if (valid[u]) s_cnt[row[u]] = found[u] ? 1u : 0u;
                }
            }
        }
        __syncthreads();

        // 4. positions
        const uint64_t total = block_scan(s_cnt, s_pre, n, s_warp);
        if (threadIdx.x == 0) {
            s_excl = lookback(a.status, a.ctl, tile, total, epoch);
            atomicAdd(&a.ctl->sum_deg, (unsigned long long)(OP == kOpK2U ? total : s_deg));
        }
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
        uint64_t bstart[kUnroll] = {a.seg.bucket_start, 0, 0, 0};
        uint64_t nbk[kUnroll] = {a.seg.num_buckets, 0, 0, 0};
        uint64_t key[kUnroll] = {a.key, 0, 0, 0};
        bool valid[kUnroll] = {threadIdx.x < kGroup, false, false, false};
        uint64_t ptr[kUnroll];
        group_probe(a.store, bstart, nbk, key, valid, ptr, &a.ctl->err);
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
    cudaError_t e;
    e = cudaFuncSetAttribute(step_kernel<kOpK2U>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(step_kernel<kOpK2K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(step_kernel<kOpK2C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
}

int step_blocks_per_sm(int cols, int op) {
    size_t smem = step_smem_bytes(cols, op, nullptr);
    int nb = 0;
    cudaError_t e;
    if (op == kOpK2U)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<kOpK2U>, kStepThreads, smem);
    else if (op == kOpK2K)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<kOpK2K>, kStepThreads, smem);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel<kOpK2C>, kStepThreads, smem);
    if (e != cudaSuccess || nb < 1) nb = 1;
    return nb;
}

cudaError_t launch_step(const StepArgs& a, int grid, cudaStream_t s) {
    int chunk = 0;
    size_t smem = step_smem_bytes(a.cols, a.op, &chunk);
    if (grid < 1) grid = 1;
    switch (a.op) {
    case kOpK2U: step_kernel<kOpK2U><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case kOpK2K: step_kernel<kOpK2K><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case kOpK2C: step_kernel<kOpK2C><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_list(const ListArgs& a, int grid, cudaStream_t s) {
    if (grid < 1) grid = 1;
    list_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace wk
