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

#include "wk_kernels.h"

namespace wk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kUnroll = 4;                                // rows per lane group in flight
constexpr int kMaxProbeIters = 1 << 14;                   // chain walk limit
constexpr unsigned long long kFlagAgg = 1, kFlagPrefix = 2;
constexpr unsigned long long kValMask = (1ull << 46) - 1;
constexpr unsigned long long kSpinLimit = 1ull << 24;     // look-back polls before giving up
constexpr unsigned kTmaWaitLimit = 1u << 24;              // mbarrier polls before giving up
constexpr int kChunkBytes = 32 * 1024;                    // staging of one output chunk
constexpr int kLinear = 8;                                // list entries checked by ballot

static_assert(kTileRows % kStepThreads == 0, "rows per thread");

__device__ __forceinline__ unsigned long long pack_status(unsigned epoch, unsigned long long flag,
                                                          unsigned long long v) {
    return ((unsigned long long)epoch << 48) | (flag << 46) | (v & kValMask);
}

__device__ __forceinline__ ulonglong2 load_slot(const Slot* p) {
    return __ldg(reinterpret_cast<const ulonglong2*>(p));
}

// ---------------------------------------------------------------- mbarrier + TMA bulk copy
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Global -> shared bulk copy; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes,
                                            uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait for the current phase; a timeout sets kErrTimeout and waits once more (bounded)
// so no copy is left in flight when the CTA moves on.
__device__ __forceinline__ void mbar_wait(uint64_t* bar, unsigned parity, unsigned* err) {
    unsigned n = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++n > kTmaWaitLimit) {
            if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
            for (unsigned m = 0; m < kTmaWaitLimit && !mbar_try_wait(bar, parity); ++m) __nanosleep(256);
            return;
        }
    }
}

// ---------------------------------------------------------------- probe
__device__ __forceinline__ uint64_t bucket_of(uint64_t key, const SegDesc& s) {
    return s.bucket_start + mod_barrett(hash_u64(key), s.num_buckets, s.magic);
}

// Probe kUnroll keys per group of L lanes.  Every lane of the warp must call this (ballots and
// shuffles are warp-wide).  On entry bucket[u] is the key's home bucket and pending[u] says
// whether to look; on return ptr[u] is the slot's pointer word in every lane of the group, or 0
// when the key is absent.
template <int L>
__device__ __forceinline__ void group_probe(const DevStore& st, const uint64_t (&key)[kUnroll],
                                            uint64_t (&bucket)[kUnroll], bool (&pending)[kUnroll],
                                            uint64_t (&ptr)[kUnroll], unsigned* err) {
    const int lane = threadIdx.x & 31;
    const int h = lane & (L - 1);
    const int gbase = lane & ~(L - 1);
    const unsigned gmask = (1u << L) - 1;
    int round[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        ptr[u] = 0;
        round[u] = 0;
    }
    for (int it = 0;; ++it) {
        bool any = false;
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) any |= pending[u];
        if (!__any_sync(kFull, any)) break;
        if (it >= kMaxProbeIters) {
            if (any && h == 0) atomicOr(err, kErrCorrupt);
            break;
        }
        ulonglong2 s[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            s[u] = make_ulonglong2(~0ull, 0);
            if (pending[u]) {
                if (bucket[u] >= st.n_buckets) {
                    pending[u] = false;
                    if (h == 0) atomicOr(err, kErrCorrupt);
                } else {
                    s[u] = load_slot(st.slots + bucket[u] * kAssoc + round[u] * L + h);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const bool data = round[u] * L + h < kAssoc - 1;
            const bool hit = pending[u] && data && s[u].x == key[u];
            const bool emp = pending[u] && data && s[u].x == 0;
            const unsigned hm = (__ballot_sync(kFull, hit) >> gbase) & gmask;
            const unsigned em = (__ballot_sync(kFull, emp) >> gbase) & gmask;
            const int src = hm ? gbase + __ffs(hm) - 1 : gbase + L - 1;
            const uint64_t kx = __shfl_sync(kFull, s[u].x, src);
            const uint64_t py = __shfl_sync(kFull, s[u].y, src);
            if (pending[u]) {
                if (hm) {
                    ptr[u] = py;
                    pending[u] = false;
                } else if (em) {
                    pending[u] = false;           // first empty slot: the key is absent
                } else if ((round[u] + 1) * L >= kAssoc) {
                    if (kx == 0) {
                        pending[u] = false;       // no extension bucket
                    } else {
                        bucket[u] = key_vid(kx);  // follow slot 7 (kvstore.hpp:303-310)
                        round[u] = 0;
                    }
                } else {
                    round[u]++;
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

// Membership of target[u] in the (ascending, unique when `sorted`) list edges[off, off+deg):
// the first kLinear entries by a group ballot, the rest by binary search (sorted) or a scan.
template <int L>
__device__ __forceinline__ void group_member(const uint32_t* edges, const uint64_t (&off)[kUnroll],
                                             const uint64_t (&deg)[kUnroll],
                                             const uint32_t (&target)[kUnroll],
                                             const bool (&valid)[kUnroll], bool sorted,
                                             bool (&found)[kUnroll]) {
    const int lane = threadIdx.x & 31;
    const int h = lane & (L - 1);
    const int gbase = lane & ~(L - 1);
    const unsigned gmask = (1u << L) - 1;
    constexpr int per = kLinear / L;
    uint32_t v[kUnroll][per];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
        for (int j = 0; j < per; ++j) {
            const uint64_t k = (uint64_t)j * L + h;
            v[u][j] = (valid[u] && k < deg[u]) ? __ldg(edges + off[u] + k) : ~target[u];
        }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        bool hit = false;
#pragma unroll
        for (int j = 0; j < per; ++j) hit |= (v[u][j] == target[u]);
        found[u] = ((__ballot_sync(kFull, hit && valid[u]) >> gbase) & gmask) != 0;
    }
    // long lists: one lane per group continues
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        bool more = valid[u] && !found[u] && deg[u] > (uint64_t)kLinear;
        bool f = false;
        if (more && h == 0) {
            const uint32_t* p = edges + off[u];
            if (sorted) {
                uint64_t lo = kLinear, hi = deg[u];
                while (lo < hi) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (__ldg(p + mid) < target[u]) lo = mid + 1; else hi = mid;
                }
                f = lo < deg[u] && __ldg(p + lo) == target[u];
            } else {
                for (uint64_t k = kLinear; k < deg[u] && !f; ++k) f = __ldg(p + k) == target[u];
            }
        }
        f = __shfl_sync(kFull, f, gbase);
        found[u] = found[u] || f;
    }
}

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
        if (threadIdx.x == 0) {
            s_excl = lookback(a.status, a.ctl, tile, total, epoch);
            atomicAdd(&a.ctl->sum_deg, (unsigned long long)(OP == kOpK2U ? total : s_deg));
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
