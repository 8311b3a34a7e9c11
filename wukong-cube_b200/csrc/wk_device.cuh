// Device-side building blocks shared by the single-query and the batched step kernels:
// bounded mbarrier waits and TMA bulk copies, the sector-granular group probe of the key table,
// the block scan, the warp-parallel decoupled look-back, 16-byte stores from shared memory,
// list membership and the self-resetting exit protocol of a launch.
#pragma once
#include <cuda_runtime.h>

#include "wk_kernels.h"

namespace wk {
namespace dev {
namespace {   // internal linkage: every .cu that includes this gets its own copy
constexpr unsigned kFull = 0xffffffffu;
constexpr int kUnroll = 4;                                // rows per lane group in flight
constexpr int kMaxProbeIters = 1 << 14;                   // chain walk limit
constexpr unsigned long long kFlagAgg = 1, kFlagPrefix = 2;
constexpr unsigned long long kValMask = (1ull << 46) - 1;
constexpr unsigned kTmaWaitLimit = 1u << 24;              // mbarrier polls before giving up
constexpr int kChunkBytes = 32 * 1024;                    // staging of one output chunk
constexpr int kLinear = 8;                                // list entries checked by ballot

static_assert(kTileRows % kStepThreads == 0, "rows per thread");

__device__ __forceinline__ unsigned long long pack_status(unsigned epoch, unsigned long long flag,
                                                          unsigned long long v) {
    return ((unsigned long long)epoch << 48) | (flag << 46) | (v & kValMask);
}

// 16 bytes from a random place in a large array, read once: no L1 allocation, first out of L2
// (the probes' lines would otherwise push out the lines the streaming reads and writes reuse).
__device__ __forceinline__ uint4 load16_once(const void* p) {
    uint4 v;
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_first.b64 pol, 1.0;\n\t"
        "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], pol;\n\t}"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
}

__device__ __forceinline__ ulonglong2 load_slot(const Slot* p) {
    const uint4 v = load16_once(p);
    return make_ulonglong2((unsigned long long)v.y << 32 | v.x, (unsigned long long)v.w << 32 | v.z);
}

// Slots p[0] and p[1] (one 32-byte sector) by one 256-bit load.  p must be 32-byte aligned: an
// even slot of a bucket (buckets are 128-byte lines of a cudaMalloc'd array).
__device__ __forceinline__ void load_sector(const Slot* p, ulonglong2* s0, ulonglong2* s1) {
    unsigned long long a, b, c, d;
    // a probe's line is seldom read again: no L1 allocation, first out of L2
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_first.b64 pol, 1.0;\n\t"
        "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u64 {%0, %1, %2, %3}, [%4], pol;\n\t}"
        : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
        : "l"(p));
    *s0 = make_ulonglong2(a, b);
    *s1 = make_ulonglong2(c, d);
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

// ---------------------------------------------------------------- single-entry lists
// The device copy of the store keeps a one-entry list in its key's own pointer word: iptr_t's
// type field (bits 62-63, 0 for the ids this path reads) is set to 3, the size stays 1 and the
// offset field holds the entry itself (inline_kernel, run at upload; the original pointer words
// are kept aside for wk_store_export).  A probe that finds the key then has the entry without a
// second random read of the edge array.  Within a step, a list offset with kInlineTag set
// carries that entry in its low 32 bits instead of an edge-array offset (list_at).
constexpr uint64_t kInlineTag = 1ull << 63;
constexpr uint64_t kInlinePtrType = 3ull << 62;

__host__ __device__ __forceinline__ bool ptr_is_inline(uint64_t p) { return (p >> 62) == 3; }
__host__ __device__ __forceinline__ uint64_t make_inline_ptr(uint32_t entry) {
    return kInlinePtrType | ((uint64_t)entry << kNbitsSize) | 1;
}

// The list a pointer word names: *off an edge-array offset or a tagged entry, *deg its length;
// an offset past the edge array sets kErrCorrupt and an empty list.
__device__ __forceinline__ void list_of_ptr(uint64_t p, uint64_t n_edges, unsigned* err, uint64_t* off,
                                            uint64_t* deg) {
    *deg = ptr_size(p);
    if (ptr_is_inline(p)) {
        *off = kInlineTag | (uint32_t)(p >> kNbitsSize);
        return;
    }
    *off = ptr_off(p);
    if (*off + *deg > n_edges) {
        if (*deg) atomicOr(err, kErrCorrupt);
        *deg = 0;
    }
}

// Entry k of the list at `off` (an edge-array offset, or a tagged single entry).
__device__ __forceinline__ uint32_t list_at(const uint32_t* edges, uint64_t off, uint64_t k) {
    return (off & kInlineTag) ? (uint32_t)off : __ldg(edges + off + k);
}

// Probe kUnroll keys per group of L lanes.  Every lane of the warp must call this (ballots and
// shuffles are warp-wide).  On entry bucket[u] is the key's home bucket and pending[u] says
// whether to look; on return ptr[u] is the slot's pointer word in every lane of the group, or 0
// when the key is absent.  Bucket ids may be held in 32 bits (BucketT): a device's store has
// fewer than 2^32 buckets, and a chain link at or past the bucket count is reported as
// corruption before it is followed.
template <int L, class BucketT>
__device__ __forceinline__ void group_probe(const DevStore& st, const uint64_t (&key)[kUnroll],
                                            BucketT (&bucket)[kUnroll], bool (&pending)[kUnroll],
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
                    // 64-bit index: slot numbers pass 2^32 from bucket 2^29 on
                    s[u] = load_slot(st.slots + (uint64_t)bucket[u] * kAssoc + round[u] * L + h);
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
                    } else if (key_vid(kx) >= st.n_buckets) {
                        pending[u] = false;       // a link out of range: corrupt chain
                        if (h == 0) atomicOr(err, kErrCorrupt);
                    } else {
                        bucket[u] = (BucketT)key_vid(kx);   // follow slot 7 (kvstore.hpp:303-310)
                        round[u] = 0;
                    }
                } else {
                    round[u]++;
                }
            }
        }
    }
}

// Probe one key by one thread: the home bucket's slots two at a time (one 32-byte sector),
// then the chain through slot 7.  Returns the pointer word, 0 when absent.  `first` skips the
// home bucket's slots a caller has already compared (0 or an even slot).
__device__ __forceinline__ uint64_t thread_probe(const DevStore& st, uint64_t key, uint64_t bucket,
                                                 unsigned* err, int first = 0) {
    for (int hop = 0; hop < kMaxProbeIters; ++hop) {
        if (bucket >= st.n_buckets) {
            atomicOr(err, kErrCorrupt);
            return 0;
        }
        const Slot* b = st.slots + bucket * kAssoc;
#pragma unroll
        for (int s = 0; s < kAssoc - 1; s += 2) {
            if (hop == 0 && s < first) continue;
            ulonglong2 s0, s1;
            load_sector(b + s, &s0, &s1);   // both slots: one 32-byte sector
            if (s0.x == key) return s0.y;
            if (s0.x == 0) return 0;   // first empty slot: absent (insert-only store)
            if (s + 1 == kAssoc - 1) {   // slot 7: the chain link
                if (s1.x == 0) return 0;
                bucket = key_vid(s1.x);
                break;
            }
            if (s1.x == key) return s1.y;
            if (s1.x == 0) return 0;
        }
    }
    atomicOr(err, kErrCorrupt);
    return 0;
}

// Is `target` in the list edges[off, off + deg)?  Binary search when lists are sorted.  `off`
// may be a tagged single entry.
__device__ __forceinline__ bool thread_member(const uint32_t* edges, uint64_t off, uint64_t deg,
                                              uint32_t target, bool sorted) {
    if (off & kInlineTag) return deg == 1 && (uint32_t)off == target;
    const uint32_t* p = edges + off;
    if (sorted) {
        uint64_t lo = 0, hi = deg;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (__ldg(p + mid) < target) lo = mid + 1; else hi = mid;
        }
        return lo < deg && __ldg(p + lo) == target;
    }
    for (uint64_t k = 0; k < deg; ++k)
        if (__ldg(p + k) == target) return true;
    return false;
}

// Exclusive block scan of f(s_cnt[0..n)) into s_pre[0..n]; returns the tile total.
template <class Out, class F>
__device__ __forceinline__ uint64_t block_scan(const uint32_t* s_cnt, Out* s_pre, int n, uint64_t* s_warp,
                                               F f) {
    constexpr int per = kTileRows / kStepThreads;
    constexpr int nwarps = kStepThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = threadIdx.x * per;
    uint64_t v[per];
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        v[i] = (base + i < n) ? f(s_cnt[base + i]) : 0;
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
        if (base + i < n) s_pre[base + i] = (Out)run;
        run += v[i];
    }
    const uint64_t total = s_warp[nwarps - 1];
    if (threadIdx.x == 0) s_pre[n] = (Out)total;
    __syncthreads();
    return total;
}

__device__ __forceinline__ uint64_t block_scan(const uint32_t* s_cnt, uint64_t* s_pre, int n,
                                               uint64_t* s_warp) {
    return block_scan(s_cnt, s_pre, n, s_warp, [](uint32_t c) { return (uint64_t)c; });
}

// Decoupled look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", 2016) by one warp: each round reads the 32 nearest unvisited predecessors at once,
// waits until all of them have published at least their aggregate, adds the aggregates up to
// the nearest inclusive prefix and stops there.  Tiles are claimed in order from the tile
// counter, so every predecessor is held by a running CTA and the wait ends; it is still bounded.
// The tile's own entry is published first (publish_aggregate, by one thread, as soon as the
// tile's total is known) and resolved later (resolve_prefix, by all 32 lanes of one warp, which
// returns the exclusive prefix in every lane).
__device__ __forceinline__ void publish_aggregate(unsigned long long* status, uint64_t tile,
                                                  uint64_t agg, unsigned epoch) {
    volatile unsigned long long* st = status;
    st[tile] = pack_status(epoch, tile == 0 ? kFlagPrefix : kFlagAgg, agg);
}

__device__ uint64_t resolve_prefix(unsigned long long* status, StepCtl* ctl, uint64_t tile,
                                   uint64_t agg, unsigned epoch, unsigned long long spin_limit) {
    volatile unsigned long long* st = status;
    const int lane = threadIdx.x & 31;
    if (tile == 0) return 0;   // tile 0 published its inclusive prefix already
    uint64_t excl = 0;
    int64_t base = (int64_t)tile - 1;
    unsigned long long spins = 0;
    for (;;) {
        const int64_t p = base - lane;
        const unsigned long long s = p >= 0 ? st[p] : pack_status(epoch, kFlagPrefix, 0);
        const unsigned long long flag = (s >> 46) & 3ull;
        const bool ready = (unsigned)(s >> 48) == epoch && flag != 0;
        if (!__all_sync(kFull, ready)) {
            if (++spins > spin_limit) {
                if (lane == 0) atomicOr(&ctl->err, kErrTimeout);
                break;
            }
            if (spins > 32) __nanosleep(32);
            continue;
        }
        const unsigned pm = __ballot_sync(kFull, flag == kFlagPrefix);
        const int first = pm ? __ffs(pm) - 1 : 32;   // nearest predecessor holding a prefix
        uint64_t v = lane <= first ? (s & kValMask) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        excl += v;
        if (pm) break;
        base -= 32;
    }
    if (lane == 0) st[tile] = pack_status(epoch, kFlagPrefix, excl + agg);
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
// `tags` / `tag_stride` / `n_tags`: epoch-tagged words of the long-list slice queue, cleared with
// the status array when the epoch wraps.
__device__ void exit_protocol(StepCtl* ctl, unsigned long long* status, unsigned epoch,
                              unsigned* tags, unsigned tag_stride, unsigned long long n_tags) {
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
        for (unsigned long long i = threadIdx.x; i < n_tags; i += blockDim.x) tags[i * tag_stride] = 0;
        next = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->tile_counter = 0;
        ctl->exit_counter = 0;
        ctl->heavy_n = 0;
        ctl->heavy_claim = 0;
        ctl->tiles_done = 0;
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
            v[u][j] = (valid[u] && k < deg[u]) ? list_at(edges, off[u], k) : ~target[u];
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

// ---------------------------------------------------------------- block-wide exclusive sum
// Every thread of a kThreads-thread block passes x and gets the sum of x over the threads
// before it.  s_warp holds kThreads / 32 words; the call synchronises the block.
template <int kThreads>
__device__ __forceinline__ uint64_t block_exclusive_sum(uint64_t x, uint64_t* s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) s_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < kThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const uint64_t before = warp ? s_warp[warp - 1] : 0;
    __syncthreads();   // s_warp may be reused by the caller's next round
    return before + v - x;
}

// ---------------------------------------------------------------- segmented gather
// Copy n tables laid out back to back in `out` (table i fills out[off[i], off[i+1]), row-major,
// cols(i) columns) from their rows in strided arenas (src(i): first row, stride(i) words).
// The output is cut into fixed chunks spread over the grid, so one long table is copied by
// many CTAs and the stores are coalesced; each element finds its table by a binary search of
// `off` narrowed to the chunk's first and last table.
constexpr int kGatherSpan = 1024;   // output elements per warp segment

// Each warp copies contiguous segments of kGatherSpan elements, lane i taking elements i,
// i + 32, ...: it finds the segment's first table once (binary search), then every lane walks
// forward through the tables it crosses.  A lane keeps its element's (row, column) in its
// table and steps it by 32 elements with a carry, so the only division is at a table change.
// Eight elements' source addresses are worked out first, then their eight loads are issued
// together, then the stores (coalesced).  One long table is spread over many warps.
constexpr int kGatherUnroll = 8;

template <class Src>
__device__ void segmented_gather(uint32_t n, const uint64_t* __restrict__ off, Src src,
                                 uint32_t* __restrict__ out) {
    const uint64_t total = off[n];
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t seg = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
         seg * kGatherSpan < total; seg += warps) {
        const uint64_t base = seg * kGatherSpan;
        const uint64_t end = min(total, base + (uint64_t)kGatherSpan);
        uint32_t lo = 0, hi = n - 1;   // last table whose offset is <= base (same in every lane)
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(off + mid) <= base) lo = mid; else hi = mid - 1;
        }
        uint32_t q = lo;
        uint64_t q_lo = __ldg(off + q), q_hi = __ldg(off + q + 1);
        const uint32_t* row0 = nullptr;
        uint32_t stride = 1, cols = 1, step_r = 0, step_c = 0;
        uint64_t r = 0;
        uint32_t c = 0;
        bool placed = false;   // (r, c) hold the position of the lane's current element
        for (uint64_t p0 = base + lane; p0 < end; p0 += 32 * kGatherUnroll) {
            const uint32_t* a[kGatherUnroll];
#pragma unroll
            for (int u = 0; u < kGatherUnroll; ++u) {
                const uint64_t p = p0 + 32ull * u;
                a[u] = nullptr;
                if (p >= end) continue;
                if (p >= q_hi) {   // tables are back to back: step to the one holding p
                    do {
                        ++q;
                        q_lo = q_hi;
                        q_hi = __ldg(off + q + 1);
                    } while (p >= q_hi);
                    placed = false;
                }
                if (!placed) {
                    src(q, row0, stride, cols);
                    const uint64_t e = p - q_lo;
                    r = e / cols;
                    c = (uint32_t)(e - r * cols);
                    step_r = 32 / cols;
                    step_c = 32 % cols;
                    placed = true;
                } else {
                    r += step_r;
                    c += step_c;
                    if (c >= cols) {
                        c -= cols;
                        ++r;
                    }
                }
                a[u] = row0 + r * stride + c;
            }
            uint32_t v[kGatherUnroll];
#pragma unroll
            for (int u = 0; u < kGatherUnroll; ++u) v[u] = a[u] ? __ldg(a[u]) : 0u;
#pragma unroll
            for (int u = 0; u < kGatherUnroll; ++u)
                if (a[u]) out[p0 + 32ull * u] = v[u];
        }
    }
}

}  // namespace
}  // namespace dev
}  // namespace wk
