// The static segment store built on the device from id triples: the same layout, byte for byte,
// as the host builder wk_gstore_build_ex (wk_gstore.cpp), which restates the reference's loader
// sort + dedup (base_loader.hpp:90-103, 481-496) and SegmentRDFGraph::init_gstore
// (segment_rdf_dgraph.hpp:1182-1269): one normal segment per (predicate, direction), the two
// index segments, optionally the vertex-predicate segments, keys placed by hash into the first
// free slot of their bucket in insertion order, chains through slot 7 into extension buckets
// appended in the order they are first needed.
//
// On the device every ordering the host builder gets from sequential insertion comes from a
// sort instead:
//   1. pack: each direction's (vid << 32 | value, predicate) items, filtered as the loader
//      filters them (no PREDICATE_ID triples; in the IN direction no type-id objects);
//   2. sort: LSD radix passes over the offsets of vid and value from their minima, then of the
//      predicate (8-bit digits, only the bits in which the items differ), then dedup;
//   3. the key runs (predicate, vid) of the sorted items give each segment's keys in insertion
//      order and its neighbour lists; the index lists are the key vids (and, for types, the
//      type triples re-sorted by type); the vertex-predicate lists are the key (vid, predicate)
//      pairs re-sorted by vid;
//   4. placement: the keys in insertion order are stably sorted by home bucket; a key's rank
//      in its bucket run is its slot (0-6), or its place in the bucket's chain of extension
//      buckets, whose numbers follow the order in which the host builder would append them
//      (an exclusive scan over the keys that open one, in insertion order).
// The small tables (segments, per-predicate counts) are worked out on the host between steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "wk_ctx.h"
#include "wk_device.cuh"

namespace wk {
namespace {
using namespace dev;

constexpr int kT = 256;       // threads per CTA of every build kernel
constexpr int kDigits = 256;  // 8-bit radix digits

__device__ __forceinline__ void span_of(uint64_t n, uint64_t* lo, uint64_t* hi) {
    const uint64_t c = (n + gridDim.x - 1) / gridDim.x;
    *lo = min(n, (uint64_t)blockIdx.x * c);
    *hi = min(n, *lo + c);
}

// ---------------------------------------------------------------- 1. pack
// Items of one direction; the order of the output is arbitrary (the sort fixes it).
__global__ void __launch_bounds__(kT) pack_kernel(const uint32_t* t, uint64_t n, int dir,
                                                  unsigned long long* key, uint32_t* pred,
                                                  unsigned long long* count) {
    const int lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * kT; base < n; base += (uint64_t)gridDim.x * kT) {
        const uint64_t i = base + threadIdx.x;
        bool keep = false;
        uint32_t s = 0, p = 0, o = 0;
        if (i < n) {
            s = __ldg(t + 3 * i);
            p = __ldg(t + 3 * i + 1);
            o = __ldg(t + 3 * i + 2);
            keep = p != kPredicateId && p < (1u << kNbitsIdx) && !(dir == kIn && is_tpid(o));
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        unsigned long long at = 0;
        if (lane == 0 && m) at = atomicAdd(count, (unsigned long long)__popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (keep) {
            const uint64_t j = at + __popc(m & ((1u << lane) - 1));
            key[j] = dir == kOut ? ((uint64_t)s << 32 | o) : ((uint64_t)o << 32 | s);
            pred[j] = p;
        }
    }
}

// Ranges of vid, value and predicate over the items: mm[0..5] = lo/hi of each.
__global__ void __launch_bounds__(kT) range_kernel(const unsigned long long* key, const uint32_t* pred,
                                                   uint64_t n, uint32_t* mm) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
    for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
        const uint64_t k = key[i];
        const uint32_t v[3] = {(uint32_t)(k >> 32), (uint32_t)k, pred[i]};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            lo[j] = min(lo[j], v[j]);
            hi[j] = max(hi[j], v[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[j] = min(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
            hi[j] = max(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&mm[2 * j], lo[j]);
            atomicMax(&mm[2 * j + 1], hi[j]);
        }
    }
}

// (vid << 32 | value) -> ((vid - vlo) << wbits | (value - wlo)); pred -> pred - plo (and back).
__global__ void __launch_bounds__(kT) shift_kernel(unsigned long long* key, uint32_t* pred, uint64_t n,
                                                   uint32_t vlo, uint32_t wlo, int wbits, uint32_t plo,
                                                   int back) {
    const uint64_t wmask = wbits >= 64 ? ~0ull : ((1ull << wbits) - 1);
    for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
        const uint64_t k = key[i];
        if (!back) {
            key[i] = ((uint64_t)((uint32_t)(k >> 32) - vlo) << wbits) | (uint64_t)((uint32_t)k - wlo);
            pred[i] -= plo;
        } else {
            key[i] = ((uint64_t)((uint32_t)(k >> wbits) + vlo) << 32) | (uint64_t)((uint32_t)(k & wmask) + wlo);
            pred[i] += plo;
        }
    }
}

// ---------------------------------------------------------------- 2. radix passes
// One stable 8-bit counting pass over (key, value) pairs; the digit comes from the key or from
// the value.  Every CTA owns a contiguous span.
struct Pass {
    const unsigned long long* k_in;
    const uint32_t* v_in;
    unsigned long long* k_out;
    uint32_t* v_out;
    uint64_t n;
    int shift;
    int from_value;
    uint32_t* hist;   // [kDigits][grid], digit-major
};

__device__ __forceinline__ uint32_t digit(const Pass& a, uint64_t i) {
    return a.from_value ? (a.v_in[i] >> a.shift) & 0xFFu : (uint32_t)(a.k_in[i] >> a.shift) & 0xFFu;
}

__global__ void __launch_bounds__(kT) hist_kernel(const Pass a) {
    __shared__ uint32_t s_h[kDigits];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    uint64_t lo, hi;
    span_of(a.n, &lo, &hi);
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kT) atomicAdd(&s_h[digit(a, i)], 1u);
    __syncthreads();
    a.hist[threadIdx.x * gridDim.x + blockIdx.x] = s_h[threadIdx.x];
}

// Exclusive scan of n words in place by one CTA of 1,024 threads.
__global__ void __launch_bounds__(1024) scan32_kernel(uint32_t* v, uint32_t n) {
    __shared__ uint64_t s_warp[32];
    __shared__ uint64_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t r0 = 0; r0 < n; r0 += 1024) {
        const uint32_t i = r0 + threadIdx.x;
        const uint64_t x = i < n ? v[i] : 0;
        const uint64_t ex = block_exclusive_sum<1024>(x, s_warp);
        const uint64_t carry = s_carry;
        if (i < n) v[i] = (uint32_t)(carry + ex);
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = carry + ex + x;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kT) scatter_kernel(const Pass a) {
    __shared__ uint32_t s_run[kDigits];
    __shared__ uint32_t s_cnt[kT / 32][kDigits];
    __shared__ uint32_t s_tile[kDigits];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_run[threadIdx.x] = a.hist[threadIdx.x * gridDim.x + blockIdx.x];
    uint64_t lo, hi;
    span_of(a.n, &lo, &hi);
    for (uint64_t base = lo; base < hi; base += kT) {
        for (int w = 0; w < kT / 32; ++w) s_cnt[w][threadIdx.x] = 0;
        __syncthreads();
        const uint64_t i = base + threadIdx.x;
        const bool live = i < hi;
        const uint32_t dg = live ? digit(a, i) : kDigits + lane;   // lone sentinel
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const int rank = __popc(peers & ((1u << lane) - 1));
        if (live && rank == 0) s_cnt[warp][dg] = __popc(peers);
        __syncthreads();
        {
            uint32_t acc = 0;
            for (int w = 0; w < kT / 32; ++w) {
                const uint32_t c = s_cnt[w][threadIdx.x];
                s_cnt[w][threadIdx.x] = acc;
                acc += c;
            }
            s_tile[threadIdx.x] = acc;
        }
        __syncthreads();
        if (live) {
            const uint32_t at = s_run[dg] + s_cnt[warp][dg] + rank;
            a.k_out[at] = a.k_in[i];
            a.v_out[at] = a.v_in[i];
        }
        __syncthreads();
        s_run[threadIdx.x] += s_tile[threadIdx.x];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- compaction
// Stable compaction of the items whose flag(i) holds: counts per CTA span, then (after a scan
// of those) placement.  `mode` picks the flag and what is written:
//   0: first of a run of equal (key, value) pairs (dedup): the pair;
//   1: first item of a (vid, value) key run: the item index;
//   2: an item of the type predicate whose value is a type id: the pair (key, vid);
//   3: first item of a value (predicate) run: the item index;
//   4: first item of a run of equal low key words (type runs): the item index.
struct Compact {
    const unsigned long long* k;
    const uint32_t* v;
    uint64_t n;
    int mode;
    uint32_t type_pred;           // mode 2: the TYPE_ID predicate
    uint32_t* part;               // [grid + 1]
    unsigned long long* k_out;
    uint32_t* v_out;
};

__device__ __forceinline__ bool cflag(const Compact& a, uint64_t i) {
    if (a.mode == 2) return a.v[i] == a.type_pred && is_tpid((uint32_t)a.k[i]);
    if (i == 0) return true;
    if (a.mode == 0) return a.k[i] != a.k[i - 1] || a.v[i] != a.v[i - 1];
    if (a.mode == 3) return a.v[i] != a.v[i - 1];
    if (a.mode == 4) return (uint32_t)a.k[i] != (uint32_t)a.k[i - 1];
    return a.v[i] != a.v[i - 1] || (a.k[i] >> 32) != (a.k[i - 1] >> 32);
}

__global__ void __launch_bounds__(kT) compact_count_kernel(const Compact a) {
    __shared__ uint64_t s_warp[kT / 32];
    uint64_t lo, hi;
    span_of(a.n, &lo, &hi);
    uint64_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kT) c += cflag(a, i);
    const uint64_t ex = block_exclusive_sum<kT>(c, s_warp);
    if (threadIdx.x == kT - 1) a.part[blockIdx.x] = (uint32_t)(ex + c);
}

__global__ void __launch_bounds__(kT) compact_place_kernel(const Compact a) {
    __shared__ uint64_t s_warp[kT / 32];
    __shared__ uint64_t s_carry;
    uint64_t lo, hi;
    span_of(a.n, &lo, &hi);
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint64_t base = lo; base < hi; base += kT) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t m = i < hi ? cflag(a, i) : 0;
        const uint64_t ex = block_exclusive_sum<kT>(m, s_warp);
        const uint64_t carry = s_carry;
        if (m) {
            const uint64_t at = carry + ex;
            if (a.mode == 0) {
                a.k_out[at] = a.k[i];
                a.v_out[at] = a.v[i];
            } else if (a.mode == 2) {
                a.k_out[at] = a.k[i];   // (vid << 32 | type): re-sorted by the type later
                a.v_out[at] = (uint32_t)(a.k[i] >> 32);
            } else {
                a.k_out[at] = i;
            }
        }
        __syncthreads();
        if (threadIdx.x == kT - 1) s_carry = carry + ex + m;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- 3. lists and keys
// A group: the items of one (direction, predicate) or one vertex-predicate segment, and where
// they go.  Items [item_lo, item_hi) of the sorted array; key runs [key_lo, key_hi); the group's
// first edge and first insertion slot; its segment's hash space.
struct Group {
    unsigned long long item_lo, item_hi, key_lo, key_hi;
    unsigned long long edge_base, ins_base;
    unsigned long long bucket_start, num_buckets, magic;
    uint32_t pid, dir;
};

// Key record in insertion order: the key, its pointer, its home bucket.
struct KeyRec {
    unsigned long long key, ptr, bucket;
};

__device__ __forceinline__ uint32_t group_of_key(const Group* g, uint32_t ng, uint64_t k) {
    uint32_t lo = 0, hi = ng;   // last group with key_lo <= k
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (g[mid].key_lo <= k) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t group_of_item(const Group* g, uint32_t ng, uint64_t i) {
    uint32_t lo = 0, hi = ng;   // last group with item_lo <= i
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (g[mid].item_lo <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Every item's value (the low word of its key) goes to its group's edge range, in item order.
__global__ void __launch_bounds__(kT) values_kernel(const unsigned long long* key, uint64_t n,
                                                    const Group* groups, uint32_t ng, uint32_t* edges) {
    for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
        const Group& g = groups[group_of_item(groups, ng, i)];
        edges[g.edge_base + (i - g.item_lo)] = (uint32_t)key[i];
    }
}

// One record per key run: [vid|pid|dir] (vid the high word of the run's items), its list's
// place in the edges, its home bucket; at the group's insertion base plus its rank in the group.
// kstart holds the item index of each key run's first item, and kstart[nkeys] = n.
__global__ void __launch_bounds__(kT) keys_kernel(const unsigned long long* key, const uint64_t* kstart,
                                                  uint64_t nkeys, const Group* groups, uint32_t ng,
                                                  KeyRec* recs) {
    for (uint64_t k = blockIdx.x * (uint64_t)kT + threadIdx.x; k < nkeys; k += (uint64_t)gridDim.x * kT) {
        const Group& g = groups[group_of_key(groups, ng, k)];
        const uint64_t i0 = kstart[k], i1 = kstart[k + 1];
        KeyRec r;
        r.key = make_key(key[i0] >> 32, g.pid, g.dir);
        r.ptr = make_ptr(i1 - i0, g.edge_base + (i0 - g.item_lo));
        r.bucket = g.bucket_start + mod_barrett(hash_u64(r.key), g.num_buckets, g.magic);
        recs[g.ins_base + (k - g.key_lo)] = r;
    }
}

// For each group start (an item index), the index of the key run it opens.
__global__ void key_of_item_kernel(const uint64_t* kstart, uint64_t nkeys, const uint64_t* items, uint64_t n,
                                   uint64_t* keys) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = nkeys;   // first key run starting at or after items[j]
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (kstart[mid] < items[j]) lo = mid + 1; else hi = mid;
        }
        keys[j] = lo;
    }
}

// Index-segment lists: out[k - k_lo] = vid of key run k, for key runs [k_lo, k_hi).
__global__ void __launch_bounds__(kT) key_vids_kernel(const unsigned long long* key, const uint64_t* kstart,
                                                      uint64_t k_lo, uint64_t k_hi, uint32_t* out) {
    for (uint64_t k = k_lo + blockIdx.x * (uint64_t)kT + threadIdx.x; k < k_hi; k += (uint64_t)gridDim.x * kT)
        out[k - k_lo] = (uint32_t)(key[kstart[k]] >> 32);
}

__global__ void __launch_bounds__(kT) copy32_kernel(const uint32_t* src, uint64_t n, uint32_t* dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) dst[i] = src[i];
}

// (vid << 32 | predicate) of every key run of a direction, with the vid as the sort value, for
// the vertex-predicate lists.
__global__ void __launch_bounds__(kT) vp_pairs_kernel(const unsigned long long* key, const uint32_t* pred,
                                                      const uint64_t* kstart, uint64_t nkeys,
                                                      unsigned long long* out_k, uint32_t* out_v) {
    for (uint64_t k = blockIdx.x * (uint64_t)kT + threadIdx.x; k < nkeys; k += (uint64_t)gridDim.x * kT) {
        const uint64_t i = kstart[k];
        out_k[k] = (key[i] >> 32) << 32 | pred[i];
        out_v[k] = (uint32_t)(key[i] >> 32);
    }
}

// Records of the index keys worked out on the host (few): their buckets.
__global__ void index_recs_kernel(KeyRec* recs, uint64_t n, unsigned long long bucket_start,
                                  unsigned long long num_buckets, unsigned long long magic) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        recs[i].bucket = bucket_start + mod_barrett(hash_u64(recs[i].key), num_buckets, magic);
}

// ---------------------------------------------------------------- 4. placement
__global__ void __launch_bounds__(kT) bucket_keys_kernel(const KeyRec* recs, uint64_t n,
                                                         unsigned long long* k, uint32_t* v) {
    for (uint64_t i = blockIdx.x * (uint64_t)kT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kT) {
        k[i] = recs[i].bucket;
        v[i] = (uint32_t)i;
    }
}

// Rank of sorted position j within its bucket's run (runs are short: walk back).
__device__ __forceinline__ uint32_t run_rank(const unsigned long long* b, uint64_t j) {
    uint32_t r = 0;
    while (r < j && b[j - r - 1] == b[j]) ++r;
    return r;
}

// Keys past the seventh of their bucket that open an extension bucket (ranks 7, 14, ...):
// flag[insertion index] = 1.
__global__ void __launch_bounds__(kT) creators_kernel(const unsigned long long* b, const uint32_t* ins,
                                                      uint64_t n, uint32_t* flag) {
    for (uint64_t j = blockIdx.x * (uint64_t)kT + threadIdx.x; j < n; j += (uint64_t)gridDim.x * kT) {
        const uint32_t r = run_rank(b, j);
        flag[ins[j]] = (r >= kAssoc - 1 && (r - (kAssoc - 1)) % (kAssoc - 1) == 0) ? 1u : 0u;
    }
}

// Exclusive scan of n words in place by CTA spans: span sums into part, a scan of part, then
// each span's scan from its offset.
__global__ void __launch_bounds__(kT) span_sum_kernel(const uint32_t* v, uint64_t n, uint32_t* part) {
    __shared__ uint64_t s_warp[kT / 32];
    uint64_t lo, hi;
    span_of(n, &lo, &hi);
    uint64_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kT) c += v[i];
    const uint64_t ex = block_exclusive_sum<kT>(c, s_warp);
    if (threadIdx.x == kT - 1) part[blockIdx.x] = (uint32_t)(ex + c);
}

__global__ void __launch_bounds__(kT) span_scan_kernel(uint32_t* v, uint64_t n, const uint32_t* part) {
    __shared__ uint64_t s_warp[kT / 32];
    __shared__ uint64_t s_carry;
    uint64_t lo, hi;
    span_of(n, &lo, &hi);
    if (threadIdx.x == 0) s_carry = part[blockIdx.x];
    __syncthreads();
    for (uint64_t base = lo; base < hi; base += kT) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t x = i < hi ? v[i] : 0;
        const uint64_t ex = block_exclusive_sum<kT>(x, s_warp);
        const uint64_t carry = s_carry;
        if (i < hi) v[i] = (uint32_t)(carry + ex);
        __syncthreads();
        if (threadIdx.x == kT - 1) s_carry = carry + ex + x;
        __syncthreads();
    }
}

// Every key's slot and every chain link.  ext_id[ins] is the exclusive scan of the creator flags
// (an extension bucket's number, less main_buckets).
__global__ void __launch_bounds__(kT) place_kernel(const unsigned long long* b, const uint32_t* ins,
                                                   uint64_t n, const KeyRec* recs, const uint32_t* ext_id,
                                                   uint64_t main_buckets, Slot* slots) {
    for (uint64_t j = blockIdx.x * (uint64_t)kT + threadIdx.x; j < n; j += (uint64_t)gridDim.x * kT) {
        const uint32_t r = run_rank(b, j);
        const KeyRec& rec = recs[ins[j]];
        uint64_t slot;
        if (r < kAssoc - 1) {
            slot = b[j] * kAssoc + r;
        } else {
            const uint32_t e = r - (kAssoc - 1);
            const uint64_t creator = j - r + (kAssoc - 1) + (uint64_t)(e / (kAssoc - 1)) * (kAssoc - 1);
            const uint64_t bucket = main_buckets + ext_id[ins[creator]];
            slot = bucket * kAssoc + e % (kAssoc - 1);
            if (e % (kAssoc - 1) == 0) {   // this key opened the bucket: link it from the previous
                const uint64_t prev = e == 0 ? b[j] : main_buckets + ext_id[ins[creator - (kAssoc - 1)]];
                slots[prev * kAssoc + kAssoc - 1].key = make_key(bucket, 0, 0);
            }
        }
        slots[slot].key = rec.key;
        slots[slot].ptr = rec.ptr;
    }
}

int grid_for(uint64_t n, int sm_count) {
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + kT - 1) / kT, (uint64_t)sm_count * 8));
}

}  // namespace

cudaError_t gbuild_kernel_attrs() {
    cudaError_t e = use_max_shared_carveout(pack_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(hist_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(scatter_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(scan32_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(compact_count_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(compact_place_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(values_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(keys_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(place_kernel);
    return e;
}

}  // namespace wk

// ---------------------------------------------------------------- host orchestration
namespace {

using wk::Group;
using wk::KeyRec;

#define WKG_CUDA(ctx, call)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call); \
    } while (0)

// Device buffers of one build, freed together at the end, or one by one (release) as soon as
// nothing reads them any more, so the build's peak stays within the device at a billion keys.
struct Bufs {
    std::vector<void*> ptrs;
    ~Bufs() {
        for (void* p : ptrs) cudaFree(p);
    }
    // Frees p (one of this set's buffers; cudaFree waits for the work that may still read it).
    void release(const void* p) {
        if (!p) return;
        for (size_t i = 0; i < ptrs.size(); ++i)
            if (ptrs[i] == p) {
                cudaFree(ptrs[i]);
                ptrs.erase(ptrs.begin() + i);
                return;
            }
    }
    template <class T>
    bool get(T** p, uint64_t n) {
        void* q = nullptr;
        if (wk::dev_malloc(&q, std::max<uint64_t>(n, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        ptrs.push_back(q);
        *p = static_cast<T*>(q);
        return true;
    }
};

struct Builder {
    wk_ctx* ctx;
    cudaStream_t s;
    Bufs& B;
    int sm;

    int sync() {
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        return e == cudaSuccess ? WK_SUCCESS : ctx->cuda_fail(e, "store build");
    }
    int grid_for(uint64_t n) const { return wk::grid_for(n, sm); }

    // Stable LSD sort of (k, v) pairs: key bits [0, kbits), then value bits [0, vbits) (the
    // value digits are the more significant).  Ping-pongs with (k2, v2); *where says which pair
    // holds the result (0: k/v, 1: k2/v2).
    int sort(unsigned long long* k, uint32_t* v, unsigned long long* k2, uint32_t* v2, uint64_t n, int kbits,
             int vbits, uint32_t* hist, int* where) {
        *where = 0;
        if (n < 2) return WK_SUCCESS;
        const int grid = grid_for(n);
        unsigned long long *ka = k, *kb = k2;
        uint32_t *va = v, *vb = v2;
        auto pass = [&](int shift, int from_value) {
            wk::Pass p{ka, va, kb, vb, n, shift, from_value, hist};
            wk::hist_kernel<<<grid, wk::kT, 0, s>>>(p);
            wk::scan32_kernel<<<1, 1024, 0, s>>>(hist, (uint32_t)(wk::kDigits * grid));
            wk::scatter_kernel<<<grid, wk::kT, 0, s>>>(p);
            std::swap(ka, kb);
            std::swap(va, vb);
            *where ^= 1;
        };
        for (int sh = 0; sh < kbits; sh += 8) pass(sh, 0);
        for (int sh = 0; sh < vbits; sh += 8) pass(sh, 1);
        return sync();
    }

    // Stable compaction (see wk::Compact); *count receives the number kept.
    int compact(wk::Compact c, uint32_t* part, uint64_t* count) {
        *count = 0;
        if (c.n == 0) return WK_SUCCESS;
        const int grid = grid_for(c.n);
        c.part = part;
        wk::compact_count_kernel<<<grid, wk::kT, 0, s>>>(c);
        cudaError_t e = cudaMemsetAsync(part + grid, 0, 4, s);   // part[grid] = total after the scan
        if (e != cudaSuccess) return ctx->cuda_fail(e, "store build");
        wk::scan32_kernel<<<1, 1024, 0, s>>>(part, (uint32_t)grid + 1);
        wk::compact_place_kernel<<<grid, wk::kT, 0, s>>>(c);
        uint32_t tot = 0;
        e = cudaMemcpyAsync(&tot, part + grid, 4, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "store build");
        int rc = sync();
        *count = tot;
        return rc;
    }
};

// One direction's sorted, deduplicated items, and their key runs.
struct DirItems {
    unsigned long long* key = nullptr;   // (vid << 32 | value), sorted by (pred, vid, value)
    uint32_t* pred = nullptr;
    uint64_t n = 0;
    uint64_t* kstart = nullptr;          // item index of each key run's first item, then n
    uint64_t nkeys = 0;
    std::vector<uint32_t> preds;         // per predicate present, ascending:
    std::vector<uint64_t> item_lo, key_lo;   // its first item and first key run
};

int bits_of(uint64_t span) { return span ? 64 - __builtin_clzll(span) : 0; }

uint64_t buckets_for(uint64_t keys, double load) {   // as the host builder sizes a segment
    if (keys == 0) return 1;
    const double nb = std::ceil((double)keys / ((wk::kAssoc - 1) * load));
    return std::max<uint64_t>(1, (uint64_t)nb);
}

// The starts of the runs a compaction mode marks (3: predicate groups, 4: type runs), read back
// to the host, and with kstart the key run each one opens.
int group_starts(Builder& bd, unsigned long long* key, uint32_t* pred, uint64_t n, int mode,
                 const uint64_t* kstart, uint64_t nkeys, uint32_t* part, std::vector<uint64_t>& item_lo,
                 std::vector<uint64_t>& key_lo) {
    item_lo.clear();
    key_lo.clear();
    if (n == 0) return WK_SUCCESS;
    uint64_t g = 0;
    uint64_t* pos = nullptr;
    // the starts are few, but their count is only known after the compaction: room for all
    if (!bd.B.get(&pos, n + 1)) return bd.ctx->fail(WK_E_OOM, "store build groups");
    wk::Compact c{key, pred, n, mode, 0, nullptr, reinterpret_cast<unsigned long long*>(pos), nullptr};
    int rc = bd.compact(c, part, &g);
    if (rc) return rc;
    item_lo.resize(g);
    cudaError_t e = cudaMemcpyAsync(item_lo.data(), pos, g * 8, cudaMemcpyDeviceToHost, bd.s);
    uint64_t* kk = nullptr;
    if (e == cudaSuccess && kstart) {
        if (!bd.B.get(&kk, g)) return bd.ctx->fail(WK_E_OOM, "store build groups");
        wk::key_of_item_kernel<<<(int)std::min<uint64_t>((g + 255) / 256, 1024), 256, 0, bd.s>>>(kstart, nkeys, pos,
                                                                                             g, kk);
        key_lo.resize(g);
        e = cudaMemcpyAsync(key_lo.data(), kk, g * 8, cudaMemcpyDeviceToHost, bd.s);
    }
    if (e != cudaSuccess) return bd.ctx->cuda_fail(e, "store build groups");
    rc = bd.sync();
    bd.B.release(pos);   // room for every item, of which a few were used
    bd.B.release(kk);
    return rc;
}

// The first n words of `p` (a buffer of this build) moved to a buffer of exactly n words; p is
// freed.  For the arrays whose length is only known once a compaction has filled them.
template <class T>
int shrink_to(Builder& bd, T** p, uint64_t n, const char* what) {
    T* q = nullptr;
    if (!bd.B.get(&q, n)) return bd.ctx->fail(WK_E_OOM, what);
    cudaError_t e = cudaMemcpyAsync(q, *p, std::max<uint64_t>(n, 1) * sizeof(T), cudaMemcpyDeviceToDevice, bd.s);
    if (e != cudaSuccess) return bd.ctx->cuda_fail(e, what);
    const int rc = bd.sync();
    bd.B.release(*p);
    *p = q;
    return rc;
}

struct SegPlan {
    wk_seg_meta m;
    uint64_t ins_base;
};

// An index list: the key [0|pid|dir] and where its values come from (a range of key runs of a
// direction, or a range of the type-sorted instances).
struct IdxEntry {
    uint32_t pid;
    uint64_t count;
    int from_types;
    const unsigned long long* key;
    const uint64_t* kstart;
    uint64_t lo;
};

// Steps 3 and 4 once each direction's items are sorted: vertex-predicate lists, type instances,
// the segment table, lists and key records, placement.
// spare_k / spare_v: the sort's free pair of buffers (room for every item), reused by the type
// index.  Every buffer of the sorted items is freed once the lists and key records are made.
int gbuild_segments(wk_ctx* ctx, Builder& bd, DirItems* D, unsigned long long* spare_k, uint32_t* spare_v,
                    double load, bool versatile, uint32_t* hist, uint32_t* part, wk::Slot** out_slots,
                    uint64_t* out_n_slots, uint32_t** out_edges, uint64_t* out_n_edges,
                    std::vector<wk_seg_meta>& segs) {
    using namespace wk;
    Bufs& B = bd.B;
    cudaStream_t s = bd.s;
    int rc;

    std::vector<const void*> dead;   // freed once the lists and key records are made
    for (int di = 0; di < 2; ++di)
        for (const void* q : {(const void*)D[di].key, (const void*)D[di].pred, (const void*)D[di].kstart})
            dead.push_back(q);

    // ---- vertex-predicate lists: each direction's key runs as (vid << 32 | predicate) pairs,
    // stably re-sorted by vid (each vertex's predicates stay ascending), then runs by vertex
    DirItems VP[2];
    if (versatile) {
        for (int di = 0; di < 2; ++di) {
            DirItems& V = VP[di];
            const uint64_t nk = D[di].nkeys;
            unsigned long long *k = nullptr, *kk = nullptr;
            uint32_t *v = nullptr, *vv = nullptr;
            if (!B.get(&k, nk) || !B.get(&v, nk) || !B.get(&kk, nk) || !B.get(&vv, nk) || !B.get(&V.kstart, nk + 1))
                return ctx->fail(WK_E_OOM, "store build vertex predicates");
            for (const void* q : {(const void*)k, (const void*)v, (const void*)kk, (const void*)vv,
                                  (const void*)V.kstart})
                dead.push_back(q);
            if (nk)
                vp_pairs_kernel<<<bd.grid_for(nk), kT, 0, s>>>(D[di].key, D[di].pred, D[di].kstart, nk, k, v);
            int where = 0;
            if ((rc = bd.sort(k, v, kk, vv, nk, 0, 32, hist, &where))) return rc;
            V.key = where ? kk : k;
            V.pred = where ? vv : v;
            V.n = nk;
            uint64_t nv = 0;
            Compact kc{V.key, V.pred, nk, 1, 0, nullptr, reinterpret_cast<unsigned long long*>(V.kstart), nullptr};
            if ((rc = bd.compact(kc, part, &nv))) return rc;
            V.nkeys = nv;
            WKG_CUDA(ctx, cudaMemcpyAsync(V.kstart + nv, &V.n, 8, cudaMemcpyHostToDevice, s));
            if ((rc = bd.sync())) return rc;
            V.item_lo.assign(1, 0);
            V.key_lo.assign(1, 0);
        }
    }

    // ---- type instances: the (TYPE_ID, type-id object) items of the OUT direction, stably
    // re-sorted by type (each type's subjects stay ascending), and the runs by type
    unsigned long long* tk = nullptr;
    uint32_t* tv = nullptr;
    uint64_t ntype = 0;
    std::vector<uint64_t> trun;
    std::vector<uint32_t> tids;
    {
        // the spare pair has room for every item; the ping-pong pair is sized once the type
        // items are counted
        unsigned long long *k = spare_k, *kk = nullptr;
        uint32_t *v = spare_v, *vv = nullptr;
        const uint64_t n0 = D[0].n;
        Compact c{D[0].key, D[0].pred, n0, 2, (uint32_t)kTypeId, nullptr, k, v};
        if ((rc = bd.compact(c, part, &ntype))) return rc;
        if (!B.get(&kk, ntype) || !B.get(&vv, ntype)) return ctx->fail(WK_E_OOM, "store build type index");
        for (const void* q : {(const void*)k, (const void*)v, (const void*)kk, (const void*)vv}) dead.push_back(q);
        int where = 0;
        if ((rc = bd.sort(k, v, kk, vv, ntype, kNbitsIdx, 0, hist, &where))) return rc;
        tk = where ? kk : k;
        tv = where ? vv : v;
        std::vector<uint64_t> unused;
        if ((rc = group_starts(bd, tk, tv, ntype, 4, nullptr, 0, part, trun, unused))) return rc;
        tids.resize(trun.size());
        for (size_t i = 0; i < trun.size(); ++i)
            WKG_CUDA(ctx, cudaMemcpyAsync(&tids[i], reinterpret_cast<const uint32_t*>(tk + trun[i]), 4,
                                          cudaMemcpyDeviceToHost, s));
        if ((rc = bd.sync())) return rc;
    }

    // ---- the segment table, in the host builder's order
    auto group_counts = [](const DirItems& d, size_t gi, uint64_t* items, uint64_t* keys) {
        const uint64_t ihi = gi + 1 < d.item_lo.size() ? d.item_lo[gi + 1] : d.n;
        const uint64_t khi = gi + 1 < d.key_lo.size() ? d.key_lo[gi + 1] : d.nkeys;
        *items = ihi - d.item_lo[gi];
        *keys = khi - d.key_lo[gi];
    };
    auto find = [](const DirItems& d, uint32_t p) -> int {
        auto it = std::lower_bound(d.preds.begin(), d.preds.end(), p);
        return (it != d.preds.end() && *it == p) ? (int)(it - d.preds.begin()) : -1;
    };
    std::vector<uint32_t> preds(D[0].preds);
    preds.insert(preds.end(), D[1].preds.begin(), D[1].preds.end());
    std::sort(preds.begin(), preds.end());
    preds.erase(std::unique(preds.begin(), preds.end()), preds.end());

    std::vector<SegPlan> plan;
    uint64_t bucket_off = 0, edge_off = 0, ins_off = 0;
    auto add_seg = [&](int index, uint32_t pid, int dir, uint64_t keys, uint64_t edges) {
        SegPlan sp{};
        sp.m.index = index;
        sp.m.pid = pid;
        sp.m.dir = dir;
        sp.m.num_keys = keys;
        sp.m.num_buckets = buckets_for(keys, load);
        sp.m.bucket_start = bucket_off;
        sp.m.num_edges = edges;
        sp.m.edge_start = edge_off;
        sp.ins_base = ins_off;
        bucket_off += sp.m.num_buckets;
        edge_off += edges;
        ins_off += keys;
        plan.push_back(sp);
        return plan.size() - 1;
    };
    size_t vp_seg[2] = {0, 0};
    if (versatile) {
        vp_seg[0] = add_seg(0, kPredicateId, kOut, VP[0].nkeys, VP[0].n);
        vp_seg[1] = add_seg(0, kPredicateId, kIn, VP[1].nkeys, VP[1].n);
    }
    std::vector<size_t> seg_out(preds.size()), seg_in(preds.size());
    std::vector<IdxEntry> idx_in, idx_out;
    for (size_t i = 0; i < preds.size(); ++i) {
        const uint32_t p = preds[i];
        uint64_t io = 0, ko = 0, ii = 0, ki = 0;
        const int go = find(D[0], p), gi = find(D[1], p);
        if (go >= 0) group_counts(D[0], go, &io, &ko);
        if (gi >= 0) group_counts(D[1], gi, &ii, &ki);
        seg_out[i] = add_seg(0, p, kOut, ko, io);
        seg_in[i] = add_seg(0, p, kIn, ki, ii);
        if (p == kTypeId) continue;   // rdf:type has no predicate index
        if (ko) idx_in.push_back(IdxEntry{p, ko, 0, D[0].key, D[0].kstart, D[0].key_lo[go]});
        if (ki) idx_out.push_back(IdxEntry{p, ki, 0, D[1].key, D[1].kstart, D[1].key_lo[gi]});
    }
    for (size_t r = 0; r < trun.size(); ++r) {
        const uint64_t hi = r + 1 < trun.size() ? trun[r + 1] : ntype;
        idx_in.push_back(IdxEntry{tids[r], hi - trun[r], 1, nullptr, nullptr, trun[r]});
    }
    uint64_t eo = 0, ei = 0;
    for (auto& e : idx_out) eo += e.count;
    for (auto& e : idx_in) ei += e.count;
    const size_t idx_seg_out = add_seg(1, kPredicateId, kOut, idx_out.size(), eo);
    const size_t idx_seg_in = add_seg(1, kPredicateId, kIn, idx_in.size(), ei);
    const uint64_t main_buckets = bucket_off, n_edges = edge_off, n_keys = ins_off;

    // ---- edges and key records
    uint32_t* d_edges = nullptr;
    if (wk::dev_malloc(&d_edges, (n_edges + 16) * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return ctx->fail(WK_E_OOM, "store edges");
    }
    *out_edges = d_edges;   // the caller's from here on, built or not
    *out_n_edges = n_edges;
    WKG_CUDA(ctx, cudaMemsetAsync(d_edges, 0, (n_edges + 16) * sizeof(uint32_t), s));
    KeyRec* recs = nullptr;
    if (!B.get(&recs, n_keys)) return ctx->fail(WK_E_OOM, "store build key records");
    auto run_set = [&](const DirItems& d, const std::vector<Group>& groups) -> int {
        if (groups.empty() || d.n == 0) return WK_SUCCESS;
        Group* dg = nullptr;
        if (!B.get(&dg, groups.size())) return ctx->fail(WK_E_OOM, "store build groups");
        cudaError_t e = cudaMemcpyAsync(dg, groups.data(), groups.size() * sizeof(Group), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return ctx->cuda_fail(e, "store build groups");
        values_kernel<<<bd.grid_for(d.n), kT, 0, s>>>(d.key, d.n, dg, (uint32_t)groups.size(), d_edges);
        if (d.nkeys)
            keys_kernel<<<bd.grid_for(d.nkeys), kT, 0, s>>>(d.key, d.kstart, d.nkeys, dg, (uint32_t)groups.size(), recs);
        return bd.sync();   // the host group table lives until the copy is done
    };
    auto group_for = [&](const DirItems& d, size_t gi, const SegPlan& sp) {
        Group g{};
        g.item_lo = d.item_lo[gi];
        g.item_hi = gi + 1 < d.item_lo.size() ? d.item_lo[gi + 1] : d.n;
        g.key_lo = d.key_lo[gi];
        g.key_hi = gi + 1 < d.key_lo.size() ? d.key_lo[gi + 1] : d.nkeys;
        g.edge_base = sp.m.edge_start;
        g.ins_base = sp.ins_base;
        g.bucket_start = sp.m.bucket_start;
        g.num_buckets = sp.m.num_buckets;
        g.magic = barrett_magic(sp.m.num_buckets);
        g.pid = sp.m.pid;
        g.dir = (uint32_t)sp.m.dir;
        return g;
    };
    for (int di = 0; di < 2; ++di) {
        std::vector<Group> groups;
        for (size_t gi = 0; gi < D[di].preds.size(); ++gi) {
            const size_t pi = std::lower_bound(preds.begin(), preds.end(), D[di].preds[gi]) - preds.begin();
            groups.push_back(group_for(D[di], gi, plan[di == 0 ? seg_out[pi] : seg_in[pi]]));
        }
        if ((rc = run_set(D[di], groups))) return rc;
    }
    if (versatile)
        for (int di = 0; di < 2; ++di)
            if (VP[di].n) {
                std::vector<Group> groups{group_for(VP[di], 0, plan[vp_seg[di]])};
                if ((rc = run_set(VP[di], groups))) return rc;
            }
    // index segments: lists from key vids or type instances; their few records made here
    for (int which = 0; which < 2; ++which) {
        const std::vector<IdxEntry>& L = which == 0 ? idx_out : idx_in;
        const SegPlan& sp = plan[which == 0 ? idx_seg_out : idx_seg_in];
        std::vector<KeyRec> hr;
        uint64_t off = sp.m.edge_start;
        for (const IdxEntry& e : L) {
            uint32_t* dst = d_edges + off;
            if (e.from_types)
                copy32_kernel<<<bd.grid_for(e.count), kT, 0, s>>>(tv + e.lo, e.count, dst);
            else
                key_vids_kernel<<<bd.grid_for(e.count), kT, 0, s>>>(e.key, e.kstart, e.lo, e.lo + e.count, dst);
            KeyRec r{};
            r.key = make_key(0, e.pid, sp.m.dir);
            r.ptr = make_ptr(e.count, off);
            hr.push_back(r);
            off += e.count;
        }
        if (!hr.empty()) {
            WKG_CUDA(ctx, cudaMemcpyAsync(recs + sp.ins_base, hr.data(), hr.size() * sizeof(KeyRec),
                                          cudaMemcpyHostToDevice, s));
            index_recs_kernel<<<1, 256, 0, s>>>(recs + sp.ins_base, hr.size(), sp.m.bucket_start, sp.m.num_buckets,
                                                barrett_magic(sp.m.num_buckets));
        }
        if ((rc = bd.sync())) return rc;   // hr lives until the copy is done
    }

    // the items, key runs and type instances are all in the edges and key records now
    for (const void* q : dead) B.release(q);

    // ---- placement
    unsigned long long *bk = nullptr, *bk2 = nullptr;
    uint32_t *ins = nullptr, *ins2 = nullptr, *ext = nullptr;
    if (!B.get(&bk, n_keys) || !B.get(&bk2, n_keys) || !B.get(&ins, n_keys) || !B.get(&ins2, n_keys) ||
        !B.get(&ext, n_keys + 1))
        return ctx->fail(WK_E_OOM, "store build placement");
    if (n_keys) bucket_keys_kernel<<<bd.grid_for(n_keys), kT, 0, s>>>(recs, n_keys, bk, ins);
    int where = 0;
    if ((rc = bd.sort(bk, ins, bk2, ins2, n_keys, bits_of(main_buckets ? main_buckets - 1 : 0), 0, hist, &where)))
        return rc;
    const unsigned long long* sb = where ? bk2 : bk;
    const uint32_t* si = where ? ins2 : ins;
    uint64_t n_ext = 0;
    if (n_keys) {
        const int grid = bd.grid_for(n_keys);
        creators_kernel<<<grid, kT, 0, s>>>(sb, si, n_keys, ext);
        span_sum_kernel<<<grid, kT, 0, s>>>(ext, n_keys, part);
        WKG_CUDA(ctx, cudaMemsetAsync(part + grid, 0, 4, s));
        scan32_kernel<<<1, 1024, 0, s>>>(part, (uint32_t)grid + 1);
        span_scan_kernel<<<grid, kT, 0, s>>>(ext, n_keys, part);
        uint32_t tot = 0;
        WKG_CUDA(ctx, cudaMemcpyAsync(&tot, part + grid, 4, cudaMemcpyDeviceToHost, s));
        if ((rc = bd.sync())) return rc;
        n_ext = tot;
    }
    // extension buckets per segment: the scan at each segment's first key
    std::vector<uint32_t> ext_at(plan.size() + 1, (uint32_t)n_ext);
    for (size_t i = 0; i < plan.size(); ++i)
        if (plan[i].ins_base < n_keys)
            WKG_CUDA(ctx, cudaMemcpyAsync(&ext_at[i], ext + plan[i].ins_base, 4, cudaMemcpyDeviceToHost, s));
    if ((rc = bd.sync())) return rc;

    const uint64_t n_slots = (main_buckets + n_ext) * kAssoc;
    Slot* d_slots = nullptr;
    if (wk::dev_malloc(&d_slots, std::max<uint64_t>(n_slots, kAssoc) * sizeof(Slot)) != cudaSuccess) {
        cudaGetLastError();
        return ctx->fail(WK_E_OOM, "store slots");
    }
    *out_slots = d_slots;
    *out_n_slots = n_slots;
    WKG_CUDA(ctx, cudaMemsetAsync(d_slots, 0, std::max<uint64_t>(n_slots, kAssoc) * sizeof(Slot), s));
    if (n_keys)
        place_kernel<<<bd.grid_for(n_keys), kT, 0, s>>>(sb, si, n_keys, recs, ext, main_buckets, d_slots);
    if ((rc = bd.sync())) return rc;

    segs.clear();
    uint64_t ext_off = main_buckets;
    for (size_t i = 0; i < plan.size(); ++i) {
        wk_seg_meta m = plan[i].m;
        // a segment without keys has its insertion base at the next segment's first key
        m.ext_num = ext_at[i + 1] - ext_at[i];
        m.ext_start = m.ext_num ? ext_off : 0;
        ext_off += m.ext_num;
        segs.push_back(m);
    }
    return WK_SUCCESS;
}

// The build: `d_tr` holds n (s, p, o) triples on the device.
int gbuild(wk_ctx* ctx, const uint32_t* d_tr, uint64_t n, double load, bool versatile, Bufs& B,
           wk::Slot** out_slots, uint64_t* out_n_slots, uint32_t** out_edges, uint64_t* out_n_edges,
           std::vector<wk_seg_meta>& segs) {
    using namespace wk;
    if (load <= 0) load = 0.1;
    if (load > 1) return ctx->fail(WK_E_BADARG, "load factor above 1");
    if (n >= (1ull << 32)) return ctx->fail(WK_E_CAPACITY, "at most 2^32 - 1 triples per device build");
    Builder bd{ctx, ctx->stream, B, ctx->sm_count};
    cudaStream_t s = ctx->stream;
    const int gmax = ctx->sm_count * 8;
    uint32_t* hist = nullptr;
    uint32_t* part = nullptr;
    unsigned long long* d_count = nullptr;
    uint32_t* d_mm = nullptr;
    if (!B.get(&hist, (uint64_t)kDigits * gmax) || !B.get(&part, gmax + 2) || !B.get(&d_count, 1) ||
        !B.get(&d_mm, 8))
        return ctx->fail(WK_E_OOM, "store build scratch");

    // ---- 1-2: items of each direction, sorted and deduplicated.  Both directions are packed
    // first, so the triples are freed before the sort's second pair of buffers is needed.
    DirItems D[2];   // [0] OUT, [1] IN
    unsigned long long* pk[2] = {nullptr, nullptr};
    uint32_t* pv[2] = {nullptr, nullptr};
    unsigned long long pcnt[2] = {0, 0};
    int rc;
    for (int di = 0; di < 2; ++di) {
        if (!B.get(&pk[di], n) || !B.get(&pv[di], n)) return ctx->fail(WK_E_OOM, "store build items");
        WKG_CUDA(ctx, cudaMemsetAsync(d_count, 0, 8, s));
        if (n) pack_kernel<<<bd.grid_for(n), kT, 0, s>>>(d_tr, n, di == 0 ? kOut : kIn, pk[di], pv[di], d_count);
        WKG_CUDA(ctx, cudaMemcpyAsync(&pcnt[di], d_count, 8, cudaMemcpyDeviceToHost, s));
        if ((rc = bd.sync())) return rc;
    }
    B.release(d_tr);
    unsigned long long* k2 = nullptr;
    uint32_t* v2 = nullptr;
    if (!B.get(&k2, n) || !B.get(&v2, n)) return ctx->fail(WK_E_OOM, "store build sort buffers");
    for (int di = 0; di < 2; ++di) {
        DirItems& Dd = D[di];
        unsigned long long* k = pk[di];
        uint32_t* v = pv[di];
        const unsigned long long cnt = pcnt[di];
        uint32_t mm[6] = {0xFFFFFFFFu, 0, 0xFFFFFFFFu, 0, 0xFFFFFFFFu, 0};
        if (cnt) {
            WKG_CUDA(ctx, cudaMemcpyAsync(d_mm, mm, sizeof(mm), cudaMemcpyHostToDevice, s));
            range_kernel<<<bd.grid_for(cnt), kT, 0, s>>>(k, v, cnt, d_mm);
            WKG_CUDA(ctx, cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, s));
            if ((rc = bd.sync())) return rc;
        }
        const int vbits = bits_of(mm[1] - mm[0]), wbits = bits_of(mm[3] - mm[2]), pbits = bits_of(mm[5] - mm[4]);
        if (cnt) shift_kernel<<<bd.grid_for(cnt), kT, 0, s>>>(k, v, cnt, mm[0], mm[2], wbits, mm[4], 0);
        int where = 0;
        if ((rc = bd.sort(k, v, k2, v2, cnt, vbits + wbits, pbits, hist, &where))) return rc;
        unsigned long long* ks = where ? k2 : k;
        uint32_t* vs = where ? v2 : v;
        if (cnt) shift_kernel<<<bd.grid_for(cnt), kT, 0, s>>>(ks, vs, cnt, mm[0], mm[2], wbits, mm[4], 1);
        // dedup into the other pair; the next direction sorts with the pair left free
        unsigned long long* kd = where ? k : k2;
        uint32_t* vd = where ? v : v2;
        uint64_t nd = 0;
        Compact c{ks, vs, cnt, 0, 0, nullptr, kd, vd};
        if ((rc = bd.compact(c, part, &nd))) return rc;
        Dd.key = kd;
        Dd.pred = vd;
        Dd.n = nd;
        if (kd == k2) {
            k2 = k;
            v2 = v;
        }
        // key runs
        if (!B.get(&Dd.kstart, nd + 1)) return ctx->fail(WK_E_OOM, "store build keys");
        uint64_t nk = 0;
        Compact kc{Dd.key, Dd.pred, nd, 1, 0, nullptr, reinterpret_cast<unsigned long long*>(Dd.kstart), nullptr};
        if ((rc = bd.compact(kc, part, &nk))) return rc;
        Dd.nkeys = nk;
        if ((rc = shrink_to(bd, &Dd.kstart, nk + 1, "store build keys"))) return rc;
        WKG_CUDA(ctx, cudaMemcpyAsync(Dd.kstart + nk, &Dd.n, 8, cudaMemcpyHostToDevice, s));
        // groups: where the predicate changes (few), and the key run each one opens
        if ((rc = group_starts(bd, Dd.key, Dd.pred, Dd.n, 3, Dd.kstart, Dd.nkeys, part, Dd.item_lo, Dd.key_lo)))
            return rc;
        Dd.preds.resize(Dd.item_lo.size());
        for (size_t gi = 0; gi < Dd.item_lo.size(); ++gi)
            WKG_CUDA(ctx, cudaMemcpyAsync(&Dd.preds[gi], Dd.pred + Dd.item_lo[gi], 4, cudaMemcpyDeviceToHost, s));
        if ((rc = bd.sync())) return rc;
    }
    return gbuild_segments(ctx, bd, D, k2, v2, load, versatile, hist, part, out_slots, out_n_slots, out_edges,
                           out_n_edges, segs);
}

}  // namespace

// Device build from host triples: the store replaces the context's store.
extern "C" int wk_store_build_device(wk_ctx* ctx, const uint32_t* triples, uint64_t n_triples, double load_factor,
                                     int32_t versatile) {
    if (!ctx || (!triples && n_triples)) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->borrowed_store) return ctx->fail(WK_E_BADARG, "a serving lane's store belongs to its parent");
    if (load_factor < 0 || load_factor > 1) return ctx->fail(WK_E_BADARG, "load factor outside (0, 1]");
    WKG_CUDA(ctx, cudaSetDevice(ctx->device));
    WKG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // the old store goes first: a build needs the room
    if (ctx->d_slots) cudaFree(ctx->d_slots);
    if (ctx->d_edges) cudaFree(ctx->d_edges);
    ctx->d_slots = nullptr;
    ctx->d_edges = nullptr;
    ctx->n_slots = ctx->n_edges = 0;
    ctx->has_store = false;
    ctx->drop_graphs();
    wk::Slot* slots = nullptr;
    uint32_t* edges = nullptr;
    uint64_t n_slots = 0, n_edges = 0;
    std::vector<wk_seg_meta> segs;
    int rc;
    {
        Bufs B;   // the build's scratch, freed before the store is adopted
        uint32_t* d_tr = nullptr;
        if (!B.get(&d_tr, std::max<uint64_t>(n_triples, 1) * 3)) return ctx->fail(WK_E_OOM, "store build triples");
        if (n_triples)
            WKG_CUDA(ctx, cudaMemcpyAsync(d_tr, triples, n_triples * 12, cudaMemcpyHostToDevice, ctx->stream));
        rc = gbuild(ctx, d_tr, n_triples, load_factor, versatile != 0, B, &slots, &n_slots, &edges, &n_edges, segs);
        cudaStreamSynchronize(ctx->stream);
    }
    if (rc) {
        if (slots) cudaFree(slots);
        if (edges) cudaFree(edges);
        return rc;
    }
    return wk::store_adopt(ctx, slots, n_slots, edges, n_edges, segs);
}
