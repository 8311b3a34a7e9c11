// Flat pipeline for large single-query steps: count -> scan -> scatter.
//
// The tile launch (wk_explore.cu) keeps a whole step in one persistent launch, which suits the
// many small tables of a batch but pays per-tile barriers and look-back waits, and runs at
// the occupancy its shared memory allows.  For one large table (index-start queries: 1e5 to
// 1e8 rows) the same step runs here as three short launches at full occupancy, each a
// streaming pass except for the probes themselves:
//   1. count: one thread per input row probes the key table (two 16-byte slots per load, the
//      chain followed through slot 7), records the row's output count (list size for
//      known_to_unknown, 0/1 membership for known_to_known / known_to_const) and its list offset;
//      each CTA owns a contiguous chunk of rows and publishes the chunk total;
//   2. scan: the last count CTA to finish scans the chunk totals, checks the output capacity
//      (overflow sets kErrOverflow and the rows needed, as the tile launch does) and sets the
//      row count;
//   3. place: each CTA scans its chunk into per-row output positions; filters copy their
//      surviving rows straight to the output here (a chunk without survivors returns at once);
//   4. expand (known_to_unknown only): the output rows are split evenly over the CTAs; each CTA
//      finds its first input row by a 32-way search of the positions and writes its rows in
//      row-major then edge order (sparql.hpp:328-370), consecutive threads on consecutive rows.
// When every input row of a known_to_unknown step has exactly one output row (a functional
// predicate such as memberOf), output row r is input row r: the count pass writes it as it
// goes (every row with one output row does, speculatively), and place and expand return at once.
// Row counts are read on the device, so the launches chain without a host round trip and can
// be captured in a graph.  Every launch returns at once unless the input has at least
// `min_rows` rows; the tile launch of the same step is given the complementary bound, so
// exactly one of the two writes the output.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/wukong_b200.h"
#include "wk_device.cuh"
#include "wk_flat.h"

namespace wk {
namespace {
using namespace dev;

constexpr int kFlatThreads = 256;
constexpr int kWindow = 256;   // input rows staged per expand round
// part[] flag bit set by a count CTA whose rows do not each have exactly one output row; the
// scan clears it from the totals and leaves part[nparts + 1] = 1 when every row has one
// (known_to_unknown on a functional predicate: output row r is then input row r, and the
// place pass and the expand search are skipped).  part has 256 spare bytes past nparts.
constexpr uint64_t kNotOneToOne = 1ull << 63;

__device__ __forceinline__ uint64_t flat_rows(const FlatArgs& a) {
    uint64_t R = *(volatile const uint64_t*)a.in_rows;
    return R > a.in_cap_rows ? 0 : R;   // past capacity: the step before overflowed
}

__device__ __forceinline__ void chunk_of(uint64_t R, uint64_t* lo, uint64_t* hi) {
    const uint64_t chunk = (R + gridDim.x - 1) / gridDim.x;
    *lo = min(R, (uint64_t)blockIdx.x * chunk);
    *hi = min(R, *lo + chunk);
}

__device__ __forceinline__ uint64_t block_sum(uint64_t x, uint64_t* s_warp) {
    const uint64_t ex = block_exclusive_sum<kFlatThreads>(x, s_warp);
    __shared__ uint64_t s_tot;
    if (threadIdx.x == kFlatThreads - 1) s_tot = ex + x;
    __syncthreads();
    const uint64_t t = s_tot;
    __syncthreads();
    return t;
}

// Scan of the count CTAs' chunk totals, run by the last count CTA to finish (its kFlatThreads
// threads): part[] becomes the exclusive scan, part[nparts] the total, part[nparts + 1] the
// one-to-one flag; the capacity check sets the output row count or the overflow bit.  The
// totals of other CTAs are read from L2 (they were written by other SMs).
__device__ void flat_scan_parts(const FlatArgs& a, uint32_t nparts, uint64_t R, uint64_t* s_warp) {
    __shared__ uint64_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    bool not_ones = false;
    for (uint32_t r0 = 0; r0 < nparts; r0 += kFlatThreads) {
        const uint32_t i = r0 + threadIdx.x;
        const uint64_t pv = i < nparts ? __ldcg((const unsigned long long*)a.part + i) : 0;
        not_ones |= (pv & kNotOneToOne) != 0;
        const uint64_t x = pv & ~kNotOneToOne;
        const uint64_t ex = block_exclusive_sum<kFlatThreads>(x, s_warp);
        const uint64_t carry = s_carry;
        if (i < nparts) a.part[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == kFlatThreads - 1) s_carry = carry + ex + x;
        __syncthreads();
    }
    const bool one_to_one = !__syncthreads_or(not_ones);
    if (threadIdx.x == 0) {
        const uint64_t total = s_carry;
        a.part[nparts] = total;
        a.part[nparts + 1] = one_to_one ? 1 : 0;
        a.pos[R] = total;
        if (total > a.out_cap_rows) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)total);
            *a.out_rows = 0;
        } else {
            *a.out_rows = total;
            atomicAdd(&a.ctl->alg_bytes, (unsigned long long)(total * a.step.cout * 4ull));
        }
    }
}

// Called by every thread of a count CTA once its chunk total is in part[blockIdx.x]: true in the
// last CTA to get here, which then runs the scan (and leaves the counter at 0 for the next pass).
__device__ __forceinline__ bool last_count_cta(StepCtl* ctl) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        s_last = atomicAdd(&ctl->flat_done, 1u) == gridDim.x - 1;
        if (s_last) ctl->flat_done = 0;
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last != 0;
}

// Key of a row of the count pass: the step's start key (const_to_known / index_to_known) or
// [cur|pid|dir] (the index key of get_index for the TYPE_ID/IN form, and for vid 0); *look is
// false where there is nothing to probe.
__device__ __forceinline__ uint64_t count_key(const FlatArgs& a, const StepDesc& d, bool from_const, uint32_t cur,
                                              bool* valid, bool* look, uint64_t* bucket) {
    uint64_t key;
    SegDesc sg = d.seg;   // by value: registers, not a pointer into the parameter block
    *valid = from_const || cur != kBlankId;
    if (from_const) {
        key = d.start_key;
    } else if (d.op == kXK2U && d.type_index) {
        // get_index(cur, IN) (sparql.hpp:342-345); only 17-bit ids can be keys
        key = make_key(0, cur, kIn);
        sg = a.seg_index[kIn];
        if (cur >= (1u << kNbitsIdx)) *valid = false;
    } else {
        key = make_key(cur, d.pid, d.dir);
        if (cur == 0) sg = a.seg_index[d.dir & 1];   // vid 0 names the index
    }
    *look = *valid && sg.num_buckets != 0 && key != 0;
    *bucket = *look ? bucket_of(key, sg) : 0;
    if (*look && *bucket >= a.store.n_buckets) {
        atomicOr(&a.ctl->err, kErrCorrupt);
        *look = false;
    }
    return key;
}

// Pointer word of `key` given its home bucket's slots 0 and 1 (one 32-byte sector, loaded
// together); the walk goes on from slot 2 only when they do not settle the key.
__device__ __forceinline__ uint64_t settle_slot(const DevStore& st, uint64_t key, uint64_t b, ulonglong2 s0,
                                                ulonglong2 s1, unsigned* err) {
    if (s0.x == key) return s0.y;
    if (s0.x == 0) return 0;   // first empty slot: absent (insert-only store)
    if (s1.x == key) return s1.y;
    if (s1.x == 0) return 0;
    return thread_probe(st, key, b, err, 2);
}

// kRowsPerThread rows per thread at a time: their keys are worked out and their home slots
// loaded before any is compared, and the neighbour words of their one-to-one rows are loaded
// before any output row is written, so a thread has that many random reads in flight.
// Registers are capped for kCountCtas CTAs per SM.  One row per thread at 8 CTAs (2,048 threads
// per SM) measured best: more rows per thread at fewer CTAs (2-8 rows, 2-6 CTAs) ran 1-35%
// slower on the heavy star and triangle, so resident warps, not reads per thread, set the rate.
// kFilter: the membership steps (known_to_known, known_to_const, const_to_known,
// index_to_known); the other instance (starts and known_to_unknown) carries no membership search.
constexpr int kRowsPerThread = 1;
constexpr int kCountCtas = 8;

template <bool kFilter>
__global__ void __launch_bounds__(kFlatThreads, kCountCtas) flat_count_kernel(const FlatArgs a) {
    __shared__ uint64_t s_warp[kFlatThreads / 32];
    const uint64_t R = flat_rows(a);
    if (R < a.min_rows) return;
    uint64_t lo, hi;
    chunk_of(R, &lo, &hi);
    const StepDesc& d = a.step;
    const bool from_const = d.op == kXC2K || d.op == kXI2K;   // every row looks up one list
    const int tcol = (d.op == kXK2K || from_const) ? d.ce : -1;   // the row's membership target
    uint64_t sum = 0, sd = 0, nvalid = 0;
    bool ones = true;   // every row of this thread has exactly one output row
    const bool spec = R <= a.out_cap_rows;   // output row r exists: one-to-one rows written here
    constexpr int K = kRowsPerThread;
    constexpr uint64_t kStride = (uint64_t)K * kFlatThreads;
    for (uint64_t r0 = lo + threadIdx.x; r0 < hi; r0 += kStride) {
        uint64_t key[K], bkt[K], p[K];
        bool valid[K], look[K];
        ulonglong2 s0[K], s1[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint64_t r = r0 + (uint64_t)k * kFlatThreads;
            const uint32_t cur = r < hi ? __ldg(a.in + r * (uint64_t)a.w_in + d.cs) : kBlankId;
            key[k] = count_key(a, d, from_const, cur, &valid[k], &look[k], &bkt[k]);
            if (r >= hi) valid[k] = look[k] = false;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            s0[k] = s1[k] = make_ulonglong2(0, 0);
            if (look[k]) load_sector(a.store.slots + bkt[k] * kAssoc, &s0[k], &s1[k]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
            p[k] = look[k] ? settle_slot(a.store, key[k], bkt[k], s0[k], s1[k], &a.ctl->err) : 0;
        // counts and list offsets
        uint32_t c[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint64_t r = r0 + (uint64_t)k * kFlatThreads;
            uint64_t off, deg;
            list_of_ptr(p[k], a.store.n_edges, &a.ctl->err, &off, &deg);
            if (d.op == kXI2K && valid[k]) {   // index_to_known reads its mt slice of the list
                uint64_t s_lo, s_hi;
                mt_slice(d.mt, deg, &s_lo, &s_hi);
                off += s_lo;
                deg = s_hi - s_lo;
            }
            c[k] = (uint32_t)deg;
            if (kFilter && valid[k] && deg) {
                // the membership target shares the row's sector with its start column
                const uint32_t target = tcol >= 0 ? __ldg(a.in + r * (uint64_t)a.w_in + tcol) : d.end_const;
                c[k] = thread_member(a.store.edges, off, deg, target, a.sorted_lists != 0) ? 1u : 0u;
            }
            if (!valid[k]) c[k] = 0;
            p[k] = off;   // from here on p holds the list offset
            if (r < hi) {
                a.pos[r] = c[k];   // the count; flat_place_kernel turns it into the row's position
                if (!kFilter) a.off[r] = off;
                if (c[k] != 1) ones = false;
                sum += c[k];
            }
            if (valid[k]) {
                sd += deg;
                ++nvalid;
            }
        }
        if (!kFilter && spec) {
            // A row with exactly one output row writes it now, at output row r: when every row
            // has one (a functional predicate), that is the step's output and the place and
            // expand passes return at once; otherwise expand overwrites these rows.  The rows'
            // neighbour words are all loaded before any row is written.
            uint32_t nb[K];
#pragma unroll
            for (int k = 0; k < K; ++k) nb[k] = c[k] == 1 ? list_at(a.store.edges, p[k], 0) : 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (c[k] != 1) continue;
                const uint64_t r = r0 + (uint64_t)k * kFlatThreads;
                const uint32_t* src = a.in + r * (uint64_t)a.w_in;
                uint32_t* dst = a.out + r * (uint64_t)a.w_out;
                for (int j = 0; j < d.cin; ++j) dst[j] = __ldg(src + j);
                dst[d.cin] = nb[k];
            }
        }
    }
    const bool all_ones = __syncthreads_and(ones);
    sum = block_sum(sum, s_warp);
    sd = block_sum(sd, s_warp);
    nvalid = block_sum(nvalid, s_warp);
    if (threadIdx.x == 0) {
        a.part[blockIdx.x] = sum | (all_ones ? 0 : kNotOneToOne);
        if (nvalid) {
            atomicAdd(&a.ctl->sum_deg, (unsigned long long)sd);
            atomicAdd(&a.ctl->alg_bytes, (unsigned long long)(nvalid * (d.cin * 4ull + 16) + sd * 4));
        }
    }
    if (last_count_cta(a.ctl)) flat_scan_parts(a, gridDim.x, R, s_warp);
}

__global__ void __launch_bounds__(kFlatThreads) flat_place_kernel(const FlatArgs a, uint32_t nparts) {
    __shared__ uint64_t s_warp[kFlatThreads / 32];
    __shared__ uint64_t s_carry;
    const uint64_t R = flat_rows(a);
    if (R < a.min_rows || a.part[nparts] > a.out_cap_rows) return;
    uint64_t lo, hi;
    chunk_of(R, &lo, &hi);
    const bool filt = is_filter_op(a.step.op);
    if (!filt && a.part[nparts + 1] == 1) return;   // one output row per input row, in order
    // a filter's chunk without survivors has nothing to copy (part holds the exclusive scan of
    // the chunk totals, part[nparts] the total)
    if (filt && a.part[blockIdx.x + 1] == a.part[blockIdx.x]) return;
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint64_t r0 = lo; r0 < hi; r0 += kFlatThreads) {
        const uint64_t r = r0 + threadIdx.x;
        const uint64_t c = r < hi ? a.pos[r] : 0;
        const uint64_t ex = block_exclusive_sum<kFlatThreads>(c, s_warp);
        const uint64_t p = s_carry + ex;
        if (r < hi) {
            if (!filt) {
                a.pos[r] = p;
            } else if (c) {   // a surviving row keeps its columns (w_out == w_in)
                const uint32_t* src = a.in + r * (uint64_t)a.w_in;
                uint32_t* dst = a.out + p * (uint64_t)a.w_out;
                for (int k = 0; k < a.w_in; ++k) dst[k] = __ldg(src + k);
            }
        }
        __syncthreads();
        if (threadIdx.x == kFlatThreads - 1) s_carry = p + c;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kFlatThreads, 8) flat_expand_kernel(const FlatArgs a, uint32_t nparts) {
    __shared__ uint64_t s_pos[kWindow + 1];
    __shared__ uint64_t s_off[kWindow];
    __shared__ uint64_t s_i0;
    const uint64_t R = flat_rows(a);
    if (R < a.min_rows) return;
    const uint64_t total = a.pos[R];
    if (total > a.out_cap_rows || total == 0) return;
    // one output row per input row: the count pass wrote output row r for input row r (the
    // total fits, so R does too)
    if (a.part[nparts + 1] == 1) return;
    const uint64_t per = (total + gridDim.x - 1) / gridDim.x;
    const uint64_t j0 = min(total, (uint64_t)blockIdx.x * per), j1 = min(total, j0 + per);
    if (j0 >= j1) return;
    // first input row whose outputs reach j0: the last r with pos[r] <= j0 (pos[R] = total > j0)
    if (threadIdx.x < 32) {
        uint64_t lo = 0, hi = R;   // invariant: pos[lo] <= j0 < pos[hi]
        while (hi - lo > 1) {
            const uint64_t step = (hi - lo + 31) / 32;
            const uint64_t probe = min(hi, lo + (uint64_t)(threadIdx.x + 1) * step);
            const bool le = probe < hi && a.pos[probe] <= j0;
            const unsigned m = __ballot_sync(0xffffffffu, le);
            const int k = m ? 31 - __clz(m) : -1;   // last lane whose probe is still <= j0
            const uint64_t nlo = k >= 0 ? min(hi, lo + (uint64_t)(k + 1) * step) : lo;
            const uint64_t nhi = min(hi, nlo + step);
            lo = nlo;
            hi = max(nhi, lo + 1);
        }
        if (threadIdx.x == 0) s_i0 = lo;
    }
    __syncthreads();
    const int wo = a.w_out, ecol = a.step.cin;
    uint64_t i = s_i0;
    uint64_t j = j0;
    // the window's positions and offsets are loaded into registers one window ahead (a thread
    // holds entries t = threadIdx.x and, for the end position, t = kWindow)
    static_assert(kWindow == kFlatThreads, "one window entry per thread");
    uint64_t nx_pos = 0, nx_off = 0, nx_end = 0;
    {
        const uint64_t n = min((uint64_t)kWindow, R - i);
        if (threadIdx.x < n) {
            nx_pos = a.pos[i + threadIdx.x];
            nx_off = a.off[i + threadIdx.x];
        }
        if (threadIdx.x == 0) nx_end = a.pos[i + n];
    }
    constexpr int U = 4;   // output rows per thread with their neighbour loads in flight
    while (j < j1 && i < R) {
        const uint64_t n = min((uint64_t)kWindow, R - i);
        if (threadIdx.x < n) {
            s_pos[threadIdx.x] = nx_pos;
            s_off[threadIdx.x] = nx_off;
        }
        if (threadIdx.x == 0) s_pos[n] = nx_end;
        __syncthreads();
        const uint64_t i2 = i + n;
        if (i2 < R) {   // the next window's entries, while this one is written
            const uint64_t n2 = min((uint64_t)kWindow, R - i2);
            if (threadIdx.x < n2) {
                nx_pos = a.pos[i2 + threadIdx.x];
                nx_off = a.off[i2 + threadIdx.x];
            }
            if (threadIdx.x == 0) nx_end = a.pos[i2 + n2];
        }
        const uint64_t wend = min(j1, s_pos[n]);
        for (uint64_t jb = j + threadIdx.x; jb < wend; jb += (uint64_t)U * kFlatThreads) {
            int row[U];
            uint32_t nb[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t jj = jb + (uint64_t)u * kFlatThreads;
                row[u] = -1;
                if (jj >= wend) continue;
                int lo = 0, hi = (int)n;   // last t with s_pos[t] <= jj
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_pos[mid] <= jj) lo = mid; else hi = mid;
                }
                row[u] = lo;
                nb[u] = list_at(a.store.edges, s_off[lo], jj - s_pos[lo]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (row[u] < 0) continue;
                const uint64_t jj = jb + (uint64_t)u * kFlatThreads;
                const uint32_t* src = a.in + (i + row[u]) * (uint64_t)a.w_in;
                uint32_t* dst = a.out + jj * (uint64_t)wo;
                for (int k = 0; k < ecol; ++k) dst[k] = __ldg(src + k);
                dst[ecol] = nb[u];
            }
        }
        j = max(j, wend);
        i += n;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- batch levels
// The same four passes over one level of a batch: every row carries its owner query, whose
// step at this level (start, known_to_unknown, known_to_known, known_to_const or done) comes
// from the level's descriptor array.  Rows keep their order, so each query's output rows stay
// contiguous and its range is recorded from the runs of its rows.

__device__ __forceinline__ uint64_t level_rows(const FlatLevelArgs& a) {
    if (a.virtual_rows) return a.n_queries;
    uint64_t R = *(volatile const uint64_t*)a.in_rows;
    return R > a.in_cap_rows ? 0 : R;   // past capacity: the step before overflowed
}

__device__ __forceinline__ uint32_t level_owner(const FlatLevelArgs& a, uint64_t r) {
    return a.virtual_rows ? (uint32_t)r : __ldg(a.owner_in + r);
}

// The level pass's scan of the chunk totals, run by the last count CTA (as flat_scan_parts).
__device__ void flat_level_scan_parts(const FlatLevelArgs& a, uint32_t nparts, uint64_t R,
                                      uint64_t* s_warp) {
    __shared__ uint64_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t r0 = 0; r0 < nparts; r0 += kFlatThreads) {
        const uint32_t i = r0 + threadIdx.x;
        const uint64_t x = i < nparts ? __ldcg((const unsigned long long*)a.part + i) : 0;
        const uint64_t ex = block_exclusive_sum<kFlatThreads>(x, s_warp);
        const uint64_t carry = s_carry;
        if (i < nparts) a.part[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == kFlatThreads - 1) s_carry = carry + ex + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint64_t total = s_carry;
        a.part[nparts] = total;
        a.pos[R] = total;
        if (total > a.out_cap_rows) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)total);
            *a.out_rows = 0;
        } else {
            *a.out_rows = total;
        }
    }
}

// kRowsPerThread rows per thread at a time, their home slots loaded before any is compared (as
// in flat_count_kernel).
__global__ void __launch_bounds__(kFlatThreads, kCountCtas) flat_level_count_kernel(const FlatLevelArgs a) {
    __shared__ uint64_t s_warp[kFlatThreads / 32];
    const uint64_t R = level_rows(a);
    uint64_t lo, hi;
    chunk_of(R, &lo, &hi);
    uint64_t sum = 0, sd = 0, alg = 0;
    constexpr int K = kRowsPerThread;
    constexpr uint64_t kStride = (uint64_t)K * kFlatThreads;
    for (uint64_t r0 = lo + threadIdx.x; r0 < hi; r0 += kStride) {
        uint64_t key[K], bkt[K];
        uint32_t target[K];
        bool valid[K], look[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint64_t r = r0 + (uint64_t)k * kFlatThreads;
            key[k] = 0;
            bkt[k] = 0;
            target[k] = 0;
            valid[k] = look[k] = false;
            if (r >= hi) continue;
            const StepDesc* d = a.desc + level_owner(a, r);
            const uint32_t op = d->op;
            const SegDesc* sg = &d->seg;
            bool v = op != kXDone;
            target[k] = d->end_const;
            if (v && op == kXStart) {
                key[k] = d->start_key;
            } else if (v && (op == kXC2K || op == kXI2K)) {   // one list for every row
                key[k] = d->start_key;
                target[k] = __ldg(a.in + r * (uint64_t)a.w_in + d->ce);
            } else if (v) {
                const uint32_t* row = a.in + r * (uint64_t)a.w_in;
                const uint32_t cur = __ldg(row + d->cs);
                if (op == kXK2K) target[k] = __ldg(row + d->ce);
                if (cur == kBlankId) v = false;
                if (op == kXK2U && d->type_index) {
                    // get_index(cur, IN) (sparql.hpp:342-345); only 17-bit ids can be keys
                    key[k] = make_key(0, cur, kIn);
                    sg = &a.seg_index[kIn];
                    if (cur >= (1u << kNbitsIdx)) v = false;
                } else {
                    key[k] = make_key(cur, d->pid, d->dir);
                    if (cur == 0) sg = &a.seg_index[d->dir & 1];   // vid 0 names the index
                }
            }
            valid[k] = v;
            look[k] = v && sg->num_buckets != 0 && key[k] != 0;
            if (look[k]) bkt[k] = bucket_of(key[k], *sg);
            if (look[k] && bkt[k] >= a.store.n_buckets) {
                atomicOr(&a.ctl->err, kErrCorrupt);
                look[k] = false;
            }
        }
        ulonglong2 s0[K], s1[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            s0[k] = s1[k] = make_ulonglong2(0, 0);
            if (look[k]) load_sector(a.store.slots + bkt[k] * kAssoc, &s0[k], &s1[k]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint64_t r = r0 + (uint64_t)k * kFlatThreads;
            if (r >= hi) continue;
            const StepDesc* d = a.desc + level_owner(a, r);
            const uint32_t op = d->op;
            uint64_t off = 0, deg = 0;
            if (look[k]) {
                const uint64_t p = settle_slot(a.store, key[k], bkt[k], s0[k], s1[k], &a.ctl->err);
                list_of_ptr(p, a.store.n_edges, &a.ctl->err, &off, &deg);
                if (op == kXI2K) {
                    uint64_t s_lo, s_hi;
                    mt_slice(d->mt, deg, &s_lo, &s_hi);
                    off += s_lo;
                    deg = s_hi - s_lo;
                }
            }
            const bool filt = is_filter_op(op);
            uint32_t c = (uint32_t)deg;
            if (filt) c = (valid[k] && deg && thread_member(a.store.edges, off, deg, target[k], a.sorted_lists != 0)) ? 1u : 0u;
            if (!valid[k]) c = 0;
            a.pos[r] = c;   // the count; flat_level_place_kernel turns it into the row's position
            a.off[r] = off;
            sum += c;
            if (valid[k]) {
                const uint32_t cin = op == kXStart ? 0u : d->cin;
                sd += deg;
                alg += cin * 4ull + 16 + deg * 4 + (uint64_t)c * d->cout * 4;
            }
        }
    }
    sum = block_sum(sum, s_warp);
    sd = block_sum(sd, s_warp);
    alg = block_sum(alg, s_warp);
    if (threadIdx.x == 0) {
        a.part[blockIdx.x] = sum;
        if (alg) {
            atomicAdd(&a.ctl->sum_deg, (unsigned long long)sd);
            atomicAdd(&a.ctl->alg_bytes, (unsigned long long)alg);
        }
    }
    if (last_count_cta(a.ctl)) flat_level_scan_parts(a, gridDim.x, R, s_warp);
}

__global__ void __launch_bounds__(kFlatThreads) flat_level_place_kernel(const FlatLevelArgs a, uint32_t nparts) {
    __shared__ uint64_t s_warp[kFlatThreads / 32];
    __shared__ uint64_t s_carry;
    const uint64_t R = level_rows(a);
    if (a.part[nparts] > a.out_cap_rows) return;
    uint64_t lo, hi;
    chunk_of(R, &lo, &hi);
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint64_t r0 = lo; r0 < hi; r0 += kFlatThreads) {
        const uint64_t r = r0 + threadIdx.x;
        const uint64_t c = r < hi ? a.pos[r] : 0;
        const uint64_t ex = block_exclusive_sum<kFlatThreads>(c, s_warp);
        const uint64_t p = s_carry + ex;
        if (r < hi) {
            a.pos[r] = p;
            const uint32_t q = level_owner(a, r);
            // the query's output range: (end - start) of every run of its rows
            const bool first = r == lo || level_owner(a, r - 1) != q;
            const bool last = r + 1 == hi || level_owner(a, r + 1) != q;
            if (first) {
                atomicMin(a.qfirst + q, (unsigned long long)p);
                atomicAdd(a.qcount + q, (unsigned long long)(0 - p));
            }
            if (last) atomicAdd(a.qcount + q, (unsigned long long)(p + c));
            const uint32_t op = a.desc[q].op;
            if (c && is_filter_op(op)) {   // a surviving row keeps its columns
                const int cin = a.desc[q].cin;
                const uint32_t* src = a.in + r * (uint64_t)a.w_in;
                uint32_t* dst = a.out + p * (uint64_t)a.w_out;
                for (int k = 0; k < cin; ++k) dst[k] = __ldg(src + k);
                a.owner_out[p] = q;
            }
        }
        __syncthreads();
        if (threadIdx.x == kFlatThreads - 1) s_carry = p + c;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kFlatThreads) flat_level_expand_kernel(const FlatLevelArgs a) {
    __shared__ uint64_t s_pos[kWindow + 1];
    __shared__ uint64_t s_off[kWindow];
    __shared__ uint32_t s_q[kWindow];
    __shared__ int32_t s_ecol[kWindow];   // column the edge goes to; -1: not an expanding row
    __shared__ uint64_t s_i0;
    const uint64_t R = level_rows(a);
    const uint64_t total = a.pos[R];
    if (total > a.out_cap_rows || total == 0) return;
    const uint64_t per = (total + gridDim.x - 1) / gridDim.x;
    const uint64_t j0 = min(total, (uint64_t)blockIdx.x * per), j1 = min(total, j0 + per);
    if (j0 >= j1) return;
    if (threadIdx.x < 32) {   // the last r with pos[r] <= j0 (pos[R] = total > j0)
        uint64_t lo = 0, hi = R;
        while (hi - lo > 1) {
            const uint64_t step = (hi - lo + 31) / 32;
            const uint64_t probe = min(hi, lo + (uint64_t)(threadIdx.x + 1) * step);
            const bool le = probe < hi && a.pos[probe] <= j0;
            const unsigned m = __ballot_sync(0xffffffffu, le);
            const int k = m ? 31 - __clz(m) : -1;
            const uint64_t nlo = k >= 0 ? min(hi, lo + (uint64_t)(k + 1) * step) : lo;
            const uint64_t nhi = min(hi, nlo + step);
            lo = nlo;
            hi = max(nhi, lo + 1);
        }
        if (threadIdx.x == 0) s_i0 = lo;
    }
    __syncthreads();
    const int wo = a.w_out;
    uint64_t i = s_i0;
    uint64_t j = j0;
    while (j < j1 && i < R) {
        const uint64_t n = min((uint64_t)kWindow, R - i);
        for (int t = threadIdx.x; t <= (int)n; t += kFlatThreads) s_pos[t] = a.pos[i + t];
        for (int t = threadIdx.x; t < (int)n; t += kFlatThreads) {
            // the window's rows once: list offset, owner, and where its step puts the edge
            s_off[t] = a.off[i + t];
            const uint32_t q = level_owner(a, i + t);
            s_q[t] = q;
            const StepDesc* d = a.desc + q;
            const uint32_t op = d->op;
            s_ecol[t] = op == kXStart ? 0 : op == kXK2U ? (int32_t)d->cin : -1;   // filters: -1
        }
        __syncthreads();
        const uint64_t wend = min(j1, s_pos[n]);
        constexpr int U = 4;   // output rows per thread with their neighbour loads in flight
        for (uint64_t jb = j + threadIdx.x; jb < wend; jb += (uint64_t)U * kFlatThreads) {
            int row[U];
            uint32_t nb[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t jj = jb + (uint64_t)u * kFlatThreads;
                row[u] = -1;
                if (jj >= wend) continue;
                int lo = 0, hi = (int)n;   // last t with s_pos[t] <= jj
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_pos[mid] <= jj) lo = mid; else hi = mid;
                }
                if (s_ecol[lo] < 0) continue;   // filters wrote their rows already
                row[u] = lo;
                nb[u] = list_at(a.store.edges, s_off[lo], jj - s_pos[lo]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (row[u] < 0) continue;
                const uint64_t jj = jb + (uint64_t)u * kFlatThreads;
                const int lo = row[u], ecol = s_ecol[lo];
                const uint32_t* src = a.in + (i + lo) * (uint64_t)a.w_in;
                uint32_t* dst = a.out + jj * (uint64_t)wo;
                for (int k = 0; k < ecol; ++k) dst[k] = __ldg(src + k);
                dst[ecol] = nb[u];
                a.owner_out[jj] = s_q[lo];
            }
        }
        j = max(j, wend);
        i += n;
        __syncthreads();
    }
}

}  // namespace

int flat_grid(int sm_count) { return sm_count * (2048 / kFlatThreads); }

int flat_grid_beside(int sm_count, const CtaUse& other, int other_ctas) {
    cudaFuncAttributes fa{}, fb{};
    int regs = 255;
    if (cudaFuncGetAttributes(&fa, flat_count_kernel<true>) == cudaSuccess &&
        cudaFuncGetAttributes(&fb, flat_count_kernel<false>) == cudaSuccess)
        regs = std::max(fa.numRegs, fb.numRegs);
    int dev = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    CtaUse me{(size_t)std::max(fa.sharedSizeBytes, fb.sharedSizeBytes) + (size_t)reserved,
              ((regs * 32 + 255) / 256) * 256 * (kFlatThreads / 32), kFlatThreads};
    const int alone = 2048 / kFlatThreads;
    return blocks_beside(me, alone, other, other_ctas) * sm_count;
}

cudaError_t launch_flat(const FlatArgs& a, int grid, cudaStream_t s) {
    // its last CTA scans the totals
    if (is_filter_op(a.step.op)) flat_count_kernel<true><<<grid, kFlatThreads, 0, s>>>(a);
    else flat_count_kernel<false><<<grid, kFlatThreads, 0, s>>>(a);
    flat_place_kernel<<<grid, kFlatThreads, 0, s>>>(a, (uint32_t)grid);
    if (a.step.op == kXK2U) flat_expand_kernel<<<grid, kFlatThreads, 0, s>>>(a, (uint32_t)grid);
    return cudaGetLastError();
}

cudaError_t launch_flat_level(const FlatLevelArgs& a, int grid, cudaStream_t s) {
    flat_level_count_kernel<<<grid, kFlatThreads, 0, s>>>(a);   // its last CTA scans the totals
    flat_level_place_kernel<<<grid, kFlatThreads, 0, s>>>(a, (uint32_t)grid);
    flat_level_expand_kernel<<<grid, kFlatThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t flat_kernel_attrs() {
    cudaError_t e;
    if ((e = use_max_shared_carveout(flat_count_kernel<true>)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(flat_count_kernel<false>)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(flat_place_kernel)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(flat_expand_kernel)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(flat_level_count_kernel)) != cudaSuccess) return e;
    if ((e = use_max_shared_carveout(flat_level_place_kernel)) != cudaSuccess) return e;
    return use_max_shared_carveout(flat_level_expand_kernel);
}

}  // namespace wk
