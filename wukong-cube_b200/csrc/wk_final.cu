// Post-pattern stage on the device: DISTINCT, OFFSET, LIMIT and the projection onto the
// required variables, as SPARQLEngine::final_process applies them (sparql.hpp:1419-1546), so a
// query's table can be finished without leaving the GPU.  ORDER BY is not here: the reference
// orders by the strings of the ids (sparql.hpp:1378-1400), which needs the string server.
//
// DISTINCT follows the reference step for step: the rows are sorted by all their columns,
// compared as signed 32-bit values (ReduceCmp over an int table, sparql.hpp:1403-1417), then
// of each run of neighbours equal on the required columns the first is kept.  The sort is an
// LSD radix sort of (packed key, row index) pairs over only the bits in which the rows differ
// (see "DISTINCT sort" below); rows equal in every column are interchangeable, so the result
// does not depend on how the reference's std::sort orders them.  A table found to be in that
// order already (one pass over it, rows_sorted_kernel) skips the sort.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "wk_ctx.h"
#include "wk_device.cuh"

namespace wk {
namespace {
using namespace dev;

#define WKF_CUDA(ctx, call)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call); \
    } while (0)

constexpr int kFinThreads = 256;
constexpr int kDigits = 256;

// ---------------------------------------------------------------- DISTINCT sort
// The sort orders rows by all their columns as signed 32-bit values.  A column is first mapped
// to its offset from the column's smallest value (in signed order), so a column spanning d
// distinct-order values needs only ceil(log2(d)) bits, and a constant column none.  Columns are
// packed, last column in the lowest bits, into 64-bit keys ("chunks" of consecutive columns that
// fit in 64 bits); the LSD sort runs the chunks from the last columns to the first, and within a
// chunk one stable 8-bit counting pass per byte of the chunk's bits.  Every pass reads the keys
// and row indices with coalesced loads; the table itself is read once per chunk, to build its
// keys.

// Smallest and largest value of every column (signed order, stored with the sign bit flipped).
__global__ void __launch_bounds__(kFinThreads) minmax_kernel(const uint32_t* table, uint64_t elems, int cols,
                                                             uint32_t* mm /* [2 * cols] */) {
    __shared__ uint32_t s_lo[64], s_hi[64];
    for (int c = threadIdx.x; c < cols; c += kFinThreads) {
        s_lo[c] = 0xFFFFFFFFu;
        s_hi[c] = 0;
    }
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * kFinThreads;
    uint64_t e = blockIdx.x * (uint64_t)kFinThreads + threadIdx.x;
    int c = (int)(e % cols);
    const int step = (int)(stride % cols);
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    int cur = c;
    // eight loads in flight per thread; the host makes the grid's stride a multiple of cols where
    // it can, so a thread's elements stay in one column and the fold below never runs in the loop
    constexpr int kPer = 8;
    for (; e + (kPer - 1) * stride < elems; e += kPer * stride) {
        uint32_t v[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) v[r] = __ldg(table + e + r * stride) ^ 0x80000000u;
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            if (c != cur) {
                atomicMin(&s_lo[cur], lo);
                atomicMax(&s_hi[cur], hi);
                lo = 0xFFFFFFFFu;
                hi = 0;
                cur = c;
            }
            lo = min(lo, v[r]);
            hi = max(hi, v[r]);
            c += step;
            if (c >= cols) c -= cols;
        }
    }
    for (; e < elems; e += stride) {
        const uint32_t v = __ldg(table + e) ^ 0x80000000u;
        if (c != cur) {   // column changed: fold the run so far into shared memory
            atomicMin(&s_lo[cur], lo);
            atomicMax(&s_hi[cur], hi);
            lo = 0xFFFFFFFFu;
            hi = 0;
            cur = c;
        }
        lo = min(lo, v);
        hi = max(hi, v);
        c += step;
        if (c >= cols) c -= cols;
    }
    if (lo <= hi) {
        atomicMin(&s_lo[cur], lo);
        atomicMax(&s_hi[cur], hi);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < cols; k += kFinThreads) {
        if (s_lo[k] <= s_hi[k]) {
            atomicMin(&mm[2 * k], s_lo[k]);
            atomicMax(&mm[2 * k + 1], s_hi[k]);
        }
    }
}

// One chunk's key layout: columns ccol[0..nc), most significant first, ccol[j] in cbits[j]
// bits above the next, offset by cmin[j].
struct ChunkDesc {
    int nc;
    int ccol[32];
    int cbits[32];
    uint32_t cmin[32];
};

// keys[i] = the chunk key of row idx_in[i] (row i when idx_in is null); idx_out[i] = that row.
__global__ void __launch_bounds__(kFinThreads) key_kernel(const uint32_t* table, int cols, ChunkDesc cd,
                                                          const uint32_t* idx_in, uint32_t n,
                                                          unsigned long long* keys, uint32_t* idx_out) {
    for (uint32_t i = blockIdx.x * kFinThreads + threadIdx.x; i < n; i += gridDim.x * kFinThreads) {
        const uint32_t r = idx_in ? idx_in[i] : i;
        const uint32_t* row = table + (uint64_t)r * cols;
        unsigned long long k = 0;
        for (int j = 0; j < cd.nc; ++j)
            k = (k << cd.cbits[j]) | (unsigned long long)((__ldg(row + cd.ccol[j]) ^ 0x80000000u) - cd.cmin[j]);
        keys[i] = k;
        idx_out[i] = r;
    }
}

// *flag = 1 when some row is greater than the next one, every column compared as a signed 32-bit
// value in column order (ReduceCmp).  A table already in that order is what the sort would
// return (rows equal in every column are interchangeable), so the sort is skipped for it: the
// exploration writes rows in input order and each row's new column from a sorted list, so a
// table started from an index or a constant with unique rows comes out in this order.
// A CTA stages `tile_rows` consecutive rows and the row after them in shared memory with
// coalesced loads, eight in flight per thread, then each thread compares one row with the next
// out of shared memory; a CTA that finds a pair out of order stops.
constexpr int kCheckWords = 8192;   // 32 KiB of rows per tile

__global__ void __launch_bounds__(kFinThreads) rows_sorted_kernel(const uint32_t* table, int cols, uint32_t n,
                                                                  uint32_t tile_rows, unsigned* flag) {
    __shared__ uint32_t s_t[kCheckWords];
    const uint32_t pairs = n - 1;   // pair i is rows (i, i + 1); n >= 2
    for (uint64_t t0 = (uint64_t)blockIdx.x * tile_rows; t0 < pairs; t0 += (uint64_t)gridDim.x * tile_rows) {
        const uint32_t here = (uint32_t)min((uint64_t)tile_rows, pairs - t0);   // pairs of this tile
        const uint32_t words = (here + 1) * (uint32_t)cols;                     // <= kCheckWords
        const uint32_t* src = table + t0 * cols;
        constexpr int kPer = 8;
        uint32_t w = threadIdx.x;
        for (; w + (kPer - 1) * kFinThreads < words; w += kPer * kFinThreads) {
            uint32_t v[kPer];
#pragma unroll
            for (int r = 0; r < kPer; ++r) v[r] = __ldg(src + w + r * kFinThreads);
#pragma unroll
            for (int r = 0; r < kPer; ++r) s_t[w + r * kFinThreads] = v[r];
        }
        for (; w < words; w += kFinThreads) s_t[w] = __ldg(src + w);
        __syncthreads();
        bool bad = false;
        for (uint32_t i = threadIdx.x; i < here && !bad; i += kFinThreads) {
            const uint32_t* r = s_t + i * cols;
            for (int c = 0; c < cols; ++c) {
                const int32_t x = (int32_t)r[c], y = (int32_t)r[cols + c];
                if (x != y) {
                    bad = x > y;
                    break;
                }
            }
        }
        // also the barrier before the next tile overwrites s_t
        if (__syncthreads_or(bad)) {
            if (threadIdx.x == 0) atomicOr(flag, 1u);
            return;
        }
    }
}

struct SortPass {
    const unsigned long long* key_in;
    const uint32_t* idx_in;
    unsigned long long* key_out;
    uint32_t* idx_out;
    int shift;
    uint32_t n;
    uint32_t* hist;          // [kDigits][grid]: digit-major, so one scan gives the offsets
    uint32_t* dtot;          // [kDigits]: elements of each digit
};
static_assert(kFinThreads == kDigits, "the counting passes give each digit one thread");

__device__ __forceinline__ void chunk(uint32_t n, uint32_t* lo, uint32_t* hi) {
    const uint32_t c = (n + gridDim.x - 1) / gridDim.x;
    *lo = min(n, blockIdx.x * c);
    *hi = min(n, *lo + c);
}

__global__ void __launch_bounds__(kFinThreads) iota_kernel(uint32_t* idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * kFinThreads + threadIdx.x; i < n; i += gridDim.x * kFinThreads) idx[i] = i;
}

// Digit counts of each CTA's chunk.  A thread loads eight keys before it counts any of them, so
// eight loads per thread are in flight instead of one.
__global__ void __launch_bounds__(kFinThreads) hist_kernel(const SortPass a) {
    constexpr int kPer = 8;
    __shared__ uint32_t s_h[kDigits];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    uint64_t i = lo + threadIdx.x;
    for (; i + (kPer - 1) * kFinThreads < hi; i += kPer * kFinThreads) {
        unsigned long long k[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) k[r] = a.key_in[i + r * kFinThreads];
#pragma unroll
        for (int r = 0; r < kPer; ++r) atomicAdd(&s_h[(uint32_t)(k[r] >> a.shift) & 0xFFu], 1u);
    }
    for (; i < hi; i += kFinThreads) atomicAdd(&s_h[(uint32_t)(a.key_in[i] >> a.shift) & 0xFFu], 1u);
    __syncthreads();
    a.hist[threadIdx.x * gridDim.x + blockIdx.x] = s_h[threadIdx.x];
}

// Exclusive scan of n words in place by one CTA of 1,024 threads.
__global__ void __launch_bounds__(1024) scan_kernel(uint32_t* v, uint32_t n, uint32_t* total) {
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
    if (threadIdx.x == 0 && total) *total = (uint32_t)s_carry;
}

// Offsets of a counting pass: digit d of CTA b starts at the elements of smaller digits plus the
// digit-d elements of CTAs before b.  CTA d of this launch scans digit d's row of hist (one
// contiguous row of `grid` words, digit-major) in place into exclusive offsets within the digit,
// with coalesced loads, and writes the digit's total to dtot[d]; each scatter CTA then adds the
// elements of smaller digits (an exclusive scan of dtot) itself.
__global__ void __launch_bounds__(kFinThreads) digit_rows_kernel(uint32_t* hist, uint32_t grid, uint32_t* dtot) {
    __shared__ uint64_t s_warp[kFinThreads / 32];
    __shared__ uint64_t s_carry;
    uint32_t* row = hist + (size_t)blockIdx.x * grid;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < grid; b0 += kFinThreads) {
        const uint32_t b = b0 + threadIdx.x;
        const uint64_t x = b < grid ? row[b] : 0;
        const uint64_t ex = block_exclusive_sum<kFinThreads>(x, s_warp);
        const uint64_t carry = s_carry;
        if (b < grid) row[b] = (uint32_t)(carry + ex);
        __syncthreads();
        if (threadIdx.x == kFinThreads - 1) s_carry = carry + ex + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) dtot[blockIdx.x] = (uint32_t)s_carry;
}

// Stable scatter of 2,048-element tiles: warp w of the CTA takes elements [w * 256, w * 256 + 256)
// of the tile in 8 rounds of 32 consecutive ones, so the warp's rounds follow the elements'
// order.  Within a round, an element's rank among the lanes with its digit comes from a match,
// and the warp's running count of each digit (shared memory, updated by one lane per digit)
// gives its place in the warp; one barrier then turns the warps' counts into per-warp digit
// offsets.  The tile is placed in shared memory sorted by digit (stable), and then written out
// in that order, consecutive threads on consecutive elements, so each digit's run goes to
// global memory in contiguous, coalesced stores.  Built for 4 CTAs per SM (64 registers, no
// spills; 34.9 KB of shared memory each), so the pass's 4 CTAs per SM run in one wave.
constexpr int kScatterPer = 8;                                // elements per thread per tile
constexpr int kScatterTile = kFinThreads * kScatterPer;       // 2,048

__global__ void __launch_bounds__(kFinThreads, 4) scatter_kernel(const SortPass a) {
    constexpr int kWarps = kFinThreads / 32;
    __shared__ uint32_t s_run[kDigits];
    __shared__ uint32_t s_cnt[kWarps][kDigits];
    __shared__ uint32_t s_tbase[kDigits];
    __shared__ unsigned long long s_key[kScatterTile];
    __shared__ uint32_t s_idx[kScatterTile];
    __shared__ uint64_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // thread d: digit d's first place for this CTA = the elements of smaller digits plus the
    // digit-d elements of the CTAs before this one
    const uint32_t smaller = (uint32_t)block_exclusive_sum<kFinThreads>(a.dtot[threadIdx.x], s_warp);
    s_run[threadIdx.x] = smaller + a.hist[threadIdx.x * gridDim.x + blockIdx.x];
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    for (uint32_t base = lo; base < hi; base += kScatterTile) {
        for (int w = 0; w < kWarps; ++w) s_cnt[w][threadIdx.x] = 0;
        __syncthreads();
        unsigned long long key[kScatterPer];
        uint32_t row[kScatterPer], dg[kScatterPer], at[kScatterPer];
        const uint32_t wbase = base + (uint32_t)warp * (32 * kScatterPer);
#pragma unroll
        for (int r = 0; r < kScatterPer; ++r) {
            const uint32_t i = wbase + r * 32 + lane;
            const bool live = i < hi;
            key[r] = live ? a.key_in[i] : 0;
            row[r] = live ? a.idx_in[i] : 0;
            dg[r] = live ? (uint32_t)(key[r] >> a.shift) & 0xFFu : kDigits + lane;   // lone sentinel
        }
#pragma unroll
        for (int r = 0; r < kScatterPer; ++r) {
            const unsigned peers = __match_any_sync(0xffffffffu, dg[r]);
            const int rank = __popc(peers & ((1u << lane) - 1));
            const bool live = dg[r] < kDigits;
            at[r] = live ? s_cnt[warp][dg[r]] + rank : 0;
            __syncwarp();
            if (live && rank == 0) s_cnt[warp][dg[r]] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t tile_cnt = 0;   // per digit (thread = digit): prefix over the warps
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = s_cnt[w][threadIdx.x];
            s_cnt[w][threadIdx.x] = tile_cnt;
            tile_cnt += c;
        }
        // the tile sorted by digit in shared memory: digit d's elements start at s_tbase[d]
        const uint32_t tbase = (uint32_t)block_exclusive_sum<kFinThreads>(tile_cnt, s_warp);
        s_tbase[threadIdx.x] = tbase;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kScatterPer; ++r) {
            if (dg[r] >= kDigits) continue;
            const uint32_t lp = s_tbase[dg[r]] + s_cnt[warp][dg[r]] + at[r];
            s_key[lp] = key[r];
            s_idx[lp] = row[r];
        }
        __syncthreads();
        // consecutive threads write consecutive elements: each digit's run goes out contiguous
        const uint32_t m = min((uint32_t)kScatterTile, hi - base);
        for (uint32_t j = threadIdx.x; j < m; j += kFinThreads) {
            const unsigned long long k = s_key[j];
            const uint32_t d = (uint32_t)(k >> a.shift) & 0xFFu;
            const uint32_t pos = s_run[d] + (j - s_tbase[d]);
            a.key_out[pos] = k;
            a.idx_out[pos] = s_idx[j];
        }
        __syncthreads();
        s_run[threadIdx.x] += tile_cnt;
    }
}

// out row i = table row idx[i]: the table in sorted order, so the run compaction and the
// projection read consecutive rows instead of gathering each row (and its neighbour) through
// the index array.  One thread per element, consecutive threads on consecutive elements.
__global__ void __launch_bounds__(kFinThreads) gather_rows_kernel(const uint32_t* table, int cols,
                                                                  const uint32_t* idx, uint32_t n, uint32_t* out) {
    const uint64_t total = (uint64_t)n * cols;
    for (uint64_t e = blockIdx.x * (uint64_t)kFinThreads + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * kFinThreads) {
        const uint64_t i = e / cols;
        const int c = (int)(e - i * cols);
        out[e] = __ldg(table + (uint64_t)__ldg(idx + i) * cols + c);
    }
}

struct UniqueArgs {
    const uint32_t* table;
    int cols;
    const int32_t* keep;   // required columns
    int n_keep;
    const uint32_t* idx;   // sorted row indices
    uint32_t n;
    uint32_t* part;        // [grid + 1] kept rows per CTA, then their exclusive scan
    uint32_t* out;         // kept row indices
};

// Row i of the sorted order (idx null: the table was in order already).
__device__ __forceinline__ uint32_t sorted_row(const UniqueArgs& a, uint32_t i) { return a.idx ? a.idx[i] : i; }

__device__ __forceinline__ bool starts_run(const UniqueArgs& a, uint32_t i) {
    if (i == 0) return true;
    const uint32_t* r = a.table + (uint64_t)sorted_row(a, i) * a.cols;
    const uint32_t* p = a.table + (uint64_t)sorted_row(a, i - 1) * a.cols;
    for (int k = 0; k < a.n_keep; ++k)
        if (r[a.keep[k]] != p[a.keep[k]]) return true;
    return false;
}

__global__ void __launch_bounds__(kFinThreads) unique_count_kernel(const UniqueArgs a) {
    __shared__ uint64_t s_warp[kFinThreads / 32];
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    uint64_t c = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += kFinThreads) c += starts_run(a, i);
    const uint64_t ex = block_exclusive_sum<kFinThreads>(c, s_warp);
    if (threadIdx.x == kFinThreads - 1) a.part[blockIdx.x] = (uint32_t)(ex + c);
}

__global__ void __launch_bounds__(kFinThreads) unique_place_kernel(const UniqueArgs a) {
    __shared__ uint64_t s_warp[kFinThreads / 32];
    __shared__ uint64_t s_carry;
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint32_t base = lo; base < hi; base += kFinThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint64_t m = i < hi ? starts_run(a, i) : 0;
        const uint64_t ex = block_exclusive_sum<kFinThreads>(m, s_warp);
        const uint64_t carry = s_carry;
        if (m) a.out[carry + ex] = sorted_row(a, i);
        __syncthreads();
        if (threadIdx.x == kFinThreads - 1) s_carry = carry + ex + m;
        __syncthreads();
    }
}

// out row j = the required columns of input row idx[start + j] (idx null: row start + j).
__global__ void __launch_bounds__(kFinThreads) project_kernel(const uint32_t* table, int cols,
                                                              const int32_t* keep, int n_keep,
                                                              const uint32_t* idx, uint64_t start,
                                                              uint64_t count, uint32_t* out,
                                                              uint64_t* out_rows) {
    const uint64_t total = count * n_keep;
    for (uint64_t e = blockIdx.x * (uint64_t)kFinThreads + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * kFinThreads) {
        const uint64_t j = e / n_keep;
        const int k = (int)(e - j * n_keep);
        const uint64_t row = idx ? idx[start + j] : start + j;
        out[e] = table[row * cols + keep[k]];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *out_rows = count;
}

// ---------------------------------------------------------------- BOUND filter
// SPARQLEngine::bound_filter (sparql.hpp:1222-1234) for every BOUND(?x) of a query at once, as
// execute_filter ANDs them (:1356-1376): a row survives when none of the named columns holds
// BLANK_ID, and the survivors keep their order (append_row_to in row order).
struct BoundArgs {
    const uint32_t* table;
    int cols;
    const int32_t* bcols;   // columns that must be bound
    int nb;
    uint32_t n;
    uint32_t* part;         // [grid + 1] survivors per CTA, then their exclusive scan
    uint32_t* out;
};

__device__ __forceinline__ bool row_bound(const BoundArgs& a, uint32_t i) {
    const uint32_t* r = a.table + (uint64_t)i * a.cols;
    for (int k = 0; k < a.nb; ++k)
        if (__ldg(r + a.bcols[k]) == kBlankId) return false;
    return true;
}

__global__ void __launch_bounds__(kFinThreads) bound_count_kernel(const BoundArgs a) {
    __shared__ uint64_t s_warp[kFinThreads / 32];
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    uint64_t c = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += kFinThreads) c += row_bound(a, i);
    const uint64_t ex = block_exclusive_sum<kFinThreads>(c, s_warp);
    if (threadIdx.x == kFinThreads - 1) a.part[blockIdx.x] = (uint32_t)(ex + c);
}

// Each CTA walks its chunk 256 rows at a time; a surviving row goes to its CTA's offset plus the
// survivors before it, and its words are copied by consecutive threads.
__global__ void __launch_bounds__(kFinThreads) bound_place_kernel(const BoundArgs a) {
    __shared__ uint64_t s_warp[kFinThreads / 32];
    __shared__ uint64_t s_carry;
    __shared__ uint32_t s_src[kFinThreads], s_dst[kFinThreads];
    __shared__ uint32_t s_m;
    uint32_t lo, hi;
    chunk(a.n, &lo, &hi);
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint32_t base = lo; base < hi; base += kFinThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint64_t m = i < hi ? row_bound(a, i) : 0;
        const uint64_t ex = block_exclusive_sum<kFinThreads>(m, s_warp);
        const uint64_t carry = s_carry;
        if (m) {
            s_src[ex] = i;
            s_dst[ex] = (uint32_t)(carry + ex);
        }
        if (threadIdx.x == kFinThreads - 1) s_m = (uint32_t)(ex + m);
        __syncthreads();
        const uint32_t cnt = s_m;
        for (uint32_t e = threadIdx.x; e < cnt * (uint32_t)a.cols; e += kFinThreads) {
            const uint32_t j = e / a.cols, c = e - j * a.cols;
            a.out[(uint64_t)s_dst[j] * a.cols + c] = __ldg(a.table + (uint64_t)s_src[j] * a.cols + c);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + cnt;
        __syncthreads();
    }
}

}  // namespace

cudaError_t final_kernel_attrs() {
    cudaError_t e = use_max_shared_carveout(iota_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(minmax_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(key_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(hist_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(scan_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(digit_rows_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(rows_sorted_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(scatter_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(unique_count_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(unique_place_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(project_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(bound_count_kernel);
    if (e == cudaSuccess) e = use_max_shared_carveout(bound_place_kernel);
    return e;
}

}  // namespace wk

extern "C" int wk_table_final_process(wk_ctx* ctx, const wk_table* in, const int32_t* keep_cols,
                                      int32_t n_keep, int32_t distinct, int64_t offset, int64_t limit,
                                      wk_table* out) {
    using namespace wk;
    if (!ctx || !in || !out || in == out || (!keep_cols && n_keep) || n_keep < 0 || offset < 0)
        return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const int cols = in->cols;
    cudaStream_t s = ctx->stream;
    uint64_t R = 0;
    WKF_CUDA(ctx, cudaMemcpyAsync(ctx->h_rows, in->d_rows, 8, cudaMemcpyDeviceToHost, s));
    WKF_CUDA(ctx, cudaStreamSynchronize(s));
    R = ctx->h_rows[0];
    // a row count past the capacity marks a table whose writing step overflowed: refused before
    // any launch (and before any scratch is sized from it), as wk_table_download refuses it
    if (cols > 0 && R > in->cap / (uint64_t)cols)
        return ctx->fail(WK_E_CORRUPT, "row count beyond table capacity");
    if (R == 0) {   // an empty table is left as it is, columns included (sparql.hpp:1420-1421)
        int rc = ctx->table_reserve(out, 1);
        if (rc) return rc;
        out->cols = cols;
        WKF_CUDA(ctx, cudaMemsetAsync(out->d_rows, 0, 8, s));
        WKF_CUDA(ctx, cudaStreamSynchronize(s));
        return WK_SUCCESS;
    }
    if (n_keep == 0) return ctx->fail(WK_NO_REQUIRED_VAR, "no required variable");
    // tables hold at most 32 columns (the context's column limit); the sort's chunk layout and
    // the order check's row tiles are sized for that
    if (cols > 32) return ctx->fail(WK_E_CAPACITY, "more than 32 columns");
    for (int k = 0; k < n_keep; ++k)
        if (keep_cols[k] < 0 || keep_cols[k] >= cols) return ctx->fail(WK_E_BADARG, "required column out of range");
    if (R >= (1ull << 32)) return ctx->fail(WK_E_CAPACITY, "table too long for the post-pattern stage");
    const uint32_t n = (uint32_t)R;
    const int grid = std::max(1, std::min<int>(ctx->sm_count * 4, (int)((n + 2047) / 2048)));
    // scratch: the required columns, two index arrays, two key arrays (DISTINCT only), the
    // digit histogram, the CTA counts and the distinct total, the column ranges, the digit totals
    const bool sort = distinct && n > 1;
    const size_t keep_bytes = ((size_t)n_keep * 4 + 255) & ~(size_t)255;
    const size_t idx_bytes = ((2 * (size_t)n * 4) + 255) & ~(size_t)255;
    // the two key arrays; once the sort is done the same room holds the table in sorted order
    const size_t key_bytes = sort ? std::max(2 * (size_t)n * 8, (size_t)n * cols * 4) : 0;
    const size_t bytes = keep_bytes + idx_bytes + key_bytes + (size_t)kDigits * grid * 4 +
                         ((size_t)grid + 2) * 4 + (size_t)cols * 8 + (size_t)kDigits * 4 + 64;
    // the context keeps the scratch between calls (grown, never shrunk): an allocation and a
    // cudaFree per call would cost more than the stage's own kernels
    int src = ctx->final_scratch_reserve(bytes);
    if (src) return src;
    char* scratch = static_cast<char*>(ctx->d_final_scratch);
    auto done = [&](int rc) {
        cudaStreamSynchronize(s);
        return rc;
    };
    int32_t* d_keep = reinterpret_cast<int32_t*>(scratch);
    uint32_t* idx0 = reinterpret_cast<uint32_t*>(scratch + keep_bytes);
    uint32_t* idx1 = idx0 + n;
    unsigned long long* key0 = reinterpret_cast<unsigned long long*>(scratch + keep_bytes + idx_bytes);
    unsigned long long* key1 = key0 + (sort ? n : 0);
    uint32_t* hist = reinterpret_cast<uint32_t*>(scratch + keep_bytes + idx_bytes + key_bytes);
    uint32_t* part = hist + (size_t)kDigits * grid;
    uint32_t* d_total = part + grid + 1;
    uint32_t* d_mm = d_total + 1;
    uint32_t* dtot = d_mm + 2 * (size_t)cols;
    cudaError_t e = cudaMemcpyAsync(d_keep, keep_cols, (size_t)n_keep * 4, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return done(ctx->cuda_fail(e, "post-pattern columns"));
    const uint32_t* idx = nullptr;   // null: rows in table order
    const uint32_t* table_src = in->d;   // the rows idx refers to (the sorted copy after a sort)
    uint64_t m = n;
    bool in_order = false;
    if (sort) {   // a table already in the sort's order keeps it (d_total is free until the scan)
        unsigned h_flag = 1;
        if ((e = cudaMemsetAsync(d_total, 0, 4, s)) == cudaSuccess) {
            const uint32_t tile_rows = (uint32_t)(kCheckWords / cols - 1);   // cols <= 32: >= 255 rows
            const int cgrid = (int)std::max<uint64_t>(
                1, std::min<uint64_t>((uint64_t)ctx->sm_count * 6, ((uint64_t)n - 1 + tile_rows - 1) / tile_rows));
            rows_sorted_kernel<<<cgrid, kFinThreads, 0, s>>>(in->d, cols, n, tile_rows, d_total);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_flag, d_total, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return done(ctx->cuda_fail(e, "order check"));
        in_order = h_flag == 0;
    }
    if (sort) {
        const uint32_t* sorted = nullptr;   // the sorted row order (null: the table's own)
        if (!in_order) {
            // each column's range, in signed order
            std::vector<uint32_t> mm(2 * (size_t)cols);
            for (int c = 0; c < cols; ++c) {
                mm[2 * c] = 0xFFFFFFFFu;
                mm[2 * c + 1] = 0;
            }
            if ((e = cudaMemcpyAsync(d_mm, mm.data(), mm.size() * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess)
                return done(ctx->cuda_fail(e, "column ranges"));
            int mgrid = std::max(1, std::min(ctx->sm_count * 8, (int)(((uint64_t)n * cols + 255) / 256)));
            if (mgrid >= cols) mgrid -= mgrid % cols;   // stride a multiple of cols: one column per thread
            minmax_kernel<<<mgrid, kFinThreads, 0, s>>>(in->d, (uint64_t)n * cols, cols, d_mm);
            if ((e = cudaGetLastError()) != cudaSuccess ||
                (e = cudaMemcpyAsync(mm.data(), d_mm, mm.size() * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess)
                return done(ctx->cuda_fail(e, "column ranges"));
            // chunks of columns, last column first; a constant column orders nothing and is left out
            std::vector<ChunkDesc> chunks;
            std::vector<int> chunk_bits;
            ChunkDesc cur{};
            int cur_bits = 0;
            auto flush = [&]() {
                if (!cur.nc) return;
                // columns were added least significant first; the key wants the most significant first
                std::reverse(cur.ccol, cur.ccol + cur.nc);
                std::reverse(cur.cbits, cur.cbits + cur.nc);
                std::reverse(cur.cmin, cur.cmin + cur.nc);
                chunks.push_back(cur);
                chunk_bits.push_back(cur_bits);
                cur = ChunkDesc{};
                cur_bits = 0;
            };
            for (int c = cols - 1; c >= 0; --c) {
                const uint32_t lo = mm[2 * c], hi = mm[2 * c + 1];
                if (lo >= hi) continue;
                const int b = 32 - __builtin_clz(hi - lo);
                if (cur_bits + b > 64) flush();
                cur.ccol[cur.nc] = c;
                cur.cbits[cur.nc] = b;
                cur.cmin[cur.nc] = lo;
                cur.nc++;
                cur_bits += b;
            }
            flush();
            const int kgrid = std::max(1, std::min(ctx->sm_count * 8, (int)((n + 255) / 256)));
            uint32_t* ia = idx0;
            uint32_t* ib = idx1;
            unsigned long long* ka = key0;
            unsigned long long* kb = key1;
            for (size_t k = 0; k < chunks.size(); ++k) {
                key_kernel<<<kgrid, kFinThreads, 0, s>>>(in->d, cols, chunks[k], sorted, n, ka, ia);
                for (int shift = 0; shift < chunk_bits[k]; shift += 8) {
                    SortPass p{ka, ia, kb, ib, shift, n, hist, dtot};
                    hist_kernel<<<grid, kFinThreads, 0, s>>>(p);
                    digit_rows_kernel<<<kDigits, kFinThreads, 0, s>>>(hist, (uint32_t)grid, dtot);
                    scatter_kernel<<<grid, kFinThreads, 0, s>>>(p);
                    std::swap(ka, kb);
                    std::swap(ia, ib);
                }
                sorted = ia;
                std::swap(ia, ib);   // the next chunk's keys go to the other index array
            }
            if (!sorted) {   // every column constant: every row is equal, the table order stands
                iota_kernel<<<kgrid, kFinThreads, 0, s>>>(idx0, n);
                sorted = idx0;
            }
        }
        uint32_t* kept = sorted == idx0 ? idx1 : idx0;
        // rows gathered into sorted order once (into the key arrays' room): the compaction then
        // compares consecutive rows and the projection reads the kept ones from this copy
        const uint32_t* rows_src = in->d;
        if (sorted) {
            uint32_t* sorted_rows = reinterpret_cast<uint32_t*>(key0);
            const int ggrid = std::max(1, std::min<int>(ctx->sm_count * 8, (int)(((uint64_t)n * cols + 255) / 256)));
            gather_rows_kernel<<<ggrid, kFinThreads, 0, s>>>(in->d, cols, sorted, n, sorted_rows);
            rows_src = sorted_rows;
            sorted = nullptr;
        }
        UniqueArgs u{rows_src, cols, d_keep, n_keep, sorted, n, part, kept};
        unique_count_kernel<<<grid, kFinThreads, 0, s>>>(u);
        scan_kernel<<<1, 1024, 0, s>>>(part, (uint32_t)grid, d_total);
        unique_place_kernel<<<grid, kFinThreads, 0, s>>>(u);
        if ((e = cudaGetLastError()) != cudaSuccess) return done(ctx->cuda_fail(e, "distinct launches"));
        uint32_t h_total = 0;
        if ((e = cudaMemcpyAsync(&h_total, d_total, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return done(ctx->cuda_fail(e, "distinct count"));
        m = h_total;
        idx = kept;
        table_src = rows_src;
    }
    const uint64_t start = std::min<uint64_t>((uint64_t)offset, m);
    const uint64_t count = limit < 0 ? m - start : std::min<uint64_t>((uint64_t)limit, m - start);
    const int rc = ctx->table_reserve(out, std::max<uint64_t>(count * n_keep, 1));
    if (rc) return done(rc);
    out->cols = n_keep;
    const int pgrid = std::max(1, std::min<int>(ctx->sm_count * 8, (int)((count * n_keep + 255) / 256)));
    project_kernel<<<pgrid, kFinThreads, 0, s>>>(table_src, cols, d_keep, n_keep, idx, start, count, out->d,
                                                 out->d_rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return done(ctx->cuda_fail(e, "projection launch"));
    return done(WK_SUCCESS);
}

extern "C" int wk_table_filter_bound(wk_ctx* ctx, const wk_table* in, const int32_t* bound_cols,
                                     int32_t n_bound, wk_table* out) {
    using namespace wk;
    if (!ctx || !in || !out || in == out || (!bound_cols && n_bound) || n_bound < 0) return WK_E_BADARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n_bound > 64) return ctx->fail(WK_E_BADARG, "at most 64 bound columns");
    const int cols = in->cols;
    cudaStream_t s = ctx->stream;
    WKF_CUDA(ctx, cudaMemcpyAsync(ctx->h_rows, in->d_rows, 8, cudaMemcpyDeviceToHost, s));
    WKF_CUDA(ctx, cudaStreamSynchronize(s));
    const uint64_t R = ctx->h_rows[0];
    if (cols > 0 && R > in->cap / (uint64_t)cols)
        return ctx->fail(WK_E_CORRUPT, "row count beyond table capacity");
    for (int k = 0; k < n_bound; ++k)
        if (bound_cols[k] < 0 || bound_cols[k] >= cols) return ctx->fail(WK_E_BADARG, "bound column out of range");
    if (R >= (1ull << 32)) return ctx->fail(WK_E_CAPACITY, "table too long for the filter stage");
    int rc = ctx->table_reserve(out, std::max<uint64_t>(R * (uint64_t)std::max(cols, 1), 1));
    if (rc) return rc;
    out->cols = cols;
    if (R == 0 || n_bound == 0) {   // nothing to drop: the table as it is
        if (R) WKF_CUDA(ctx, cudaMemcpyAsync(out->d, in->d, R * (uint64_t)cols * 4, cudaMemcpyDeviceToDevice, s));
        WKF_CUDA(ctx, cudaMemcpyAsync(out->d_rows, in->d_rows, 8, cudaMemcpyDeviceToDevice, s));
        WKF_CUDA(ctx, cudaStreamSynchronize(s));
        return WK_SUCCESS;
    }
    const uint32_t n = (uint32_t)R;
    const int grid = std::max(1, std::min<int>(ctx->sm_count * 4, (int)((n + 2047) / 2048)));
    const size_t bytes = 256 + ((size_t)grid + 2) * 4 + 64;
    int src = ctx->final_scratch_reserve(bytes);
    if (src) return src;
    char* scratch = static_cast<char*>(ctx->d_final_scratch);
    auto done = [&](int code) {
        cudaStreamSynchronize(s);
        return code;
    };
    int32_t* d_cols = reinterpret_cast<int32_t*>(scratch);
    uint32_t* part = reinterpret_cast<uint32_t*>(scratch + 256);
    uint32_t* d_total = part + grid + 1;
    cudaError_t e = cudaMemcpyAsync(d_cols, bound_cols, (size_t)n_bound * 4, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return done(ctx->cuda_fail(e, "filter columns"));
    BoundArgs b{in->d, cols, d_cols, n_bound, n, part, out->d};
    bound_count_kernel<<<grid, kFinThreads, 0, s>>>(b);
    scan_kernel<<<1, 1024, 0, s>>>(part, (uint32_t)grid, d_total);
    bound_place_kernel<<<grid, kFinThreads, 0, s>>>(b);
    if ((e = cudaGetLastError()) != cudaSuccess) return done(ctx->cuda_fail(e, "filter launches"));
    uint32_t h_total = 0;
    if ((e = cudaMemcpyAsync(&h_total, d_total, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return done(ctx->cuda_fail(e, "filter count"));
    ctx->h_rows[1] = h_total;
    e = cudaMemcpyAsync(out->d_rows, ctx->h_rows + 1, 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return done(ctx->cuda_fail(e, "filter row count"));
    return done(WK_SUCCESS);
}
