// Patterns with an unknown predicate (the versatile operators of the reference's default
// VERSATILE build, sparql.hpp:554-739), on a store that holds every vertex's predicate list
// [v|PREDICATE_ID|d] (wk_gstore_build_ex):
//   ?X ?P ?Y (known_unknown_unknown): every row times its start's (p, y) pairs;
//   ?X ?P C  (known_unknown_const):   every row times each predicate of its start reaching C;
//   C ?P ?X  (const_unknown_unknown): the (p, x) pairs of the constant;
//   C1 ?P C2 (const_unknown_const):   the predicates of C1 that reach C2.
// Each row reads its vertex's predicate list and then its list for each of those predicates,
// so a row's output count is only known after a walk of several lists.  Two launches at full
// occupancy, one thread per row:
//   1. count: the row's output rows; the last CTA to finish scans the chunk totals, checks the
//      output capacity (overflow sets kErrOverflow and the rows needed) and sets the row count;
//   2. write: each CTA scans its chunk's counts into positions, and each thread walks its row's
//      lists again and writes its rows: row-major, then predicate-list order, then list order,
//      the order the reference appends them in.
// A vertex's predicates are few (the predicates of the data set), so one thread per row does
// not leave work unbalanced the way a hub's neighbour list would.  The constant forms run the
// same launches over one virtual row.
#include <cuda_runtime.h>

#include <algorithm>

#include "wk_device.cuh"
#include "wk_versatile.h"

namespace wk {
namespace {
using namespace dev;

constexpr int kVThreads = 256;

__device__ __forceinline__ uint64_t vers_rows(const VersArgs& a) {
    if (a.virtual_row) return 1;
    const uint64_t R = *(volatile const uint64_t*)a.in_rows;
    return R > a.in_cap_rows ? 0 : R;   // past capacity: the step before overflowed
}

// Segment of normal keys [v|pid|dir]: a binary search of the store's predicate segments.
__device__ __forceinline__ bool pred_seg(const VersArgs& a, uint32_t pid, int dir, SegDesc* out) {
    const uint32_t want = pid * 2 + (uint32_t)dir;
    uint32_t lo = 0, hi = a.n_pseg;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.pseg[mid].key < want) lo = mid + 1; else hi = mid;
    }
    if (lo >= a.n_pseg || a.pseg[lo].key != want) return false;
    *out = a.pseg[lo].seg;
    return true;
}

// The list of key (vid, pid, dir): offset and length (0 when absent).
__device__ __forceinline__ void list_of(const VersArgs& a, uint64_t vid, uint32_t pid, const SegDesc& sg,
                                        uint64_t* off, uint64_t* deg) {
    *off = 0;
    *deg = 0;
    const uint64_t key = make_key(vid, pid, a.dir);
    if (sg.num_buckets == 0 || key == 0) return;
    const uint64_t p = thread_probe(a.store, key, bucket_of(key, sg), &a.ctl->err);
    list_of_ptr(p, a.store.n_edges, &a.ctl->err, off, deg);   // *off may be a tagged entry
}

__device__ __forceinline__ uint32_t row_start(const VersArgs& a, uint64_t r) {
    return a.virtual_row ? a.start_const : __ldg(a.in + r * (uint64_t)a.w_in + a.cs);
}

// Output rows of a row whose start vertex is `cur`; with `write`, also writes them from
// output row `at` on.
__device__ uint64_t walk_row(const VersArgs& a, uint64_t r, uint32_t cur, bool write, uint64_t at) {
    const bool to_const = a.op == kVKUC || a.op == kVCUC;
    uint64_t poff, npred;
    list_of(a, cur, kPredicateId, a.vp_seg, &poff, &npred);
    uint64_t n = 0;
    for (uint64_t k = 0; k < npred; ++k) {
        const uint32_t p = list_at(a.store.edges, poff, k);
        SegDesc sg;
        if (!pred_seg(a, p, a.dir, &sg)) continue;
        uint64_t off, deg;
        list_of(a, cur, p, sg, &off, &deg);
        if (to_const) {
            if (!deg || !thread_member(a.store.edges, off, deg, a.end_const, a.sorted_lists != 0)) continue;
            if (write) {   // row ++ [p]
                uint32_t* dst = a.out + (at + n) * (uint64_t)a.w_out;
                const uint32_t* src = a.in + r * (uint64_t)a.w_in;
                for (int c = 0; c < a.cin; ++c) dst[c] = __ldg(src + c);
                dst[a.cin] = p;
            }
            ++n;
        } else {
            if (write) {   // row ++ [p, y] for every neighbour y
                const uint32_t* src = a.in + r * (uint64_t)a.w_in;
                for (uint64_t j = 0; j < deg; ++j) {
                    uint32_t* dst = a.out + (at + n + j) * (uint64_t)a.w_out;
                    for (int c = 0; c < a.cin; ++c) dst[c] = __ldg(src + c);
                    dst[a.cin] = p;
                    dst[a.cin + 1] = list_at(a.store.edges, off, j);
                }
            }
            n += deg;
        }
    }
    return n;
}

__device__ __forceinline__ void vchunk(uint64_t R, uint64_t* lo, uint64_t* hi) {
    const uint64_t c = (R + gridDim.x - 1) / gridDim.x;
    *lo = min(R, (uint64_t)blockIdx.x * c);
    *hi = min(R, *lo + c);
}

__global__ void __launch_bounds__(kVThreads) vers_count_kernel(const VersArgs a) {
    __shared__ uint64_t s_warp[kVThreads / 32];
    __shared__ uint64_t s_carry;
    __shared__ int s_last;
    const uint64_t R = vers_rows(a);
    uint64_t lo, hi;
    vchunk(R, &lo, &hi);
    uint64_t sum = 0;
    for (uint64_t r = lo + threadIdx.x; r < hi; r += kVThreads) {
        const uint32_t cur = row_start(a, r);
        const uint64_t n = cur == kBlankId ? 0 : walk_row(a, r, cur, false, 0);
        a.pos[r] = n;
        sum += n;
    }
    const uint64_t ex = block_exclusive_sum<kVThreads>(sum, s_warp);
    if (threadIdx.x == kVThreads - 1) a.part[blockIdx.x] = ex + sum;
    // the last CTA to finish scans the chunk totals
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        s_last = atomicAdd(&a.ctl->flat_done, 1u) == gridDim.x - 1;
        if (s_last) a.ctl->flat_done = 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < gridDim.x; b0 += kVThreads) {
        const uint32_t i = b0 + threadIdx.x;
        const uint64_t x = i < gridDim.x ? __ldcg((const unsigned long long*)a.part + i) : 0;
        const uint64_t e = block_exclusive_sum<kVThreads>(x, s_warp);
        const uint64_t carry = s_carry;
        if (i < gridDim.x) a.part[i] = carry + e;
        __syncthreads();
        if (threadIdx.x == kVThreads - 1) s_carry = carry + e + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint64_t total = s_carry;
        a.part[gridDim.x] = total;
        if (total > a.out_cap_rows) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)total);
            *a.out_rows = 0;
        } else {
            *a.out_rows = total;
        }
    }
}

__global__ void __launch_bounds__(kVThreads) vers_write_kernel(const VersArgs a) {
    __shared__ uint64_t s_warp[kVThreads / 32];
    __shared__ uint64_t s_carry;
    const uint64_t R = vers_rows(a);
    if (a.part[gridDim.x] > a.out_cap_rows) return;
    uint64_t lo, hi;
    vchunk(R, &lo, &hi);
    if (threadIdx.x == 0) s_carry = a.part[blockIdx.x];
    __syncthreads();
    for (uint64_t r0 = lo; r0 < hi; r0 += kVThreads) {
        const uint64_t r = r0 + threadIdx.x;
        const uint64_t c = r < hi ? a.pos[r] : 0;
        const uint64_t ex = block_exclusive_sum<kVThreads>(c, s_warp);
        const uint64_t at = s_carry + ex;
        if (c) walk_row(a, r, row_start(a, r), true, at);
        __syncthreads();
        if (threadIdx.x == kVThreads - 1) s_carry = at + c;
        __syncthreads();
    }
}

}  // namespace

int vers_grid(uint64_t rows, int sm_count) {
    const uint64_t want = (rows + kVThreads - 1) / kVThreads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count * 8));
}

cudaError_t launch_versatile(const VersArgs& a, int grid, cudaStream_t s) {
    vers_count_kernel<<<grid, kVThreads, 0, s>>>(a);   // its last CTA scans the totals
    vers_write_kernel<<<grid, kVThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t versatile_kernel_attrs() {
    cudaError_t e = use_max_shared_carveout(vers_count_kernel);
    return e != cudaSuccess ? e : use_max_shared_carveout(vers_write_kernel);
}

}  // namespace wk
