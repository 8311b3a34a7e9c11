// Small kernels of the single-query path: the start-list copy of index_to_unknown /
// const_to_unknown, and the upload-time check that every neighbour list is sorted.
//
// The exploration launch itself is in wk_explore.cu.
#include <cuda_runtime.h>

#include "wk_device.cuh"
#include "wk_kernels.h"

namespace wk {
namespace {
using namespace dev;

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
    uint64_t off, sz;
    list_of_ptr(s_ptr, a.store.n_edges, &a.ctl->err, &off, &sz);
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
    if (off & kInlineTag) {   // a one-entry list kept in its key's slot
        if (n && blockIdx.x == 0 && threadIdx.x == 0) a.out[0] = (uint32_t)off;
        return;
    }
    // grid-stride copy, eight loads in flight per thread before their stores (the list starts
    // at any word, so the words are moved one by one; each warp access is 128 contiguous bytes)
    const uint32_t* srcp = a.store.edges + off + b;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (; i + 7 * stride < n; i += 8 * stride) {
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldg(srcp + i + k * stride);
#pragma unroll
        for (int k = 0; k < 8; ++k) a.out[i + k * stride] = v[k];
    }
    for (; i < n; i += stride) a.out[i] = __ldg(srcp + i);
}

// Checks that every key's list is strictly ascending (the loader's sort + dedup), which lets
// the filters binary-search long lists.
// One warp per slot; the lanes walk the slot's list together (coalesced), so a hub list costs
// len/32 steps of one warp instead of len steps of one thread.
__global__ void sorted_check_kernel(const Slot* slots, uint64_t n_slots, const uint32_t* edges,
                                    uint64_t n_edges, unsigned* unsorted) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t i = blockIdx.x * (uint64_t)(blockDim.x / 32) + threadIdx.x / 32; i < n_slots; i += warps) {
        if ((i & (kAssoc - 1)) == kAssoc - 1) continue;   // chain link
        const Slot s = slots[i];
        if (s.key == 0) continue;
        if (ptr_is_inline(s.ptr)) continue;   // a one-entry list (none before inline_kernel)
        const uint64_t off = ptr_off(s.ptr), sz = ptr_size(s.ptr);
        if (off + sz > n_edges) {
            if (lane == 0) atomicOr(unsorted, 2u);
            continue;
        }
        bool bad = false;
        for (uint64_t k = 1 + lane; k < sz && !bad; k += 32) bad = __ldg(edges + off + k - 1) >= __ldg(edges + off + k);
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(unsorted, 1u);
    }
}

// One-entry lists into their keys' own pointer words (see kInlinePtrType): for every data slot
// (slots 0-6) whose list has one entry, the original pointer word goes to the side table
// `orig` (slot index, pointer word; wk_store_export puts them back) and the slot's pointer word
// becomes the entry with the inline type.  With orig null the kernel only counts such slots
// (into *n) and whether any pointer word already carries type 3 (into *clash; the store is then
// refused, since that type cannot be told apart).
__global__ void inline_kernel(Slot* slots, uint64_t n_slots, const uint32_t* edges, uint64_t n_edges,
                              unsigned long long* n, unsigned* clash, uint64_t* orig) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_slots; i += stride) {
        if ((i & (kAssoc - 1)) == kAssoc - 1) continue;   // chain link
        const Slot sl = slots[i];
        if (sl.key == 0) continue;
        if (!orig && ptr_is_inline(sl.ptr)) atomicOr(clash, 1u);
        if ((sl.ptr >> 62) != 0 || ptr_size(sl.ptr) != 1 || ptr_off(sl.ptr) >= n_edges) continue;
        const unsigned long long at = atomicAdd(n, 1ull);
        if (!orig) continue;
        orig[2 * at] = i;
        orig[2 * at + 1] = sl.ptr;
        slots[i].ptr = make_inline_ptr(__ldg(edges + ptr_off(sl.ptr)));
    }
}

// Random-read calibration: every thread makes `per` independent 16-byte reads at pseudo-random
// 16-byte-aligned positions of buf (the splitmix64 finaliser of thread and read index), eight in
// flight at a time, in the probes' own load form (no L1 allocation, first out of L2).  With buf
// much larger than L2 each read moves a whole DRAM line (about 123 B measured), as a probe of a
// distinct key does.  The words read are summed and stored only if the sum is one the fill
// cannot produce, which keeps the reads live.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__global__ void __launch_bounds__(256) random_read_kernel(const uint4* __restrict__ buf, uint64_t n16,
                                                          int per, uint64_t seed, uint32_t* sink) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t acc = 0;
#pragma unroll 8
    for (int i = 0; i < per; ++i) {
        const uint4 v = dev::load16_once(buf + mix64(seed + t * 0x9e3779b97f4a7c15ull + (uint64_t)i) % n16);
        acc += v.x + v.y + v.z + v.w;
    }
    if (acc == 1u) sink[0] = acc;
}

}  // namespace

cudaError_t launch_random_reads(const void* buf, uint64_t bytes, int per, uint64_t seed,
                                uint32_t* sink, int grid, cudaStream_t s) {
    random_read_kernel<<<grid, 256, 0, s>>>((const uint4*)buf, bytes / 16, per, seed, sink);
    return cudaGetLastError();
}

cudaError_t launch_list(const ListArgs& a, int grid, cudaStream_t s) {
    if (grid < 1) grid = 1;
    list_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sorted_check(const DevStore& st, unsigned* d_flag, cudaStream_t s) {
    sorted_check_kernel<<<4096, 256, 0, s>>>(st.slots, st.n_buckets * kAssoc, st.edges, st.n_edges, d_flag);
    return cudaGetLastError();
}

cudaError_t launch_inline(const DevStore& st, unsigned long long* n, unsigned* clash, uint64_t* orig,
                          cudaStream_t s) {
    if (st.n_buckets)
        inline_kernel<<<4096, 256, 0, s>>>(const_cast<Slot*>(st.slots), st.n_buckets * kAssoc, st.edges, st.n_edges,
                                           n, clash, orig);
    return cudaGetLastError();
}

cudaError_t small_kernel_attrs() {
    cudaError_t e = use_max_shared_carveout(list_kernel);
    return e != cudaSuccess ? e : use_max_shared_carveout(sorted_check_kernel);
}

}  // namespace wk