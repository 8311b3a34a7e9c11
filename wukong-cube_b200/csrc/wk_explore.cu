// Exploration launch for sm_100a: one pattern level over a whole table (single query) or over
// the tables of every query of a batch.
//
// The reference chains five kernels, a Thrust scan and two host syncs per pattern
// (gpu_engine_cuda.hpp:169-177, gpu_hash.cu:96-836).  Here CTAs claim 512-row tiles from a
// device counter and, per tile:
//   1. start a TMA bulk copy (cp.async.bulk + mbarrier) of the tile's rows into shared memory
//      and, while it is in flight, read each row's start column straight from global memory;
//   2. probe the key table with groups of L lanes, one 16-byte slot per lane, four rows per group
//      in flight; since the static store only ever inserts into the first empty slot
//      (kvstore.hpp:163-180, segment_rdf_dgraph.hpp:216-233) an empty slot ends the search, so
//      most probes read one 32- or 64-byte slice of the bucket;
//   3. count each row's output rows: the neighbour count (start / known_to_unknown) or a 0/1
//      membership flag (known_to_known / known_to_const: a group ballot over the first entries,
//      then a binary search of the rest of a sorted list);
//   4. scan the counts (block scan + warp-parallel decoupled look-back, 64-bit positions);
//   5. write the rows whose lists are short through shared memory with coalesced stores, in
//      row-major then edge order (what the CPU engine appends, sparql.hpp:328-370), and hand
//      rows with long lists to the slice launch as kHeavyChunk-row slices so a hub vertex is
//      spread over every CTA instead of holding one.
// Sizes are read from device memory, so levels chain without a host round trip; an output that
// would not fit sets kErrOverflow and records the size needed instead of writing.
#include <cuda_runtime.h>

#include "wk_device.cuh"
#include "wk_explore.h"

namespace wk {
namespace {
using namespace dev;

template <int L>
__global__ void __launch_bounds__(kStepThreads, 3) explore_kernel(const ExploreArgs a, int chunk_rows) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ unsigned long long s_tile, s_excl, s_alg, s_sd;
    __shared__ uint64_t s_warp[kStepThreads / 32];
    __shared__ int s_has_heavy;
    constexpr int kGroups = kStepThreads / L;
    constexpr int kBatches = kTileRows / (kGroups * kUnroll);
    static_assert(kBatches * kGroups * kUnroll == kTileRows, "tile shape");

    const int wi = a.virtual_rows ? 0 : a.w_in, wo = a.w_out;
    uint32_t* s_in = reinterpret_cast<uint32_t*>(smem);
    uint64_t* s_pre = reinterpret_cast<uint64_t*>(s_in + ((kTileRows * wi + 3) & ~3));
    uint64_t* s_lpre = s_pre + kTileRows + 2;
    uint64_t* s_off = s_lpre + kTileRows + 2;
    uint64_t* s_pos = s_off + kTileRows;
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_pos + chunk_rows);
    uint32_t* s_lcnt = s_cnt + kTileRows;
    uint32_t* s_q = s_lcnt + kTileRows;
    uint32_t* s_meta = s_q + kTileRows;   // op | cin << 8 | cout << 16
    uint32_t* s_out = s_meta + kTileRows;

    const unsigned epoch = *(volatile unsigned*)&a.ctl->epoch;
    uint64_t R = a.virtual_rows ? a.n_queries : *(volatile const uint64_t*)a.in_rows;
    if (!a.virtual_rows && R > a.in_cap_rows) R = a.in_cap_rows;
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
        const uint32_t* src = a.in + r0 * (uint64_t)wi;

        // 1. rows -> shared memory, asynchronously; owners; zero counts
        if (threadIdx.x == 0) {
            if (wi) {
                const unsigned bytes = (unsigned)(((uint64_t)n * wi * 4 + 15) & ~15ull);
                mbar_expect_tx(&s_bar, bytes);
                tma_load_1d(s_in, src, bytes, &s_bar);
            }
            s_alg = 0;
            s_sd = 0;
            s_has_heavy = 0;
        }
        for (int i = threadIdx.x; i < n; i += kStepThreads) {
            s_q[i] = a.virtual_rows ? (uint32_t)(r0 + i) : (a.owner_in ? __ldg(a.owner_in + r0 + i) : 0u);
            s_cnt[i] = 0;
        }
        __syncthreads();

        // 2-3. probe and count; start columns straight from global memory
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
                const StepDesc* d = a.desc ? a.desc + (valid[u] ? s_q[row[u]] : 0) : &a.one;
                op[u] = valid[u] ? d->op : kXDone;
                if (op[u] == kXDone) valid[u] = false;
                const SegDesc* sg = &d->seg;
                target[u] = d->end_const;
                if (op[u] == kXStart) {
                    key[u] = d->start_key;
                } else {
                    const uint32_t* rin = src + (uint64_t)row[u] * wi;
                    const uint32_t cur = valid[u] ? __ldg(rin + d->cs) : kBlankId;
                    if (op[u] == kXK2K && valid[u]) target[u] = __ldg(rin + d->ce);
                    if (op[u] == kXK2U && d->type_index) {
                        // get_index(cur, IN) (sparql.hpp:342-345); only 17-bit ids can be keys
                        key[u] = make_key(0, cur, kIn);
                        sg = &a.seg_index[kIn];
                        if (cur >= (1u << kNbitsIdx)) valid[u] = false;
                    } else {
                        key[u] = make_key(cur, d->pid, d->dir);
                        if (cur == 0) sg = &a.seg_index[d->dir & 1];   // vid 0 names the index
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
                has[u] = valid[u] && deg[u] > 0 && (op[u] == kXK2K || op[u] == kXK2C);
            }
            group_member<L>(a.store.edges, off, deg, target, has, a.sorted_lists != 0, found);
            if (h == 0) {
                unsigned long long alg = 0, sd = 0;
#pragma unroll
                for (int u = 0; u < kUnroll; ++u)
                    if (valid[u]) {
                        const bool filt = op[u] == kXK2K || op[u] == kXK2C;
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
        for (int i = threadIdx.x; i < n; i += kStepThreads) {
            const uint32_t c = s_cnt[i];
            const bool heavy = c > (uint32_t)kHeavyRows;
            s_lcnt[i] = heavy ? 0u : c;
            if (heavy) s_has_heavy = 1;
        }
        __syncthreads();

        // 4. positions
        const uint64_t total = block_scan(s_cnt, s_pre, n, s_warp);
        const uint64_t ltotal = s_has_heavy ? block_scan(s_lcnt, s_lpre, n, s_warp) : total;
        if (threadIdx.x < 32) {
            const uint64_t ex = lookback_warp(a.status, a.ctl, tile, total, epoch);
            if (threadIdx.x == 0) {
                s_excl = ex;
                atomicAdd(&a.ctl->alg_bytes, s_alg);
                atomicAdd(&a.ctl->sum_deg, s_sd);
            }
        }
        if (wi) mbar_wait(&s_bar, phase, &a.ctl->err);   // the tile's rows are in shared memory
        phase ^= wi ? 1u : 0u;
        __syncthreads();
        const uint64_t excl = s_excl;
        if (tile == ntiles - 1 && threadIdx.x == 0) *a.out_rows = excl + total;
        const bool fits = excl + total <= a.out_cap_rows;
        if (!fits && threadIdx.x == 0) {
            atomicOr(&a.ctl->err, kErrOverflow);
            atomicMax(&a.ctl->need, (unsigned long long)(excl + total));
        }
        // per-query output ranges: each run of one query's rows adds (end - start)
        if (a.qcount && fits) {
            for (int i = threadIdx.x; i < n; i += kStepThreads) {
                const uint32_t q = s_q[i];
                if (i == 0 || s_q[i - 1] != q) {
                    atomicMin(a.qfirst + q, (unsigned long long)(excl + s_pre[i]));
                    atomicAdd(a.qcount + q, (unsigned long long)(0 - (excl + s_pre[i])));
                }
                if (i == n - 1 || s_q[i + 1] != q) atomicAdd(a.qcount + q, (unsigned long long)(excl + s_pre[i + 1]));
            }
        }
        // long lists -> slices on the queue (fields first, then the epoch tag)
        if (s_has_heavy && fits) {
            for (int i = threadIdx.x; i < n; i += kStepThreads) {
                const uint32_t c = s_cnt[i];
                if (c <= (uint32_t)kHeavyRows) continue;
                const uint32_t nch = (c + kHeavyChunk - 1) / kHeavyChunk;
                const unsigned long long at = atomicAdd(&a.ctl->heavy_n, (unsigned long long)nch);
                for (uint32_t k = 0; k < nch; ++k) {
                    if (at + k >= a.heavy_cap) {
                        atomicOr(&a.ctl->err, kErrOverflow);
                        break;
                    }
                    HeavyItem* it = a.heavy + at + k;
                    it->in_row = r0 + i;
                    it->off = s_off[i] + (uint64_t)k * kHeavyChunk;
                    it->out_pos = excl + s_pre[i] + (uint64_t)k * kHeavyChunk;
                    it->count = min((uint32_t)kHeavyChunk, c - k * kHeavyChunk);
                    it->q = s_q[i];
                    __threadfence();
                    *(volatile uint32_t*)&it->tag = epoch;
                }
            }
        }

        // 5. write the short-list rows: stride w_out, zero past the query's width
        if (fits && ltotal) {
            const bool contiguous = !s_has_heavy;
            const uint64_t* lp = contiguous ? s_pre : s_lpre;
            for (uint64_t c0 = 0; c0 < ltotal; c0 += chunk_rows) {
                const int m = (int)min((uint64_t)chunk_rows, ltotal - c0);
                for (int j = threadIdx.x; j < m; j += kStepThreads) {
                    const uint64_t o = c0 + j;
                    int lo = 0, hi = n;   // lp[lo] <= o < lp[hi]
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (lp[mid] <= o) lo = mid; else hi = mid;
                    }
                    const uint64_t k = o - lp[lo];
                    const uint32_t meta = s_meta[lo];
                    const int opv = meta & 0xFF, cin = (meta >> 8) & 0xFF;
                    uint32_t* dst = s_out + (size_t)j * wo;
                    const uint32_t* sr = s_in + lo * wi;
                    int c = 0;
                    if (opv != kXStart)
                        for (; c < cin; ++c) dst[c] = sr[c];
                    if (opv == kXStart || opv == kXK2U) dst[c++] = __ldg(a.store.edges + s_off[lo] + k);
                    for (; c < wo; ++c) dst[c] = 0;
                    const uint64_t pos = excl + s_pre[lo] + k;
                    s_pos[j] = pos;
                    if (a.owner_out) a.owner_out[pos] = s_q[lo];
                }
                __syncthreads();
                if (contiguous) {
                    store_words(a.out + (excl + c0) * wo, s_out, (uint64_t)m * wo);
                } else {
                    for (int e = threadIdx.x; e < m * wo; e += kStepThreads) {
                        const int j = e / wo, c = e - j * wo;
                        a.out[s_pos[j] * wo + c] = s_out[e];
                    }
                }
                __syncthreads();
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {   // this tile's slices are all reserved
            __threadfence();
            atomicAdd(&a.ctl->tiles_done, 1ull);
        }
    }

    // Out of tiles: write queued long-list slices until every tile is done and the queue is
    // drained.  A claimed index either gets reserved by a tile still running (wait for its
    // tag) or lies past the final count (stop).  Every wait is bounded.
    __syncthreads();   // every thread has read the last s_tile before it is reused
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long idx = atomicAdd(&a.ctl->heavy_claim, 1ull);
            int state = 0;
            unsigned long long spins = 0;
            for (;;) {
                unsigned long long hn = *(volatile unsigned long long*)&a.ctl->heavy_n;
                if (idx < hn) {
                    if (idx >= a.heavy_cap) {
                        state = 2;   // the queue overflowed; kErrOverflow is already set
                        break;
                    }
                    if (*(volatile uint32_t*)&a.heavy[idx].tag == epoch) {
                        __threadfence();
                        state = 1;
                        break;
                    }
                } else if (*(volatile unsigned long long*)&a.ctl->tiles_done >= ntiles) {
                    __threadfence();
                    hn = *(volatile unsigned long long*)&a.ctl->heavy_n;
                    if (idx >= hn) {
                        state = 2;
                        break;
                    }
                    continue;
                }
                if (++spins > kSpinLimit) {
                    atomicOr(&a.ctl->err, kErrTimeout);
                    state = 2;
                    break;
                }
                if (spins > 32) __nanosleep(64);
            }
            s_tile = state == 1 ? idx : ~0ull;
        }
        __syncthreads();
        const unsigned long long idx = s_tile;
        if (idx == ~0ull) break;
        const HeavyItem* it = a.heavy + idx;
        const uint64_t in_row = __ldcg((const unsigned long long*)&it->in_row);
        const uint64_t off = __ldcg((const unsigned long long*)&it->off);
        const uint64_t out_pos = __ldcg((const unsigned long long*)&it->out_pos);
        const uint32_t count = __ldcg((const unsigned int*)&it->count);
        const uint32_t q = __ldcg((const unsigned int*)&it->q);
        const StepDesc* d = a.desc ? a.desc + q : &a.one;
        const int opv = d->op, cin = d->cin;
        if (opv != kXStart && threadIdx.x < cin) s_out[threadIdx.x] = __ldg(a.in + in_row * (uint64_t)a.w_in + threadIdx.x);
        __syncthreads();
        const int ecol = opv == kXStart ? 0 : cin;
        const uint64_t ne = (uint64_t)count * wo;
        uint32_t* dst = a.out + out_pos * wo;
        for (uint64_t e = threadIdx.x; e < ne; e += kStepThreads) {
            const uint64_t j = e / wo;
            const int c = (int)(e - j * wo);
            uint32_t v = 0;
            if (c < ecol) v = s_out[c];
            else if (c == ecol) v = __ldg(a.store.edges + off + j);
            dst[e] = v;
        }
        if (a.owner_out)
            for (uint32_t j = threadIdx.x; j < count; j += kStepThreads) a.owner_out[out_pos + j] = q;
        __syncthreads();
    }
    exit_protocol(a.ctl, a.status, epoch, a.heavy ? &a.heavy[0].tag : nullptr,
                  sizeof(HeavyItem) / sizeof(uint32_t), a.heavy ? a.heavy_cap : 0);
}

template <int L>
cudaError_t set_attr(int bytes) {
    return cudaFuncSetAttribute(explore_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace

size_t explore_smem_bytes(int w_in, int w_out, int* chunk_rows) {
    int chunk = 16 * 1024 / (w_out > 0 ? w_out * 4 : 4);
    if (chunk > 1024) chunk = 1024;
    if (chunk < 64) chunk = 64;
    size_t in_words = ((size_t)kTileRows * w_in + 3) & ~(size_t)3;
    size_t bytes = in_words * 4 + 2 * (kTileRows + 2) * 8 + kTileRows * 8 + (size_t)chunk * 8 +
                   4 * kTileRows * 4 + (size_t)chunk * w_out * 4;
    if (chunk_rows) *chunk_rows = chunk;
    return bytes;
}

cudaError_t explore_kernel_attrs() {
    const int bytes = (int)explore_smem_bytes(32, 32, nullptr);
    cudaError_t e;
    if ((e = set_attr<2>(bytes)) != cudaSuccess) return e;
    if ((e = set_attr<4>(bytes)) != cudaSuccess) return e;
    return set_attr<8>(bytes);
}

int explore_blocks_per_sm(int w_in, int w_out, int lanes) {
    size_t smem = explore_smem_bytes(w_in, w_out, nullptr);
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    if (lanes == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<2>, kStepThreads, smem);
    if (lanes == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<4>, kStepThreads, smem);
    if (lanes == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<8>, kStepThreads, smem);
    return (e == cudaSuccess && nb > 0) ? nb : 1;
}

cudaError_t launch_explore(const ExploreArgs& a, int grid, cudaStream_t s) {
    int chunk = 0;
    const int wi = a.virtual_rows ? 0 : a.w_in;
    size_t smem = explore_smem_bytes(wi, a.w_out, &chunk);
    if (grid < 1) grid = 1;
    switch (a.lanes) {
    case 2: explore_kernel<2><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    case 8: explore_kernel<8><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    default: explore_kernel<4><<<grid, kStepThreads, smem, s>>>(a, chunk); break;
    }
    return cudaGetLastError();
}

}  // namespace wk
