// Exploration launch for sm_100a: one pattern level over a whole table (single query) or over
// the tables of every query of a batch.
//
// The reference chains five kernels, a Thrust scan and two host syncs per pattern
// (gpu_engine_cuda.hpp:169-177, gpu_hash.cu:96-836).  Here CTAs claim 256-row tiles from a
// device counter, two at a time (the probes of the next tile run while the current one waits for
// its position), and per tile:
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
//      rows with long lists to a device queue as kHeavyChunk-row slices that CTAs out of tiles
//      drain, so a hub vertex is spread over every CTA instead of holding one.
// Sizes are read from device memory, so levels chain without a host round trip; an output that
// would not fit sets kErrOverflow and records the size needed instead of writing.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/wukong_b200.h"
#include "wk_device.cuh"
#include "wk_explore.h"

namespace wk {

// Optional per-phase cycle counters (build with -DWK_PHASE_TIMING): thread 0 of every CTA adds
// the clock64() time spent in each phase of the launch; read with wk_debug_phase_cycles.
__device__ unsigned long long g_phase_cycles[kPhaseSlots];

namespace {
using namespace dev;

#ifdef WK_PHASE_TIMING
__shared__ unsigned long long s_ph[kPhaseSlots];
__shared__ long long s_ph_t;
#define WK_PH_DECL                                              \
    if (threadIdx.x < kPhaseSlots) s_ph[threadIdx.x] = 0;       \
    if (threadIdx.x == 0) s_ph_t = clock64();
#define WK_PH(k)                                                \
    do {                                                        \
        if (threadIdx.x == 0) {                                 \
            const long long t_ = clock64();                     \
            s_ph[k] += (unsigned long long)(t_ - s_ph_t);       \
            s_ph_t = t_;                                        \
        }                                                       \
    } while (0)
#define WK_PH_FLUSH                                                                              \
    do {                                                                                         \
        __syncthreads();                                                                         \
        if (threadIdx.x < kPhaseSlots) atomicAdd(&g_phase_cycles[threadIdx.x], s_ph[threadIdx.x]); \
    } while (0)
#else
#define WK_PH_DECL
#define WK_PH(k) \
    do {         \
    } while (0)
#define WK_PH_FLUSH \
    do {            \
    } while (0)
#endif

// The step every row of a finished query runs: nothing.
__constant__ StepDesc c_done = {{0, 0, 0, 0}, 0, 0, 0, kXDone, 0, 0, 0, 0, 0, 0, 0, 0};

// Rows with more output rows than this are written as slices from the queue.  At most 2^23, so
// a tile's short-row outputs (256 rows) stay below 2^31 and their scan fits 32 bits.
__device__ __forceinline__ uint32_t slice_threshold(const ExploreArgs& a) {
    return a.slice_rows ? min(max(a.slice_rows, (uint32_t)kMinSliceRows), 1u << 23) : (uint32_t)kHeavyRows;
}

// Polls of a bounded wait on another CTA (look-back, slice queue) before it gives up.
__device__ __forceinline__ unsigned long long spin_limit(const ExploreArgs& a) {
    return a.spin_limit ? a.spin_limit : kDefaultSpinLimit;
}

// Step of query q at this launch.
__device__ __forceinline__ const StepDesc* step_desc(const ExploreArgs& a, uint32_t q) {
    if (!a.desc) return &a.one;
    if (!a.desc_stride) return a.desc + q;
    const uint32_t st = a.iter - __ldg(a.q_admit + q);
    return st < a.desc_stride ? a.desc + (size_t)q * a.desc_stride + st : &c_done;
}

// How a launch's rows are cut into tiles: kTileRows-row tiles, then (when the status array has
// room for them) the last rows in kTailTileRows-row tiles, at most kTailRowsPerCta rows per CTA
// of the grid.  Tiles are claimed in order, so the small ones come last: they shorten the wait
// of CTAs that run out of tiles for the last ones to finish.
constexpr int kTailTileRows = 64;
constexpr int kTailRowsPerCta = 128;
struct Tiling {
    uint64_t ntiles, nbig, big_rows;
    __device__ __forceinline__ uint64_t r0(uint64_t t) const {
        return t < nbig ? t * kTileRows : big_rows + (t - nbig) * kTailTileRows;
    }
    __device__ __forceinline__ int rows(uint64_t t, uint64_t R) const {
        return (int)min((uint64_t)(t < nbig ? kTileRows : kTailTileRows), R - r0(t));
    }
};

__device__ __forceinline__ Tiling make_tiling(uint64_t R, uint64_t cap_tiles) {
    Tiling T;
    T.nbig = (R + kTileRows - 1) / kTileRows;
    T.big_rows = T.nbig * kTileRows;
    T.ntiles = T.nbig;
    const uint64_t tail = min(R, (uint64_t)kTailRowsPerCta * gridDim.x);
    const uint64_t big = (R - tail) / kTileRows;   // whole big tiles before the tail
    const uint64_t nt = big + (R - big * kTileRows + kTailTileRows - 1) / kTailTileRows;
    if (nt <= cap_tiles) {
        T.nbig = big;
        T.big_rows = big * kTileRows;
        T.ntiles = nt;
    }
    return T;
}

// Per-tile state kept in shared memory while the tile is between its front and back halves.
struct TileState {
    unsigned long long tile;
    unsigned long long r0;       // its first row
    unsigned long long total;    // output rows of the tile
    unsigned long long ltotal;   // output rows written by the tile itself (short lists)
    int n;
    int has_heavy;
};

// Words of one tile buffer: its rows (rounded to 16 bytes, the TMA copy's unit), pre and off
// (64-bit), lpre (kTileRows + 4 words, so the next buffer starts on 16 bytes) and three
// per-row words.
__host__ __device__ constexpr size_t tile_buf_words(int wi) {
    return (((size_t)kTileRows * wi + 3) & ~(size_t)3) + 2 * (kTileRows + 2) + 2 * kTileRows + (kTileRows + 4) +
           3 * kTileRows;
}
static_assert(tile_buf_words(1) % 4 == 0, "tile buffers start on 16 bytes");

// Widest input rows the launch's shared-memory attribute is set for (explore_kernel_attrs): two
// tile buffers of 100-column rows are 221 KB of the 227 KB a CTA may have.
constexpr int kMaxSmemCols = 100;

// Shared-memory arrays of one tile buffer (tile_buf_words() words).
struct TileBuf {
    uint32_t* in;     // kTileRows * w_in words (TMA destination)
    uint64_t* pre;    // kTileRows + 2: exclusive scan of cnt, pre[n] = total
    uint64_t* off;    // kTileRows: first edge of each row's list
    uint32_t* lpre;   // kTileRows + 4: exclusive scan of the short rows' counts (0 for a row
                      // whose list goes to the slice queue); filled only when the tile has one
    uint32_t* cnt;    // kTileRows: output rows of each input row
    uint32_t* q;      // kTileRows: owner query
    uint32_t* meta;   // kTileRows: op | cin << 8 | cout << 16
};

__device__ __forceinline__ TileBuf tile_buf(uint32_t* base, int wi) {
    TileBuf b;
    b.in = base;
    b.pre = reinterpret_cast<uint64_t*>(base + (((size_t)kTileRows * wi + 3) & ~(size_t)3));
    b.off = b.pre + kTileRows + 2;
    b.lpre = reinterpret_cast<uint32_t*>(b.off + kTileRows);
    b.cnt = b.lpre + kTileRows + 4;
    b.q = b.cnt + kTileRows;
    b.meta = b.q + kTileRows;
    return b;
}

// Setup of one row of a tile: its step (descriptor), probe key, home bucket and filter target,
// and the flag op | valid << 8 | pending << 9 | cin << 16 | cout << 24; records the row's meta.
__device__ __forceinline__ void row_setup(const ExploreArgs& a, const TileBuf& B, int row, int wi,
                                          uint64_t* key_out, uint32_t* bkt_out, uint32_t* tgt_out,
                                          uint32_t* flag_out) {
    const StepDesc* d = step_desc(a, B.q[row]);
    const uint32_t op = d->op;
    bool valid = op != kXDone;
    const SegDesc* sg = &d->seg;
    uint32_t target = d->end_const;
    uint64_t key = 0;
    if (op == kXStart) {
        key = d->start_key;
    } else if (valid && (op == kXC2K || op == kXI2K)) {
        // const_to_known / index_to_known: every row looks up the same list
        key = d->start_key;
        target = B.in[row * wi + d->ce];   // shared memory: plain loads
    } else if (valid) {
        const uint32_t* rin = B.in + row * wi;   // shared memory: plain loads
        const uint32_t cur = rin[d->cs];
        if (op == kXK2K) target = rin[d->ce];
        if (op == kXK2U && d->type_index) {
            // get_index(cur, IN) (sparql.hpp:342-345); only 17-bit ids can be keys
            key = make_key(0, cur, kIn);
            sg = &a.seg_index[kIn];
            if (cur >= (1u << kNbitsIdx)) valid = false;
        } else {
            key = make_key(cur, d->pid, d->dir);
            if (cur == 0) sg = &a.seg_index[d->dir & 1];   // vid 0 names the index
        }
        if (cur == kBlankId) valid = false;
    }
    const bool pending = valid && sg->num_buckets != 0 && key != 0;
    const uint32_t cin = d->cin, cout = d->cout;
    *key_out = key;
    *bkt_out = pending ? (uint32_t)bucket_of(key, *sg) : 0;   // 32 bits (stores are refused at 2^32)
    *tgt_out = target;
    *flag_out = op | (valid ? 0x100u : 0u) | (pending ? 0x200u : 0u) | (cin << 16) | (cout << 24);
    B.meta[row] = op | (cin << 8) | (cout << 16);
}

// A row's count and list offset (an edge-array offset or a tagged single entry) once its list
// is known (filters test membership of the target): written to B.cnt / B.off, bytes added to
// the accounting.
__device__ __forceinline__ uint32_t row_count(const ExploreArgs& a, const TileBuf& B, TileState& S, int row,
                                              uint32_t flag, uint64_t off, uint64_t deg, bool found,
                                              unsigned long long& acc_alg, unsigned long long& acc_sd) {
    const uint32_t op = flag & 0xFFu;
    const bool filt = is_filter_op(op);
    const uint32_t cnt = filt ? (found ? 1u : 0u) : (uint32_t)deg;
    B.off[row] = off;
    B.cnt[row] = cnt;
    if (cnt > slice_threshold(a)) S.has_heavy = 1;   // its rows go to the slice queue
    // byte accounting, kept in registers until the CTA leaves
    acc_sd += deg;
    acc_alg += ((flag >> 16) & 0xFF) * 4ull + 16 + deg * 4 + (unsigned long long)cnt * (flag >> 24) * 4;
    return cnt;
}

// One thread per row (the L = 1 launch): each thread sets up its tile rows, loads every row's
// home sector (slots 0 and 1, 32 bytes) before comparing any, and walks on from slot 2 only
// where that sector does not settle the key; filters then search the list themselves.  No
// ballots or shuffles.
__device__ __forceinline__ void tile_probe_rows(const ExploreArgs& a, const TileBuf& B, TileState& S, int n, int wi,
                                                unsigned long long& acc_alg, unsigned long long& acc_sd) {
    constexpr int kRows = kTileRows / kStepThreads;
    uint64_t key[kRows];
    uint32_t bkt[kRows], tgt[kRows], flag[kRows];
#pragma unroll
    for (int k = 0; k < kRows; ++k) {
        const int row = threadIdx.x + k * kStepThreads;
        key[k] = 0;
        bkt[k] = 0;
        tgt[k] = 0;
        flag[k] = kXDone;
        if (row < n) row_setup(a, B, row, wi, &key[k], &bkt[k], &tgt[k], &flag[k]);
        if ((flag[k] & 0x200u) && bkt[k] >= a.store.n_buckets) {
            atomicOr(&a.ctl->err, kErrCorrupt);
            flag[k] &= ~0x200u;
        }
    }
    ulonglong2 s0[kRows], s1[kRows];
#pragma unroll
    for (int k = 0; k < kRows; ++k) {
        s0[k] = make_ulonglong2(0, 0);
        s1[k] = make_ulonglong2(0, 0);
        if (flag[k] & 0x200u) load_sector(a.store.slots + (uint64_t)bkt[k] * kAssoc, &s0[k], &s1[k]);
    }
#pragma unroll
    for (int k = 0; k < kRows; ++k) {
        const int row = threadIdx.x + k * kStepThreads;
        if (row >= n || !(flag[k] & 0x100u)) continue;
        uint64_t p = 0;
        if (flag[k] & 0x200u) {
            if (s0[k].x == key[k]) p = s0[k].y;
            else if (s0[k].x == 0) p = 0;   // first empty slot: absent (insert-only store)
            else if (s1[k].x == key[k]) p = s1[k].y;
            else if (s1[k].x != 0) p = thread_probe(a.store, key[k], bkt[k], &a.ctl->err, 2);
        }
        uint64_t off, deg;
        list_of_ptr(p, a.store.n_edges, &a.ctl->err, &off, &deg);
        const uint32_t op = flag[k] & 0xFFu;
        if (op == kXI2K) {   // index_to_known reads its mt slice of the list (a one-entry list
            uint64_t lo, hi;   // keeps its entry: its slice starts at 0)
            mt_slice(step_desc(a, B.q[row])->mt, deg, &lo, &hi);
            off += lo;
            deg = hi - lo;
        }
        const bool found = is_filter_op(op) && deg &&
                           thread_member(a.store.edges, off, deg, tgt[k], a.sorted_lists != 0);
        row_count(a, B, S, row, flag[k], off, deg, found, acc_alg, acc_sd);
    }
}

// Front half of a tile: start the TMA copy of its rows, probe, count, scan, publish the tile's
// aggregate.  Nothing here waits on another CTA.
template <int L>
__device__ __forceinline__ void tile_front(const ExploreArgs& a, const TileBuf& B, TileState& S,
                                           uint64_t* bar, unsigned phase, uint64_t tile, const Tiling& T,
                                           uint64_t R, int wi, unsigned epoch, uint64_t* s_warp,
                                           unsigned long long& acc_alg, unsigned long long& acc_sd) {
    constexpr int kGroups = kStepThreads / L;
    constexpr int kBatches = L > 1 ? kTileRows / (kGroups * kUnroll) : 1;   // L = 1: tile_probe_rows
    static_assert(L == 1 || kBatches * kGroups * kUnroll == kTileRows, "tile shape");
    const int grp = threadIdx.x / L;
    const int h = threadIdx.x & (L - 1);
    const int gbase = (threadIdx.x & 31) & ~(L - 1);
    const uint64_t r0 = T.r0(tile);
    const int n = T.rows(tile, R);
    const uint32_t* src = a.in + r0 * (uint64_t)wi;
    if (threadIdx.x == 0) {
        if (wi) {
            const unsigned bytes = (unsigned)(((uint64_t)n * wi * 4 + 15) & ~15ull);
            mbar_expect_tx(bar, bytes);
            tma_load_1d(B.in, src, bytes, bar);
        }
        S.tile = tile;
        S.r0 = r0;
        S.n = n;
    }
    for (int i = threadIdx.x; i < n; i += kStepThreads) {
        B.q[i] = a.virtual_rows ? (a.virt_owner ? __ldg(a.virt_owner + r0 + i) : (uint32_t)(r0 + i))
                                : (a.owner_in ? __ldg(a.owner_in + r0 + i) : 0u);
        B.cnt[i] = 0;
    }
    // the one-thread-per-row probe reads only the rows this thread just set up; the group probes
    // share rows across threads
    if constexpr (L > 1) __syncthreads();
    // the rows' copy ran alongside the owner loads; read the rows from shared memory
    if (wi) mbar_wait(bar, phase, &a.ctl->err);
    if constexpr (L == 1) {
        tile_probe_rows(a, B, S, n, wi, acc_alg, acc_sd);
    } else {
    constexpr int kOwn = (kUnroll + L - 1) / L;   // rows of a batch each lane works out
#pragma unroll 1
    for (int b = 0; b < kBatches; ++b) {
        // Row setup, split over the group's lanes: lane h works out the rows u = h, h + L, ...
        // of the batch (row_setup), then the group shares them by shuffles, so no row's hash or
        // descriptor is worked out twice.
        uint64_t mkey[kOwn];
        uint32_t mbkt[kOwn], mtgt[kOwn], mflag[kOwn];   // buckets in 32 bits (group_probe)
#pragma unroll
        for (int j = 0; j < kOwn; ++j) {
            const int u = j * L + h;
            const int row = (b * kUnroll + u) * kGroups + grp;
            mkey[j] = 0;
            mbkt[j] = 0;
            mtgt[j] = 0;
            mflag[j] = kXDone;
            if (u < kUnroll && row < n) row_setup(a, B, row, wi, &mkey[j], &mbkt[j], &mtgt[j], &mflag[j]);
        }
        uint64_t key[kUnroll], ptr[kUnroll];
        uint32_t bucket[kUnroll];
        bool valid[kUnroll], pending[kUnroll];
        int row[kUnroll];
        uint32_t target[kUnroll], flag[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int src = gbase + u % L;
            row[u] = (b * kUnroll + u) * kGroups + grp;
            key[u] = __shfl_sync(kFull, mkey[u / L], src);
            bucket[u] = __shfl_sync(kFull, mbkt[u / L], src);
            target[u] = __shfl_sync(kFull, mtgt[u / L], src);
            flag[u] = __shfl_sync(kFull, mflag[u / L], src);
            valid[u] = (flag[u] & 0x100u) != 0;
            pending[u] = (flag[u] & 0x200u) != 0;
        }
        WK_PH(8);
        group_probe<L>(a.store, key, bucket, pending, ptr, &a.ctl->err);
        WK_PH(9);
        uint64_t off[kUnroll], deg[kUnroll];
        bool has[kUnroll], found[kUnroll], any_filter = false;
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint32_t op = flag[u] & 0xFFu;
            list_of_ptr(ptr[u], a.store.n_edges, &a.ctl->err, &off[u], &deg[u]);
            if (op == kXI2K && valid[u]) {   // index_to_known reads its mt slice of the list
                uint64_t lo, hi;
                mt_slice(step_desc(a, B.q[row[u]])->mt, deg[u], &lo, &hi);
                off[u] += lo;
                deg[u] = hi - lo;
            }
            has[u] = valid[u] && deg[u] > 0 && is_filter_op(op);
            any_filter |= has[u];
            found[u] = false;
        }
        // membership only where a row of the warp filters (the test is warp-uniform)
        if (__any_sync(kFull, any_filter))
            group_member<L>(a.store.edges, off, deg, target, has, a.sorted_lists != 0, found);
        WK_PH(10);
        if (h == 0) {
#pragma unroll
            for (int u = 0; u < kUnroll; ++u)
                if (valid[u]) row_count(a, B, S, row[u], flag[u], off[u], deg[u], found[u], acc_alg, acc_sd);
        }
    }
    }
    __syncthreads();
    WK_PH(2);
    const uint32_t thr = slice_threshold(a);   // S.has_heavy was set by row_count
    const uint64_t total = block_scan(B.cnt, B.pre, n, s_warp);
    const uint64_t ltotal =
        S.has_heavy ? block_scan(B.cnt, B.lpre, n, s_warp, [thr](uint32_t c) { return (uint64_t)(c > thr ? 0u : c); })
                    : total;
    if (threadIdx.x == 0) {
        S.total = total;
        S.ltotal = ltotal;
        publish_aggregate(a.status, tile, total, epoch);
    }
    __syncthreads();
    WK_PH(3);
}

// Back half of a tile: resolve its position (look-back), wait for its rows, record per-query
// ranges, queue long lists, write the short ones.
template <int L>
__device__ __forceinline__ void tile_back(const ExploreArgs& a, const TileBuf& B, TileState& S,
                                          uint64_t* bar, unsigned phase, uint64_t ntiles, int wi,
                                          int wo, unsigned epoch, unsigned long long* s_excl, uint64_t obase) {
    const uint64_t tile = S.tile;
    const int n = S.n;
    const uint64_t total = S.total, ltotal = S.ltotal;
    const uint64_t r0 = S.r0;
    if (threadIdx.x < 32) {
        const uint64_t ex = resolve_prefix(a.status, a.ctl, tile, total, epoch, spin_limit(a));
        if (threadIdx.x == 0) *s_excl = ex;
    }
    if (wi) mbar_wait(bar, phase, &a.ctl->err);   // the tile's rows are in shared memory
    __syncthreads();
    WK_PH(4);
    const uint64_t excl = *s_excl + obase;   // output positions start at the launch's base row
    if (tile == ntiles - 1 && threadIdx.x == 0) *a.out_rows = excl + total;
    const bool fits = excl + total <= a.out_cap_rows;
    if (!fits && threadIdx.x == 0) {
        atomicOr(&a.ctl->err, kErrOverflow);
        atomicMax(&a.ctl->need, (unsigned long long)(excl + total));
    }
    // per-query output ranges: each run of one query's rows adds (end - start)
    if (a.qcount && fits) {
        for (int i = threadIdx.x; i < n; i += kStepThreads) {
            const uint32_t q = B.q[i];
            if (i == 0 || B.q[i - 1] != q) {
                atomicMin(a.qfirst + q, (unsigned long long)(excl + B.pre[i]));
                atomicAdd(a.qcount + q, (unsigned long long)(0 - (excl + B.pre[i])));
            }
            if (i == n - 1 || B.q[i + 1] != q) atomicAdd(a.qcount + q, (unsigned long long)(excl + B.pre[i + 1]));
        }
    }
    // long lists -> slices on the queue (fields first, then the epoch tag)
    if (S.has_heavy && fits) {
        for (int i = threadIdx.x; i < n; i += kStepThreads) {
            const uint32_t c = B.cnt[i];
            if (c <= slice_threshold(a)) continue;
            const uint32_t nch = (c + kHeavyChunk - 1) / kHeavyChunk;
            const unsigned long long at = atomicAdd(&a.ctl->heavy_n, (unsigned long long)nch);
            for (uint32_t k = 0; k < nch; ++k) {
                if (at + k >= a.heavy_cap) {
                    atomicOr(&a.ctl->err, kErrOverflow);
                    break;
                }
                HeavyItem* it = a.heavy + at + k;
                it->in_row = r0 + i;
                it->off = B.off[i] + (uint64_t)k * kHeavyChunk;
                it->out_pos = excl + B.pre[i] + (uint64_t)k * kHeavyChunk;
                it->count = min((uint32_t)kHeavyChunk, c - k * kHeavyChunk);
                it->q = B.q[i];
                __threadfence();
                *(volatile uint32_t*)&it->tag = epoch;
            }
        }
    }
    WK_PH(5);
    // Write the short-list rows (stride w_out), each warp on its own with no block barrier: warp
    // w takes the outputs of input rows [w * 64, w * 64 + 64), 32 rows at a time, one output row
    // per lane.  Lane l holds row l's first short output st_l; the output o belongs to the last
    // row with st <= o (a row without outputs has the next row's st), which a 5-step search over
    // the lanes' st values finds.  Consecutive lanes write consecutive output rows, in row-major
    // then list order, straight to global memory.
    if (fits && ltotal) {
        const bool contiguous = !S.has_heavy;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        constexpr int kWarpRows = kTileRows / (kStepThreads / 32);
        for (int h0 = warp * kWarpRows; h0 < warp * kWarpRows + kWarpRows; h0 += 32) {
            if (h0 >= n) break;
            const int r = min(h0 + lane, n);   // rows past n read the end entry
            const uint64_t st = contiguous ? B.pre[r] : (uint64_t)B.lpre[r];
            const int last = min(h0 + 32, n);
            const uint64_t o_begin = __shfl_sync(kFull, st, 0);
            const uint64_t o_end = contiguous ? B.pre[last] : (uint64_t)B.lpre[last];
            for (uint64_t o0 = o_begin; o0 < o_end; o0 += 32) {
                const uint64_t o = o0 + lane;
                int own = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const uint64_t sv = __shfl_sync(kFull, st, own + step);
                    if (own + step < 32 && sv <= o) own += step;
                }
                const uint64_t st_own = __shfl_sync(kFull, st, own);
                if (o >= o_end) continue;
                const int row = h0 + own;
                const uint64_t k = o - st_own;
                const uint32_t meta = B.meta[row];
                const int opv = meta & 0xFF, cin = (meta >> 8) & 0xFF;
                const uint64_t pos = excl + B.pre[row] + k;
                uint32_t* dst = a.out + pos * wo;
                const uint32_t* sr = B.in + row * wi;
                int c = 0;
                if (opv != kXStart)
                    for (; c < cin; ++c) dst[c] = sr[c];
                // columns past the query's own width are never read (later levels and the
                // result gather use only the query's columns), so they are left as they are
                if (opv == kXStart || opv == kXK2U) dst[c] = list_at(a.store.edges, B.off[row], k);
                if (a.owner_out) a.owner_out[pos] = B.q[row];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // this tile's slices are all reserved
        __threadfence();
        atomicAdd(&a.ctl->tiles_done, 1ull);
        S.has_heavy = 0;      // the buffer's next tile starts without long lists
    }
    WK_PH(6);
}

// Resident CTAs per SM each launch shape is built for: registers are capped for this many.  The
// one-thread-per-row probe holds fewer registers than the group probes.
__host__ __device__ constexpr int explore_min_blocks(int lanes) { return lanes == 1 ? 9 : 7; }

template <int L>
__global__ void __launch_bounds__(kStepThreads, explore_min_blocks(L)) explore_kernel(const ExploreArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ unsigned long long s_claim, s_excl;
    __shared__ uint64_t s_warp[kStepThreads / 32];
    __shared__ TileState s_ts[2];

    const int wi = a.virtual_rows ? 0 : a.w_in, wo = a.w_out;
    const size_t buf_words = tile_buf_words(wi);
    uint32_t* base = reinterpret_cast<uint32_t*>(smem);

    const unsigned epoch = *(volatile unsigned*)&a.ctl->epoch;
    uint64_t R = a.virtual_rows ? a.n_queries : *(volatile const uint64_t*)a.in_rows;
    // an input count past its capacity means the step before overflowed (and said so): its rows
    // were never written, so this step does no work and reports no size of its own
    if (!a.virtual_rows && R > a.in_cap_rows) R = 0;
    const bool handed_off = !a.virtual_rows && a.max_rows && R >= a.max_rows;   // flat pipeline's
    const Tiling T = make_tiling(handed_off ? 0 : R, a.ctl->status_cap);
    uint64_t ntiles = T.ntiles;
    if (ntiles > a.ctl->status_cap) {
        if (threadIdx.x == 0) atomicOr(&a.ctl->err, kErrStatus);
        ntiles = 0;
    }
    const uint64_t obase = a.out_base_rows ? *(volatile const uint64_t*)a.out_base_rows : 0;
    if (ntiles == 0 && !handed_off && blockIdx.x == 0 && threadIdx.x == 0) *a.out_rows = obase;
    // Nothing to do (an empty input, or the flat passes run this step): leave at once.  No CTA
    // claims a tile or a slice or publishes a status word, so the counters stay as the last
    // launch reset them and the epoch need not move (it tags only published words).  A launch
    // that returns at once costs a few microseconds instead of every CTA's counter atomics.
    if (ntiles == 0) return;
    WK_PH_DECL
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        s_ts[0].has_heavy = s_ts[1].has_heavy = 0;   // row_count sets them; tile_back clears them
    }
    unsigned phases = 0;   // mbarrier phase bit of each tile buffer
    unsigned long long acc_alg = 0, acc_sd = 0;   // this thread's share of the byte accounting

    // Two tiles in flight per CTA: the front half of the next tile runs before the back half
    // of the current one, so the look-back and the row copy of one overlap the other's probes.
    if (threadIdx.x == 0) s_claim = atomicAdd(&a.ctl->tile_counter, 1ull);
    __syncthreads();
    uint64_t cur = s_claim;
    int b = 0;
    WK_PH(0);
    if (cur < ntiles)
        tile_front<L>(a, tile_buf(base, wi), s_ts[0], &s_bar[0], phases & 1u, cur, T, R, wi, epoch, s_warp,
                      acc_alg, acc_sd);
    while (cur < ntiles) {
        if (threadIdx.x == 0) s_claim = atomicAdd(&a.ctl->tile_counter, 1ull);
        __syncthreads();
        const uint64_t next = s_claim;
        WK_PH(0);
        if (next < ntiles)
            tile_front<L>(a, tile_buf(base + (b ^ 1) * buf_words, wi), s_ts[b ^ 1], &s_bar[b ^ 1],
                          (phases >> (b ^ 1)) & 1u, next, T, R, wi, epoch, s_warp, acc_alg, acc_sd);
        tile_back<L>(a, tile_buf(base + b * buf_words, wi), s_ts[b], &s_bar[b], (phases >> b) & 1u, ntiles, wi,
                     wo, epoch, &s_excl, obase);
        if (wi) phases ^= 1u << b;
        cur = next;
        b ^= 1;
    }

    // Out of tiles: write queued long-list slices until every tile is done and the queue is
    // drained.  A claimed index either gets reserved by a tile still running (wait for its
    // tag) or lies past the final count (stop).  Every wait is bounded.
    __syncthreads();
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
                if (++spins > spin_limit(a)) {
                    atomicOr(&a.ctl->err, kErrTimeout);
                    state = 2;
                    break;
                }
                if (spins > 32) __nanosleep(64);
            }
            s_claim = state == 1 ? idx : ~0ull;
        }
        __syncthreads();
        const unsigned long long idx = s_claim;
        if (idx == ~0ull) break;
        const HeavyItem* it = a.heavy + idx;
        const uint64_t in_row = __ldcg((const unsigned long long*)&it->in_row);
        const uint64_t off = __ldcg((const unsigned long long*)&it->off);
        const uint64_t out_pos = __ldcg((const unsigned long long*)&it->out_pos);
        const uint32_t count = __ldcg((const unsigned int*)&it->count);
        const uint32_t q = __ldcg((const unsigned int*)&it->q);
        const StepDesc* d = step_desc(a, q);
        const int opv = d->op, cin = d->cin;
        const uint32_t* src = a.in + in_row * (uint64_t)a.w_in;   // the row's columns: L1 hits
        const int ecol = opv == kXStart ? 0 : cin;
        const uint64_t ne = (uint64_t)count * wo;
        uint32_t* dst = a.out + out_pos * wo;
        for (uint64_t e = threadIdx.x; e < ne; e += kStepThreads) {
            const uint64_t j = e / wo;
            const int c = (int)(e - j * wo);
            uint32_t v = 0;
            if (c < ecol) v = __ldg(src + c);
            else if (c == ecol) v = __ldg(a.store.edges + off + j);
            dst[e] = v;
        }
        if (a.owner_out)
            for (uint32_t j = threadIdx.x; j < count; j += kStepThreads) a.owner_out[out_pos + j] = q;
        __syncthreads();
    }
    WK_PH(7);
    WK_PH_FLUSH;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc_alg += __shfl_xor_sync(0xffffffffu, acc_alg, o);
        acc_sd += __shfl_xor_sync(0xffffffffu, acc_sd, o);
    }
    if ((threadIdx.x & 31) == 0 && acc_alg) {
        atomicAdd(&a.ctl->alg_bytes, acc_alg);
        atomicAdd(&a.ctl->sum_deg, acc_sd);
    }
    exit_protocol(a.ctl, a.status, epoch, a.heavy ? &a.heavy[0].tag : nullptr,
                  sizeof(HeavyItem) / sizeof(uint32_t), a.heavy ? a.heavy_cap : 0);
}

template <int L>
cudaError_t set_attr(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(explore_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e != cudaSuccess ? e : use_max_shared_carveout(explore_kernel<L>);
}

}  // namespace

size_t explore_smem_bytes(int w_in) {
    // two tile buffers: rows, the two scans, list offsets and three per-row words (the writes go
    // straight to global memory, with no staging)
    return 2 * tile_buf_words(w_in) * 4;
}

cudaError_t explore_kernel_attrs() {
    const int bytes = (int)explore_smem_bytes(kMaxSmemCols);
    cudaError_t e;
    if ((e = set_attr<1>(bytes)) != cudaSuccess) return e;
    if ((e = set_attr<2>(bytes)) != cudaSuccess) return e;
    if ((e = set_attr<4>(bytes)) != cudaSuccess) return e;
    return set_attr<8>(bytes);
}

CtaUse explore_cta_use(int w_in, int w_out, int lanes) {
    CtaUse u{0, 0, kStepThreads};
    cudaFuncAttributes fa{};
    cudaError_t e = cudaErrorInvalidValue;
    if (lanes == 1) e = cudaFuncGetAttributes(&fa, explore_kernel<1>);
    if (lanes == 2) e = cudaFuncGetAttributes(&fa, explore_kernel<2>);
    if (lanes == 4) e = cudaFuncGetAttributes(&fa, explore_kernel<4>);
    if (lanes == 8) e = cudaFuncGetAttributes(&fa, explore_kernel<8>);
    int dev = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e != cudaSuccess) fa.numRegs = 255;   // unknown: assume the worst
    u.smem = explore_smem_bytes(w_in) + fa.sharedSizeBytes + (size_t)reserved;
    // registers are allocated per warp in units of 256
    u.regs = ((fa.numRegs * 32 + 255) / 256) * 256 * (kStepThreads / 32);
    return u;
}

int blocks_beside(const CtaUse& me, int alone, const CtaUse& other, int other_ctas) {
    if (other_ctas <= 0) return alone;
    int dev = 0, smem_sm = 0, regs_sm = 0, thr_sm = 0, blk_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    long long n = alone;
    auto fit = [&](long long limit, long long theirs, long long mine) {
        if (mine <= 0) return;
        const long long left = limit - (long long)other_ctas * theirs;
        n = std::min(n, left > 0 ? left / mine : 0ll);
    };
    fit(smem_sm, (long long)other.smem, (long long)me.smem);
    fit(regs_sm, other.regs, me.regs);
    fit(thr_sm, other.threads, me.threads);
    fit(blk_sm, 1, 1);
    return (int)std::max(1ll, n);
}

int explore_blocks_beside(int w_in, int w_out, int lanes, const CtaUse& other, int other_ctas) {
    const int alone = explore_blocks_per_sm(w_in, w_out, lanes);
    if (other_ctas <= 0) return alone;
    return blocks_beside(explore_cta_use(w_in, w_out, lanes), alone, other, other_ctas);
}

int explore_blocks_per_sm(int w_in, int w_out, int lanes) {
    size_t smem = explore_smem_bytes(w_in);
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    if (lanes == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<1>, kStepThreads, smem);
    if (lanes == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<2>, kStepThreads, smem);
    if (lanes == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<4>, kStepThreads, smem);
    if (lanes == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, explore_kernel<8>, kStepThreads, smem);
    return (e == cudaSuccess && nb > 0) ? nb : 1;
}

cudaError_t launch_explore(const ExploreArgs& a, int grid, cudaStream_t s) {
    const int wi = a.virtual_rows ? 0 : a.w_in;
    const size_t smem = explore_smem_bytes(wi);
    if (grid < 1) grid = 1;
    switch (a.lanes) {
    case 1: explore_kernel<1><<<grid, kStepThreads, smem, s>>>(a); break;
    case 2: explore_kernel<2><<<grid, kStepThreads, smem, s>>>(a); break;
    case 8: explore_kernel<8><<<grid, kStepThreads, smem, s>>>(a); break;
    default: explore_kernel<4><<<grid, kStepThreads, smem, s>>>(a); break;
    }
    return cudaGetLastError();
}

}  // namespace wk

// Phase cycle counters of an instrumented build (all zero otherwise); reset clears them.
extern "C" int wk_debug_phase_cycles(unsigned long long* out, int32_t n, int32_t reset) {
    if (!out || n < wk::kPhaseSlots) return WK_E_BADARG;
    if (cudaMemcpyFromSymbol(out, wk::g_phase_cycles, sizeof(unsigned long long) * wk::kPhaseSlots) !=
        cudaSuccess)
        return WK_E_CUDA;
    if (reset) {
        unsigned long long z[wk::kPhaseSlots] = {0};
        if (cudaMemcpyToSymbol(wk::g_phase_cycles, z, sizeof(z)) != cudaSuccess) return WK_E_CUDA;
    }
    return WK_SUCCESS;
}
