// The exploration launch shared by single queries and batches.
//
// One launch runs one pattern level: for a single query every input row runs the same step;
// for a batch each input row belongs to one query (owner_in) whose step for this level is
// desc[owner].  Output rows keep their query's rows contiguous and in input order.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_kernels.h"

namespace wk {

// kXC2K: const_to_known, kXI2K: index_to_known (the row survives when its `ce` value is in the
// constant's / index's list, the index list cut to the step's mt slice).
enum ExploreOp : uint8_t { kXStart = 0, kXK2U = 1, kXK2K = 2, kXK2C = 3, kXDone = 4, kXC2K = 5, kXI2K = 6 };

__host__ __device__ inline bool is_filter_op(uint32_t op) {
    return op == kXK2K || op == kXK2C || op == kXC2K || op == kXI2K;
}

// One query's step at one level (64 bytes).
struct StepDesc {
    SegDesc seg;            // segment of the step's normal key, or of the start key
    uint64_t start_key;     // kXStart: the constant / index key whose list starts the table
    uint32_t pid;
    uint32_t end_const;     // kXK2C
    uint8_t op, dir, cin, cout;
    uint8_t cs, ce, type_index, pad;
    uint32_t mt;            // kXI2K: mt_tid | mt_factor << 16, the slice of the index list
};

// The part of a list of `deg` entries that slice mt_tid of mt_factor reads (sparql.hpp:105-116,
// 213-224): equal shares of deg / mt_factor, the last slice also taking the remainder.
__host__ __device__ inline void mt_slice(uint32_t mt, uint64_t deg, uint64_t* lo, uint64_t* hi) {
    const uint64_t tid = mt & 0xFFFF, factor = (mt >> 16) ? (mt >> 16) : 1;
    const uint64_t len = deg / factor;
    *lo = (tid % factor) * len;
    *hi = (tid % factor) == factor - 1 ? deg : *lo + len;
}
static_assert(sizeof(StepDesc) == 64, "StepDesc is 64 bytes");

// A slice of a long neighbour list.  Rows whose count exceeds kHeavyRows are not written by
// the CTA that scanned them: it queues them as kHeavyChunk-row slices, and CTAs that run out of
// tiles take slices from the queue, so a hub vertex is spread over every CTA.
struct HeavyItem {
    uint64_t in_row;        // physical input row (virtual rows: unused)
    uint64_t off;           // first edge of the slice
    uint64_t out_pos;       // first output row of the slice
    uint32_t count;         // output rows in the slice
    uint32_t q;             // owner query
    uint32_t tag;           // launch epoch, written last: the slice is ready
    uint32_t pad;
};
static_assert(sizeof(HeavyItem) == 40, "HeavyItem is 40 bytes");

constexpr int kHeavyRows = 128;     // slice threshold when a launch sets none
constexpr int kMinSliceRows = 8;    // lowest threshold a launch may set (queues are sized for it)
constexpr int kHeavyChunk = 2048;
constexpr int kPhaseSlots = 12;  // phase cycle counters of an instrumented build

struct ExploreArgs {
    DevStore store;
    SegDesc seg_index[2];        // index segment of each direction
    StepDesc one;                // the step of every row when desc is null
    const StepDesc* desc;        // [n_queries] this level's step per query, or null
    // Continuous batching: when desc_stride > 0, query q's step is
    // desc[q * desc_stride + (iter - q_admit[q])] (kXDone past the plan).
    uint32_t desc_stride;
    uint32_t iter;
    const uint32_t* q_admit;
    uint32_t n_queries;
    int32_t virtual_rows;        // input row r is a start row (no input table)
    const uint32_t* virt_owner;  // owner query of virtual row r, or null (query r)
    const uint64_t* out_base_rows;   // first output row, read at launch (null: 0)
    const uint64_t* in_rows;     // device row count of the input (unused for virtual rows)
    const uint32_t* owner_in;    // owner query of each input row, or null (query 0)
    const uint32_t* in;          // input rows, stride w_in (tables carry >= 64 B of padding)
    int32_t w_in;
    uint64_t in_cap_rows;
    uint32_t* out;               // output rows, stride w_out
    int32_t w_out;
    uint64_t out_cap_rows;
    uint32_t* owner_out;         // owner query of each output row, or null
    uint64_t* out_rows;          // rows written (set by the launch)
    unsigned long long* qfirst;  // [n_queries] first output row per query (min), or null
    unsigned long long* qcount;  // [n_queries] output rows per query (sum), or null
    HeavyItem* heavy;
    uint64_t heavy_cap;
    StepCtl* ctl;
    unsigned long long* status;
    int32_t sorted_lists;
    int32_t lanes;
    // Rows with more output rows than this go to the slice queue (spread over every CTA);
    // shorter ones are written by the CTA that scanned them.  0 means kHeavyRows; values below
    // kMinSliceRows are raised to it (the queues of a context are sized for that).
    uint32_t slice_rows;
    // When nonzero and the input has at least this many rows, the launch does nothing (the
    // flat pipeline of wk_flat.cu runs the step instead).
    uint64_t max_rows;
    // Polls a look-back on a predecessor tile or a wait for the slice queue makes before it
    // gives up and sets kErrTimeout (0: kDefaultSpinLimit).  Tests lower it to make the waits
    // run out; the wait for the launch's own bulk copies keeps its fixed limit.
    uint64_t spin_limit;
};

constexpr uint64_t kDefaultSpinLimit = 1ull << 24;

size_t explore_smem_bytes(int w_in);
cudaError_t explore_kernel_attrs();
int explore_blocks_per_sm(int w_in, int w_out, int lanes);

// Resources one CTA of the exploration launch holds on its SM.
struct CtaUse {
    size_t smem;   // dynamic + static + the per-block reservation, bytes
    int regs;      // registers, in the per-warp allocation granularity
    int threads;
};
CtaUse explore_cta_use(int w_in, int w_out, int lanes);
// CTAs per SM of this launch that fit beside `other_ctas` resident CTAs using `other` each
// (at least 1), so two persistent launches can be resident on every SM at once.
int explore_blocks_beside(int w_in, int w_out, int lanes, const CtaUse& other, int other_ctas);
// CTAs of shape `me` (at most `alone`) that fit on an SM beside other_ctas CTAs of shape
// `other`: shared memory, registers, threads and CTA slots; at least 1.
int blocks_beside(const CtaUse& me, int alone, const CtaUse& other, int other_ctas);
cudaError_t launch_explore(const ExploreArgs& a, int grid, cudaStream_t s);

}  // namespace wk
