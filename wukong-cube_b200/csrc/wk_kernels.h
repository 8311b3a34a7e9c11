// Host-visible launch interface of the exploration-step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_format.h"

namespace wk {

// Error bits a kernel ORs into StepCtl::err (sticky until the host clears them).
enum : uint32_t {
    kErrOverflow = 1u,   // an output did not fit; StepCtl::need holds the elements required
    kErrTimeout = 2u,    // a bounded wait (tile look-back) gave up
    kErrCorrupt = 4u,    // a key-table chain left the slot array or exceeded the hop limit
    kErrStatus = 8u,     // more tiles than the status array holds (host grows it and reruns)
};

// Per-stream control block of the single-pass scan.  Kernels that use it reset the tile and
// exit counters themselves on their way out (the last CTA to leave does it) and advance the
// epoch, so back-to-back launches and CUDA-graph replays need no memset in between.
struct StepCtl {
    unsigned long long tile_counter;
    unsigned int exit_counter;
    unsigned int epoch;          // 1..65535, tags valid status words of the running launch
    unsigned int err;
    unsigned int pad;
    unsigned long long need;     // largest output (elements) a launch asked for
    unsigned long long status_cap;   // entries in the status array that follows
    unsigned long long sum_deg;  // neighbour-list lengths the probes found (profiling)
    unsigned long long alg_bytes;   // algorithmic bytes of the launches: rows in * cols * 4
                                    // + 16 per probe + 4 per list entry read + rows out * cols * 4
};

// Where the store lives on the device.
struct DevStore {
    const Slot* slots;
    uint64_t n_buckets;   // slots / 8
    const uint32_t* edges;
    uint64_t n_edges;
};

enum StepOp : int32_t { kOpK2U = 0, kOpK2K = 1, kOpK2C = 2 };

struct StepArgs {
    DevStore store;
    SegDesc seg;             // segment of [vid|pid|dir]
    SegDesc seg_index;       // index segment of `dir` (rows whose value is 0 and TYPE_ID/IN)
    const uint32_t* in;      // input table, row-major
    const uint64_t* in_rows; // device row count of the input
    uint64_t in_cap;         // elements the input buffer holds (reads never pass it)
    uint32_t* out;
    uint64_t* out_rows;      // written by the launch: rows of the output
    uint64_t out_cap;        // elements the output buffer holds
    StepCtl* ctl;
    unsigned long long* status;
    int32_t op;
    int32_t cols;
    int32_t col_start;
    int32_t col_end;         // K2K
    uint32_t end_const;      // K2C
    uint32_t pid;
    int32_t dir;
    int32_t type_index;      // K2U with pid == TYPE_ID and dir == IN: key = [0|cur|IN]
    int32_t sorted_lists;    // every list ascending + unique (checked at upload)
    int32_t lanes;           // lanes per probe group: 2, 4 or 8 (slots read per request)
};

struct ListArgs {
    DevStore store;
    SegDesc seg;
    uint64_t key;            // the single key to expand
    int32_t mt_tid, mt_factor;
    uint32_t* out;
    uint64_t* out_rows;
    uint64_t out_cap;
    StepCtl* ctl;
};

// Launch geometry helpers.
constexpr int kStepThreads = 256;
constexpr int kTileRows = 512;
size_t step_smem_bytes(int cols, int op, int* out_chunk_rows);
int step_blocks_per_sm(int cols, int op, int lanes);

cudaError_t launch_step(const StepArgs& a, int grid, cudaStream_t s);
cudaError_t launch_list(const ListArgs& a, int grid, cudaStream_t s);
cudaError_t launch_sorted_check(const DevStore& st, unsigned* d_flag, cudaStream_t s);
cudaError_t step_kernel_attrs(int max_cols);

}  // namespace wk
