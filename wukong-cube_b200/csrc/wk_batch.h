// Batched execution of many planned queries: the small launches after the last level.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_explore.h"
#include "wk_kernels.h"

namespace wk {

constexpr int kMaxBatchLevels = 16;

struct ResultScanArgs {
    uint32_t n;
    const uint32_t* nsteps;              // [n] patterns per query (0 = failed / empty plan)
    const unsigned long long* qfirst;    // [levels][n]
    const unsigned long long* qcount;    // [levels][n]
    const uint32_t* final_cols;          // [n]
    int32_t* final_level;                // [n] level holding the final table, -1 if empty
    uint64_t* final_base;                // [n] its first row there
    uint64_t* final_rows;                // [n]
    uint64_t* res_off;                   // [n + 1] element offsets of the compact results
};

struct GatherArgs {
    uint32_t n;
    const int32_t* final_level;
    const uint64_t* final_base;
    const uint64_t* final_rows;
    const uint32_t* final_cols;
    const uint64_t* res_off;
    const uint32_t* region[kMaxBatchLevels];   // base of each level's rows
    int32_t width[kMaxBatchLevels];            // their stride
    uint32_t* out;
    uint64_t out_cap;
    StepCtl* ctl;
};

cudaError_t launch_result_scan(const ResultScanArgs& a, cudaStream_t s);
cudaError_t launch_gather(const GatherArgs& a, int grid, cudaStream_t s);

}  // namespace wk
