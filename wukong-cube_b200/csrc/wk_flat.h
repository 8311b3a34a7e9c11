// Host-visible interface of the flat count / scan / scatter pipeline (wk_flat.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_explore.h"

namespace wk {

struct FlatArgs {
    DevStore store;
    SegDesc seg_index[2];        // index segment of each direction
    StepDesc step;               // a known_to_unknown / known_to_known / known_to_const step
    const uint64_t* in_rows;     // device row count of the input
    const uint32_t* in;
    int32_t w_in;
    uint64_t in_cap_rows;
    uint32_t* out;
    int32_t w_out;
    uint64_t out_cap_rows;
    uint64_t* out_rows;
    uint64_t min_rows;           // every launch returns at once for smaller inputs
    // scratch, sized for in_cap_rows input rows and `grid` CTAs
    uint64_t* pos;               // [in_cap_rows + 1] output rows of each input row, then (in
                                 // place) its first output row; pos[R] = the total
    uint64_t* off;               // [in_cap_rows] list offset of each input row
    uint64_t* part;              // [grid + 1] chunk totals, then their exclusive scan
    StepCtl* ctl;
    int32_t sorted_lists;
};

// Scratch bytes for `rows` input rows and `grid` CTAs.
inline size_t flat_scratch_bytes(uint64_t rows, int grid) {
    return (size_t)(rows + 1) * 8 + (size_t)rows * 8 + (size_t)(grid + 1) * 8 + 256;
}
int flat_grid(int sm_count);
// The grid of a serving lane's flat passes: the CTAs per SM of the count pass (the one that holds
// the most registers) that fit beside other_ctas CTAs of shape `other`, times the SMs (at most
// flat_grid).
int flat_grid_beside(int sm_count, const CtaUse& other, int other_ctas);
cudaError_t launch_flat(const FlatArgs& a, int grid, cudaStream_t s);
cudaError_t flat_kernel_attrs();

// One level of a batch through the flat passes: every row's step comes from its owner query's
// descriptor.  Writes owner_out and each query's output range (qfirst / qcount, which the
// caller has reset).  Level 0 has virtual rows: row r is query r's start.
struct FlatLevelArgs {
    DevStore store;
    SegDesc seg_index[2];
    const StepDesc* desc;        // [n_queries] this level's step per query
    uint32_t n_queries;
    int32_t virtual_rows;
    const uint64_t* in_rows;
    const uint32_t* owner_in;
    const uint32_t* in;
    int32_t w_in;
    uint64_t in_cap_rows;
    uint32_t* out;
    int32_t w_out;
    uint64_t out_cap_rows;
    uint64_t* out_rows;
    uint32_t* owner_out;
    unsigned long long* qfirst;
    unsigned long long* qcount;
    uint64_t* pos;               // [max(in_cap_rows, n_queries) + 1]
    uint64_t* off;               // [max(in_cap_rows, n_queries)]
    uint64_t* part;              // [grid + 1]
    StepCtl* ctl;
    int32_t sorted_lists;
};
cudaError_t launch_flat_level(const FlatLevelArgs& a, int grid, cudaStream_t s);

}  // namespace wk
