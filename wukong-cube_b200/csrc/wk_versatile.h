// Host-visible interface of the unknown-predicate (versatile) operators (wk_versatile.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_kernels.h"

namespace wk {

enum VersOp : int32_t { kVKUU = 0, kVKUC = 1, kVCUU = 2, kVCUC = 3 };

// The segment of the normal keys of one predicate and direction, keyed pid * 2 + dir; the
// store's table of these is sorted by key.
struct PredSeg {
    uint32_t key;
    uint32_t pad;
    SegDesc seg;
};

struct VersArgs {
    DevStore store;
    SegDesc vp_seg;              // segment of the vertex-predicate keys [v|PREDICATE_ID|dir]
    const PredSeg* pseg;         // the store's predicate segments
    uint32_t n_pseg;
    int32_t op;                  // VersOp
    int32_t dir;
    int32_t virtual_row;         // the constant forms: one row whose start is start_const
    uint32_t start_const;
    uint32_t end_const;          // kVKUC / kVCUC
    int32_t cs;                  // start column (kVKUU / kVKUC)
    int32_t cin;                 // input columns copied to every output row (0: constant forms)
    const uint64_t* in_rows;
    const uint32_t* in;
    int32_t w_in;
    uint64_t in_cap_rows;
    uint32_t* out;
    int32_t w_out;
    uint64_t out_cap_rows;
    uint64_t* out_rows;
    uint64_t* pos;               // [rows + 1] output rows of each row
    uint64_t* part;              // [grid + 1] chunk totals, then their exclusive scan
    StepCtl* ctl;
    int32_t sorted_lists;
};

int vers_grid(uint64_t rows, int sm_count);
cudaError_t launch_versatile(const VersArgs& a, int grid, cudaStream_t s);
cudaError_t versatile_kernel_attrs();

}  // namespace wk
