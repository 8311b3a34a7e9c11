// Batched execution of many planned queries: host-visible descriptors and launch interface.
//
// All queries of a batch advance one pattern per level.  A level's input rows are the
// concatenation, in query order, of every active query's current table (a query at its first,
// constant- or index-start pattern contributes one virtual row: its start key).  One
// persistent launch per level probes, counts, scans and writes all of them; a small prep launch
// between levels turns the scanned row positions into each query's next table.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wk_kernels.h"

namespace wk {

enum BatchOp : uint8_t { kBStart = 0, kBK2U = 1, kBK2K = 2, kBK2C = 3, kBDone = 4 };

// One query at one level (64 bytes).
struct BatchDesc {
    SegDesc seg;            // segment of the step's normal key (or of the start key)
    uint64_t start_key;     // kBStart: the constant / index key whose list starts the table
    uint32_t pid;
    uint32_t end_const;     // kBK2C
    uint8_t op, dir, cin, cout;
    uint8_t cs, ce, type_index, pad;
    uint32_t pad2;
};
static_assert(sizeof(BatchDesc) == 64, "BatchDesc is 64 bytes");

struct LevelArgs {
    DevStore store;
    SegDesc seg_index[2];        // index segment per direction
    const BatchDesc* desc;       // [n] this level
    const uint64_t* row_start;   // [n + 1] flattened first input row per query; [n] = total
    const uint64_t* src_base;    // [n] physical row of the query's first input row
    uint32_t n;
    const uint32_t* in;          // previous level's region (stride w_in); null at level 0
    int32_t w_in;
    uint32_t* out;               // this level's region (stride w_out)
    int32_t w_out;
    uint64_t out_cap_rows;
    uint64_t* pref;              // [rows + 1] exclusive output-row prefix per input row
    uint64_t pref_cap;           // entries pref holds
    uint64_t* total_out;         // rows this level produced
    StepCtl* ctl;
    unsigned long long* status;
    int32_t sorted_lists;
    int32_t lanes;
};

struct PrepArgs {
    int32_t level;               // level about to run (== n_levels for the final pass)
    uint32_t n;
    const uint32_t* nsteps;      // [n] patterns of each query (0 = failed / empty plan)
    const uint64_t* prev_row_start;   // [n + 1] of the previous level (null at level 0)
    const uint64_t* prev_pref;        // previous level's pref
    const uint64_t* prev_total_out;
    uint64_t prev_pref_cap;           // entries of prev_pref
    uint64_t* row_start;         // [n + 1] this level
    uint64_t* src_base;          // [n]
    int32_t* final_level;        // [n]
    uint64_t* final_base;        // [n]
    uint64_t* final_rows;        // [n]
    const uint32_t* final_cols;  // [n] (final pass)
    uint64_t* res_off;           // [n + 1] element offsets of the compact results (final pass)
};

struct GatherArgs {
    uint32_t n;
    const int32_t* final_level;
    const uint64_t* final_base;
    const uint64_t* final_rows;
    const uint32_t* final_cols;
    const uint64_t* res_off;
    const uint32_t* region[16];  // base of each level's region
    int32_t width[16];           // its row stride
    uint32_t* out;
    uint64_t out_cap;
    StepCtl* ctl;
};

size_t level_smem_bytes(int w_in, int w_out, int* chunk_rows);
cudaError_t level_kernel_attrs();
int level_blocks_per_sm(int w_in, int w_out, int lanes);
cudaError_t launch_level(const LevelArgs& a, int grid, cudaStream_t s);
cudaError_t launch_prep(const PrepArgs& a, cudaStream_t s);
cudaError_t launch_gather(const GatherArgs& a, int grid, cudaStream_t s);

}  // namespace wk
