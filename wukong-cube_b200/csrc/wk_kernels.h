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
    kErrResult = 16u,    // a result gather did not fit its buffer (host grows it and reruns)
};

// Per-stream control block of the single-pass scan.  Kernels that use it reset the tile and
// exit counters themselves on their way out (the last CTA to leave does it) and advance the
// epoch, so back-to-back launches and CUDA-graph replays need no memset in between.
struct StepCtl {
    unsigned long long tile_counter;
    unsigned int exit_counter;
    unsigned int epoch;          // 1..65535, tags valid status words of the running launch
    unsigned int err;
    unsigned int flat_done;      // count CTAs of a flat pass that have published their chunk
                                 // total; the last one scans them and resets this to 0
    unsigned long long need;     // largest output (elements) a launch asked for
    unsigned long long status_cap;   // entries in the status array that follows
    unsigned long long sum_deg;  // neighbour-list lengths the probes found (profiling)
    unsigned long long alg_bytes;   // algorithmic bytes of the launches: rows in * cols * 4
                                    // + 16 per probe + 4 per list entry read + rows out * cols * 4
    unsigned long long heavy_n;     // long-list slices reserved by the running launch
    unsigned long long heavy_claim; // slices claimed by CTAs that ran out of tiles
    unsigned long long tiles_done;  // tiles whose slices are all reserved
};

// Where the store lives on the device.
struct DevStore {
    const Slot* slots;
    uint64_t n_buckets;   // slots / 8
    const uint32_t* edges;
    uint64_t n_edges;
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

// Launch geometry of the exploration launch.
constexpr int kStepThreads = 128;
constexpr int kTileRows = 256;

cudaError_t launch_list(const ListArgs& a, int grid, cudaStream_t s);
cudaError_t launch_sorted_check(const DevStore& st, unsigned* d_flag, cudaStream_t s);
// One-entry lists into their keys' pointer words (inline_kernel): with orig null, counts them
// into *n and flags pointer words that already carry the inline type in *clash; with orig (two
// words per counted slot), converts them and keeps the original pointer words there.  *n must
// be 0 on entry.
cudaError_t launch_inline(const DevStore& st, unsigned long long* n, unsigned* clash, uint64_t* orig,
                          cudaStream_t s);
// `grid` CTAs of 256 threads, `per` random 16-byte reads each from a `bytes`-byte buffer.
cudaError_t launch_random_reads(const void* buf, uint64_t bytes, int per, uint64_t seed,
                                uint32_t* sink, int grid, cudaStream_t s);

// Every device allocation of the library goes through dev_malloc, which counts it, so a caller
// (and the tests) can see that a call allocated nothing (wk_debug_device_allocs).
uint64_t device_alloc_count();
void note_device_alloc();
template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    note_device_alloc();
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

// Every kernel of the library asks for the same L1 / shared-memory split, the largest shared
// carveout.  The split is an SM-wide setting, so CTAs of launches that ask for different
// splits cannot share an SM; with one split everywhere, a serving lane's launches and the
// iteration launches run side by side instead of one draining SMs for the other.
template <class K>
inline cudaError_t use_max_shared_carveout(K kernel) {
    return cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}
// Set that attribute on the kernels of each translation unit (called at context creation).
cudaError_t small_kernel_attrs();    // wk_kernels.cu
cudaError_t batch_kernel_attrs();    // wk_batch.cu
cudaError_t serve_kernel_attrs();    // wk_serve.cu
cudaError_t final_kernel_attrs();    // wk_final.cu

}  // namespace wk
