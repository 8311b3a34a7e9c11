// Batched light queries and the serving loop (filled in below the single-query path).
#include "wk_ctx.h"

void wk_batch_release(wk_ctx* ctx) { (void)ctx; }

extern "C" int wk_batch_execute(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t* host_out,
                                uint64_t cap_elems, wk_qresult* results) {
    (void)ctx; (void)queries; (void)n; (void)host_out; (void)cap_elems; (void)results;
    return WK_E_UNSUPPORTED;
}

extern "C" int wk_batch_execute_device(wk_ctx* ctx, const wk_query* queries, uint32_t n,
                                       uint64_t* total_rows) {
    (void)ctx; (void)queries; (void)n; (void)total_rows;
    return WK_E_UNSUPPORTED;
}

extern "C" int wk_serve_run_open_loop(wk_ctx* ctx, const wk_serve_config* cfg, const wk_query* queries,
                                      uint32_t n, const double* arrival_us, uint32_t* host_out,
                                      uint64_t cap_elems, wk_qresult* results) {
    (void)ctx; (void)cfg; (void)queries; (void)n; (void)arrival_us; (void)host_out; (void)cap_elems;
    (void)results;
    return WK_E_UNSUPPORTED;
}
