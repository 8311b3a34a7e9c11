/*
 * wukong_b200.h — C ABI of the B200-native triple-pattern exploration step.
 *
 * This is the boundary a Wukong host binds to in place of the reference's src/gpu path.
 * Every call returns an int status: 0..13 keep the numbering of Wukong's
 * src/core/common/errors.hpp:30-45 (SUCCESS, UNKNOWN_ERROR, ... FILE_NOT_FOUND); codes from
 * 100 up are new (the reference aborts instead: gpu_utils.hpp:28-37, assertion.hpp:89-100).
 * No call takes or returns a torch type; pointers are plain host pointers unless a parameter
 * says "device".
 *
 * Threading: one wk_ctx per host thread (the reference runs one GPUAgent thread per GPU,
 * gpu_agent.hpp:248).  Calls on one context are serialised by an internal mutex.
 */
#ifndef WUKONG_B200_H
#define WUKONG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum {
    WK_SUCCESS = 0,             /* errors.hpp:31 */
    WK_UNKNOWN_ERROR = 1,
    WK_SYNTAX_ERROR = 2,
    WK_UNKNOWN_PATTERN = 3,     /* unsupported pattern shape / operator */
    WK_ATTR_DISABLE = 4,        /* attribute (non-SID) predicate */
    WK_NO_REQUIRED_VAR = 5,
    WK_UNSUPPORT_UNION = 6,
    WK_OBJ_ERROR = 7,           /* index pattern whose predicate is not TYPE/PREDICATE */
    WK_VERTEX_INVALID = 8,      /* variable id out of range */
    WK_UNKNOWN_SUB = 9,         /* pattern starts from an unknown variable */
    WK_SETTING_ERROR = 10,
    WK_FIRST_PATTERN_ERROR = 11,/* const/index start that is not the first pattern */
    WK_UNKNOWN_FILTER = 12,
    WK_FILE_NOT_FOUND = 13,
    WK_E_OOM = 100,             /* device allocation failed */
    WK_E_CAPACITY = 101,        /* a result or working set would exceed a configured cap */
    WK_E_TIMEOUT = 102,         /* a bounded device-side wait gave up */
    WK_E_BADARG = 103,          /* null pointer, bad column, bad direction, ... */
    WK_E_CUDA = 104,            /* a CUDA runtime call failed (see wk_last_error) */
    WK_E_NOSTORE = 105,         /* no GStore uploaded yet */
    WK_E_CORRUPT = 106,         /* key table chain out of range or too long */
    WK_E_UNSUPPORTED = 107      /* legal in Wukong but outside this path (e.g. versatile) */
};

/* Directions (type.hpp:50) and reserved ids (vertex.hpp:52-53). */
#define WK_IN 0
#define WK_OUT 1
#define WK_PREDICATE_ID 0
#define WK_TYPE_ID 1
#define WK_NO_RESULT 0xFFFF      /* v2c_map entry of an unbound variable (query.hpp:63) */

/* Execution modes of wk_query_execute. */
#define WK_MODE_PLAIN 0     /* one launch per pattern, host sync + size read-back per step */
#define WK_MODE_RESIDENT 1  /* all steps enqueued back to back, sizes stay on the device */
#define WK_MODE_GRAPH 2     /* as RESIDENT, replayed from a cached CUDA graph per plan shape */

typedef struct wk_ctx wk_ctx;
typedef struct wk_table wk_table;
typedef struct wk_gstore wk_gstore;
typedef struct wk_serve wk_serve;

/* ---------------------------------------------------------------- plain data types */

/* Device context configuration.  Zero fields take defaults. */
typedef struct wk_config {
    int32_t device;                   /* CUDA device ordinal */
    int32_t max_cols;                 /* widest result table accepted (default 64) */
    uint64_t rbuf_bytes;              /* initial size of each of the two ping-pong result
                                         buffers (GPUMem rbuf, gpu_mem.hpp:53-60); they grow */
    uint64_t working_set_cap_bytes;   /* serving admission cap (default 40 GiB) */
    int32_t tune;                     /* 1 = run the tile autotuner at store upload */
    int32_t reserved[7];
} wk_config;

/* One segment: segid_t (segment_meta.hpp:159-178) + rdf_seg_meta_t (:87-154), GPU build
 * with one ext-bucket extent (EXT_BUCKET_LIST_CAPACITY 1, :43-45). */
typedef struct wk_seg_meta {
    int32_t index;          /* 0 = normal segment [vid|pid|dir]; 1 = index segment [0|*|dir] */
    uint32_t pid;           /* predicate id (PREDICATE_ID for index segments) */
    int32_t dir;            /* WK_IN / WK_OUT */
    uint32_t reserved;
    uint64_t num_keys;
    uint64_t num_buckets;   /* main-header buckets of the segment (hash space) */
    uint64_t bucket_start;  /* absolute bucket id of its first main-header bucket */
    uint64_t num_edges;
    uint64_t edge_start;
    uint64_t ext_start;     /* ext_bucket_list[0].start (absolute bucket id) */
    uint64_t ext_num;       /* ext_bucket_list[0].num_ext_buckets */
} wk_seg_meta;

/* SPARQLQuery::Pattern (query.hpp:145-170).  Variables are negative (-1, -2, ...),
 * constants are ids >= 0.  pred_type must be 0 (SID_t). */
typedef struct wk_pattern {
    int32_t subject;
    int32_t predicate;
    int32_t object;
    int32_t direction;
    int32_t pred_type;
} wk_pattern;

/* A planned basic graph pattern: SPARQLQuery::pattern_group.patterns after
 * Planner::set_direction (planner.hpp:667-699), plus Result::nvars and the mt_factor split
 * of an index start (sparql.hpp:213-224). */
typedef struct wk_query {
    const wk_pattern* patterns;
    int32_t n_patterns;
    int32_t nvars;
    int32_t mt_tid;         /* 0 unless the caller splits an index start */
    int32_t mt_factor;      /* 1 unless the caller splits an index start */
} wk_query;

/* Synthetic LUBM-shaped graph generator parameters. */
typedef struct wk_synth_params {
    uint64_t seed;
    uint32_t n_orgs;
    int32_t zipf;           /* 0 = uniform degreeFrom targets / course choice, 1 = Zipf */
    double zipf_s;          /* Zipf exponent when zipf = 1 (default 1.1) */
} wk_synth_params;

/* Ids the generator assigned; entity classes are written in this order per org. */
typedef struct wk_synth_vocab {
    uint32_t t_org, t_unit, t_person_a, t_person_b, t_person_c, t_course, t_doc;
    uint32_t p_sub_org_of, p_member_of, p_takes, p_degree_from, p_author;
    uint32_t first_vid;     /* first vertex id (2^17) */
    uint32_t next_vid;      /* one past the last vertex id */
} wk_synth_vocab;

/* Serving configuration (wk_serve_run_open_loop).  Zero fields take defaults. */
typedef struct wk_serve_config {
    uint64_t working_set_cap_bytes;   /* admission cap on projected table bytes (40 GiB) */
    uint64_t arena_bytes;             /* initial bytes of each of the two table arenas (1 GiB);
                                         they grow up to the cap when a step needs more */
    uint64_t min_proj_bytes;          /* floor of one query's projected bytes (64 KiB).  A
                                         query's projection is the input + output table bytes of
                                         its widest step, with rows taken from the store's
                                         metadata: an index start's exact list length, a mean
                                         degree (edges / keys of the segment) for a constant
                                         start and each known_to_unknown step, and unchanged
                                         rows through a filter step */
    uint64_t lane_table_bytes;        /* table bytes each lane is sized for before the run
                                         (0: the largest projection among the run's index-start
                                         queries, at most 1 GiB) */
    uint32_t max_inflight;            /* constant-start queries resident at once (default 65536) */
    uint32_t max_heavy_inflight;      /* index-start queries running at once (default 1); each
                                         runs whole on its own lane: a stream of the lowest
                                         priority with its own tables, beside the iterations */
    int32_t light_ctas_per_sm;        /* exploration CTAs per SM of the iteration launches; the
                                         lanes leave these slots free so iterations never wait
                                         for an index-start step (default 2) */
    int32_t blind;                    /* 1: tables stay on the device and only row counts come
                                         back, as the reference's emulator runs its queries
                                         (result.blind, console_proxy.hpp:395) */
    int32_t reserved[2];
} wk_serve_config;

/* Per-query outcome of a batch or a serving run. */
typedef struct wk_qresult {
    uint64_t rows;           /* rows of the final table */
    uint64_t elem_offset;    /* where its table starts in the caller's output buffer */
    int32_t cols;            /* Result::col_num */
    int32_t status;          /* WK_* status of this query */
    double t_arrive_us;      /* serving: arrival time (open-loop schedule) */
    double t_done_us;        /* serving: completion time (result on the host) */
} wk_qresult;

/* ---------------------------------------------------------------- errors */
const char* wk_strerror(int code);                 /* message for a status (errors.hpp:48-62) */
const char* wk_last_error(const wk_ctx* ctx);      /* detail of the context's last failure */

/* ---------------------------------------------------------------- synthetic data + host store */

/* Generate the seeded LUBM-shaped triple set as n x (s, p, o) uint32 rows.  *triples is
 * allocated by the library and released with wk_free.  (Stands in for the loader's id
 * files, base_loader.hpp:236-280.) */
int wk_synth_generate(const wk_synth_params* p, uint32_t** triples, uint64_t* n_triples,
                      wk_synth_vocab* vocab);
void wk_free(void* p);

/* Build the static segment store on the host from id triples, as
 * SegmentRDFGraph::init_gstore does (segment_rdf_dgraph.hpp:1182-1269) after the loader's
 * sort + dedup (base_loader.hpp:481-496).  pso and pos are the triples to insert in the OUT
 * and IN directions (normally the same array; n x 3 uint32 each).  load_factor is the mean
 * fraction of the 7 data slots of a bucket in use (0 < f <= 1; 0 = default 0.1). */
int wk_gstore_build(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos, uint64_t n_pos,
                    double load_factor, wk_gstore** out);
/* The same, and with versatile != 0 also every vertex's predicate list, as the reference's
 * default (VERSATILE) build inserts it (insert_vp, segment_rdf_dgraph.hpp:365-455): key
 * [vid|PREDICATE_ID|OUT] lists the distinct predicates of subject vid ascending, key
 * [vid|PREDICATE_ID|IN] those of object vid (type ids are never IN keys).  A context whose
 * store holds them runs patterns with an unknown predicate (wk_query_execute and the
 * wk_step_*_unknown_* steps); without them those patterns are WK_UNKNOWN_PATTERN, as in a
 * reference build without VERSATILE.  The global sets [0|TYPE_ID|*] and [0|PREDICATE_ID|OUT]
 * are not built: no pattern operator reads them. */
int wk_gstore_build_ex(const uint32_t* pso, uint64_t n_pso, const uint32_t* pos, uint64_t n_pos,
                       double load_factor, int32_t versatile, wk_gstore** out);
void wk_gstore_free(wk_gstore* g);
int wk_gstore_info(const wk_gstore* g, uint64_t* n_slots, uint64_t* n_edges, uint32_t* n_segs,
                   uint64_t* n_keys);
/* Borrowed views of the built arrays (valid until wk_gstore_free). */
int wk_gstore_arrays(const wk_gstore* g, const void** slots, const uint32_t** edges,
                     const wk_seg_meta** segs);
/* Host-side DGraph::get_triples / get_index (segment_rdf_dgraph.hpp:1114-1129):
 * *sz = 0 and *edges = NULL on a miss. */
int wk_gstore_get_triples(const wk_gstore* g, uint32_t vid, uint32_t pid, int32_t dir,
                          const uint32_t** edges, uint64_t* sz);
int wk_gstore_get_index(const wk_gstore* g, uint32_t tpid, int32_t dir, const uint32_t** edges,
                        uint64_t* sz);

/* ---------------------------------------------------------------- datasets and plans */

/* Read an ID-format dataset directory as the POSIX loader does (posix_loader.hpp:49-70,
 * base_loader.hpp:235-280, 548): every entry whose name starts with "id_" (dot entries
 * skipped), in sorted path order, each read as whitespace-separated decimal "s p o" triples up
 * to the first token that is not a number in [0, 2^32).  *triples (n x 3 uint32) is allocated
 * by the library and released with wk_free; pass it to wk_gstore_build, which sorts and
 * dedups.  Attribute files ("attr_") are not read.  WK_E_BADARG if the directory or a file
 * cannot be opened. */
int wk_load_id_dir(const char* dir, uint32_t** triples, uint64_t* n_triples);

/* Apply a user-defined plan (.fmt text) to a pattern group in written order, as
 * Planner::set_plan and set_direction do (planner.hpp:667-699, 723-770): each line "k dir"
 * takes pattern k (1-based) in that position; dir ">" keeps it (OUT), "<" swaps subject and
 * object (IN), ">>" and "<<" turn it into a predicate-index pattern (OUT / IN).  A line
 * without a direction keeps the previous one (initially ">"); "#" lines, blank lines and "{"
 * are skipped, "}" ends the group.  WK_E_BADARG when fewer lines than patterns or a line names
 * no pattern, WK_E_UNSUPPORTED for union / optional groups, WK_E_CAPACITY when out_cap is too
 * small.  *n_out = the number of planned patterns. */
int wk_plan_apply_fmt(const wk_pattern* patterns, int32_t n_patterns, const char* fmt_text,
                      wk_pattern* out, int32_t out_cap, int32_t* n_out);

/* ---------------------------------------------------------------- device context */
int wk_ctx_create(const wk_config* cfg, wk_ctx** out);
int wk_ctx_destroy(wk_ctx* ctx);
int wk_ctx_sync(wk_ctx* ctx);
/* The context's CUDA stream (cudaStream_t), for callers that time or order work on it. */
int wk_ctx_stream(wk_ctx* ctx, void** stream);
/* Read and clear the sticky device-side error bits of the context stream (syncs); returns
 * WK_E_CORRUPT / WK_E_TIMEOUT / WK_E_CAPACITY or 0. */
int wk_ctx_check(wk_ctx* ctx);

/* Upload a static segment store in Wukong's layout: slots = vertex_t[n_slots] (16 B each),
 * edges = edge_t[n_edges] (uint32), segs = one entry per segment.  Replaces
 * GPUCache::load_segment paging (gpu_cache.hpp:341-425): the whole store stays resident. */
int wk_store_upload(wk_ctx* ctx, const wk_seg_meta* segs, uint32_t n_segs, const void* slots,
                    uint64_t n_slots, const uint32_t* edges, uint64_t n_edges);
int wk_store_upload_gstore(wk_ctx* ctx, const wk_gstore* g);
/* Build the store on the device from n x 3 (s, p, o) id triples in host memory (used for both
 * directions, as wk_gstore_build is normally called): the same layout, byte for byte, as
 * wk_gstore_build_ex with the same load factor and versatile flag, in place of the host build
 * and upload.  The loader's sort + dedup (base_loader.hpp:481-496) and
 * SegmentRDFGraph::init_gstore (segment_rdf_dgraph.hpp:1182-1269) run as radix sorts, scans and
 * a placement pass on the device.  Replaces the context's store.  At most 2^32 - 1 triples;
 * load_factor 0 takes the default 0.1. */
int wk_store_build_device(wk_ctx* ctx, const uint32_t* triples, uint64_t n_triples, double load_factor,
                          int32_t versatile);
/* Copy the context's store to host memory in wk_store_upload's layout.  With all three array
 * pointers null only the sizes are returned; otherwise each non-null array must hold its size
 * (WK_E_CAPACITY).  No reference counterpart. */
int wk_store_export(wk_ctx* ctx, void* slots, uint64_t slots_cap, uint32_t* edges, uint64_t edges_cap,
                    wk_seg_meta* segs, uint32_t segs_cap, uint64_t* n_slots, uint64_t* n_edges, uint32_t* n_segs);
/* Device bytes held by the store (slots + edges + segment table). */
int wk_store_bytes(const wk_ctx* ctx, uint64_t* bytes);

/* ---------------------------------------------------------------- result tables */
/* A device result table: row-major uint32, col_num * r + c (query.hpp:501-509). */
int wk_table_alloc(wk_ctx* ctx, uint64_t capacity_elems, wk_table** out);
int wk_table_free(wk_ctx* ctx, wk_table* t);
/* GPUEngineCuda::load_result_buf (gpu_engine_cuda.hpp:90-106). */
int wk_table_upload(wk_ctx* ctx, wk_table* t, const uint32_t* host, uint64_t rows, int32_t cols);
/* The final thrust::copy D2H (gpu_engine_cuda.hpp:189-193); cap_elems bounds the copy. */
int wk_table_download(wk_ctx* ctx, const wk_table* t, uint32_t* host, uint64_t cap_elems);
int wk_table_shape(wk_ctx* ctx, const wk_table* t, uint64_t* rows, int32_t* cols);
/* The post-pattern stage on the device, as SPARQLEngine::final_process applies it without
 * ORDER BY (sparql.hpp:1419-1546): with `distinct`, the rows sorted by all their columns
 * (signed 32-bit order) and, of each run of neighbours equal on the required columns, the first
 * kept; then `offset` rows dropped and at most `limit` kept (limit < 0: all); then the
 * projection onto keep_cols, the required variables' columns in their order.  The result goes
 * to `out` (grown as needed; not `in`).  An empty input comes back empty with its columns
 * unchanged, as the reference leaves it; WK_NO_REQUIRED_VAR if n_keep == 0; WK_E_CAPACITY for a
 * table of more than 32 columns (the context's column limit) or of 2^32 rows or more;
 * WK_E_CORRUPT for an input whose row count is past its capacity.  ORDER BY compares the ids'
 * strings in the reference and is not offered. */
int wk_table_final_process(wk_ctx* ctx, const wk_table* in, const int32_t* keep_cols, int32_t n_keep,
                           int32_t distinct, int64_t offset, int64_t limit, wk_table* out);
/* The BOUND filters of a query on the device: SPARQLEngine::bound_filter (sparql.hpp:1222-1234)
 * for each column in bound_cols, ANDed as execute_filter applies a query's filters
 * (sparql.hpp:1356-1376).  A row of `in` is kept when none of those columns holds BLANK_ID
 * (0xFFFFFFFF, an unbound variable); kept rows keep their order and all their columns and go to
 * `out` (grown as needed; not `in`).  n_bound == 0 copies the table.  At most 64 columns;
 * WK_E_BADARG for a column out of range, WK_E_CORRUPT for an input whose row count is past its
 * capacity. */
int wk_table_filter_bound(wk_ctx* ctx, const wk_table* in, const int32_t* bound_cols, int32_t n_bound,
                          wk_table* out);
/* Device address of the table's first element (for callers that keep data on the GPU). */
int wk_table_device_ptr(wk_ctx* ctx, const wk_table* t, uint32_t** dptr);

/* ---------------------------------------------------------------- one exploration step
 * Each call runs one planned pattern over `in` and writes the next table to `out`
 * (grown if needed), then synchronises.  Column indices are Result::var2col values. */

/* IDX P ?X — GPUEngine::index_to_unknown (gpu_engine.hpp:65-100; CPU-only in the reference,
 * GPU stub gpu_engine_cuda.hpp:108-111).  dir picks [0|tpid|dir]. */
int wk_step_index_to_unknown(wk_ctx* ctx, uint32_t tpid, int32_t dir, int32_t mt_tid,
                             int32_t mt_factor, wk_table* out);
/* C P ?X — GPUEngine::const_to_unknown (gpu_engine.hpp:102-125). */
int wk_step_const_to_unknown(wk_ctx* ctx, uint32_t vid, uint32_t pid, int32_t dir, wk_table* out);
/* ?X P ?Y — GPUEngineCuda::known_to_unknown (gpu_engine_cuda.hpp:113-198). */
int wk_step_known_to_unknown(wk_ctx* ctx, const wk_table* in, int32_t col_start, uint32_t pid,
                             int32_t dir, wk_table* out);
/* ?X P ?Y, both known — GPUEngineCuda::known_to_known (gpu_engine_cuda.hpp:200-282). */
int wk_step_known_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_start, int32_t col_end,
                           uint32_t pid, int32_t dir, wk_table* out);
/* ?X P C — GPUEngineCuda::known_to_const (gpu_engine_cuda.hpp:284-363). */
int wk_step_known_to_const(wk_ctx* ctx, const wk_table* in, int32_t col_start, uint32_t end_vid,
                           uint32_t pid, int32_t dir, wk_table* out);
/* C P ?X with ?X known (a column of `in`): SPARQLEngine::const_to_known (sparql.hpp:132-189).
 * Keeps the rows whose col_end value is in the list of [vid|pid|dir], in order.  (The GPU
 * engine has no counterpart; the dispatch reaches it for a constant subject whose object an
 * earlier pattern bound.) */
int wk_step_const_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_end, uint32_t vid, uint32_t pid,
                           int32_t dir, wk_table* out);
/* IDX P ?X with ?X known: SPARQLEngine::index_to_known (sparql.hpp:83-130), the first pattern of
 * a group that inherited `in` (a union / optional sub-query).  Keeps the rows whose col_end
 * value is in slice mt_tid of mt_factor of the index list [0|tpid|dir]: equal shares of
 * length / mt_factor, the last slice with the remainder (sparql.hpp:105-116). */
int wk_step_index_to_known(wk_ctx* ctx, const wk_table* in, int32_t col_end, uint32_t tpid, int32_t dir,
                           int32_t mt_tid, int32_t mt_factor, wk_table* out);
/* The unknown-predicate (versatile) steps, on a store built with wk_gstore_build_ex(versatile):
 *   ?X ?P ?Y  known_unknown_unknown (sparql.hpp:600-640): each row of `in` times every (p, y) of
 *             its col_start vertex: the row, then p, then y (two new columns);
 *   ?X ?P C   known_unknown_const (:649-689): each row times every predicate p of its vertex
 *             whose list holds end_vid (one new column);
 *   C ?P ?X   const_unknown_unknown (:559-592): the (p, x) pairs of vid (two columns);
 *   C1 ?P C2  const_unknown_const (:697-739): the predicates of vid reaching end_vid (one).
 * Rows come row-major, then in the vertex's predicate order, then in list order.
 * WK_UNKNOWN_PATTERN on a store without the vertex-predicate lists. */
int wk_step_known_unknown_unknown(wk_ctx* ctx, const wk_table* in, int32_t col_start, int32_t dir,
                                  wk_table* out);
int wk_step_known_unknown_const(wk_ctx* ctx, const wk_table* in, int32_t col_start, uint32_t end_vid,
                                int32_t dir, wk_table* out);
int wk_step_const_unknown_unknown(wk_ctx* ctx, uint32_t vid, int32_t dir, wk_table* out);
int wk_step_const_unknown_const(wk_ctx* ctx, uint32_t vid, uint32_t end_vid, int32_t dir, wk_table* out);

/* known_to_unknown that allocates nothing.  No reference counterpart: the reference allocates
 * its buffers up front (GPUMem) and aborts when they overflow.
 *
 * For callers that must not allocate device memory during a step. Examples: a loop that runs
 * while other streams of the device must not be stalled (cudaFree waits for the whole device),
 * and code that budgets every device byte up front.
 *
 * The scan scratch (control block, per-tile status words, long-list slice queue) is one fixed
 * 448 KiB device array per device, inside the library. The output table must already be large
 * enough, and nothing is grown.
 *
 * Limits:
 * - inputs of at most 4,193,792 rows (16,382 tiles of 256 rows);
 * - at most 8,192 long-list slices.  Every input row whose list is longer than the context's
 *   slice threshold (knob 2: 128 rows unless tuned) takes ceil(length / 2,048) slices, so the
 *   queue holds between 8,192 such rows (about 1 M output rows of 129-row lists) and 16.7 M
 *   output rows of long lists.
 * Beyond them, or when the output does not fit, the call returns WK_E_CAPACITY and
 * wk_last_error says which limit was hit.  An input whose row count is past its capacity (a
 * table left by a step that overflowed) is refused with WK_E_CORRUPT, as wk_table_download
 * refuses it.
 *
 * The first call on a device sets the scratch up: it takes its address and clears it, and
 * leaves the calling thread's current device as it found it. Make that first call before any
 * stream capture on the device.
 *
 * The scratch is shared by every context and stream of the device, so calls that overlap in
 * time on one device race; serialise them.
 *
 * Same arguments and results as wk_step_known_to_unknown. */
int wk_step_known_to_unknown_noalloc(wk_ctx* ctx, const wk_table* in, int32_t col_start, uint32_t pid,
                                     int32_t dir, wk_table* out);

/* ---------------------------------------------------------------- whole query
 * GPUAgent::execute_sparql_query's pattern loop (gpu_agent.hpp:173-246) driving
 * GPUEngine::execute_one_pattern (gpu_engine.hpp:265-338).  On success *out_table holds the
 * final table (owned by the context until the next query on it, or pass a table of your
 * own via wk_query_execute_into), v2c_map[nvars] and *col_num describe its columns. */
int wk_query_execute(wk_ctx* ctx, const wk_query* q, int32_t mode, const wk_table** out_table,
                     int32_t* v2c_map, int32_t* col_num, uint64_t* rows);
/* Check a plan without a device: the dispatch of GPUEngine::execute_one_pattern
 * (gpu_engine.hpp:265-338) over var_stat (query.hpp:409-416) for every pattern.  Returns the
 * status the query would end with for a malformed plan, else 0 with the final v2c_map[nvars]
 * and *col_num. */
int wk_query_validate(const wk_query* q, int32_t max_cols, int32_t* v2c_map, int32_t* col_num);
/* The same for a store with (versatile != 0) or without the vertex-predicate lists: with them a
 * pattern with an unknown predicate dispatches to the versatile operators (sparql.hpp:954-1012);
 * without them it is WK_UNKNOWN_PATTERN (wk_query_validate).  Batches and serving runs refuse
 * plans with versatile steps (WK_E_UNSUPPORTED): those run as single queries. */
int wk_query_validate_ex(const wk_query* q, int32_t max_cols, int32_t versatile, int32_t* v2c_map,
                         int32_t* col_num);
/* Same, with the final table copied to host memory (the reference's new_table vector). */
int wk_query_execute_host(wk_ctx* ctx, const wk_query* q, int32_t mode, uint32_t* host_out,
                          uint64_t cap_elems, int32_t* v2c_map, int32_t* col_num, uint64_t* rows);
/* Enqueue a query on the context stream and return without waiting (RESIDENT or GRAPH mode).
 * The result buffers must already be large enough for it, i.e. the same plan has completed
 * once through wk_query_execute; device-side errors surface through wk_ctx_check. */
int wk_query_enqueue(wk_ctx* ctx, const wk_query* q, int32_t mode);

/* Per-step profile of one query: each step runs alone between CUDA events on the context
 * stream, `iters` times after one warm-up run; kind is 0 index, 1 const, 2 known_to_unknown,
 * 3 known_to_known, 4 known_to_const.  sum_deg = total neighbour-list length the step's
 * probes found (the edges an exhaustive list scan reads). */
typedef struct wk_step_prof {
    int32_t kind;            /* 0..4 as above; 5 = one level of a batch */
    int32_t cols_in;
    int32_t cols_out;
    int32_t reserved;
    uint64_t rows_in;
    uint64_t rows_out;
    uint64_t sum_deg;
    uint64_t alg_bytes;      /* rows in * cols * 4 + 16 per probe + 4 per list entry read
                                + rows out * cols * 4 */
    double ms;               /* mean kernel time of the step */
} wk_step_prof;
int wk_query_profile(wk_ctx* ctx, const wk_query* q, int32_t iters, wk_step_prof* out,
                     int32_t max_steps, int32_t* n_steps);

/* Diagnostics: clock64() cycles each phase of the exploration launch took, summed over CTAs
 * (claim, stage, probe tail, scan, look-back, ranges, write, drain, probe setup, probe walk,
 * membership), in a library built with -DWK_PHASE_TIMING; all zero otherwise.  n >= 12.
 * No reference counterpart. */
int wk_debug_phase_cycles(unsigned long long* out, int32_t n, int32_t reset);
/* Fault injection on the host, for tests: the next time the context reads its device error
 * word after a launch, it also sees `err_bits` (1 overflow, 2 bounded wait gave up, 4 corrupt
 * chain).  The same handling runs as for a real device-side error: growth and rerun for an
 * overflow, WK_E_TIMEOUT / WK_E_CORRUPT otherwise, with the context usable afterwards.  No GPU
 * fault, trap or hang is involved.  No reference counterpart (the reference aborts). */
int wk_debug_fail_next(wk_ctx* ctx, uint32_t err_bits);

/* Device allocations (cudaMalloc calls) the library has made in this process, over every
 * context.  A caller that must not allocate during some call reads it before and after.  No
 * reference counterpart. */
int wk_debug_device_allocs(uint64_t* count);

/* Tile-schedule knobs of the exploration launch (what the autotuner sets).
 *   knob 0: lanes per probe group of the single-query path (1: one thread per row reading its
 *           home bucket's first 32 bytes; 2, 4 or 8: a group of lanes staging 32-, 64- or
 *           128-byte bucket slices per request);
 *   knob 1: the same for batches and serving;
 *   knob 2: the list length above which a row's output is written as 2,048-row slices by every
 *           CTA (block-per-row) instead of by the CTA that probed it (group-per-row); 8 to
 *           2^23, default 128;
 *   knob 3: the same for batches and serving;
 *   knob 4: single-query steps of index-start plans (and single steps) whose input has at
 *           least this many rows run as the flat count / scan / expand pipeline instead of the
 *           tile launch; 0 never does (default 65,536);
 *   knob 5: a mask over batch levels; level k runs as the flat passes when bit k is set (one
 *           thread per row, full occupancy, output rows split evenly over the grid) and as
 *           the tile launch otherwise (default 0: all tile launches);
 *   knob 6: polls a bounded device-side wait on another CTA (a tile's look-back, a CTA waiting
 *           for the long-list slice queue) makes before it gives up and the call returns
 *           WK_E_TIMEOUT; 0 restores the default (2^24).  A few polls make the waits run out,
 *           which is how the timeout path is tested without hanging or faulting a GPU.
 * wk_ctx_tune_get reads a knob back.  No reference counterpart (its launch shape is fixed,
 * gpu_hash.cu:96-326). */
#define WK_KNOB_LANES 0
#define WK_KNOB_BATCH_LANES 1
#define WK_KNOB_SLICE_ROWS 2
#define WK_KNOB_BATCH_SLICE_ROWS 3
#define WK_KNOB_FLAT_ROWS 4
#define WK_KNOB_BATCH_FLAT 5
#define WK_KNOB_SPIN_LIMIT 6
int wk_ctx_tune_set(wk_ctx* ctx, int32_t knob, int32_t value);
int wk_ctx_tune_get(wk_ctx* ctx, int32_t knob, int32_t* value);

/* The autotuner: times every combination of the knobs above on the caller's own workload and
 * keeps the fastest.  Queries that start from a constant are timed as one batch (knobs 1, 3; CUDA
 * events over `iters` graph replays); index-start queries one at a time, step by step (knob 0
 * per (step kind, input columns), knob 2).  `out` receives the choice and its timings. */
typedef struct wk_tune_result {
    int32_t batch_lanes, batch_slice_rows;   /* chosen for batches */
    int32_t lanes, slice_rows;               /* chosen default for single queries */
    double batch_ms_default, batch_ms_tuned; /* one batch replay, before and after */
    double single_ms_default, single_ms_tuned;   /* sum over the index-start queries */
    int32_t candidates;                      /* configurations timed */
    int32_t batch_flat;                      /* chosen level mask of the flat passes (knob 5) */
    int32_t reserved[2];
} wk_tune_result;
int wk_ctx_autotune(wk_ctx* ctx, const wk_query* queries, uint32_t n, int32_t iters, wk_tune_result* out);

/* Calibration: the rate of independent random 16-byte reads from a fresh `region_bytes` device
 * buffer (each costs one 32-byte DRAM sector once the region is well above L2), timed with CUDA
 * events over `iters` launches on the context stream; the buffer is freed before returning.
 * The copy bandwidth overstates what random probes and short list reads can reach; this is
 * their ceiling.  region_bytes >= 1 MiB.  No reference counterpart. */
int wk_measure_random_reads(wk_ctx* ctx, uint64_t region_bytes, int32_t iters, double* reads_per_s);

/* ---------------------------------------------------------------- batching
 * Run n planned queries together: all queries advance one pattern per level inside one
 * persistent kernel fed by a device work queue, levels replayed from a CUDA graph.  No
 * counterpart in the reference (it runs one query per GPU agent at a time). */
int wk_batch_execute(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t* host_out,
                     uint64_t cap_elems, wk_qresult* results);
/* A stream of batches: queries[0..n) run as consecutive batches of `batch` queries (0: 16,384)
 * with the same launches and results as wk_batch_execute per batch, but pipelined.  While the
 * device runs one batch, the host resolves the next one's plans and the previous one's tables
 * are copied to host_out on a second stream.  Tables are laid out back to back in query
 * order.  No counterpart in the reference. */
int wk_batch_execute_stream(wk_ctx* ctx, const wk_query* queries, uint32_t n, uint32_t batch,
                            uint32_t* host_out, uint64_t cap_elems, wk_qresult* results);
/* Device-only variant: results stay on the device (for throughput timing).  *total_rows
 * receives the sum of final rows. */
int wk_batch_execute_device(wk_ctx* ctx, const wk_query* queries, uint32_t n,
                            uint64_t* total_rows);
/* Replay the last batch of this context on its stream and return without waiting (for
 * device-side timing of an identical batch; errors surface through wk_ctx_check). */
int wk_batch_replay(wk_ctx* ctx);
/* Per-level profile of a batch: each level launch between CUDA events on the context stream,
 * averaged over `iters` runs after one warm-up; out[k].kind = 5, followed by three entries
 * timing the setup memsets (kind 6), the result scan (7) and the gather (8). */
int wk_batch_profile(wk_ctx* ctx, const wk_query* queries, uint32_t n, int32_t iters,
                     wk_step_prof* out, int32_t max_levels, int32_t* n_levels);

/* ---------------------------------------------------------------- serving
 * Continuous batching over an open-loop arrival schedule (no reference counterpart; shaped
 * like ConsoleProxy::run_query_emu, console_proxy.hpp:287-439).  arrival_us[i] is when
 * query i arrives, relative to the start of the run; results are copied to host_out. */
int wk_serve_run_open_loop(wk_ctx* ctx, const wk_serve_config* cfg, const wk_query* queries,
                           uint32_t n, const double* arrival_us, uint32_t* host_out,
                           uint64_t cap_elems, wk_qresult* results);

#ifdef __cplusplus
}
#endif

#endif /* WUKONG_B200_H */
