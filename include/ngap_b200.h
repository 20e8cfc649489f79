/*
 * ngap_b200 — C ABI of the B200 automata-processing engine.
 *
 * The reference (getianao/ngAP) has no FFI; its in-process boundary is
 * `class ngap` (code/src/ngap/ngap.h:27-177) driven by the CLI
 * (code/src/ngap/main.cu:16-137). Each entry point below replaces one step of
 * that flow; the reference interface it replaces is cited beside it.
 *
 * Conventions: every function returns an int status (NGAP_OK = 0) unless
 * stated; ngap_last_error() gives the calling thread's last message. Nothing
 * here calls exit(). Objects are not shared between host threads; the CUDA
 * stream is passed explicitly. Report encoding is the reference's
 * (ngap.cu:1899-1905): ((uint64)(sid | group << 22) << 32) | input_offset,
 * sorted by (offset, id) and deduplicated (ngap.cu:19-30, 1928-1932).
 */
#ifndef NGAP_B200_H_
#define NGAP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define NGAP_OK 0
#define NGAP_E_INVALID 1          /* bad argument */
#define NGAP_E_PARSE 2            /* ANML malformed or uses an unsupported element */
#define NGAP_E_UNSUPPORTED 3      /* unsupported file type or size */
#define NGAP_E_DEGREE 4           /* a CC's out-degree could not be limited (quit requested) */
#define NGAP_E_CUDA 5             /* CUDA runtime error (message has details) */
#define NGAP_E_OVERFLOW_QUEUE 6   /* a worklist exceeded its capacity; results incomplete */
#define NGAP_E_OVERFLOW_RESULTS 7 /* more reports than result_capacity; results truncated */
#define NGAP_E_TIMEOUT 8          /* a bounded device wait gave up */
#define NGAP_E_NOMEM 9            /* allocation failed */
#define NGAP_E_IO 10              /* file could not be read */

/* ---- algorithms (the --algorithm values, code/src/ngap/main.cu:114-130) ---- */
#define NGAP_ALGO_BLOCKING 0        /* blockinggroups      (BAP, kernel_ngap_O0.cu) */
#define NGAP_ALGO_NAP 1             /* NAPgroups           (kernel_bap.cu) */
#define NGAP_ALGO_NONBLOCKING 2     /* nonblockinggroups   (O1, kernel_ngap_O1.cu) */
#define NGAP_ALGO_NONBLOCKING_R1 3  /* nonblockingr1groups (kernel_ngap_O4.cu:7) */
#define NGAP_ALGO_NONBLOCKING_R2 4  /* nonblockingr2groups (kernel_ngap_O4.cu:240) */
#define NGAP_ALGO_NONBLOCKING_PC 5  /* nonblockingpcgroups (O1+O2, kernel_ngap_O3.cu) */
#define NGAP_ALGO_NONBLOCKING_ALL 6 /* nonblockingallgroups (O1+O2+O3, kernel_ngap_OA.cu) */

typedef struct ngap_nfa ngap_nfa;       /* parsed ANML */
typedef struct ngap_groups ngap_groups; /* group graphs after preprocessing */
typedef struct ngap_tables ngap_tables; /* device-resident matching tables */
typedef struct ngap_engine ngap_engine; /* device buffers, results, timing */

/* ---- front-end ---- */

/* Replaces load_nfa_from_file / load_nfa_from_anml (code/src/commons/NFALoader.cpp:70-171). */
int ngap_nfa_load_anml(const char* path, ngap_nfa** out);
/* Same, from an in-memory ANML document. */
int ngap_nfa_parse_anml(const char* xml, size_t len, ngap_nfa** out);
void ngap_nfa_destroy(ngap_nfa* nfa);
/* Counts of NFA::size / NFA::edge_size (code/src/commons/NFA.cpp:411-417). */
int64_t ngap_nfa_num_states(const ngap_nfa* nfa);
int64_t ngap_nfa_num_edges(const ngap_nfa* nfa);

typedef struct ngap_group_opts {
  int group_num;     /* --group-num (reference default 10) */
  int max_nfa_size;  /* --max-nfa-size, -1 = no limit */
  int quit_degree;   /* --quit-degree (default 1) */
  int remove_degree; /* --remove-degree (default 0) */
} ngap_group_opts;

/* Replaces ngap::preprocessing (code/src/ngap/ngap.cu:63-91) followed by
 * nfa_utils::group_nfas_by_num (code/src/commons/nfa_utils.cpp:382-424) and
 * Graph::ReadNFA per group (code/src/commons/graph.cu:169-206). */
int ngap_groups_build(const ngap_nfa* nfa, const ngap_group_opts* opts, ngap_groups** out);
int ngap_groups_count(const ngap_groups* g);
/* CCs before limiting, CCs dropped by the degree limiter, CCs dropped by size. */
int ngap_groups_cc_stats(const ngap_groups* g, int64_t* total, int64_t* failed, int64_t* too_big);

/* Host view of one group graph; pointers stay valid until ngap_groups_destroy. */
typedef struct ngap_group_view {
  int32_t num_states;
  int32_t num_edges;
  int32_t num_aas;
  int32_t num_start;
  int32_t num_ccs;
  const int32_t* row_offsets;  /* [num_states + 1] */
  const int32_t* col_indices;  /* [num_edges], sorted by (src, dst) */
  const uint32_t* symbol_sets; /* [num_states * 8], bit s of word s/32 */
  const uint8_t* node_attrs;   /* bit0 always-active, bit1 report */
  const int32_t* always_active;/* [num_aas], ascending */
  const int32_t* start_states; /* [num_start], start-of-data, ascending */
  const int32_t* cc_begin;     /* [num_ccs + 1], first state of each CC */
  const int32_t* orig_node;    /* [num_states], index of the ANML STE each state came from */
} ngap_group_view;
int ngap_group_view_get(const ngap_groups* g, int group, ngap_group_view* out);
void ngap_groups_destroy(ngap_groups* g);

/* ---- device tables ---- */

typedef struct ngap_table_opts {
  int device;            /* CUDA device ordinal */
  int precompute_depth;  /* --precompute-depth: prefix-memoization depth 0..12 (the
                            reference allows 0..3; keys are byte-class ids, so
                            deeper tables stay small); -1 = as deep as the size
                            caps allow */
  int precompute_cutoff; /* --precompute-cutoff, -1 = mean list length (precompute_table.cu:171) */
  int tile_states;       /* max states per tile; 0 = automatic */
  int64_t max_table_entries; /* cap on prefix-table list entries per tile; 0 = automatic */
  int tile_mode;         /* NGAP_TILES_*: where tiles of acyclic CCs keep their tables */
} ngap_table_opts;

/* Tile modes. Shared: every tile is sized to stage its tables in one CTA's
 * shared memory (one group per tile). Global: the acyclic CCs of all groups
 * form few large tiles read through L2, so each input position is looked up
 * once per large tile instead of once per small one. Auto picks global when
 * the acyclic CCs need more than two shared-memory tiles. Cyclic CCs always
 * use shared-memory tiles. No mode changes any report. */
#define NGAP_TILES_AUTO 0
#define NGAP_TILES_SHARED 1
#define NGAP_TILES_GLOBAL 2

/* Replaces GroupCsr/GroupMatchset/GroupNodeAttrs/GroupAAS::init
 * (code/include/commons/group_graph.h:6-109) and ngap::initGroupCsrWithPrec
 * (code/src/ngap/ngap.cu:3086-3111, prefix tables ngap.cu:2358-2513). */
int ngap_tables_build(const ngap_groups* g, const ngap_table_opts* opts, ngap_tables** out);
void ngap_tables_destroy(ngap_tables* t);
/* The tiles ngap_tables_build would make, planned on the host only (no
 * device memory, no GPU needed): one record per tile, at most cap; *n = tile
 * count. The reference has no tiles (its unit of work is a whole group,
 * code/src/ngap/ngap.cu:1507); this exposes the partition for inspection. */
typedef struct ngap_tile_desc {
  int32_t phase;      /* 0 plain, 1 activation (dot-star CCs), 2 layered */
  int32_t pair;       /* activation/layered pair index, -1 for plain tiles */
  int32_t group;      /* group of the tile's first CC */
  int32_t num_states, num_ccs;
  int32_t nact;       /* sticky states of the pair (activation slots) */
  int32_t nsticky;    /* sticky states handled in the tile */
  int32_t global;     /* 1: tables read through L2 (several groups possible) */
  int32_t depth;      /* prefix-table depth */
  int32_t max_path;   /* longest acyclic path (chunk warm-up + 1); -1 = cyclic */
  int32_t nlive;      /* live byte classes */
  int32_t dense_levels; /* bit d-1 set: table d is dense (offsets by key), else hashed */
  int32_t naas;       /* always-active states in the tile */
  int32_t shortcuts;  /* layered tiles: successors their sticky states enable from their
                         first match on (edges of the CC's states into them dropped) */
  int64_t table_bytes; /* prefix tables and image */
} ngap_tile_desc;
int ngap_tiles_describe(const ngap_groups* g, const ngap_table_opts* opts, ngap_tile_desc* out,
                        int cap, int* n);

/* Host-only check of the prefix tables (no GPU): plans the tiles as
 * ngap_tiles_describe does, then looks up nkeys byte strings of len bytes
 * each (keys: nkeys * len bytes; 1 <= len <= the tile's depth) in table len
 * of tile `tile` the way the matching kernel does (byte -> class -> base-L
 * key; dense offsets or hash slots). Table d of the reference maps d symbols
 * to the states reached after them from the always-active states
 * (code/src/ngap/ngap.cu:2358-2468, precompute_table.h:8-101). For key k,
 * ids[off[k] .. off[k+1]) are the report ids (group-local sid | group << 22)
 * of the listed states and reports[roff[k] .. roff[k+1]) those of its report
 * states (in an activation tile, phase 1, a sticky state's id is its
 * activation slot); off and roff hold nkeys + 1 entries and ids and reports room for
 * cap entries each. When cap is too small the call returns NGAP_E_INVALID
 * with off[nkeys] and roff[nkeys] set to the entries needed. */
int ngap_tiles_lookup(const ngap_groups* g, const ngap_table_opts* opts, int tile,
                      const uint8_t* keys, int nkeys, int len, uint32_t* ids, int64_t* off,
                      uint32_t* reports, int64_t* roff, int64_t cap);

/* Bytes of device memory held by the tables. */
int64_t ngap_tables_device_bytes(const ngap_tables* t);

/* ---- engine ---- */

/* Replaces NonBlockingBuffer/BlockingBuffer allocation (code/src/ngap/ngap_buffer.cu:111-748). */
int ngap_engine_create(int device, ngap_engine** out);
void ngap_engine_destroy(ngap_engine* e);

typedef struct ngap_match_params {
  int algorithm;             /* NGAP_ALGO_* */
  int64_t num_seg;           /* input segments (main.cu:88-102) */
  int64_t seg_len;           /* bytes per segment; input holds num_seg * seg_len bytes */
  int is_dup;                /* start-of-data states in every segment (ngap_buffer.cu:479-484) */
  int unique;                /* --unique: drop duplicate worklist entries within a step */
  int active_threshold;      /* --active-threshold: busy-lane count enabling privatization */
  int report_off;            /* --report-off: count reports only */
  uint64_t result_capacity;  /* --result-capacity */
  int window;                /* positions per worklist window; 0 = automatic */
  int chunk;                 /* positions per chunk of a bounded tile; 0 = automatic */
  int64_t first_segment;     /* global index of the first segment when a stream is
                                split across GPUs (start-of-data states belong to
                                global segment 0); 0 otherwise */
} ngap_match_params;

/* Replaces ngap::launch_*_groups (code/src/ngap/ngap.cu:115-2078) up to the
 * report copy: matches `input` (host or device memory, num_seg * seg_len
 * bytes) against every group and leaves the sorted, deduplicated reports on
 * the device. Asynchronous on `stream` (a cudaStream_t, NULL = default);
 * ngap_engine_sync waits and returns the run's status. */
int ngap_match(ngap_engine* e, const ngap_tables* t, const uint8_t* input, int input_on_device,
               const ngap_match_params* p, void* stream);
int ngap_engine_sync(ngap_engine* e);

/* Results of the last ngap_match (after ngap_engine_sync). raw = reports
 * emitted by the kernel (duplicates included), unique = after sort+unique. */
int ngap_results_count(const ngap_engine* e, uint64_t* raw, uint64_t* unique);
/* Device pointer to the unique reports (valid until the next match). */
const uint64_t* ngap_results_device(const ngap_engine* e);
/* Copies up to cap unique reports to host memory; returns how many were copied. */
int64_t ngap_results_copy(ngap_engine* e, uint64_t* host, uint64_t cap);
/* Device time of the last match in milliseconds: [0] matching kernel, [1] sort+unique. */
int ngap_last_times_ms(const ngap_engine* e, float* match_ms, float* sort_ms);
/* Kernel launches issued by the last ngap_match. */
int ngap_last_launches(const ngap_engine* e);
/* Worklist entries expanded and always-active entries injected by the last match. */
int ngap_engine_work(const ngap_engine* e, uint64_t* expanded, uint64_t* injected);
/* Bytes of device memory the engine holds (input copy, reports, per-warp scratch). */
int64_t ngap_engine_device_bytes(const ngap_engine* e);
/* The same, by part. The reference allocates its buffers once per run
 * (NonBlockingBuffer::init_nfagroups, code/src/ngap/ngap_buffer.cu:475-748);
 * an engine's buffers only grow, so a caller sharing the device (the serving
 * loop's memory budget) can tell what a larger batch would add. */
typedef struct ngap_engine_mem {
  int64_t input;    /* the engine's copy of the input (largest batch so far, padded) */
  int64_t reports;  /* raw and unique report buffers, sort scratch, stream ids */
  int64_t scratch;  /* per-warp worklist scratch: overflow stacks, carry lists, bitmaps */
  int64_t plan;     /* units, tasks, activation slots, unit traces */
} ngap_engine_mem;
int ngap_engine_memory(const ngap_engine* e, ngap_engine_mem* out);

/* Test hook for the kernel's one device wait, the mbarrier of a window's
 * input copy (the reference has no bounded waits; its kernels poll their
 * worklists, kernel_ngap_OA.cu:142). For the next ngap_match only, unit
 * `unit` (in plan order) does not issue its first window's copy and every wait
 * gives up after `wait_rounds` try_wait rounds: that unit's wait runs out with
 * nothing in flight, and ngap_engine_sync returns NGAP_E_TIMEOUT. The engine
 * stays usable; the following match runs normally. */
int ngap_engine_test_wait_timeout(ngap_engine* e, int32_t unit, int32_t wait_rounds);

/* ---- worklist traces ---- */

/* Generalises --motivate-worklist-length (code/src/ngap/kernel_ngap_OA.cu:366-369,
 * code/src/ngap/ngap.cu:1843-1866), which records the fetched worklist length
 * per round: with tracing on, every later match (plain or batched) records
 * the worklist work and the duration of each unit (one tile over one chunk
 * of a segment or stream). */
typedef struct ngap_unit_trace {
  int32_t stream;   /* segment (ngap_match) or stream (ngap_batch_match) index */
  int32_t tile;     /* tile index (in the tableset for batched matches) */
  int64_t lo, hi;   /* positions whose reports the unit owns, relative to its segment/stream */
  uint64_t work;    /* worklist entries the unit expanded plus entries it injected */
  uint64_t cycles;  /* SM clock cycles from the unit's start to its end (one warp) */
} ngap_unit_trace;
int ngap_engine_set_trace(ngap_engine* e, int enable);
/* Copies up to cap of the last match's unit records (after ngap_engine_sync);
 * *n = records copied, or with out = NULL the number of records. */
int ngap_trace_copy(ngap_engine* e, ngap_unit_trace* out, int64_t cap, int64_t* n);

/* Statistics of built tables, the NFA features of the cost model. The
 * reference sizes its adaptive AAS interval from the longest table list
 * (maxkey, code/src/ngap/kernel_ngap_OA.cu:180-194). */
typedef struct ngap_tables_stats {
  int32_t tiles, states, edges, aas;
  int32_t depth;          /* deepest prefix table */
  int32_t max_nlive;      /* live byte classes (key base) */
  int32_t max_list;       /* longest list of a deepest table (maxkey) */
  int32_t cutoff;         /* sum over tiles of the mean non-empty deepest list length */
  int64_t list_entries;   /* entries of the deepest tables, all tiles */
  double exp_list;        /* sum over tiles of the deepest tables' mean list length per key
                             (all keys equally likely): states injected per position */
} ngap_tables_stats;
int ngap_tables_stats_get(const ngap_tables* t, ngap_tables_stats* out);

/* ---- batched matching: many streams, several NFAs, one launch ---- */

/* The reference matches one (duplicated) stream against one NFA per run
 * (code/src/ngap/main.cu:81-131) with a rigid (group, segment) grid
 * (code/src/ngap/ngap.cu:1507). A tableset combines the tables of several
 * NFAs so that streams of uneven length, each against its own NFA, run in one
 * persistent launch. The tables must outlive the tableset. */
typedef struct ngap_tableset ngap_tableset;
int ngap_tableset_create(const ngap_tables* const* tables, int n, ngap_tableset** out);
void ngap_tableset_destroy(ngap_tableset* ts);

typedef struct ngap_batch_stream {
  uint64_t offset;  /* first byte of the stream in the batch input */
  uint64_t length;  /* bytes; the stream is one segment (start-of-data states at its start) */
  int32_t nfa;      /* index into the tableset */
  int32_t chunk;    /* chunk length for this stream's acyclic tiles; 0 = the batch's */
} ngap_batch_stream;

typedef struct ngap_batch_params {
  int algorithm;            /* NGAP_ALGO_* */
  int unique;
  int active_threshold;
  int report_off;
  uint64_t result_capacity;
  int window;               /* 0 = automatic */
  int chunk;                /* 0 = automatic */
  int use_graph;            /* capture the pipeline in a CUDA graph; replay it while the
                               tableset, streams, parameters and input pointer repeat */
  int queue_capacity;       /* overflow-stack entries per warp (>= 1024); 0 = 65536. An
                               engine keeps the largest capacity it has held (a smaller
                               request runs with that one). A run that needs more fails
                               with NGAP_E_OVERFLOW_QUEUE */
} ngap_batch_params;

/* Matches every stream against its NFA in one persistent launch, then sorts
 * the reports by (stream, offset, id) on the device. Asynchronous on stream;
 * ngap_engine_sync waits. Offsets in the results are local to each stream. */
int ngap_batch_match(ngap_engine* e, const ngap_tableset* ts, const uint8_t* input,
                     uint64_t input_bytes, int input_on_device, const ngap_batch_stream* streams,
                     int nstreams, const ngap_batch_params* p, void* stream);
/* Copies up to cap unique reports (reference encoding) and, when stream_ids is
 * not NULL, the stream index of each; *n receives the count copied. */
int ngap_batch_results(ngap_engine* e, uint64_t* reports, uint32_t* stream_ids, uint64_t cap,
                       uint64_t* n);

/* ---- learned cost model ---- */

/* The reference has no cost model: it records the fetched worklist length per
 * round (--motivate-worklist-length, code/src/ngap/kernel_ngap_OA.cu:366-369)
 * and sizes its adaptive AAS interval from the longest table list
 * (kernel_ngap_OA.cu:180-194). These entry points compute input features and
 * train / run a small regressor on the engine's own worklist traces
 * (ngap_trace_copy); the scheduler above them (ngap_b200/cost_model.py)
 * predicts worklist entries per input byte. */
#define NGAP_FEAT_BYTES 258 /* 256-bin histogram, mean and max windowed entropy */

/* Features of n regions of data (device or host memory of `bytes` bytes):
 * region i (offsets[i], lengths[i]) gets out[i * NGAP_FEAT_BYTES + k]: the
 * symbol histogram normalised to sum 1 (k < 256), then the mean (k = 256) and
 * the largest (k = 257) Shannon entropy of its windows of `window` bytes, in
 * bits / 8. out is host memory; the call waits for the result. */
int ngap_features(const uint8_t* data, uint64_t bytes, int on_device, const uint64_t* offsets,
                  const uint64_t* lengths, int n, int window, float* out, void* stream);

/* The same features computed on the host, for bytes that are still in host
 * memory (a serving loop predicting a request's work before its batch is
 * formed): no device memory, no copy, no synchronisation. */
int ngap_features_host(const uint8_t* data, uint64_t bytes, const uint64_t* offsets,
                       const uint64_t* lengths, int n, int window, float* out);

/* A regressor with two hidden ReLU layers of `hidden` (= 64) units and one
 * linear output; FP32 parameters on the device. */
typedef struct ngap_mlp ngap_mlp;
int ngap_mlp_create(int device, int in_dim, int hidden, uint64_t seed, ngap_mlp** out);
void ngap_mlp_destroy(ngap_mlp* m);
/* Adam on the mean squared error over x[n][in_dim], y[n] (host arrays):
 * `epochs` shuffled passes in mini-batches of `batch`; *loss receives the
 * last epoch's mean squared error. FP32 throughout. */
int ngap_mlp_train(ngap_mlp* m, const float* x, const float* y, int64_t n, int epochs, int batch,
                   float lr, float* loss);
/* Gradient of the mean squared error over all n samples x[n][in_dim], y[n]
 * (host arrays) at the current parameters, in the layout of
 * ngap_mlp_get_params, into grad (host, room for every parameter); *loss
 * receives the mean squared error. Parameters are not changed: this is the
 * step ngap_mlp_train feeds to Adam, exposed for checking. */
int ngap_mlp_gradient(ngap_mlp* m, const float* x, const float* y, int64_t n, float* grad,
                      float* loss);
/* y[n] = model(x[n][in_dim]) (host arrays). bf16 = 1 rounds inputs, weights and
 * activations to bfloat16 (FP32 accumulation); 0 computes in FP32. Runs on
 * the model's own stream; allocates only when n exceeds every earlier call. */
int ngap_mlp_predict(ngap_mlp* m, const float* x, int64_t n, int bf16, float* y);
/* The same predictions computed on the host from a host copy of the
 * parameters (fetched once after each change): for a serving loop, whose GPU
 * is busy with matching kernels that leave no room for the inference kernel
 * until they end. Same bfloat16 roundings and accumulation order per unit as
 * the kernel, but products and sums rounded apart (no fused multiply-add)
 * and the output sum in another order: FP32 rounding differences, which a
 * bfloat16 activation near a rounding boundary can carry to 2^-8 of it. */
int ngap_mlp_predict_host(ngap_mlp* m, const float* x, int64_t n, int bf16, float* y);
/* Parameters as one FP32 vector; *n = count (out = NULL queries it). */
int ngap_mlp_get_params(const ngap_mlp* m, float* out, int64_t cap, int64_t* n);
int ngap_mlp_set_params(ngap_mlp* m, const float* in, int64_t n);

/* ---- report compaction ---- */

/* Sorts n packed reports (reference encoding) in device memory by (offset, id)
 * with the engine's radix sort and removes duplicates; writes the result to
 * d_out (may alias nothing) and its length to *n_out (host). */
int ngap_reports_sort_unique(ngap_engine* e, const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                             uint64_t* n_out, void* stream);

/* Same sort + unique as ngap_reports_sort_unique, but allocating nothing: it
 * has no counterpart in the reference. It is for callers that cannot call
 * cudaMalloc — a process whose device memory is owned by another allocator
 * (for example a framework's caching allocator that has reserved the GPU), or
 * a latency-critical loop where cudaMalloc's implicit synchronisation is not
 * acceptable. The caller passes device input (n reference-encoded reports)
 * and device output (room for n); n must not exceed 262,144 (larger n returns
 * NGAP_E_INVALID). d_out may be d_in. Scratch (about 2 MiB) is a static
 * device array that every GPU loading this library keeps until exit. The
 * first call on a device (and the first after the device's context changes,
 * e.g. after cudaDeviceReset) looks up that array's device address
 * (cudaGetSymbolAddress) with the device current. All calls share the
 * scratch and it keeps the last call's contents; calls that overlap on the
 * GPU race on it. Uses the calling thread's current device. The call waits
 * for `stream` before returning the unique count in *n_out, so it must not be
 * called while `stream` is being captured (it then returns NGAP_E_INVALID). */
int ngap_reports_sort_unique_noalloc(const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                                     uint64_t* n_out, void* stream);

/* ---- CPU checker used by the CLI's --validation (ngap.cu:2171-2344) ---- */

/* Runs the reference's CPU frontier simulation over the group graphs and
 * writes the sorted, deduplicated reports; returns the count or -1 if more
 * than cap. This is a checker for the CLI's --validation flag only: it never
 * produces the engine's results. */
int64_t ngap_cpu_validate_reference(const ngap_groups* g, const uint8_t* input, int64_t num_seg,
                                    int64_t seg_len, int is_dup, uint64_t* out, int64_t cap,
                                    double* elapsed_ms);

/* Message of the calling thread's last error. Returns its length. */
int ngap_last_error(char* buf, size_t n);
/* Library version string. */
const char* ngap_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NGAP_B200_H_ */
