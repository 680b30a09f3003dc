/*
 * pggc.h -- C ABI of the B200-native PGGC clustering hot path.
 *
 * The reference exposes this path as C++ templates over Kokkos types; every
 * entry point below replaces one of them with plain pointers and sizes (no
 * Kokkos, no torch types).  Citations are to the reference project.
 *
 * Conventions
 *   - Every call returns pggc_status; on failure pggc_last_error() returns a
 *     thread-local message.  PGGC_ERR_DEVICE means a device-side bounded loop
 *     (hash probe, pointer chase) gave up; the context stays usable.
 *   - mem_kind says where caller arrays live: PGGC_MEM_HOST (pageable or
 *     pinned host memory, copied in/out inside the call) or PGGC_MEM_DEVICE
 *     (device pointers on the context's device).
 *   - Weight kinds: PGGC_W_UNIFORM (unit weights, `weights` ignored),
 *     PGGC_W_INT32 (int32 weights), PGGC_W_FLOAT32 (float32 weights).
 *     Vertex weights / cluster volumes ("V" arrays) are int64 for the first two
 *     and float64 for PGGC_W_FLOAT32.  Float64 volumes are summed with
 *     order-free atomics, so results are bit-reproducible when every vertex
 *     weight is a multiple of one power of two q and the total weight stays
 *     below 2^53 q (the default weighted degrees of FP32 weights in [0.5, 1.5)
 *     meet it for nnz < 2^29); other float64 vertex weights can differ
 *     between runs in the last bits.
 *   - Graphs are symmetric CSR: int64 row offsets (n+1), int32 columns (nnz),
 *     no self-loops, no duplicate edges.
 *   - Calls on one context are serialised on the context's CUDA stream and
 *     return after the work is complete.
 */
#ifndef PGGC_H
#define PGGC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pggc_status {
    PGGC_OK = 0,
    PGGC_ERR_INVALID = 1,  /* bad argument or unsupported input            */
    PGGC_ERR_CUDA = 2,     /* CUDA runtime error (message has the details)  */
    PGGC_ERR_DEVICE = 3,   /* device-side bounded loop gave up              */
    PGGC_ERR_INTERNAL = 4
} pggc_status;

enum { PGGC_W_UNIFORM = 0, PGGC_W_INT32 = 1, PGGC_W_FLOAT32 = 2 };
/* app/io/parse_args.cpp:10-16 objective names: Mod, WMod, CPM, NLCC, LCC */
enum { PGGC_OBJ_MOD = 0, PGGC_OBJ_WMOD = 1, PGGC_OBJ_CPM = 2, PGGC_OBJ_NLCC = 3, PGGC_OBJ_LCC = 4 };
enum { PGGC_MEM_HOST = 0, PGGC_MEM_DEVICE = 1 };
/* app/CMakeLists.txt:3-7: plouvain, pleiden, pleiden+ */
enum { PGGC_METHOD_LOUVAIN = 0, PGGC_METHOD_LEIDEN = 1, PGGC_METHOD_LEIDEN_PLUS = 2 };

typedef struct pggc_context pggc_context;           /* interface/memory_store.hpp:12-91   */
typedef struct pggc_graph pggc_graph;               /* interface/weighted_graph.h:10-19   */
typedef struct pggc_cluster_data pggc_cluster_data; /* interface/cluster_data.hpp:9-181   */

typedef struct pggc_stats {
    int64_t levels;      /* ExperimentLoggerUtil level count (src/clustering_methods.cpp:123)  */
    int64_t total_nnz;   /* ExperimentLoggerUtil total nnz   (src/clustering_methods.cpp:122)  */
    int64_t sweeps;      /* local-move sweeps executed                                        */
    int64_t moves;       /* vertex moves applied                                              */
    int64_t passes;      /* leiden_part / louvain_part calls (1 + ex_iters passes)            */
    double objective;    /* cluster_data::get_objective() after the call                      */
    double raw_obj;      /* cluster_data::obj                                                 */
    int64_t label_count; /* cluster_data::label_count                                         */
    /* learned move filter judge (run_clustering with a filter enabled; 0 otherwise) */
    int64_t filtered_passes; /* passes run with the filter                                    */
    int64_t exact_passes;    /* exact (unfiltered) passes the judge ran after them              */
    double judge_gain;       /* objective change of those exact passes                         */
    int64_t fell_back;       /* 1 when the judge's first exact pass gained more than
                                PGGC_FILTER_TOLERANCE and the run fell back to exact passes
                                until stable (the plain method)                                */
} pggc_stats;

/* Modularity the learned filter may give up before its judge counts a fallback
 * to the plain sweep. */
#define PGGC_FILTER_TOLERANCE 0.001

const char* pggc_last_error(void);
/* build-time identification, e.g. "pggc-b200 sm_100a" */
const char* pggc_version(void);

/* kernels launched by this library in this process so far */
uint64_t pggc_launch_count(void);

/* Fault injection for tests: cap every hash-table probe sequence at `limit`
 * probes (0 restores the default bound, the table size).  A capped probe that
 * gives up latches a device error and the call returns PGGC_ERR_DEVICE; the
 * context stays usable. */
pggc_status pggc_debug_set_probe_limit(pggc_context* ctx, int limit);

/* Per-kernel-family timing (CUDA events on the context stream) and algorithmic
 * byte counts, for roofline reporting; the counterpart of the reference's
 * EXTRA_TIMING measurements (src/clustering_methods.cpp:78-108).  Families:
 * "select_warp", "select_block", "select_huge", "afterburner_warp",
 * "afterburner_block", "own_weights", "contract", "leiden_refine", "orderings". */
pggc_status pggc_profile_enable(pggc_context* ctx, int on); /* 2: also per level, "family@level" */
pggc_status pggc_profile_reset(pggc_context* ctx);
pggc_status pggc_profile_read(pggc_context* ctx, const char* family, int64_t* launches, double* ms, double* bytes);
/* the recorded family names, newline-separated, into buf (cap bytes, NUL
 * terminated); *needed = the size that holds them all */
pggc_status pggc_profile_names(pggc_context* ctx, char* buf, int64_t cap, int64_t* needed);

/* ---- memory_store (interface/memory_store.hpp:84-90) ---------------------- */
pggc_status pggc_context_create(int device, pggc_context** out);
pggc_status pggc_context_destroy(pggc_context* ctx);
/* the cudaStream_t all calls on this context are issued on */
pggc_status pggc_context_stream(pggc_context* ctx, void** stream_out);

/* ---- weighted_graph (interface/weighted_graph.h:10-19) --------------------
 * Copies the CSR.  vtx_w may be NULL: the objective's default vertex weights
 * are computed (degree for Mod, weighted degree for WMod, 1 otherwise;
 * app/io/vertex_weighting.cpp:27-42). */
pggc_status pggc_graph_create(pggc_context* ctx, int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col,
                              const void* weights, int weight_kind, const void* vtx_w, int objective, int mem_kind,
                              pggc_graph** out);
/* ---- graph input (app/io/io_mtx.cpp:95-345, app/io/io_metis.cpp:64-181) ---
 * pggc_graph_load replaces load_graph(g, uniform_ew, fname)
 * (app/io/io_mtx.cpp:336-345): a path ending in ".mtx" is read as a Matrix
 * Market coordinate file, anything else as a METIS file.  Mod and CPM ignore
 * file weights (uses_edge_weights, app/objective_helpers.hpp:24-29); real
 * weights and weights of non-symmetric files are ignored as in the
 * reference; pattern files have unit weights.  *edge_uniform_out (may be
 * NULL) receives the reference's uniform_ew.  Malformed files, METIS vertex
 * weights and non-square matrices return PGGC_ERR_INVALID.
 * pggc_graph_from_edges replaces construct_from_edgelist (io_mtx.cpp:95-201)
 * for 0-based edge lists: self loops and zero weights dropped, both
 * directions stored, unordered duplicates removed unless `symmetric`, rows
 * sorted by column.  weights (may be NULL) only with symmetric != 0. */
pggc_status pggc_graph_load(pggc_context* ctx, const char* path, int objective, int* edge_uniform_out,
                            pggc_graph** out);
pggc_status pggc_graph_from_edges(pggc_context* ctx, int64_t n, int64_t m, const int32_t* src, const int32_t* dst,
                                  const int32_t* weights, int symmetric, int objective, int mem_kind,
                                  pggc_graph** out);
/* replaces the vertex weights (n values: int64, or double for FP32-weighted
 * graphs), as get_vtx_weights does with -vw_file (app/io/vertex_weighting.cpp:27-30) */
pggc_status pggc_graph_set_vertex_weights(pggc_context* ctx, pggc_graph* g, const void* vtx_w, int mem_kind);
pggc_status pggc_graph_destroy(pggc_graph* g);
pggc_status pggc_graph_dims(const pggc_graph* g, int64_t* n, int64_t* nnz, int* weight_kind);
/* copies out any non-NULL array (weights only for non-uniform graphs) */
pggc_status pggc_graph_read(pggc_context* ctx, const pggc_graph* g, int64_t* rowptr, int32_t* col, void* weights,
                            void* vtx_w, int mem_kind);

/* ---- cluster_data and subclasses (interface/cluster_data.hpp:38-181,
 *      app/objective_helpers.hpp:9-22) --------------------------------------- */
pggc_status pggc_cluster_data_create(pggc_context* ctx, const pggc_graph* g, int objective, double lambda_mult,
                                     pggc_cluster_data** out);
pggc_status pggc_cluster_data_destroy(pggc_cluster_data* cd);
/* any output pointer may be NULL */
pggc_status pggc_cluster_data_get(const pggc_cluster_data* cd, double* obj, double* objective, double* lambda,
                                  double* uncut, int64_t* label_count);
/* total_deg[0..label_count) */
pggc_status pggc_cluster_data_total_deg(pggc_context* ctx, const pggc_cluster_data* cd, void* out, int mem_kind);
/* overwrite label_count / total_deg / uncut and recompute obj */
pggc_status pggc_cluster_data_set(pggc_context* ctx, pggc_cluster_data* cd, int64_t label_count, const void* total_deg,
                                  double uncut, int mem_kind);

/* ---- ordering::generate_orderings (src/header/ordering.h:21) -------------
 * offsets = {offset_large, offset_large2, offset_mid, offset_mid2} */
pggc_status pggc_generate_orderings(pggc_context* ctx, const pggc_graph* g, int32_t* order1, int32_t* order2,
                                    int64_t offsets[4], int mem_kind);

/* Allocation-free generate_orderings.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory -- a host whose framework
 * owns all device memory through its own pool and budget, or a latency-bound
 * loop that must stay out of the driver's allocator.  rowptr (n+1), order1, order2 (n) and
 * offsets (4 int64) are device pointers; work is queued on `stream` (a
 * cudaStream_t; NULL = legacy default stream) and the call returns without
 * waiting.  The scratch is a fixed 768 KiB __device__ array inside the library
 * (held by every GPU that loads it until exit), so n is limited to 16,777,216
 * (larger n returns PGGC_ERR_INVALID).  The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * All calls share the one array: calls whose work overlaps on the GPU race.
 * Output: the two orderings and the four offsets only (no maximum degree, no
 * list of the vertices above 4096 edges, which pggc_generate_orderings keeps
 * with the graph).  Precondition: rowptr is non-decreasing.  The call does not
 * check it (the offsets live on the device and the call does not wait); a
 * decreasing pair puts that vertex in the lowest degree bucket, so the outputs
 * stay permutations of 0..n-1 and no write leaves them, but they are then not
 * the reference's orderings. */
pggc_status pggc_generate_orderings_noalloc(const int64_t* rowptr, int64_t n, int32_t* order1, int32_t* order2,
                                            int64_t* offsets, void* stream);

/* ---- local_move_heuristic (src/header/local_mover.h:21-25) ----------------
 * local_move<constrained> (strict = 0) or local_move_strict<constrained>
 * (strict = 1) on partition part_io with cluster_data cd (in/out).
 * constraint_io (cluster-indexed, constraint_len entries with
 * n <= constraint_len <= 2n + 64) is used when constrained; entries for labels
 * appended by the call are written back when they fit.
 * sweep_limit < 0: the reference schedule; >= 0 caps the sweeps (test hook). */
pggc_status pggc_local_move(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int32_t* part_io,
                            int is_initial, int constrained, int32_t* constraint_io, int64_t constraint_len,
                            int enable_sa, int strict, int sweep_limit, int mem_kind, pggc_stats* stats);

/* One candidates_and_destinations pass (src/local_mover.cpp:567-634) on a given
 * state: dest_io is the dest cache in, destinations out (NO_MOVE = -3,
 * NEW_PART = -4); gain_io is save_gains in/out (skipped NO_MOVE vertices keep
 * their entries, as src/local_mover.cpp:477-479 does).  pvals: own-cluster weights
 * (V type).  initial != 0 uses the input graph as the conn graph. */
pggc_status pggc_select_pass(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, const int32_t* part,
                             const void* pvals, int32_t* dest_io, float* gain_io, float filter_ratio, int initial,
                             int constrained, const int32_t* constraint, int mem_kind, int64_t* num_candidates);

/* ---- contracter::build_coarse_graph (src/header/contract.h:20-24) --------
 * Coarse CSR with rows sorted by column, self-loops dropped, weights summed;
 * coarse vertex weights are summed vertex weights.  The new graph has int32
 * weights (integer inputs) or float32 weights (float32 input). */
pggc_status pggc_build_coarse_graph(pggc_context* ctx, const pggc_graph* g, const int32_t* vcmap, int64_t nc,
                                    int mem_kind, pggc_graph** out);

/* ---- leidenR::coarsen_leidenR (src/header/leidenR.h:26-31) ---------------
 * Refines `constraint` (the local-move partition, cd its cluster_data);
 * seed_pick / seed_order replace the two std::random_device draws. */
pggc_status pggc_coarsen_leidenR(pggc_context* ctx, const pggc_graph* g, const pggc_cluster_data* cd,
                                 const int32_t* constraint, uint32_t seed_pick, uint32_t seed_order,
                                 int32_t* vcmap_out, int64_t* nc_out, int mem_kind);

/* ---- clustering_methods (interface/clustering_methods.h:20-24) ----------- */
pggc_status pggc_leiden_part(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int plus, int improve,
                             const int32_t* input, uint64_t seed, int32_t* labels_out, int mem_kind,
                             pggc_stats* stats);
pggc_status pggc_louvain_part(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int constrained,
                              const int32_t* constraint, int32_t* labels_out, int mem_kind, pggc_stats* stats);

/* run_clustering (app/cluster_main.cpp:116-165): the method, then ex_iters
 * improvement passes (ex_iters < 0: until the objective stops rising). */
pggc_status pggc_run_clustering(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int method,
                                int ex_iters, uint64_t seed, int32_t* labels_out, int mem_kind, pggc_stats* stats);

/* ---- batched clustering (no counterpart in the reference) ------------------
 * `count` independent run_clustering jobs -- a population of seeds on one graph
 * (the memetic driver's population, app/memetic_clustering.cpp:118-219) or a
 * set of uneven-size graphs -- run concurrently on min(streams, count) CUDA
 * streams of the context's device, one host thread and one worker context
 * (stream, memory pool, scratch) per stream pulling jobs in order.
 * Graphs must belong to `ctx`; each job builds its own cluster_data
 * (objective, lambda_mult) and writes labels_out (n int32, host or device per
 * mem_kind), stats and status.  A learned filter enabled on `ctx` applies to
 * every job.  Returns the first failing job's status (its message in
 * pggc_last_error) or PGGC_OK.  Results equal those of sequential
 * pggc_run_clustering calls with the same arguments.  The workers start after
 * the work already queued on the context's stream and that stream waits for
 * all of them, so CUDA events recorded on it around the call bracket the
 * batch.  Batch calls on one context are serialised: a second call from
 * another host thread waits until the first has finished. */
typedef struct pggc_batch_job {
    const pggc_graph* graph;
    int objective;
    double lambda_mult;
    int method;
    int ex_iters;
    uint64_t seed;
    int32_t* labels_out;
    int mem_kind;
    pggc_stats stats; /* out */
    int status;       /* out: pggc_status */
} pggc_batch_job;
/* streams = 0: the context's tuned batch width (pggc_tune.streams) */
pggc_status pggc_batch_run(pggc_context* ctx, pggc_batch_job* jobs, int64_t count, int streams);

/* ---- kernel-selection knobs and the batch autotuner (no counterpart in the
 * reference) ------------------------------------------------------------------
 * The local-move select step picks a kernel per degree class: one thread per
 * vertex up to thread_max_deg (0, 8, 16 or 32), one warp per vertex up to
 * warp_max_deg (32 or 127), a block above; warp and block hash tables are
 * sized for load_factor (0.5 or 0.7).  These replace the reference's fixed
 * cut-offs (src/header/ordering.h:17-19, the 128-degree team boundary of
 * src/local_mover.cpp:591-593).  No knob changes any result.  `streams` is the
 * batch width used when pggc_batch_run is given streams = 0.  Other values
 * round to the nearest supported one. */
typedef struct pggc_tune {
    int thread_max_deg;
    int warp_max_deg;
    double load_factor;
    int streams;
} pggc_tune;
pggc_status pggc_tune_set(pggc_context* ctx, const pggc_tune* t);
pggc_status pggc_tune_get(pggc_context* ctx, pggc_tune* out);

/* One timed configuration of the autotuner: the batch's device time
 * (seconds, CUDA events on the context stream) and undirected edges / second
 * over the jobs. */
typedef struct pggc_tune_trial {
    pggc_tune config;
    double seconds;
    double edges_per_s;
} pggc_tune_trial;
/* Tunes the knobs above on a sample batch (the caller's jobs, run as they
 * are, repeatedly): after one warm-up batch at the current settings, batch
 * width over {1, 4, 8, 16, 32} (at most `count`), then the thread / warp
 * degree bounds over {(32,127), (16,127), (8,127), (0,127), (32,32), (8,32)},
 * then the load factor over {0.5, 0.7}, each step keeping the fastest (a
 * configuration's time is the better of two batches, and a challenger wins
 * only when more than 2 % faster).  The
 * best configuration is set on the context and written to *best; the trials
 * (at most trials_cap) to `trials`, their number to *n_trials.  Job outputs
 * hold the last trial's results. */
pggc_status pggc_batch_autotune(pggc_context* ctx, pggc_batch_job* jobs, int64_t count, pggc_tune_trial* trials,
                                int64_t trials_cap, int64_t* n_trials, pggc_tune* best);

/* ---- memetic driver (app/memetic_clustering.cpp:27-219) -------------------
 * meme_cluster: pop_size pLeiden+ clusterings, then offspring from the
 * intersection of two tournament-selected parents, refined by constrained
 * pLouvain and five pLeiden+ improvement passes, each replacing the most
 * similar (cut-edge signature) worse member.  The reference runs for a wall
 * time; here the loop stops after `offspring` children (< 0: no limit) or
 * `time_limit_s` seconds (<= 0: no limit), whichever comes first (at least one
 * limit must be set).  `seed` replaces std::random_device.  labels_out gets the
 * best member (n int32). */
typedef struct pggc_meme_stats {
    double objective;    /* best member's objective */
    int64_t label_count;
    int64_t offspring;   /* children made */
    int64_t replaced;    /* children that entered the population */
    double best_initial; /* best objective of the initial population */
} pggc_meme_stats;
pggc_status pggc_meme_cluster(pggc_context* ctx, const pggc_graph* g, int objective, double lambda_mult, int pop_size,
                              int64_t offspring, double time_limit_s, uint64_t seed, int32_t* labels_out,
                              int mem_kind, pggc_meme_stats* stats);
/* intersection_cluster (:27-62): out[i] = rank of (c1[i], c2[i]) among the
 * distinct pairs in ascending order (labels in [0, n)); *count_out = pairs */
pggc_status pggc_intersect_clusters(pggc_context* ctx, const int32_t* c1, const int32_t* c2, int64_t n, int32_t* out,
                                    int64_t* count_out, int mem_kind);
/* gen_signature (:64-104): bit j of sign_out (ceil(nnz / 32) words) is set when
 * edge j joins two clusters */
pggc_status pggc_cut_signature(pggc_context* ctx, const pggc_graph* g, const int32_t* labels, uint32_t* sign_out,
                               int mem_kind);

/* verify_objective<uniform> (app/verify_objective.cpp:64-89) in int64 / FP64 */
pggc_status pggc_verify_objective(pggc_context* ctx, const pggc_graph* g, const int32_t* labels, int objective,
                                  double lambda_mult, int mem_kind, double* objective_out, double* raw_obj_out);

/* ---- learned move filter (no counterpart in the reference) ----------------
 * A network that decides which vertices a local-move sweep evaluates; the
 * gains of the evaluated vertices stay exact.  8 features per vertex ->
 * 32 -> 32 (ReLU) -> 1 logit, BF16 weights and FP32 accumulation.  Parameters
 * are PGGC_MLP_PARAMS FP32 values: W1[32][8] | b1[32] | W2[32][32] | b2[32] |
 * W3[32] | b3 (weights [out][in]).  Features are rows of PGGC_MLP_FEATURES
 * floats; labels are 0/1 floats (1 = the vertex moved). */
#define PGGC_MLP_PARAMS 1377
#define PGGC_MLP_FEATURES 8

/* logits of `count` feature rows (tensor-core inference path) */
pggc_status pggc_mlp_infer(pggc_context* ctx, const float* params, const float* features, int64_t count, int mem_kind,
                           float* logits_out);
/* mean positive-weighted binary cross-entropy of the rows and its gradient
 * (PGGC_MLP_PARAMS floats); count <= 1,048,576 */
pggc_status pggc_mlp_loss_grad(pggc_context* ctx, const float* params, const float* features, const float* labels,
                               int64_t count, float pos_weight, int mem_kind, float* grad_out, float* loss_out);
/* Adam on shuffled mini-batches of `batch` rows for `epochs` epochs; params_io
 * is updated in place; epoch_loss_out (host, `epochs` floats, may be NULL)
 * receives each epoch's mean batch loss */
pggc_status pggc_mlp_train(pggc_context* ctx, float* params_io, const float* features, const float* labels,
                           int64_t count, int mem_kind, int epochs, int batch, float lr, float pos_weight,
                           uint64_t seed, float* epoch_loss_out);
/* start logging (features, label) samples from the context's plain sweeps:
 * each evaluated vertex is sampled with probability sample_rate, up to
 * `capacity` rows */
pggc_status pggc_filter_log_start(pggc_context* ctx, int64_t capacity, double sample_rate, uint64_t seed);
/* the label logged samples get: 0 (default) 1 when the vertex moves in the
 * sweep; 1 when the sweep's select step proposes a move for it (it becomes a
 * candidate of the afterburner) */
pggc_status pggc_filter_log_label(pggc_context* ctx, int label);
/* stop logging and copy out min(rows, capacity) rows; *count_out = rows logged */
pggc_status pggc_filter_log_stop(pggc_context* ctx, float* features_out, float* labels_out, int64_t capacity,
                                 int mem_kind, int64_t* count_out);
/* filter the context's sweeps with this network (host params): vertices whose
 * logit is below threshold_logit are not evaluated.  params NULL disables it.
 * The finest level's last local move of each pass always runs unfiltered. */
pggc_status pggc_filter_enable(pggc_context* ctx, const float* params, float threshold_logit);
/* where the enabled filter applies: sweeps of the passes before max_pass
 * (max_pass < 0: every pass; passes count from 0 within a run_clustering) at
 * multilevel levels >= min_level (0: the input graph).  Default: everywhere. */
pggc_status pggc_filter_scope(pggc_context* ctx, int max_pass, int min_level);
/* vertices evaluated / skipped by the filter since the last reset */
pggc_status pggc_filter_stats(pggc_context* ctx, int64_t* evaluated, int64_t* skipped, int reset);

#ifdef __cplusplus
}
#endif

#endif /* PGGC_H */
