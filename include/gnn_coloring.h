/*
 * gnn_coloring.h -- status-returning C ABI of the B200 greedy-coloring library.
 *
 * The reference program (KennethLangedal/GNN-COLORING) has no device API; its
 * operator boundary is a set of host functions (coloring.h, first_fit.h,
 * largest_degree_first.h, smallest_degree_last.h, gnn.h, fast_gnn.h) that this
 * library also exports under the reference's own names (see the other headers
 * in this directory).  Those entry points take host buffers and return void.
 * This header is the native interface underneath them: a context owns one CUDA
 * stream on one device, graphs and models live in device memory, every call
 * returns a gc_status, and nothing ever falls back to the CPU.
 *
 * Plain C types only: pointers, sizes and opaque handles.
 *
 * Arithmetic contract (what "identical to the reference" means here):
 *   - priorities are per-vertex keys; vertex v precedes u when
 *     key[v] > key[u], or key[v] == key[u] and v < u
 *     (src/coloring.c:249 of the reference);
 *   - color[u] = smallest c >= 1 not used by any predecessor of u, i.e. the
 *     Jones-Plassmann / priority-order greedy coloring of src/coloring.c:223-330;
 *   - the GraphSAGE-16 priorities reproduce src/fast_gnn.c:13-243 bit for bit
 *     (sequential FP32 neighbour sums in CSR order, IEEE division, FMA chain
 *     in input order, fixed-tree output sum).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gc_status {
    GC_OK = 0,
    GC_ERR_INVALID = 1,   /* bad argument: null pointer, size out of range, malformed CSR, NaN priority */
    GC_ERR_NOMEM = 2,     /* host or device allocation failed */
    GC_ERR_CUDA = 3,      /* a CUDA runtime call failed (message in gc_last_error) */
    GC_ERR_DEVICE = 4,    /* a kernel raised its error flag (bounded wait expired, internal bound exceeded) */
    GC_ERR_IO = 5,        /* file missing or unreadable */
    GC_ERR_FORMAT = 6,    /* malformed Matrix Market or .gnn content */
    GC_ERR_BUDGET = 7,    /* admission refused: the request does not fit the HBM budget */
    GC_ERR_NODEV = 8,     /* no usable CUDA device */
    GC_ERR_STATE = 9      /* call out of order (e.g. coloring before a priority was computed) */
} gc_status;

/* Priority heuristics, named as in the reference's output lines (src/main.c:199-208). */
typedef enum gc_heuristic {
    GC_FF = 0,   /* first fit: p[i] = N - i                       (src/first_fit.c:8-12)              */
    GC_LF = 1,   /* largest degree first: p = deg                 (src/largest_degree_first.c:12-16)  */
    GC_LLF = 2,  /* largest log degree first: p = 32 - clz(deg)   (src/largest_degree_first.c:87-97)  */
    GC_SL = 3,   /* smallest degree last (bucket peeling)          (src/smallest_degree_last.c:62-124) */
    GC_SLL = 4,  /* smallest log degree last                       (src/smallest_degree_last.c:274-328)*/
    GC_GNN = 5   /* GraphSAGE-16 inference; needs a model          (src/fast_gnn.c:297-347)            */
} gc_heuristic;

typedef struct gc_ctx gc_ctx;       /* device + stream + scratch; not shared between host threads */
typedef struct gc_graph gc_graph;   /* device-resident CSR with its key / color / work buffers    */
typedef struct gc_model gc_model;   /* device-resident GraphSAGE-16 weights (L * 528 floats)      */

const char *gc_status_string(gc_status s);

/* ---- context ------------------------------------------------------------------------------ */

/* Creates a context on `device` with its own non-blocking stream. */
gc_status gc_ctx_create(int device, gc_ctx **ctx);
/* Releases the caller's handle.  Graphs and models hold their context: its memory and stream go
 * when the last of them is freed, so handles may be released in any order. */
void gc_ctx_destroy(gc_ctx *ctx);
/* Last error message of this context ("" when none). */
const char *gc_last_error(const gc_ctx *ctx);
/* The cudaStream_t the context launches on (returned as void* to keep CUDA types out of the ABI). */
void *gc_ctx_stream(gc_ctx *ctx);
/* Blocks until the context's stream is idle; reports deferred device errors. */
gc_status gc_sync(gc_ctx *ctx);
/* Number of kernels this context has launched so far (instrumentation for benchmarks). */
uint64_t gc_ctx_launches(const gc_ctx *ctx);
/* Per-kernel timing: when on, every kernel launch group is bracketed by CUDA events on the stream
 * it runs on.  Turning it on clears earlier records. */
gc_status gc_prof_enable(gc_ctx *ctx, int on);
/* Waits for the stream, then aggregates the records by kernel name: up to `max` entries of
 * (name, total milliseconds, launches).  Returns the number of distinct names (may exceed max). */
int gc_prof_read(gc_ctx *ctx, const char **names, double *total_ms, uint64_t *launches, int max);

/* ---- graphs ------------------------------------------------------------------------------- */

/* Copies a host CSR (V[N+1], E[V[N]]) to the device.  The CSR must be simple and symmetric with
 * ascending adjacency lists, as produced by the reference's graph_sort_edges + graph_make_simple
 * (src/fast_io.c:450-477); only V's monotonicity and E's range are checked here. */
gc_status gc_graph_upload(gc_ctx *ctx, uint32_t N, const uint32_t *V, const uint32_t *E, gc_graph **g);
/* Allocates an empty graph able to hold up to cap_N vertices and cap_M directed edges; fill it
 * with gc_graph_reupload.  Lets callers reserve device memory once and reuse it per job. */
gc_status gc_graph_create(gc_ctx *ctx, uint32_t cap_N, uint32_t cap_M, gc_graph **g);
/* Same as gc_graph_upload, from pinned or pageable host memory, reusing an existing graph object whose capacity
 * (N, M) is at least the new graph's: no device allocation happens. */
gc_status gc_graph_reupload(gc_ctx *ctx, gc_graph *g, uint32_t N, const uint32_t *V, const uint32_t *E);
/* Wraps a CSR that already lives in device memory (no copy; the caller keeps ownership). */
gc_status gc_graph_wrap_device(gc_ctx *ctx, uint32_t N, uint32_t M, const uint32_t *dV,
                               const uint32_t *dE, gc_graph **g);
void gc_graph_free(gc_graph *g);
uint32_t gc_graph_num_vertices(const gc_graph *g);
uint32_t gc_graph_num_edges(const gc_graph *g);
uint32_t gc_graph_max_degree(const gc_graph *g);
/* Device pointers of the graph's buffers (for zero-copy readers such as benchmarks). */
const uint32_t *gc_graph_device_keys(const gc_graph *g);
const int32_t *gc_graph_device_colors(const gc_graph *g);

/* ---- models ------------------------------------------------------------------------------- */

/* Reads a .gnn model file: "params md" followed by `params` floats (src/gnn.c:33-40). */
gc_status gc_model_load(gc_ctx *ctx, const char *path, gc_model **m);
/* Builds a model from host parameters: params = L * 528, L >= 2 (W[32x16] row-major then b[16]
 * per layer, src/fast_gnn.c:256-258); md is the degree normaliser of the input layer. */
gc_status gc_model_create(gc_ctx *ctx, int params, int md, const float *param, gc_model **m);
void gc_model_free(gc_model *m);
int gc_model_layers(const gc_model *m);

/* ---- the hot path --------------------------------------------------------------------------- */

/* Computes the heuristic's priority keys on the device into the graph's key buffer.
 * `model` is required for GC_GNN and ignored otherwise. */
gc_status gc_priority(gc_ctx *ctx, gc_graph *g, gc_heuristic h, const gc_model *model);
/* Sets arbitrary host priorities (the reference's `double *p`); -0.0 equals +0.0, NaN is rejected. */
gc_status gc_priority_set(gc_ctx *ctx, gc_graph *g, const double *p);
/* Jones-Plassmann coloring by the current keys, then `recolor` Culberson iterations
 * (key := color, recolor), as in src/runner.c:139-152.  `colors_used` (optional) receives the
 * number of colors of the final coloring.  Colors stay on the device. */
gc_status gc_color(gc_ctx *ctx, gc_graph *g, int recolor, int *colors_used);
/* `iters` Culberson iterations on the current coloring: key := color, recolor (the loop body of
 * src/runner.c:139-152).  The color count never increases. */
gc_status gc_recolor(gc_ctx *ctx, gc_graph *g, int iters, int *colors_used);
/* Checks the current coloring on the device: *max_color = number of colors if proper and all
 * colors positive, 0 otherwise (src/coloring.c:332-352). */
gc_status gc_validate(gc_ctx *ctx, gc_graph *g, int *max_color);
/* Sets the graph's coloring from host memory (e.g. to validate an external coloring). */
gc_status gc_upload_colors(gc_ctx *ctx, gc_graph *g, const int32_t *color);
/* Copies results to host memory. */
gc_status gc_download_colors(gc_ctx *ctx, gc_graph *g, int32_t *color);
/* Priorities as the reference's doubles: FF N-i, LF deg, LLF/SL/SLL delta, GNN the FP32 sum, and
 * after Culberson the colors. */
gc_status gc_download_priority(gc_ctx *ctx, gc_graph *g, double *p);

/* ---- GraphSAGE priorities without device allocation ------------------------------------------- */

/* No counterpart in the reference: an extra entry point of this library.
 *
 * The same FP32 GraphSAGE-16 priorities as gc_priority(GC_GNN) -- the reference's fast_gnn.c
 * arithmetic, bit for bit -- for callers that may not allocate device memory: a serving loop that
 * reserved its HBM budget up front, a host framework that owns all device memory and passes only
 * its own buffers, or a latency-critical path that cannot take cudaMalloc's implicit device
 * synchronisation.  The caller passes the CSR (dV[N+1], dE[dV[N]]), the model (dparam: params
 * floats, params = L * 528, L >= 2; md its degree normaliser) and the output dp[N] (one float per
 * vertex), all in device memory, plus a cudaStream_t as void* (NULL: the default stream).  The call
 * is asynchronous on that stream and allocates nothing: its scratch is a fixed device array in the
 * library, sized for GC_NOALLOC_MAX_VERTICES vertices, held by every device that loads the library
 * until the process exits.  Larger graphs return GC_ERR_INVALID (use gc_priority).  All calls
 * share that array: calls whose kernels overlap on one device (other streams, other host threads)
 * race.  The first call on a device looks up the array's address with that device current; make
 * that first call before any stream capture. */
#define GC_NOALLOC_MAX_VERTICES 65536u
gc_status gc_gnn_priority_noalloc(uint32_t N, const uint32_t *dV, const uint32_t *dE, int params, int md,
                                  const float *dparam, float *dp, void *stream);

/* ---- batches: many independent graphs in one segmented CSR ---------------------------------- */

/* No counterpart in the reference, whose runner colors one graph per process (src/runner.c:105-153).
 *
 * A batch holds G graphs as one segmented CSR in device memory.  Graph g owns the global vertex
 * range [voff[g], voff[g+1]); V holds global row offsets (voff[G] + 1 entries, V[0] = 0), and E
 * holds each graph's LOCAL neighbour ids (0 .. n_g - 1), as a concatenation of G ordinary CSRs
 * would.  Every graph's priorities, colors and color count equal those of the same graph colored
 * alone by gc_priority + gc_color: the segments share no edge, ties still break by id inside a
 * graph, FF keys and the GNN id feature use the graph's own n and local ids.  SL and SLL are not
 * offered on batches (their peeling thresholds are per graph; color such graphs one at a time). */
typedef struct gc_batch gc_batch;

/* Vertex schedules of the split and GNN kernels. */
typedef enum gc_schedule {
    GC_SCHEDULE_DEGREE = 0,  /* all vertices by descending degree: even work per warp on skewed graphs */
    GC_SCHEDULE_SEGMENT = 1  /* graph by graph, by degree class inside: one graph's rows stay in L2 */
} gc_schedule;

/* What an autotuner may change; none of it changes a single color or priority bit. */
typedef struct gc_tuning {
    uint32_t warp_degree;   /* above this many neighbours a vertex gets a whole warp (else 4 lanes) */
    uint32_t hub_degree;    /* above this many neighbours a vertex gets a whole CTA (GNN) or split tasks */
    int schedule;           /* gc_schedule */
    int jp_ctas_per_sm;     /* resident CTAs per SM of the ordered coloring kernel */
    unsigned int jp_tight;  /* polling rounds before a coloring warp starts to sleep */
    unsigned int jp_nap;    /* first sleep of a coloring warp (ns) */
    uint32_t gnn_warp_degree;  /* GNN layers, degree schedule: above this many neighbours a vertex gets a warp */
} gc_tuning;

/* Uploads G graphs given as one segmented CSR (layout above). */
gc_status gc_batch_upload(gc_ctx *ctx, uint32_t G, const uint32_t *voff, const uint32_t *V, const uint32_t *E,
                          gc_batch **b);
/* Uploads G separate host CSRs: graph g has n[g] vertices, row offsets Vs[g] (n[g] + 1 entries
 * from 0) and local neighbour ids Es[g].  Pinned host memory makes the copies asynchronous. */
gc_status gc_batch_upload_graphs(gc_ctx *ctx, uint32_t G, const uint32_t *n, const uint32_t *const *Vs,
                                 const uint32_t *const *Es, gc_batch **b);
/* An empty batch with room for cap_G graphs, cap_N vertices and cap_M directed edges, refilled by
 * gc_batch_reupload_graphs without new device allocations. */
gc_status gc_batch_create(gc_ctx *ctx, uint32_t cap_G, uint32_t cap_N, uint32_t cap_M, gc_batch **b);
gc_status gc_batch_reupload_graphs(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *n,
                                   const uint32_t *const *Vs, const uint32_t *const *Es);
/* Refills an existing batch from a segmented CSR in host memory (the layout of gc_batch_upload)
 * without new device allocations; pinned host memory makes the copies asynchronous. */
gc_status gc_batch_reupload(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *voff, const uint32_t *V,
                            const uint32_t *E);
/* Refills an existing batch from G CSRs that already live in device memory (graph g: n[g] vertices,
 * m[g] directed edges, local row offsets dVs[g] and neighbour ids dEs[g]); one gather kernel copies
 * them into the batch, no device allocation happens.  The sources are only read. */
gc_status gc_batch_reupload_device_graphs(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *n, const uint32_t *m,
                                          const uint32_t *const *dVs, const uint32_t *const *dEs);
void gc_batch_free(gc_batch *b);
uint32_t gc_batch_num_graphs(const gc_batch *b);
uint32_t gc_batch_num_vertices(const gc_batch *b);
uint32_t gc_batch_num_edges(const gc_batch *b);
/* Device bytes a batch (or a single graph: G = 1) of this size holds once colored with heuristic
 * h: the figure admission control charges. */
uint64_t gc_batch_device_bytes(uint32_t G, uint32_t N, uint32_t M, gc_heuristic h);
/* The union of the batch's graphs as one gc_graph (global ids), for gc_download_priority,
 * gc_download_colors and gc_validate over all graphs at once.  Owned by the batch. */
gc_graph *gc_batch_graph(gc_batch *b);

/* Priorities by heuristic h (GC_FF, GC_LF, GC_LLF or GC_GNN), Jones-Plassmann, then `recolor`
 * Culberson iterations, for every graph of the batch.  The first call for a given (h, model,
 * recolor) runs the stages directly and captures them into a CUDA graph; later calls replay that
 * graph: one launch for all stages of all graphs.  colors (host, G entries, may be NULL) receives
 * each graph's color count as validate_coloring_par reports it: 0 for an improper coloring. */
gc_status gc_batch_color(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *model, int recolor,
                         int32_t *colors);
/* The same pipeline as gc_batch_color, run once without capturing it: for batches whose contents
 * change on every call (a serving loop refilling one batch), where a capture would not be replayed. */
gc_status gc_batch_color_once(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *model, int recolor,
                              int32_t *colors);
/* Colors of all vertices, graph by graph (voff[G] entries, local order inside each graph). */
gc_status gc_batch_download_colors(gc_ctx *ctx, gc_batch *b, int32_t *color);

/* Measures candidate tunings on this batch (each one a full gc_batch_color pass, timed with CUDA
 * events) and keeps the fastest; `effort` 0 tries the tier thresholds only, 1 also the schedule and
 * the coloring-kernel settings, 2 a wider grid.  *best (may be NULL) receives the tuning kept and
 * *best_ms its time per pass. */
gc_status gc_batch_autotune(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *model, int recolor,
                            int effort, gc_tuning *best, double *best_ms);
gc_status gc_batch_set_tuning(gc_ctx *ctx, gc_batch *b, const gc_tuning *t);
gc_status gc_batch_get_tuning(const gc_batch *b, gc_tuning *t);
/* The library's default tuning. */
void gc_tuning_default(gc_tuning *t);

/* ---- serving: a request loop with continuous batching ----------------------------------------- */

/* No counterpart in the reference, whose runner colors one graph per process (src/runner.c:105-153).
 *
 * A server keeps device-resident pools on one GPU and colors jobs submitted from any host thread.
 * Every job's colors and color count equal those of its graph colored alone by gc_priority +
 * gc_color; only when and beside what it runs changes.
 *
 *   lanes      `lanes` worker threads, each with its own stream, a batch slot of fixed capacity
 *              (slot_graphs graphs, slot_vertices vertices, slot_edges directed edges) and pinned
 *              staging buffers; lanes run concurrently, so their device work overlaps.
 *   batching   continuous: a free lane takes the oldest pending job and, when it is small (at most
 *              batch_max_job_vertices vertices, heuristic FF, LF, LLF or GNN), every other pending
 *              small job of the same heuristic, layer count and recolor count that fits its slot,
 *              and colors them in one pass.  Jobs arriving while the lanes are busy join the next
 *              free lane's batch, so batches grow with the load.
 *   admission  by HBM budget: the slots are charged once at creation; a job that runs alone (large,
 *              or SL / SLL) is charged gc_batch_device_bytes(1, N, M, h) while it runs and starts
 *              only when that fits what is left.  Such jobs start in arrival order.  A job that
 *              could never fit is refused at submission with GC_ERR_BUDGET.
 *   isolation  a batch that fails is re-run job by job, so a malformed job fails alone.
 *   resident   graphs registered once stay in device memory; jobs on them skip the upload.
 *   copies     CSRs of jobs that run alone go up through pinned chunks filled by several host
 *              threads while the previous chunk's DMA runs; colors come back the same way.
 *
 * The caller's V, E and color_out buffers must stay valid and unchanged until the job is done. */
typedef struct gc_server gc_server;

typedef struct gc_serve_config {
    int device;                       /* CUDA device */
    uint32_t lanes;                   /* concurrent worker lanes (default 4) */
    uint64_t hbm_budget;              /* device bytes the server may hold; 0 = 80% of the free memory */
    uint32_t slot_graphs;             /* most jobs in one batch (default 4096) */
    uint32_t slot_vertices;           /* vertex capacity of a lane's batch slot (default 2^22) */
    uint32_t slot_edges;              /* directed-edge capacity of a lane's batch slot (default 2^26) */
    uint32_t batch_max_job_vertices;  /* larger jobs run alone (default 2^17) */
} gc_serve_config;

typedef struct gc_job_info {
    int status;           /* gc_status of the job */
    int colors;           /* colors used (validate_coloring_par's figure: 0 = improper) */
    uint32_t N, M;        /* vertices, directed edges */
    uint32_t batch_jobs;  /* jobs colored in the same pass (1 = alone) */
    uint32_t lane;        /* lane that ran it */
    double queue_ms;      /* submission to start */
    double run_ms;        /* start to completion (upload, coloring, read-back) */
    double latency_ms;    /* submission to completion */
} gc_job_info;

typedef struct gc_serve_stats {
    uint64_t submitted, completed, failed, rejected;
    uint64_t edges;                /* directed edges of completed jobs */
    uint64_t launches;             /* passes run: batches plus jobs run alone */
    uint64_t batched_jobs;         /* completed jobs that shared their pass with others */
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submission-to-completion latency of completed jobs */
    double span_s;                 /* first submission to last completion */
    double edges_per_s;            /* edges / span_s */
    uint64_t budget_bytes, reserved_bytes, peak_reserved_bytes;  /* admission accounting */
    uint64_t pool_peak_bytes;      /* high-water mark of the lanes' device memory pool */
    uint32_t lanes;
} gc_serve_stats;

void gc_serve_config_default(gc_serve_config *c);
/* Starts the lanes; GC_ERR_BUDGET when the slots alone exceed the budget. */
gc_status gc_serve_create(const gc_serve_config *cfg, gc_server **s);
/* Adds the GraphSAGE-16 model GNN jobs with params / 528 layers use (before the first submission). */
gc_status gc_serve_add_model(gc_server *s, int params, int md, const float *param);
/* Queues a job: CSR (V[N+1], E[V[N]], the rules of gc_graph_upload), heuristic h (`layers` picks
 * the model for GC_GNN), `recolor` Culberson iterations; color_out (N entries, may be NULL)
 * receives the colors.  Returns at once with the job's id. */
gc_status gc_serve_submit(gc_server *s, uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h, int layers,
                          int recolor, int32_t *color_out, uint64_t *job);
/* *done = 1 when the job has finished. */
gc_status gc_serve_test(gc_server *s, uint64_t job, int *done);
/* Blocks until the job has finished, fills *info (may be NULL), releases the job's id and returns
 * the job's status. */
gc_status gc_serve_wait(gc_server *s, uint64_t job, gc_job_info *info);
/* Blocks until no job is pending or running. */
gc_status gc_serve_drain(gc_server *s);
/* Open-loop load from the calling thread: job i is submitted arrive_s[i] seconds after the call
 * starts (non-decreasing), with the arguments of gc_serve_submit taken from the arrays (layers,
 * recolor and color_out may be NULL); then waits for every job and fills info[i] (may be NULL).
 * A job's latency counts from its scheduled arrival.  Returns the first failing job's status. */
gc_status gc_serve_replay(gc_server *s, uint32_t J, const double *arrive_s, const uint32_t *N,
                          const uint32_t *const *V, const uint32_t *const *E, const int *h, const int *layers,
                          const int *recolor, int32_t *const *color_out, gc_job_info *info);
/* Device-resident graphs: gc_serve_register checks a host CSR (rows monotone, ids below N), copies
 * it to device memory once and returns its id; it stays there, charged 4 (N + 1) + 4 M bytes to the
 * budget, until gc_serve_unregister (GC_ERR_STATE while jobs on it are pending or running).  Jobs on
 * a registered graph skip the host-to-device copy; the host arrays may be freed after registering. */
gc_status gc_serve_register(gc_server *s, uint32_t N, const uint32_t *V, const uint32_t *E, uint64_t *graph);
gc_status gc_serve_unregister(gc_server *s, uint64_t graph);
/* gc_serve_submit for a registered graph. */
gc_status gc_serve_submit_registered(gc_server *s, uint64_t graph, gc_heuristic h, int layers, int recolor,
                                     int32_t *color_out, uint64_t *job);
/* gc_serve_replay for registered graphs: job i runs on graph[i]. */
gc_status gc_serve_replay_registered(gc_server *s, uint32_t J, const double *arrive_s, const uint64_t *graph,
                                     const int *h, const int *layers, const int *recolor, int32_t *const *color_out,
                                     gc_job_info *info);
gc_status gc_serve_read_stats(gc_server *s, gc_serve_stats *st);
void gc_serve_reset_stats(gc_server *s);
const char *gc_serve_last_error(gc_server *s);
/* Waits for all jobs, stops the lanes and frees everything. */
void gc_serve_destroy(gc_server *s);

/* ---- Matrix Market on the device ------------------------------------------------------------ */

/* Reads a Matrix Market file into a device-resident graph with the CSR of gc_mtx_read, built on the
 * GPU: the host reads the header and streams the data lines to the device; line splitting,
 * parsing, symmetrisation, sorting and de-duplication run there (src/fast_io.c:33-222, 450-477 are
 * the rules).  Lines with fewer than two numbers are skipped; an entry outside 1..N is
 * GC_ERR_FORMAT, as is a file with fewer entries than its header announces. */
gc_status gc_graph_load_mtx(gc_ctx *ctx, const char *path, gc_graph **g);
/* The same CSR back on the host (arrays malloc'd; free with gc_host_free). */
gc_status gc_mtx_read_device(gc_ctx *ctx, const char *path, uint32_t *N, uint32_t **V, uint32_t **E);

/* ---- host-side graph preparation (no device involved) --------------------------------------- */

/* Reads a Matrix Market file into a simple, symmetric, sorted CSR with the reference's rules:
 * N = max(rows, cols), every entry added in both directions, adjacency sorted ascending,
 * self-loops and duplicates dropped (src/fast_io.c:68-222, 450-477).  Arrays are malloc'd. */
gc_status gc_mtx_read(const char *path, uint32_t *N, uint32_t **V, uint32_t **E);
/* Reads a graph by its file extension -- .mtx (Matrix Market), .gr (PACE), .graph (METIS), .adj
 * (GBBS adjacency) -- into the simple, symmetric, sorted CSR of gc_mtx_read (the reference's
 * readers in src/fast_io.c followed by its clean-up steps).  Arrays are malloc'd. */
gc_status gc_read_graph(const char *path, uint32_t *N, uint32_t **V, uint32_t **E);
/* Builds the same CSR from L 0-based vertex pairs. */
gc_status gc_csr_from_pairs(uint32_t N, uint64_t L, const uint32_t *I, const uint32_t *J,
                            uint32_t **V, uint32_t **E);
/* Writes a CSR as a symmetric pattern Matrix Market file (each undirected edge once, 1-based). */
gc_status gc_mtx_write(const char *path, uint32_t N, const uint32_t *V, const uint32_t *E);
/* Reads a .gnn file on the host (malloc'd params). */
gc_status gc_model_read(const char *path, int *params, int *md, float **param);
void gc_host_free(void *p);

/* Seeded synthetic graphs (same seed => same graph on every host and thread count). */
/* Erdos-Renyi G(n, m): the first m distinct non-loop pairs of a splitmix64 stream. */
gc_status gc_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t **V, uint32_t **E);
/* R-MAT: ef * n samples over 2^ceil(log2 n) ids with quadrant probabilities a, b, c (d = 1-a-b-c);
 * samples with an endpoint >= n are dropped; symmetrised, deduplicated, loops removed. */
gc_status gc_gen_rmat(uint32_t n, double ef, double a, double b, double c, uint64_t seed,
                      uint32_t **V, uint32_t **E);
/* 2D random geometric graph: n uniform points in [0,1]^2, edge when distance < radius. */
gc_status gc_gen_rgg2d(uint32_t n, double radius, uint64_t seed, uint32_t **V, uint32_t **E);
/* 3D 27-point stencil on an nx * ny * nz grid (all 26 neighbours at Chebyshev distance 1). */
gc_status gc_gen_stencil27(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t **V, uint32_t **E);
/* One graph of a mixed batch, drawn from `seed` alone: n log-uniform in [n_min, n_max] (rounded);
 * even `seed`: Erdos-Renyi with average degree d uniform in [8, 32] (m = round(n d / 2) pairs);
 * odd `seed`: R-MAT with edge factor 8 and (a, b, c) = (0.57, 0.19, 0.19) over 2^ceil(log2 n)
 * ids, samples with an endpoint >= n dropped.  *kind is 0 for ER, 1 for R-MAT; *param the ER
 * degree or the R-MAT edge factor. */
gc_status gc_gen_mixed(uint64_t seed, uint32_t n_min, uint32_t n_max, uint32_t *n, int *kind, double *param,
                       uint32_t **V, uint32_t **E);
/* G graphs of gc_gen_mixed with seeds seed0 .. seed0 + G - 1, generated in parallel, as one
 * segmented CSR (the layout of gc_batch_upload): voff (G + 1), V (voff[G] + 1, global row
 * offsets), E (local ids).  All three malloc'd. */
gc_status gc_gen_mixed_batch(uint32_t G, uint64_t seed0, uint32_t n_min, uint32_t n_max, uint32_t **voff,
                             uint32_t **V, uint32_t **E);

#ifdef __cplusplus
}
#endif
