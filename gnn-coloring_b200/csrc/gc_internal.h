// Internal objects of the device library: contexts, device-resident graphs and models, and the
// host-side drivers of each kernel family.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "gc_device.cuh"
#include "gnn_coloring.h"

// Optional per-kernel timing: when enabled, each kernel launch group records an event pair on
// the stream it runs on; gc_prof_read aggregates the durations by name.
struct gc_prof_rec {
    const char *name;
    cudaEvent_t a, b;
};

// Degree tiers: above GC_GNN_HUB_DEGREE a vertex is a hub (JP split tasks; in the GNN its neighbour
// sums are evaluated exactly by whole warps before each layer); above GC_GNN_WARP_DEGREE the split
// gives it a warp.
constexpr int GC_UPLOAD_CHUNKS = 8;  // pieces of a page-locked E converted to GNN rows as they arrive
constexpr uint32_t GC_GNN_HUB_DEGREE = 16384;
// Giant hubs (GNN): at least this many neighbours, and a third of the largest degree; their staged
// rows take at most GC_GIANT_MAX_ROWS padded rows (16 floats each).
constexpr uint32_t GC_GIANT_MIN_DEGREE = 32768;
constexpr uint64_t GC_GIANT_MAX_ROWS = 1ull << 24;
constexpr uint32_t GC_GNN_WARP_DEGREE = 256;
// The GNN layers' own warp tier (degree schedule): a warp stages 32 rows through shared memory, which
// costs about 2.5 L1 wavefronts per row against 1 for the four-lane tier, so only vertices whose lists
// are long enough to need a warp's latency hiding get one (the split kernel keeps GC_GNN_WARP_DEGREE).
constexpr uint32_t GC_GNN_WIDE_DEGREE = 4096;

struct gc_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t hub_stream = nullptr;   // GNN: the hubs' kernel beside the layer kernel (high priority)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool gnn_hub_side = true;            // GNN: hubs on a high-priority stream beside the layer kernel (GC_GNN_HUB_SIDE=0: before it)
    uint32_t gnn_hub_ctas_per_sm = 0;    // GNN: persistent hub CTAs per SM at most (0: as many as fit; GC_GNN_HUB_CTAS)
    int hub_blocks_per_sm[3] = {0, 0, 0};  // resident CTAs of each hub kernel
    cudaStream_t copy_stream = nullptr;  // host copies that overlap work on `stream` (created on first use)
    cudaEvent_t ev_copy_fence = nullptr, ev_copy_done = nullptr;
    cudaEvent_t ev_chunk[GC_UPLOAD_CHUNKS] = {};  // pieces of a page-locked E that have arrived
    int color_blocks_per_sm = 0;         // resident CTAs of the coloring kernel (occupancy query)
    int jp_ctas_per_sm = 2;              // CTAs per SM of the coloring kernel: fewer pollers beat more lookahead (measured)
    unsigned int jp_tight = 32;          // coloring: unproductive polling rounds before sleeping
    unsigned int jp_nap = 32;            // coloring: first sleep between polling rounds (ns)
    bool jp_decide = true;               // coloring: early decisions from published forbidden colors
    bool jp_classes = true;              // Culberson rounds: class by class instead of tickets
    uint32_t jp_core_max = 32768;        // coloring: first tickets colored inside one cluster (0: off; GC_JP_CORE)
    int jp_core_cluster = -1;            // CTAs of that cluster (16 or 8; 0: unavailable; -1: not yet queried)
    uint32_t jp_core_block = 16;         // consecutive core tickets per CTA (GC_JP_CORE_BLOCK)
    unsigned int jp_core_nap = 0;        // core kernel: sleep between polling rounds, ns (GC_JP_CORE_NAP)
    int jp_core_warps = 16;              // core kernel: warps per CTA, 1..32 (GC_JP_CORE_WARPS)
    bool jp_core_decide = true;          // core kernel: early decisions from published seen colors (GC_JP_CORE_DECIDE)
    size_t jp_core_smem = 0;             // core kernel: shared memory per CTA (the device's opt-in maximum)
    int jp_light_warps = 2;              // coloring: warps per CTA on the light stream (0: no split; GC_JP_LIGHT_WARPS)
    int gnn_blocks_per_sm[3] = {0, 0, 0};  // resident CTAs of each GNN layer kernel
    uint32_t gnn_warp_deg = GC_GNN_WIDE_DEGREE;  // GNN: above this many neighbours a vertex gets a warp
    uint32_t hub_deg = GC_GNN_HUB_DEGREE;    // plain graphs: above this many neighbours a vertex is a hub (GC_HUB_DEGREE)
    uint32_t gnn_thin_deg = 16;          // GNN: vertices with at most this many neighbours get one lane each
    bool gnn_fuse_isolated = true;       // GNN: vertices without neighbours run all layers at once (GC_GNN_FUSE_ISOLATED)
    uint32_t gnn_grab = 2;               // GNN counter hand-out: items per grab (GC_GNN_GRAB; 1-2 best, 8 +4 %, 16 +17 %)
    uint32_t gnn_heavy = 16384;          // GNN counter hand-out: leading four-lane items taken singly (GC_GNN_HEAVY)
    cudaMemPool_t pool = nullptr;        // when set, graph buffers are stream-ordered allocations from this pool
    gc::DevState *dstate = nullptr;      // device status block
    gc::DevState *hstate = nullptr;      // pinned host mirror for read-back
    uint64_t launches = 0;
    std::string last_error;
    unsigned int spin_limit = 1u << 22;  // iterations a kernel waits on a predecessor before giving up
    bool prof = false;
    int refs = 1;                   // the owner's reference plus one per live graph and model
    bool destroy_requested = false; // gc_ctx_destroy was called; freed when refs reaches 0
    std::vector<gc_prof_rec> prof_recs;
    std::vector<cudaEvent_t> prof_pool;
};

// Records an event pair around the launches in its scope when profiling is on.
struct ProfScope {
    gc_ctx *ctx;
    cudaStream_t stream;
    const char *name;
    cudaEvent_t a = nullptr;
    ProfScope(gc_ctx *c, const char *n, cudaStream_t s);
    ~ProfScope();
};

// Hubs (more than GC_GNN_HUB_DEGREE neighbours) are split across several warps in the JP split
// pass, this many edges per warp task.
constexpr uint32_t GC_SPLIT_CHUNK = 1024;  // edges per warp task (shared-memory buffer per warp)
constexpr int GC_JP_MASK_WORDS = 8;        // published forbidden colors: 8 x 32 = colors 1..256

struct gc_graph {
    gc_ctx *ctx = nullptr;
    uint32_t N = 0, M = 0;          // current graph
    uint32_t cap_N = 0, cap_M = 0;  // allocated capacity
    uint32_t max_deg = 0;
    bool owns_csr = true;
    uint32_t *V = nullptr, *E = nullptr;
    // priorities and colors
    uint32_t *key = nullptr;   // uint32 priority keys (float bits for GNN)
    int32_t *color = nullptr;  // 1-based colors
    int key_kind = -1;         // gc_heuristic that produced the keys, 100 = our colors (Culberson),
                               // 101 = caller colors as keys, 200 = user priorities
    bool has_keys = false, has_colors = false;
    bool colors_ours = false;  // the current colors come from this library's JP (at most max degree + 1)
    // JP workspace
    uint32_t *P = nullptr;      // predecessor lists, packed at the front of each CSR segment
    uint32_t *pc = nullptr;     // predecessor counts
    uint32_t *order = nullptr;  // vertices by descending key, ascending id on ties: the ticket order
    uint32_t *leaf_list = nullptr;  // leaves too large for one thread
    uint32_t *rank = nullptr;       // ticket of each core vertex (valid for the core tickets only)
    uint4 *jprec = nullptr;         // per ticket: (vertex, first CSR entry, predecessor count, 0)
    uint4 *jpsplit = nullptr;       // the tickets after the core: heavy stream from the front, light from the back
    uint32_t *part_tiles = nullptr; // heavy tickets per tile of the split (prefix)
    uint32_t *class_first = nullptr;  // Culberson rounds: first ticket position of each key (old color)
    size_t class_cap = 0;
    // forbidden colors 1..256 published by waiting vertices of the ordered coloring kernel:
    // GC_JP_MASK_WORDS words per vertex, each (epoch << 32 | 32 color bits); the word after the
    // last vertex's holds the epoch counter, advanced once per coloring run
    unsigned long long *fmask = nullptr;
    uint32_t *sort_buf = nullptr;  // radix sort ping-pong (keys and values), 4 * cap_N words
    uint32_t *sort_hist = nullptr;
    uint32_t sort_hist_cap = 0;
    // degree classes (depend on the graph only; rebuilt on upload)
    uint32_t *big = nullptr;         // split tasks of the hubs: (vertex, first edge) pairs
    uint32_t n_big_tasks = 0;
    size_t big_cap = 0;              // words allocated for `big`
    uint32_t *hubs = nullptr;        // vertices with deg > GC_GNN_HUB_DEGREE, by descending degree
    uint32_t n_hubs = 0;
    uint32_t *hub_aux = nullptr;     // GNN: per hub 16 feature sums, then one completion counter each
    size_t hub_aux_cap = 0;
    uint32_t n_giant = 0;            // the leading hubs whose rows the GNN stages (see k_hub_stage)
    uint32_t giant_rows = 0;         // their degrees, each padded to a multiple of 1,024
    uint32_t *giant_off = nullptr;   // n_giant + 1 first padded rows
    float *hub_stage = nullptr;      // GNN: 16 x giant_rows staged feature values
    size_t hub_stage_cap = 0;
    uint32_t *gnn_ctr = nullptr;     // GNN: 8 work counters (bulk hand-out)
    uint32_t *vorder = nullptr;      // the other vertices by descending degree (GNN schedule)
    uint32_t n_vorder = 0;
    uint32_t n_wide = 0;             // leading vorder entries with more than GC_GNN_WARP_DEGREE neighbours
    uint32_t n_wide_gnn = 0;         // leading vorder entries the GNN gives a warp (more than gnn_warp_deg)
    uint32_t gnn_warp_deg = GC_GNN_WIDE_DEGREE;
    uint32_t n_thin = 0;             // trailing vorder entries with at most ctx->gnn_thin_deg neighbours
    uint32_t n_iso = 0;              // of those, the trailing entries without neighbours (degree schedule only)
                                     // (degree schedule only; 0 with the graph-major schedule)
    // GNN scratch (allocated on first use).  Feature rows (x, y, t01) are stored in degree order:
    // the hubs take rows 0 .. n_hubs-1 in hub order, vorder[i] takes row n_hubs + i, so rows that
    // many lists gather share cache lines, and a warp's own rows are consecutive.
    float *x = nullptr, *y = nullptr;
    float2 *t01 = nullptr;
    uint32_t *row_of = nullptr;  // feature row of each vertex
    uint2 *vrow = nullptr;       // per feature row: (first CSR entry, degree) of its vertex
    uint32_t *Er = nullptr;      // E with every neighbour id replaced by its feature row (same positions)
    bool rows_ready = false;     // row_of and Er describe the current CSR (cleared by gc_graph_prepare)
    bool gnn_hint = false;       // GNN priorities follow the next upload: a page-locked E is converted to
                                 // rows piece by piece while it arrives (set by the reference-named calls)
    // SL/SLL scratch (allocated on first use)
    uint32_t *deg_rem = nullptr, *frontier = nullptr, *frontier2 = nullptr, *removed = nullptr;
    // tier thresholds and vertex schedule of the split and GNN kernels (gc_graph_prepare applies them)
    uint32_t warp_deg = GC_GNN_WARP_DEGREE, hub_deg = GC_GNN_HUB_DEGREE;
    int sched = GC_SCHEDULE_DEGREE;
    // coloring-kernel overrides (0 = the context's value)
    int jp_ctas = 0;
    unsigned int jp_tight = 0, jp_nap = 0;
    // segments: n_seg independent graphs in one CSR (0 = a single graph).  Segment s owns the
    // vertices [seg_voff[s], seg_voff[s + 1]); E holds global ids after the upload.
    uint32_t n_seg = 0, seg_cap = 0;
    uint32_t *seg_voff = nullptr;    // device copy of the vertex offsets
    int32_t *seg_stat = nullptr;     // device, 2 * seg_cap: largest color, improper flag per segment
    std::vector<uint32_t> h_seg_voff;
    // stats of the last coloring
    int colors_used = 0;
    std::vector<double> user_p;  // priorities given by gc_priority_set, returned unchanged
    double *p64 = nullptr;       // device staging for gc_download_priority
};

struct gc_model {
    gc_ctx *ctx = nullptr;
    int params = 0, md = 0, layers = 0;
    float *d_param = nullptr;  // device copy
    float *h_param = nullptr;  // host copy
};

// Makes the context's device current for the scope of a call.
struct DeviceGuard {
    explicit DeviceGuard(const gc_ctx *ctx) {
        if (ctx) cudaSetDevice(ctx->device);
    }
};

// ---- helpers (api.cu) ----
gc_status gc_graph_alloc(gc_ctx *ctx, gc_graph *g, uint32_t N, uint32_t M, bool csr);  // CSR, keys, colors
gc_status gc_graph_finish_upload(gc_graph *g);  // CSR checks, then gc_graph_prepare
void gc_graph_free_buffers(gc_graph *g);
gc_status gc_fail(gc_ctx *ctx, gc_status s, const std::string &msg);
gc_status gc_check_cuda(gc_ctx *ctx, cudaError_t e, const char *what);
gc_status gc_check_launch(gc_ctx *ctx, const char *what);
gc_status gc_read_state(gc_ctx *ctx);  // syncs, copies DevState, reports device errors
gc_status gc_check_hstate(gc_ctx *ctx);  // reports device errors of an already copied DevState
gc_status gc_reset_state(gc_ctx *ctx);
gc_status gc_copy_stream(gc_ctx *ctx);  // creates ctx->copy_stream and its events once
bool gc_is_pinned(const void *host_ptr);  // page-locked (or registered) host memory
template <typename T>
gc_status gc_alloc(gc_ctx *ctx, T **p, size_t count, const char *what) {
    if (*p) return GC_OK;
    const size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync((void **)p, bytes, ctx->pool, ctx->stream)
                              : cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return gc_check_cuda(ctx, e, what);
    }
    return GC_OK;
}

// Frees a device buffer of a graph owned by ctx (stream-ordered when the context allocates from a pool).
inline void gc_dev_free(gc_ctx *ctx, void *p) {
    if (!p) return;
    if (ctx && ctx->pool) cudaFreeAsync(p, ctx->stream);
    else cudaFree(p);
}

// ---- kernel drivers ----
gc_status gc_graph_prepare(gc_graph *g);  // degree classes, max degree (k_graph.cu)
gc_status gc_priority_simple(gc_graph *g, gc_heuristic h);         // FF / LF / LLF (k_priority.cu)
gc_status gc_priority_peel(gc_graph *g, bool log_thresholds);      // SL / SLL (k_priority.cu)
gc_status gc_priority_gnn(gc_graph *g, const gc_model *m);         // GraphSAGE (k_gnn.cu)
// The GNN's feature-row order (k_gnn.cu): row_of and vrow from the hub list and the degree order,
// then E's entries [first, first + count) as rows into Er.  The conversion checks every id against
// N (ERR_BOUND, reported by the next gc_read_state) and writes row 0 for one that is out of range.
gc_status gc_gnn_rows_begin(gc_graph *g);
gc_status gc_gnn_row_ids(gc_graph *g, uint32_t first, uint32_t count);
gc_status gc_jp_color(gc_graph *g);                                // JP by current keys (k_jp.cu)
gc_status gc_keys_from_colors(gc_graph *g);                        // Culberson step (k_jp.cu)
gc_status gc_validate_device(gc_graph *g, int *max_color);         // (k_jp.cu)
// Vertex sorts (k_sort.cu): descending key, ascending id on ties, over the vertices a filter keeps.
enum { SORT_KEEP_ALL = 0, SORT_KEEP_INNER = 1, SORT_KEEP_DEG_AT_MOST = 2 };
gc_status gc_sort_vertices(gc_graph *g, const uint32_t *keys, int key_bits, int filter, uint32_t max_deg,
                           uint32_t *out, uint32_t *d_count);
gc_status gc_sort_order_bits(gc_graph *g, int key_bits, bool filter, uint32_t *d_count);
// Stable sort of n (key, value) pairs by ascending key into (kout, vout); kbuf, vbuf: n-word
// scratch; hist: gc_sort_pairs_hist_words(n) words (k_sort.cu).
size_t gc_sort_pairs_hist_words(uint32_t n);
gc_status gc_sort_pairs(gc_ctx *ctx, uint32_t n, const uint32_t *kin, const uint32_t *vin, int key_bits,
                        uint32_t *kbuf, uint32_t *vbuf, uint32_t *kout, uint32_t *vout, uint32_t *hist);
// Segments (batch.cu): per-segment largest color and improper flag into g->seg_stat.
gc_status gc_segment_stats(gc_graph *g);
