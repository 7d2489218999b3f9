// Batches of independent graphs (the "batches" section of include/gnn_coloring.h).
//
// G graphs live in one segmented CSR: global vertex ids, graph g owning [voff[g], voff[g+1]).
// After the upload turns local neighbour ids into global ones, the union is an ordinary graph
// whose connected pieces are the G graphs, so every kernel of the plain path runs on it
// unchanged, at the cost of one launch sequence for all graphs:
//   - the JP predecessor relation (key, then id) only ever compares vertices of one graph, and
//     global ids keep each graph's id order, so colors are the per-graph colors;
//   - the ticket order (all inner vertices by key, then id) is a topological order of every
//     graph's DAG at once: the ordered kernel's critical path is the deepest graph's, not the sum;
//   - the two priorities that read the graph's size (FF: N - u; GNN: u / N) look the segment up
//     (gc::seg_of) and use the graph's own N and local id.
// Per-graph color counts come from one statistics pass (k_color_stats with segments).
//
// gc_batch_color captures the whole pipeline -- priorities, split, sort, ordered coloring,
// leaves, Culberson rounds, statistics and the read-back -- into one CUDA graph per (heuristic,
// model, recolor), replayed by a single cudaGraphLaunch.  gc_batch_autotune picks the tier
// thresholds, vertex schedule and coloring-kernel settings by timing full passes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gc_internal.h"

// Where one device-resident graph goes in a batch's staging buffers.
struct gc_seg_src {
    const uint32_t *V;  // n + 1 local row offsets
    const uint32_t *E;  // m local neighbour ids
    uint32_t n, m;
    uint32_t vdst;      // voff[g] + g: its first staged row offset
    uint32_t edst;      // eoff[g]: its first edge
};

namespace {

__global__ void k_check_rows(const uint32_t *__restrict__ V, uint32_t N, uint32_t M, gc::DevState *st) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t a = V[u], b = V[u + 1];
        if (b < a || b > M) gc::raise_error(st, gc::ERR_BOUND, u);
    }
}

// Global row offsets from the staged per-graph offsets: graph s's local row i sits at
// vloc[voff[s] + s + i] (each graph contributes n_s + 1 entries).
__global__ void k_seg_rows(const uint32_t *__restrict__ vloc, const uint32_t *__restrict__ voff,
                           const uint32_t *__restrict__ eoff, uint32_t nseg, uint32_t N, uint32_t M,
                           uint32_t *__restrict__ V) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t u = tid; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t s = gc::seg_of(voff, nseg, u);
        V[u] = __ldg(eoff + s) + vloc[u + s];
    }
    if (tid == 0) V[N] = M;
}

// Local neighbour ids to global ones, one warp per row; an id outside its graph is an error.
__global__ void k_seg_globalize(const uint32_t *__restrict__ V, uint32_t *__restrict__ E,
                                const uint32_t *__restrict__ voff, uint32_t nseg, uint32_t N, gc::DevState *st) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t u = warp; u < N; u += nwarps) {
        const uint32_t s = gc::seg_of(voff, nseg, u);
        const uint32_t base = __ldg(voff + s), n = __ldg(voff + s + 1) - base;
        const uint32_t e = V[u + 1];
        for (uint32_t j = V[u] + lane; j < e; j += 32) {
            const uint32_t v = E[j];
            if (v >= n) gc::raise_error(st, gc::ERR_BOUND, j);
            else E[j] = v + base;
        }
    }
}

// Copies graph g's local row offsets to vloc[src.vdst ...] and its neighbour ids to E[src.edst ...],
// one CTA per graph (the staging layout of fill_graphs, but from device-resident CSRs).
__global__ void k_seg_gather(const gc_seg_src *__restrict__ src, uint32_t G, uint32_t *__restrict__ vloc,
                             uint32_t *__restrict__ E) {
    for (uint32_t gi = blockIdx.x; gi < G; gi += gridDim.x) {
        const gc_seg_src s = src[gi];
        for (uint32_t i = threadIdx.x; i <= s.n; i += blockDim.x) vloc[s.vdst + i] = __ldg(s.V + i);
        for (uint32_t i = threadIdx.x; i < s.m; i += blockDim.x) E[s.edst + i] = __ldg(s.E + i);
    }
}

// A captured pipeline and what it was captured for.
struct BatchCapture {
    int h = -1;
    const float *param = nullptr;
    int layers = 0, md = 0, recolor = 0;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
};

}  // namespace

struct gc_batch {
    gc_ctx *ctx = nullptr;
    gc_seg_src *d_src = nullptr;    // gather descriptors of gc_batch_reupload_device_graphs (cap_G)
    gc_seg_src *h_src = nullptr;    // pinned staging of the same
    gc_graph *g = nullptr;          // the union of the graphs (owned)
    uint32_t G = 0, cap_G = 0;
    uint32_t *d_vloc = nullptr;     // staged per-graph row offsets
    size_t vloc_cap = 0;
    uint32_t *d_eoff = nullptr;     // first directed entry of each graph (cap_G + 1)
    int32_t *h_stat = nullptr;      // pinned copy of the per-graph statistics (2 * cap_G)
    std::vector<BatchCapture> caps;
    gc_tuning tuning{};
};

namespace {

void drop_captures(gc_batch *b) {
    for (auto &c : b->caps)
        if (c.exec) cudaGraphExecDestroy(c.exec);
    b->caps.clear();
}

bool tuning_valid(const gc_tuning &t) {
    return t.hub_degree >= 1 && t.warp_degree <= t.hub_degree && t.gnn_warp_degree >= 1 &&
           (t.schedule == GC_SCHEDULE_DEGREE || t.schedule == GC_SCHEDULE_SEGMENT) && t.jp_ctas_per_sm >= 1 &&
           t.jp_ctas_per_sm <= 32;
}

// Room for `G` graphs: segment buffers (device) and the pinned statistics copy.
gc_status reserve_segments(gc_batch *b, uint32_t G) {
    gc_ctx *ctx = b->ctx;
    gc_graph *g = b->g;
    gc_status s;
    if (G <= b->cap_G && g->seg_voff) return GC_OK;
    const uint32_t cap = std::max(G, 1u);
    gc_dev_free(ctx, g->seg_voff);
    gc_dev_free(ctx, g->seg_stat);
    gc_dev_free(ctx, b->d_eoff);
    g->seg_voff = nullptr;
    g->seg_stat = nullptr;
    b->d_eoff = nullptr;
    if (b->h_stat) cudaFreeHost(b->h_stat);
    b->h_stat = nullptr;
    if ((s = gc_alloc(ctx, &g->seg_voff, (size_t)cap + 1, "segment offsets")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->seg_stat, 2 * (size_t)cap, "segment statistics")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &b->d_eoff, (size_t)cap + 1, "segment edge offsets")) != GC_OK) return s;
    if ((s = gc_check_cuda(ctx, cudaMallocHost((void **)&b->h_stat, sizeof(int32_t) * 2 * cap), "pinned statistics")) !=
        GC_OK)
        return s;
    b->cap_G = cap;
    g->seg_cap = cap;
    return GC_OK;
}

gc_status new_batch(gc_ctx *ctx, uint32_t cap_G, uint32_t cap_N, uint32_t cap_M, gc_batch **out) {
    gc_batch *b = new gc_batch();
    b->ctx = ctx;
    gc_tuning_default(&b->tuning);
    gc_status s = gc_graph_create(ctx, cap_N, cap_M, &b->g);
    if (s == GC_OK) s = reserve_segments(b, cap_G);
    if (s != GC_OK) {
        gc_batch_free(b);
        return s;
    }
    *out = b;
    return GC_OK;
}

// Checks the staged CSR's rows, makes neighbour ids global, then the plain upload checks and
// preparation (degree classes, schedule) on the union.
gc_status finish_batch_upload(gc_batch *b, uint32_t G, const uint32_t *voff_host) {
    gc_ctx *ctx = b->ctx;
    gc_graph *g = b->g;
    gc_status s;
    drop_captures(b);
    b->G = G;
    g->n_seg = G;
    g->h_seg_voff.assign(voff_host, voff_host + G + 1);
    g->has_keys = g->has_colors = false;
    g->key_kind = -1;
    if (g->N) {
        if ((s = gc_reset_state(ctx)) != GC_OK) return s;
        k_check_rows<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, g->M, ctx->dstate);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "row check")) != GC_OK) return s;
        if ((s = gc_read_state(ctx)) != GC_OK)
            return s == GC_ERR_DEVICE ? gc_fail(ctx, GC_ERR_INVALID, "malformed batch: row offsets not monotone") : s;
        if (g->M) {
            k_seg_globalize<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->V, g->E, g->seg_voff, G, g->N, ctx->dstate);
            ctx->launches++;
            if ((s = gc_check_launch(ctx, "globalize ids")) != GC_OK) return s;
            if ((s = gc_read_state(ctx)) != GC_OK)
                return s == GC_ERR_DEVICE ? gc_fail(ctx, GC_ERR_INVALID, "malformed batch: neighbour id outside its graph")
                                          : s;
        }
    }
    g->warp_deg = b->tuning.warp_degree;
    g->gnn_warp_deg = b->tuning.gnn_warp_degree;
    g->hub_deg = b->tuning.hub_degree;
    g->sched = b->tuning.schedule;
    g->jp_ctas = b->tuning.jp_ctas_per_sm;
    g->jp_tight = b->tuning.jp_tight;
    g->jp_nap = b->tuning.jp_nap;
    return gc_graph_finish_upload(g);
}

// Host-side shape checks of G separate CSRs; fills voff and eoff (G + 1 each).
gc_status shape_graphs(gc_ctx *ctx, uint32_t G, const uint32_t *n, const uint32_t *const *Vs,
                       const uint32_t *const *Es, std::vector<uint32_t> &voff, std::vector<uint32_t> &eoff) {
    if (G && (!n || !Vs || !Es)) return gc_fail(ctx, GC_ERR_INVALID, "null graph arrays");
    voff.assign((size_t)G + 1, 0);
    eoff.assign((size_t)G + 1, 0);
    uint64_t nv = 0, ne = 0;
    for (uint32_t i = 0; i < G; i++) {
        if (!Vs[i]) return gc_fail(ctx, GC_ERR_INVALID, "graph " + std::to_string(i) + ": V is NULL");
        if (Vs[i][0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "graph " + std::to_string(i) + ": V[0] must be 0");
        const uint32_t m = Vs[i][n[i]];
        if (m && !Es[i]) return gc_fail(ctx, GC_ERR_INVALID, "graph " + std::to_string(i) + ": E is NULL");
        nv += n[i];
        ne += m;
        if (nv >= 0xffffffffULL || ne > 0xffffffffULL)
            return gc_fail(ctx, GC_ERR_INVALID, "batch exceeds 2^32 vertices or edges");
        voff[i + 1] = (uint32_t)nv;
        eoff[i + 1] = (uint32_t)ne;
    }
    return GC_OK;
}

// Copies G separate host CSRs into the batch (capacity already checked).
gc_status fill_graphs(gc_batch *b, uint32_t G, const uint32_t *n, const uint32_t *const *Vs,
                      const uint32_t *const *Es, const std::vector<uint32_t> &voff, const std::vector<uint32_t> &eoff) {
    gc_ctx *ctx = b->ctx;
    gc_graph *g = b->g;
    gc_status s;
    const uint32_t N = voff[G], M = eoff[G];
    g->N = N;
    g->M = M;
    if ((s = reserve_segments(b, G)) != GC_OK) return s;
    const size_t vloc_words = (size_t)N + G;
    if (vloc_words > b->vloc_cap) {
        gc_dev_free(ctx, b->d_vloc);
        b->d_vloc = nullptr;
        if ((s = gc_alloc(ctx, &b->d_vloc, vloc_words, "staged row offsets")) != GC_OK) return s;
        b->vloc_cap = vloc_words;
    }
    for (uint32_t i = 0; i < G; i++) {
        const uint32_t m = eoff[i + 1] - eoff[i];
        if (m && (s = gc_check_cuda(ctx, cudaMemcpyAsync(g->E + eoff[i], Es[i], sizeof(uint32_t) * m,
                                                         cudaMemcpyHostToDevice, ctx->stream), "upload E")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(b->d_vloc + voff[i] + i, Vs[i], sizeof(uint32_t) * ((size_t)n[i] + 1),
                                                    cudaMemcpyHostToDevice, ctx->stream), "upload V")) != GC_OK)
            return s;
    }
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->seg_voff, voff.data(), sizeof(uint32_t) * ((size_t)G + 1),
                                                cudaMemcpyHostToDevice, ctx->stream), "upload offsets")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(b->d_eoff, eoff.data(), sizeof(uint32_t) * ((size_t)G + 1),
                                                cudaMemcpyHostToDevice, ctx->stream), "upload offsets")) != GC_OK)
        return s;
    k_seg_rows<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(b->d_vloc, g->seg_voff, b->d_eoff, G, N, M, g->V);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "segment rows")) != GC_OK) return s;
    // the host vectors must outlive the copies above
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "upload batch")) != GC_OK) return s;
    return finish_batch_upload(b, G, voff.data());
}

// Priorities, coloring, Culberson rounds, per-graph statistics and their read-back, all queued
// on the context's stream without a host synchronisation (so that it can be captured).
gc_status queue_pipeline(gc_batch *b, gc_heuristic h, const gc_model *m, int recolor) {
    gc_ctx *ctx = b->ctx;
    gc_graph *g = b->g;
    gc_status s;
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    if (h == GC_GNN) s = gc_priority_gnn(g, m);
    else s = gc_priority_simple(g, h);
    if (s != GC_OK) return s;
    g->key_kind = (int)h;
    g->has_keys = true;
    if ((s = gc_jp_color(g)) != GC_OK) return s;
    for (int it = 0; it < recolor; it++) {
        if ((s = gc_keys_from_colors(g)) != GC_OK) return s;
        if ((s = gc_jp_color(g)) != GC_OK) return s;
    }
    if ((s = gc_segment_stats(g)) != GC_OK) return s;
    if (b->G && (s = gc_check_cuda(ctx, cudaMemcpyAsync(b->h_stat, g->seg_stat, sizeof(int32_t) * 2 * b->G,
                                                        cudaMemcpyDeviceToHost, ctx->stream), "read statistics")) != GC_OK)
        return s;
    return gc_check_cuda(ctx, cudaMemcpyAsync(ctx->hstate, ctx->dstate, sizeof(gc::DevState), cudaMemcpyDeviceToHost,
                                              ctx->stream), "read device state");
}

// Waits for a queued pipeline and turns its statistics into color counts.
gc_status finish_pipeline(gc_batch *b, int32_t *colors) {
    gc_ctx *ctx = b->ctx;
    gc_status s;
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "batch execution")) != GC_OK) return s;
    if ((s = gc_check_hstate(ctx)) != GC_OK) return s;
    if (colors)
        for (uint32_t i = 0; i < b->G; i++) colors[i] = b->h_stat[2 * i + 1] ? 0 : std::max(b->h_stat[2 * i], 1);
    return GC_OK;
}

gc_status check_heuristic(gc_ctx *ctx, gc_heuristic h, const gc_model *m) {
    if (h == GC_GNN) {
        if (!m || m->layers < 2) return gc_fail(ctx, GC_ERR_INVALID, "GNN priorities need a model with at least 2 layers");
        return GC_OK;
    }
    if (h == GC_FF || h == GC_LF || h == GC_LLF) return GC_OK;
    if (h == GC_SL || h == GC_SLL)
        return gc_fail(ctx, GC_ERR_INVALID, "SL / SLL peel each graph on its own: not offered on batches");
    return gc_fail(ctx, GC_ERR_INVALID, "unknown heuristic");
}

// One uncaptured pass; with `ms` set, timed with CUDA events on the stream.
gc_status direct_pass(gc_batch *b, gc_heuristic h, const gc_model *m, int recolor, int32_t *colors, float *ms) {
    gc_ctx *ctx = b->ctx;
    gc_status s;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        if ((s = gc_check_cuda(ctx, cudaEventCreate(&e0), "event")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreate(&e1), "event")) != GC_OK) {
            cudaEventDestroy(e0);
            return s;
        }
        cudaEventRecord(e0, ctx->stream);
    }
    s = queue_pipeline(b, h, m, recolor);
    if (ms && s == GC_OK) cudaEventRecord(e1, ctx->stream);
    if (s == GC_OK) s = finish_pipeline(b, colors);
    if (ms) {
        if (s == GC_OK) s = gc_check_cuda(ctx, cudaEventElapsedTime(ms, e0, e1), "event timing");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return s;
}

gc_status capture(gc_batch *b, gc_heuristic h, const gc_model *m, int recolor, BatchCapture *out) {
    gc_ctx *ctx = b->ctx;
    gc_status s;
    if ((s = gc_check_cuda(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "begin capture")) !=
        GC_OK)
        return s;
    const uint64_t l0 = ctx->launches;
    const bool prof = ctx->prof;
    ctx->prof = false;  // no event records inside the graph
    s = queue_pipeline(b, h, m, recolor);
    ctx->prof = prof;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    out->launches = ctx->launches - l0;
    ctx->launches = l0;
    if (s == GC_OK) s = gc_check_cuda(ctx, e, "end capture");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaGraphInstantiate(&out->exec, graph, 0), "instantiate graph");
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return s;
}

gc_status apply_tuning(gc_batch *b, const gc_tuning &t) {
    gc_graph *g = b->g;
    const bool reprepare = t.warp_degree != g->warp_deg || t.hub_degree != g->hub_deg || t.schedule != g->sched ||
                           t.gnn_warp_degree != g->gnn_warp_deg;
    b->tuning = t;
    drop_captures(b);
    g->warp_deg = t.warp_degree;
    g->gnn_warp_deg = t.gnn_warp_degree;
    g->hub_deg = t.hub_degree;
    g->sched = t.schedule;
    g->jp_ctas = t.jp_ctas_per_sm;
    g->jp_tight = t.jp_tight;
    g->jp_nap = t.jp_nap;
    if (!reprepare) return GC_OK;
    g->has_keys = g->has_colors = false;
    return gc_graph_prepare(g);
}

}  // namespace

extern "C" {

void gc_tuning_default(gc_tuning *t) {
    if (!t) return;
    t->warp_degree = GC_GNN_WARP_DEGREE;
    t->hub_degree = GC_GNN_HUB_DEGREE;
    t->schedule = GC_SCHEDULE_DEGREE;
    t->jp_ctas_per_sm = 2;
    t->jp_tight = 32;
    t->jp_nap = 32;
    t->gnn_warp_degree = GC_GNN_WIDE_DEGREE;
}

uint64_t gc_batch_device_bytes(uint32_t G, uint32_t N, uint32_t M, gc_heuristic h) {
    // CSR, keys, colors, hub list, degree order, sort buffers, predecessor lists and counts, ticket
    // order, leaf list, staged offsets, published forbidden colors, ticket records; GNN feature planes, input
    // table, feature-row map and the neighbour ids as rows; segment arrays; the
    // split task list and sort histogram; allocation granularity.
    uint64_t per_vertex = 4 + 4 + 4 + 4 + 4 + 16 + 4 + 4 + 4 + 4 + 8 * GC_JP_MASK_WORDS + 16;
    uint64_t per_edge = 8;
    if (h == GC_GNN) per_vertex += 64 + 64 + 8 + 4 + 8, per_edge += 4;
    uint64_t bytes = per_edge * M + per_vertex * N + 4ull * G + 20ull * G + 64;
    bytes += 8ull * (M / GC_SPLIT_CHUNK + 1) + 4ull * (256ull * (N / 8192 + 1) + 2048);
    bytes += 24ull * (2u << 20);
    return bytes;
}

gc_status gc_batch_create(gc_ctx *ctx, uint32_t cap_G, uint32_t cap_N, uint32_t cap_M, gc_batch **out) {
    if (!ctx || !out) return GC_ERR_INVALID;
    *out = nullptr;
    DeviceGuard dg(ctx);
    return new_batch(ctx, cap_G, cap_N, cap_M, out);
}

gc_status gc_batch_upload_graphs(gc_ctx *ctx, uint32_t G, const uint32_t *n, const uint32_t *const *Vs,
                                 const uint32_t *const *Es, gc_batch **out) {
    if (!ctx || !out) return GC_ERR_INVALID;
    *out = nullptr;
    DeviceGuard dg(ctx);
    std::vector<uint32_t> voff, eoff;
    gc_status s = shape_graphs(ctx, G, n, Vs, Es, voff, eoff);
    if (s != GC_OK) return s;
    gc_batch *b = nullptr;
    if ((s = new_batch(ctx, G, voff[G], eoff[G], &b)) != GC_OK) return s;
    if ((s = fill_graphs(b, G, n, Vs, Es, voff, eoff)) != GC_OK) {
        gc_batch_free(b);
        return s;
    }
    *out = b;
    return GC_OK;
}

gc_status gc_batch_reupload_graphs(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *n, const uint32_t *const *Vs,
                                   const uint32_t *const *Es) {
    if (!ctx || !b || b->ctx != ctx) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    std::vector<uint32_t> voff, eoff;
    gc_status s = shape_graphs(ctx, G, n, Vs, Es, voff, eoff);
    if (s != GC_OK) return s;
    if (voff[G] > b->g->cap_N || eoff[G] > b->g->cap_M)
        return gc_fail(ctx, GC_ERR_INVALID, "batch exceeds the allocated capacity");
    return fill_graphs(b, G, n, Vs, Es, voff, eoff);
}

gc_status gc_batch_upload(gc_ctx *ctx, uint32_t G, const uint32_t *voff, const uint32_t *V, const uint32_t *E,
                          gc_batch **out) {
    if (!ctx || !out || !voff || !V) return GC_ERR_INVALID;
    *out = nullptr;
    DeviceGuard dg(ctx);
    if (voff[0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "voff[0] must be 0");
    for (uint32_t i = 0; i < G; i++)
        if (voff[i + 1] < voff[i]) return gc_fail(ctx, GC_ERR_INVALID, "voff not monotone");
    const uint32_t N = voff[G];
    if (V[0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "V[0] must be 0");
    const uint32_t M = V[N];
    if (M && !E) return gc_fail(ctx, GC_ERR_INVALID, "E is NULL");
    gc_batch *b = nullptr;
    gc_status s = new_batch(ctx, G, N, M, &b);
    if (s != GC_OK) return s;
    gc_graph *g = b->g;
    g->N = N;
    g->M = M;
    s = gc_check_cuda(ctx, cudaMemcpyAsync(g->V, V, sizeof(uint32_t) * ((size_t)N + 1), cudaMemcpyHostToDevice,
                                           ctx->stream), "upload V");
    if (s == GC_OK && M)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(g->E, E, sizeof(uint32_t) * (size_t)M, cudaMemcpyHostToDevice, ctx->stream),
                          "upload E");
    if (s == GC_OK)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(g->seg_voff, voff, sizeof(uint32_t) * ((size_t)G + 1),
                                               cudaMemcpyHostToDevice, ctx->stream), "upload offsets");
    if (s == GC_OK) s = finish_batch_upload(b, G, voff);
    if (s != GC_OK) {
        gc_batch_free(b);
        return s;
    }
    *out = b;
    return GC_OK;
}

gc_status gc_batch_reupload(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *voff, const uint32_t *V,
                            const uint32_t *E) {
    if (!ctx || !b || b->ctx != ctx || !voff || !V) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    if (voff[0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "voff[0] must be 0");
    for (uint32_t i = 0; i < G; i++)
        if (voff[i + 1] < voff[i]) return gc_fail(ctx, GC_ERR_INVALID, "voff not monotone");
    const uint32_t N = voff[G];
    if (V[0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "V[0] must be 0");
    const uint32_t M = V[N];
    if (M && !E) return gc_fail(ctx, GC_ERR_INVALID, "E is NULL");
    gc_graph *g = b->g;
    if (N > g->cap_N || M > g->cap_M || G > b->cap_G)
        return gc_fail(ctx, GC_ERR_INVALID, "batch exceeds the allocated capacity");
    g->N = N;
    g->M = M;
    gc_status s = gc_check_cuda(ctx, cudaMemcpyAsync(g->V, V, sizeof(uint32_t) * ((size_t)N + 1),
                                                     cudaMemcpyHostToDevice, ctx->stream), "upload V");
    if (s == GC_OK && M)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(g->E, E, sizeof(uint32_t) * (size_t)M, cudaMemcpyHostToDevice, ctx->stream),
                          "upload E");
    if (s == GC_OK)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(g->seg_voff, voff, sizeof(uint32_t) * ((size_t)G + 1),
                                               cudaMemcpyHostToDevice, ctx->stream), "upload offsets");
    if (s != GC_OK) return s;
    return finish_batch_upload(b, G, voff);
}

gc_status gc_batch_reupload_device_graphs(gc_ctx *ctx, gc_batch *b, uint32_t G, const uint32_t *n, const uint32_t *m,
                                          const uint32_t *const *dVs, const uint32_t *const *dEs) {
    if (!ctx || !b || b->ctx != ctx) return GC_ERR_INVALID;
    if (G && (!n || !m || !dVs || !dEs)) return gc_fail(ctx, GC_ERR_INVALID, "null graph arrays");
    DeviceGuard dg(ctx);
    gc_graph *g = b->g;
    std::vector<uint32_t> voff((size_t)G + 1, 0), eoff((size_t)G + 1, 0);
    uint64_t nv = 0, ne = 0;
    for (uint32_t i = 0; i < G; i++) {
        if (!dVs[i] || (m[i] && !dEs[i]))
            return gc_fail(ctx, GC_ERR_INVALID, "graph " + std::to_string(i) + ": null device CSR");
        nv += n[i];
        ne += m[i];
        if (nv >= 0xffffffffULL || ne > 0xffffffffULL)
            return gc_fail(ctx, GC_ERR_INVALID, "batch exceeds 2^32 vertices or edges");
        voff[i + 1] = (uint32_t)nv;
        eoff[i + 1] = (uint32_t)ne;
    }
    const uint32_t N = voff[G], M = eoff[G];
    if (N > g->cap_N || M > g->cap_M || G > b->cap_G)
        return gc_fail(ctx, GC_ERR_INVALID, "batch exceeds the allocated capacity");
    gc_status s;
    const size_t vloc_words = (size_t)N + G;
    if (vloc_words > b->vloc_cap) {
        gc_dev_free(ctx, b->d_vloc);
        b->d_vloc = nullptr;
        if ((s = gc_alloc(ctx, &b->d_vloc, std::max(vloc_words, (size_t)g->cap_N + b->cap_G), "staged row offsets")) !=
            GC_OK)
            return s;
        b->vloc_cap = std::max(vloc_words, (size_t)g->cap_N + b->cap_G);
    }
    if ((s = gc_alloc(ctx, &b->d_src, (size_t)b->cap_G, "gather descriptors")) != GC_OK) return s;
    if (!b->h_src && (s = gc_check_cuda(ctx, cudaMallocHost((void **)&b->h_src, sizeof(gc_seg_src) * b->cap_G),
                                        "pinned descriptors")) != GC_OK)
        return s;
    // the previous refill's descriptor copy must be done before the pinned staging is rewritten
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "batch refill")) != GC_OK) return s;
    for (uint32_t i = 0; i < G; i++) b->h_src[i] = gc_seg_src{dVs[i], dEs[i], n[i], m[i], voff[i] + i, eoff[i]};
    g->N = N;
    g->M = M;
    if (G && (s = gc_check_cuda(ctx, cudaMemcpyAsync(b->d_src, b->h_src, sizeof(gc_seg_src) * G, cudaMemcpyHostToDevice,
                                                     ctx->stream), "upload descriptors")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->seg_voff, voff.data(), sizeof(uint32_t) * ((size_t)G + 1),
                                                cudaMemcpyHostToDevice, ctx->stream), "upload offsets")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(b->d_eoff, eoff.data(), sizeof(uint32_t) * ((size_t)G + 1),
                                                cudaMemcpyHostToDevice, ctx->stream), "upload offsets")) != GC_OK)
        return s;
    if (G) {
        k_seg_gather<<<std::min<uint32_t>(G, 65535u), 256, 0, ctx->stream>>>(b->d_src, G, b->d_vloc, g->E);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "gather graphs")) != GC_OK) return s;
    }
    k_seg_rows<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(b->d_vloc, g->seg_voff, b->d_eoff, G, N, M, g->V);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "segment rows")) != GC_OK) return s;
    // the host vectors must outlive the copies above
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "batch refill")) != GC_OK) return s;
    return finish_batch_upload(b, G, voff.data());
}

void gc_batch_free(gc_batch *b) {
    if (!b) return;
    {
        DeviceGuard dg(b->ctx);
        if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
        drop_captures(b);
        if (b->g) {
            gc_dev_free(b->ctx, b->d_vloc);
            gc_dev_free(b->ctx, b->d_eoff);
            gc_dev_free(b->ctx, b->d_src);
        }
        if (b->h_stat) cudaFreeHost(b->h_stat);
        if (b->h_src) cudaFreeHost(b->h_src);
    }
    if (b->g) gc_graph_free(b->g);
    delete b;
}

uint32_t gc_batch_num_graphs(const gc_batch *b) { return b ? b->G : 0; }
uint32_t gc_batch_num_vertices(const gc_batch *b) { return b ? b->g->N : 0; }
uint32_t gc_batch_num_edges(const gc_batch *b) { return b ? b->g->M : 0; }
gc_graph *gc_batch_graph(gc_batch *b) { return b ? b->g : nullptr; }

gc_status gc_batch_color(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *m, int recolor, int32_t *colors) {
    if (!ctx || !b || b->ctx != ctx || recolor < 0) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s = check_heuristic(ctx, h, m);
    if (s != GC_OK) return s;
    gc_graph *g = b->g;
    if (g->N == 0) {
        if (colors)
            for (uint32_t i = 0; i < b->G; i++) colors[i] = 1;
        g->has_colors = true;
        return GC_OK;
    }
    const float *param = h == GC_GNN ? m->d_param : nullptr;
    const int layers = h == GC_GNN ? m->layers : 0, md = h == GC_GNN ? m->md : 0;
    BatchCapture *hit = nullptr;
    for (auto &c : b->caps)
        if (c.h == (int)h && c.param == param && c.layers == layers && c.md == md && c.recolor == recolor) hit = &c;
    if (!hit) {
        // first pass: runs directly (this also allocates every lazily allocated buffer), then the
        // same sequence is captured for the next calls
        if ((s = direct_pass(b, h, m, recolor, colors, nullptr)) != GC_OK) return s;
        BatchCapture c;
        c.h = (int)h;
        c.param = param;
        c.layers = layers;
        c.md = md;
        c.recolor = recolor;
        if ((s = capture(b, h, m, recolor, &c)) != GC_OK) return s;
        b->caps.push_back(c);
        g->has_colors = true;
        return GC_OK;
    }
    if ((s = gc_check_cuda(ctx, cudaGraphLaunch(hit->exec, ctx->stream), "graph launch")) != GC_OK) return s;
    ctx->launches += hit->launches;
    g->key_kind = (int)h;
    g->has_keys = g->has_colors = true;
    return finish_pipeline(b, colors);
}

gc_status gc_batch_color_once(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *m, int recolor,
                              int32_t *colors) {
    if (!ctx || !b || b->ctx != ctx || recolor < 0) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s = check_heuristic(ctx, h, m);
    if (s != GC_OK) return s;
    gc_graph *g = b->g;
    if (g->N == 0) {
        if (colors)
            for (uint32_t i = 0; i < b->G; i++) colors[i] = 1;
        g->has_colors = true;
        return GC_OK;
    }
    if ((s = direct_pass(b, h, m, recolor, colors, nullptr)) != GC_OK) return s;
    g->key_kind = (int)h;
    g->has_keys = g->has_colors = true;
    return GC_OK;
}

gc_status gc_batch_download_colors(gc_ctx *ctx, gc_batch *b, int32_t *color) {
    if (!b) return GC_ERR_INVALID;
    return gc_download_colors(ctx, b->g, color);
}

gc_status gc_batch_set_tuning(gc_ctx *ctx, gc_batch *b, const gc_tuning *t) {
    if (!ctx || !b || b->ctx != ctx || !t) return GC_ERR_INVALID;
    if (!tuning_valid(*t)) return gc_fail(ctx, GC_ERR_INVALID, "invalid tuning");
    DeviceGuard dg(ctx);
    return apply_tuning(b, *t);
}

gc_status gc_batch_get_tuning(const gc_batch *b, gc_tuning *t) {
    if (!b || !t) return GC_ERR_INVALID;
    *t = b->tuning;
    return GC_OK;
}

gc_status gc_batch_autotune(gc_ctx *ctx, gc_batch *b, gc_heuristic h, const gc_model *m, int recolor, int effort,
                            gc_tuning *best_out, double *best_ms_out) {
    if (!ctx || !b || b->ctx != ctx || recolor < 0) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s = check_heuristic(ctx, h, m);
    if (s != GC_OK) return s;
    gc_tuning best = b->tuning;
    double best_ms = INFINITY;
    // one warm pass, then the faster of two timed passes
    auto measure = [&](const gc_tuning &t, double *ms) -> gc_status {
        gc_status st = apply_tuning(b, t);
        if (st != GC_OK) return st;
        if ((st = direct_pass(b, h, m, recolor, nullptr, nullptr)) != GC_OK) return st;
        float a = 0.0f, c = 0.0f;
        if ((st = direct_pass(b, h, m, recolor, nullptr, &a)) != GC_OK) return st;
        if ((st = direct_pass(b, h, m, recolor, nullptr, &c)) != GC_OK) return st;
        *ms = std::min(a, c);
        return GC_OK;
    };
    std::vector<gc_tuning> seen;
    auto consider = [&](const gc_tuning &t) -> gc_status {
        if (!tuning_valid(t)) return GC_OK;
        for (const gc_tuning &o : seen)
            if (!memcmp(&o, &t, sizeof t)) return GC_OK;
        seen.push_back(t);
        double ms = 0;
        gc_status st = measure(t, &ms);
        if (st != GC_OK) return st;
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
        return GC_OK;
    };
    if (b->g->N == 0) {
        if (best_out) *best_out = best;
        if (best_ms_out) *best_ms_out = 0.0;
        return GC_OK;
    }
    if ((s = consider(best)) != GC_OK) return s;
    std::vector<uint32_t> warp_degs = {64, 128, 256, 512};
    if (effort >= 2) warp_degs = {16, 32, 64, 128, 256, 512, 1024, 4096};
    std::vector<uint32_t> hub_degs = {best.hub_degree};
    if (effort >= 2) hub_degs = {4096, 16384, 65536};
    std::vector<int> scheds = {best.schedule};
    if (effort >= 1 && b->G > 1) scheds = {GC_SCHEDULE_DEGREE, GC_SCHEDULE_SEGMENT};
    // stage 1: vertex-to-thread mapping (tier thresholds) and schedule
    {
        const gc_tuning base = best;
        for (int sc : scheds)
            for (uint32_t hd : hub_degs)
                for (uint32_t wd : warp_degs) {
                    gc_tuning t = base;
                    t.schedule = sc;
                    t.hub_degree = hd;
                    t.warp_degree = wd;
                    if ((s = consider(t)) != GC_OK) return s;
                }
    }
    if (effort >= 1 && (h == GC_GNN) && best.schedule == GC_SCHEDULE_DEGREE) {
        // stage 1b: the GNN layers' own warp tier
        const gc_tuning base = best;
        for (uint32_t gw : {256u, 1024u, 4096u}) {
            gc_tuning t = base;
            t.gnn_warp_degree = gw;
            if ((s = consider(t)) != GC_OK) return s;
        }
    }
    if (effort >= 1) {
        // stage 2: resident CTAs of the ordered coloring kernel
        const gc_tuning base = best;
        for (int c : {1, 2, 3, 4}) {
            gc_tuning t = base;
            t.jp_ctas_per_sm = c;
            if ((s = consider(t)) != GC_OK) return s;
        }
        // stage 3: its polling rhythm
        const gc_tuning base2 = best;
        const unsigned int polls[][2] = {{32, 32}, {8, 32}, {128, 32}, {32, 128}, {4, 8}};
        for (auto &p : polls) {
            gc_tuning t = base2;
            t.jp_tight = p[0];
            t.jp_nap = p[1];
            if ((s = consider(t)) != GC_OK) return s;
        }
    }
    if ((s = apply_tuning(b, best)) != GC_OK) return s;
    if (best_out) *best_out = best;
    if (best_ms_out) *best_ms_out = best_ms;
    return GC_OK;
}

}  // extern "C"
