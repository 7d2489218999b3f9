// Native C ABI (include/gnn_coloring.h): contexts, device-resident graphs and models, and the
// hot-path entry points.  Every call returns a status; nothing falls back to the CPU.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gc_internal.h"
#include "host_graph.h"
#include "overlap.h"


// ---- errors ------------------------------------------------------------------------------------

gc_status gc_fail(gc_ctx *ctx, gc_status s, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return s;
}

gc_status gc_check_cuda(gc_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return GC_OK;
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return gc_fail(ctx, GC_ERR_NOMEM, m);
    return gc_fail(ctx, GC_ERR_CUDA, m);
}

gc_status gc_check_launch(gc_ctx *ctx, const char *what) { return gc_check_cuda(ctx, cudaGetLastError(), what); }

gc_status gc_reset_state(gc_ctx *ctx) {
    return gc_check_cuda(ctx, cudaMemsetAsync(ctx->dstate, 0, sizeof(gc::DevState), ctx->stream), "reset device state");
}

gc_status gc_read_state(gc_ctx *ctx) {
    gc_status s = gc_check_cuda(
        ctx, cudaMemcpyAsync(ctx->hstate, ctx->dstate, sizeof(gc::DevState), cudaMemcpyDeviceToHost, ctx->stream),
        "read device state");
    if (s != GC_OK) return s;
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "kernel execution")) != GC_OK) return s;
    return gc_check_hstate(ctx);
}

gc_status gc_check_hstate(gc_ctx *ctx) {
    unsigned int err = ctx->hstate->err;
    if (err) {
        char buf[160];
        snprintf(buf, sizeof buf, "device error 0x%x at index %u (%s)", err, ctx->hstate->err_info,
                 (err & gc::ERR_WAIT_EXPIRED) ? "wait for a predecessor color expired"
                 : (err & gc::ERR_BOUND)      ? "bound exceeded"
                                              : "ordering invariant");
        return gc_fail(ctx, GC_ERR_DEVICE, buf);
    }
    return GC_OK;
}

ProfScope::ProfScope(gc_ctx *c, const char *n, cudaStream_t s) : ctx(c), stream(s), name(n) {
    if (!ctx->prof) return;
    if (ctx->prof_pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        ctx->prof_pool.push_back(e);
    }
    a = ctx->prof_pool.back();
    ctx->prof_pool.pop_back();
    cudaEventRecord(a, stream);
}

ProfScope::~ProfScope() {
    if (!a) return;
    cudaEvent_t b;
    if (ctx->prof_pool.empty()) {
        if (cudaEventCreate(&b) != cudaSuccess) return;
    } else {
        b = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
    }
    cudaEventRecord(b, stream);
    ctx->prof_recs.push_back({name, a, b});
}

namespace {

__global__ void k_check_csr(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E, uint32_t N, uint32_t M,
                            gc::DevState *st) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += stride) {
        uint32_t a = V[u], b = V[u + 1];
        if (b < a || b > M) gc::raise_error(st, gc::ERR_BOUND, u);
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride)
        if (E[i] >= N) gc::raise_error(st, gc::ERR_BOUND, i);
}

// The two halves of k_check_csr, for uploads that check V before E has arrived.
__global__ void k_check_offsets(const uint32_t *__restrict__ V, uint32_t N, uint32_t M, gc::DevState *st) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        uint32_t a = V[u], b = V[u + 1];
        if (b < a || b > M) gc::raise_error(st, gc::ERR_BOUND, u);
    }
}
__global__ void k_check_ids(const uint32_t *__restrict__ E, uint32_t N, uint32_t M, gc::DevState *st) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x)
        if (E[i] >= N) gc::raise_error(st, gc::ERR_BOUND, i);
}

__global__ void k_keys_to_double(const uint32_t *__restrict__ key, uint32_t N, int float_bits, double *__restrict__ p) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
        p[u] = float_bits ? (double)__uint_as_float(key[u]) : (double)key[u];
}

}  // namespace

void gc_graph_free_buffers(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    if (g->owns_csr) {
        gc_dev_free(ctx, g->V);
        gc_dev_free(ctx, g->E);
    }
    void *bufs[] = {g->key,       g->color,  g->P,        g->pc,       g->order,    g->sort_buf, g->sort_hist,
                    g->big,       g->hubs,   g->x,        g->y,        g->t01,      g->deg_rem,  g->frontier,
                    g->frontier2, g->removed, g->leaf_list, g->vorder, g->rank,     g->p64,      g->seg_voff,
                    g->seg_stat,  g->fmask,    g->jprec, g->class_first,
                    g->gnn_ctr,   g->hub_aux, g->jpsplit, g->part_tiles, g->giant_off, g->hub_stage,
                    g->row_of,    g->Er,      g->vrow};
    for (void *p : bufs) gc_dev_free(ctx, p);
}

gc_status gc_graph_alloc(gc_ctx *ctx, gc_graph *g, uint32_t N, uint32_t M, bool csr) {
    gc_status s;
    g->cap_N = N;
    g->cap_M = M;
    if (csr) {
        if ((s = gc_alloc(ctx, &g->V, (size_t)N + 1, "graph V")) != GC_OK) return s;
        if ((s = gc_alloc(ctx, &g->E, (size_t)M, "graph E")) != GC_OK) return s;
    }
    if ((s = gc_alloc(ctx, &g->key, (size_t)N, "keys")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->color, (size_t)N, "colors")) != GC_OK) return s;
    return GC_OK;
}

namespace {

gc_status check_host_csr(gc_ctx *ctx, uint32_t N, const uint32_t *V, const uint32_t *E) {
    if (!V) return gc_fail(ctx, GC_ERR_INVALID, "V is NULL");
    if (V[0] != 0) return gc_fail(ctx, GC_ERR_INVALID, "V[0] must be 0");
    if (V[N] > 0 && !E) return gc_fail(ctx, GC_ERR_INVALID, "E is NULL");
    return GC_OK;
}

}  // namespace

gc_status gc_graph_finish_upload(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    g->has_keys = g->has_colors = false;
    g->key_kind = -1;
    if (g->N == 0) return gc_graph_prepare(g);
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    k_check_csr<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->E, g->N, g->M, ctx->dstate);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "csr check")) != GC_OK) return s;
    if ((s = gc_read_state(ctx)) != GC_OK)
        return s == GC_ERR_DEVICE ? gc_fail(ctx, GC_ERR_INVALID, "malformed CSR: V not monotone or E out of range") : s;
    return gc_graph_prepare(g);
}

gc_status gc_copy_stream(gc_ctx *ctx) {
    if (ctx->copy_stream) return GC_OK;
    gc_status s = gc_check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream");
    if (s == GC_OK)
        s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_copy_fence, cudaEventDisableTiming), "copy events");
    if (s == GC_OK)
        s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_copy_done, cudaEventDisableTiming), "copy events");
    for (int k = 0; k < GC_UPLOAD_CHUNKS && s == GC_OK; k++)
        s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_chunk[k], cudaEventDisableTiming), "copy events");
    return s;
}

void gc_graph_gnn_hint(gc_graph *g, int on) {
    if (g) g->gnn_hint = on != 0;
}

bool gc_is_pinned(const void *host_ptr) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, host_ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

namespace {

// Upload of a CSR whose E is page-locked host memory: E goes up on the copy stream while V is
// checked and the graph prepared on the context's stream (preparation reads V only); E is checked
// once it has arrived.  When GNN priorities follow (gnn_hint), E goes up in GC_UPLOAD_CHUNKS pieces
// and, once the graph is prepared, each piece is converted to feature rows (which checks its ids)
// as soon as it has arrived, beside the rest of the copy.  Returns only after the copy has
// finished, so the caller may reuse E.
gc_status reupload_overlapped(gc_ctx *ctx, gc_graph *g, const uint32_t *V, const uint32_t *E) {
    const uint32_t N = g->N, M = g->M;
    gc_status s = gc_copy_stream(ctx);
    if (s != GC_OK) return s;
    g->has_keys = g->has_colors = false;
    g->key_kind = -1;
    const bool rows = g->gnn_hint;
    const uint32_t piece = (M + GC_UPLOAD_CHUNKS - 1) / GC_UPLOAD_CHUNKS;
    // E may still be read by earlier work on the context's stream
    if ((s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_copy_fence, ctx->stream), "upload E")) != GC_OK) return s;
    if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_copy_fence, 0), "upload E")) != GC_OK)
        return s;
    for (int k = 0; k < (rows ? GC_UPLOAD_CHUNKS : 1) && s == GC_OK; k++) {
        const uint32_t first = rows ? std::min<uint32_t>(M, (uint32_t)k * piece) : 0u;
        const uint32_t count = rows ? std::min<uint32_t>(M - first, piece) : M;
        if (count)
            s = gc_check_cuda(ctx, cudaMemcpyAsync(g->E + first, E + first, sizeof(uint32_t) * (size_t)count,
                                                   cudaMemcpyHostToDevice, ctx->copy_stream), "upload E");
        if (s == GC_OK && rows)
            s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_chunk[k], ctx->copy_stream), "upload E");
    }
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_copy_done, ctx->copy_stream), "upload E");
    if (s != GC_OK) {
        cudaStreamSynchronize(ctx->copy_stream);
        return s;
    }
    s = gc_check_cuda(ctx, cudaMemcpyAsync(g->V, V, sizeof(uint32_t) * ((size_t)N + 1), cudaMemcpyHostToDevice,
                                           ctx->stream), "upload V");
    if (s == GC_OK) s = gc_reset_state(ctx);
    if (s == GC_OK) {
        k_check_offsets<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, N, M, ctx->dstate);
        ctx->launches++;
        s = gc_check_launch(ctx, "csr check");
    }
    if (s == GC_OK && (s = gc_read_state(ctx)) == GC_ERR_DEVICE)
        s = gc_fail(ctx, GC_ERR_INVALID, "malformed CSR: V not monotone or E out of range");
    if (s == GC_OK) s = gc_graph_prepare(g);
    // GNN priorities follow: the feature-row order now, then each piece of E as rows once it has
    // arrived (the conversion checks the piece's ids)
    bool rows_queued = false;
    if (s == GC_OK && rows) {
        s = gc_reset_state(ctx);
        if (s == GC_OK) s = gc_gnn_rows_begin(g);
        for (int k = 0; k < GC_UPLOAD_CHUNKS && s == GC_OK; k++) {
            const uint32_t first = std::min<uint32_t>(M, (uint32_t)k * piece);
            const uint32_t count = std::min<uint32_t>(M - first, piece);
            s = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_chunk[k], 0), "upload E");
            if (s == GC_OK) s = gc_gnn_row_ids(g, first, count);
        }
        rows_queued = s == GC_OK;
    }
    // from here on the context's stream follows the copy
    const gc_status w = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_copy_done, 0), "upload E");
    if (w != GC_OK) {
        cudaStreamSynchronize(ctx->copy_stream);
        return s != GC_OK ? s : w;
    }
    if (s != GC_OK) {
        cudaStreamSynchronize(ctx->copy_stream);
        return s;
    }
    if (!rows_queued) {
        if ((s = gc_reset_state(ctx)) == GC_OK) {
            k_check_ids<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->E, N, M, ctx->dstate);
            ctx->launches++;
            s = gc_check_launch(ctx, "csr check");
        }
        if (s != GC_OK) {
            cudaStreamSynchronize(ctx->copy_stream);
            return s;
        }
    }
    if ((s = gc_read_state(ctx)) != GC_OK)
        return s == GC_ERR_DEVICE ? gc_fail(ctx, GC_ERR_INVALID, "malformed CSR: V not monotone or E out of range") : s;
    g->rows_ready = rows_queued;
    return GC_OK;
}

}  // namespace


extern "C" {

const char *gc_status_string(gc_status s) {
    switch (s) {
        case GC_OK: return "ok";
        case GC_ERR_INVALID: return "invalid argument";
        case GC_ERR_NOMEM: return "out of memory";
        case GC_ERR_CUDA: return "CUDA error";
        case GC_ERR_DEVICE: return "device-side error";
        case GC_ERR_IO: return "I/O error";
        case GC_ERR_FORMAT: return "format error";
        case GC_ERR_BUDGET: return "HBM budget exceeded";
        case GC_ERR_NODEV: return "no CUDA device";
        case GC_ERR_STATE: return "call out of order";
    }
    return "unknown status";
}

gc_status gc_ctx_create(int device, gc_ctx **out) {
    if (!out) return GC_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return GC_ERR_NODEV;
    }
    if (device < 0 || device >= n) return GC_ERR_INVALID;
    gc_ctx *ctx = new gc_ctx();
    ctx->device = device;
    gc_status s = gc_check_cuda(ctx, cudaSetDevice(device), "set device");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaMalloc((void **)&ctx->dstate, sizeof(gc::DevState)), "device state");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaMallocHost((void **)&ctx->hstate, sizeof(gc::DevState)), "host state");
    if (s == GC_OK) s = gc_reset_state(ctx);
    if (const char *lim = getenv("GC_SPIN_LIMIT")) ctx->spin_limit = (unsigned int)strtoul(lim, nullptr, 10);
    // tuning of the coloring kernel's polling (defaults measured on B200)
    if (const char *e = getenv("GC_JP_CTAS_PER_SM")) ctx->jp_ctas_per_sm = atoi(e);
    if (const char *e = getenv("GC_JP_TIGHT")) ctx->jp_tight = (unsigned int)strtoul(e, nullptr, 10);
    if (const char *e = getenv("GC_JP_CLASSES")) ctx->jp_classes = atoi(e) != 0;
    if (const char *e = getenv("GC_JP_DECIDE")) ctx->jp_decide = atoi(e) != 0;
    if (const char *e = getenv("GC_JP_LIGHT_WARPS")) ctx->jp_light_warps = atoi(e);
    if (const char *e = getenv("GC_GNN_HUB_SIDE")) ctx->gnn_hub_side = atoi(e) != 0;
    if (const char *e = getenv("GC_GNN_HUB_CTAS")) ctx->gnn_hub_ctas_per_sm = std::max<uint32_t>(1u, (uint32_t)strtoul(e, nullptr, 10));
    if (const char *e = getenv("GC_JP_CORE_BLOCK")) ctx->jp_core_block = std::max<uint32_t>(1u, (uint32_t)strtoul(e, nullptr, 10));
    if (const char *e = getenv("GC_JP_CORE_WARPS")) ctx->jp_core_warps = atoi(e);
    if (const char *e = getenv("GC_JP_CORE_NAP")) ctx->jp_core_nap = (unsigned int)strtoul(e, nullptr, 10);
    if (const char *e = getenv("GC_JP_CORE_DECIDE")) ctx->jp_core_decide = atoi(e) != 0;
    if (const char *e = getenv("GC_JP_CORE"))
        ctx->jp_core_max = std::min<uint32_t>((uint32_t)strtoul(e, nullptr, 10), 32768u);
    if (const char *e = getenv("GC_JP_NAP")) ctx->jp_nap = (unsigned int)strtoul(e, nullptr, 10);
    if (const char *e = getenv("GC_GNN_WARP_DEGREE")) ctx->gnn_warp_deg = (uint32_t)strtoul(e, nullptr, 10);
    if (const char *e = getenv("GC_HUB_DEGREE")) ctx->hub_deg = std::max<uint32_t>(256u, (uint32_t)strtoul(e, nullptr, 10));
    if (const char *e = getenv("GC_GNN_GRAB")) ctx->gnn_grab = std::max<uint32_t>(1u, (uint32_t)strtoul(e, nullptr, 10));
    if (const char *e = getenv("GC_GNN_HEAVY")) ctx->gnn_heavy = (uint32_t)strtoul(e, nullptr, 10);
    if (const char *e = getenv("GC_GNN_FUSE_ISOLATED")) ctx->gnn_fuse_isolated = atoi(e) != 0;
    if (const char *e = getenv("GC_GNN_THIN_DEGREE")) ctx->gnn_thin_deg = (uint32_t)strtoul(e, nullptr, 10);
    if (s != GC_OK) {
        gc_ctx_destroy(ctx);
        return s;
    }
    *out = ctx;
    return GC_OK;
}

// Graphs and models keep their context alive: destruction order is free.
static void ctx_release(gc_ctx *ctx);

void gc_ctx_destroy(gc_ctx *ctx) {
    if (!ctx || ctx->destroy_requested) return;
    ctx->destroy_requested = true;
    ctx_release(ctx);
}

static void ctx_retain(gc_ctx *ctx) { ctx->refs++; }

static void ctx_release(gc_ctx *ctx) {
    if (--ctx->refs > 0) return;
    DeviceGuard dg(ctx);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &r : ctx->prof_recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : ctx->prof_pool) cudaEventDestroy(e);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->hub_stream) {
        cudaStreamSynchronize(ctx->hub_stream);
        cudaStreamDestroy(ctx->hub_stream);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->ev_copy_fence) cudaEventDestroy(ctx->ev_copy_fence);
    if (ctx->ev_copy_done) cudaEventDestroy(ctx->ev_copy_done);
    for (auto e : ctx->ev_chunk)
        if (e) cudaEventDestroy(e);
    if (ctx->dstate) cudaFree(ctx->dstate);
    if (ctx->hstate) cudaFreeHost(ctx->hstate);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

gc_status gc_prof_enable(gc_ctx *ctx, int on) {
    if (!ctx) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    cudaStreamSynchronize(ctx->stream);
    for (auto &r : ctx->prof_recs) {
        ctx->prof_pool.push_back(r.a);
        ctx->prof_pool.push_back(r.b);
    }
    ctx->prof_recs.clear();
    ctx->prof = on != 0;
    return GC_OK;
}

int gc_prof_read(gc_ctx *ctx, const char **names, double *total_ms, uint64_t *launches, int max) {
    if (!ctx) return 0;
    DeviceGuard dg(ctx);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->hub_stream) cudaStreamSynchronize(ctx->hub_stream);
    std::vector<const char *> nm;
    std::vector<double> ms;
    std::vector<uint64_t> cnt;
    for (auto &r : ctx->prof_recs) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        size_t i = 0;
        while (i < nm.size() && strcmp(nm[i], r.name) != 0) i++;
        if (i == nm.size()) {
            nm.push_back(r.name);
            ms.push_back(0.0);
            cnt.push_back(0);
        }
        ms[i] += t;
        cnt[i]++;
    }
    for (size_t i = 0; i < nm.size() && (int)i < max; i++) {
        if (names) names[i] = nm[i];
        if (total_ms) total_ms[i] = ms[i];
        if (launches) launches[i] = cnt[i];
    }
    return (int)nm.size();
}

const char *gc_last_error(const gc_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }
void *gc_ctx_stream(gc_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
uint64_t gc_ctx_launches(const gc_ctx *ctx) { return ctx ? ctx->launches : 0; }

gc_status gc_sync(gc_ctx *ctx) {
    if (!ctx) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    return gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

// ---- graphs ---------------------------------------------------------------------------------

gc_status gc_graph_upload(gc_ctx *ctx, uint32_t N, const uint32_t *V, const uint32_t *E, gc_graph **out) {
    if (!ctx || !out) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    *out = nullptr;
    gc_status s = check_host_csr(ctx, N, V, E);
    if (s != GC_OK) return s;
    gc_graph *g = new gc_graph();
    g->ctx = ctx;
    g->gnn_warp_deg = ctx->gnn_warp_deg;
    g->hub_deg = ctx->hub_deg;
    ctx_retain(ctx);
    if ((s = gc_graph_alloc(ctx, g, N, V[N], true)) != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    if ((s = gc_graph_reupload(ctx, g, N, V, E)) != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    *out = g;
    return GC_OK;
}

gc_status gc_graph_create(gc_ctx *ctx, uint32_t cap_N, uint32_t cap_M, gc_graph **out) {
    if (!ctx || !out) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    *out = nullptr;
    gc_graph *g = new gc_graph();
    g->ctx = ctx;
    g->gnn_warp_deg = ctx->gnn_warp_deg;
    g->hub_deg = ctx->hub_deg;
    ctx_retain(ctx);
    gc_status s = gc_graph_alloc(ctx, g, cap_N, cap_M, true);
    if (s != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    *out = g;
    return GC_OK;
}

gc_status gc_graph_reupload(gc_ctx *ctx, gc_graph *g, uint32_t N, const uint32_t *V, const uint32_t *E) {
    if (!ctx || !g || !g->owns_csr) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s = check_host_csr(ctx, N, V, E);
    if (s != GC_OK) return s;
    const uint32_t M = V[N];
    if (N > g->cap_N || M > g->cap_M) return gc_fail(ctx, GC_ERR_INVALID, "graph exceeds the allocated capacity");
    g->N = N;
    g->M = M;
    if (M && !ctx->pool && gc_is_pinned(E)) return reupload_overlapped(ctx, g, V, E);
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->V, V, sizeof(uint32_t) * ((size_t)N + 1), cudaMemcpyHostToDevice,
                                                ctx->stream), "upload V")) != GC_OK)
        return s;
    if (M && (s = gc_check_cuda(ctx, cudaMemcpyAsync(g->E, E, sizeof(uint32_t) * (size_t)M, cudaMemcpyHostToDevice,
                                                     ctx->stream), "upload E")) != GC_OK)
        return s;
    return gc_graph_finish_upload(g);
}

gc_status gc_graph_wrap_device(gc_ctx *ctx, uint32_t N, uint32_t M, const uint32_t *dV, const uint32_t *dE,
                               gc_graph **out) {
    if (!ctx || !out || !dV || (M && !dE)) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    *out = nullptr;
    gc_graph *g = new gc_graph();
    g->ctx = ctx;
    g->gnn_warp_deg = ctx->gnn_warp_deg;
    g->hub_deg = ctx->hub_deg;
    ctx_retain(ctx);
    g->owns_csr = false;
    g->V = const_cast<uint32_t *>(dV);
    g->E = const_cast<uint32_t *>(dE);
    gc_status s = gc_graph_alloc(ctx, g, N, M, false);
    if (s == GC_OK) {
        g->N = N;
        g->M = M;
        s = gc_graph_finish_upload(g);
    }
    if (s != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    *out = g;
    return GC_OK;
}

void gc_graph_free(gc_graph *g) {
    if (!g) return;
    gc_ctx *ctx = g->ctx;
    {
        DeviceGuard dg(ctx);
        if (ctx) cudaStreamSynchronize(ctx->stream);
        gc_graph_free_buffers(g);
    }
    delete g;
    if (ctx) ctx_release(ctx);
}

uint32_t gc_graph_num_vertices(const gc_graph *g) { return g ? g->N : 0; }
uint32_t gc_graph_num_edges(const gc_graph *g) { return g ? g->M : 0; }
uint32_t gc_graph_max_degree(const gc_graph *g) { return g ? g->max_deg : 0; }
const uint32_t *gc_graph_device_keys(const gc_graph *g) { return g ? g->key : nullptr; }
const int32_t *gc_graph_device_colors(const gc_graph *g) { return g ? g->color : nullptr; }

// ---- models ---------------------------------------------------------------------------------

gc_status gc_model_create(gc_ctx *ctx, int params, int md, const float *param, gc_model **out) {
    if (!ctx || !out || !param) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    *out = nullptr;
    if (params / gc::LAYER_PARAMS < 2)
        return gc_fail(ctx, GC_ERR_INVALID, "a GraphSAGE-16 model needs at least 2 layers (1056 parameters)");
    gc_model *m = new gc_model();
    m->ctx = ctx;
    ctx_retain(ctx);
    m->params = params;
    m->md = md;
    m->layers = params / gc::LAYER_PARAMS;
    m->h_param = (float *)malloc(sizeof(float) * params);
    if (!m->h_param) {
        delete m;
        return gc_fail(ctx, GC_ERR_NOMEM, "model host copy");
    }
    memcpy(m->h_param, param, sizeof(float) * params);
    gc_status s = gc_alloc(ctx, &m->d_param, (size_t)params, "model parameters");
    if (s == GC_OK)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(m->d_param, param, sizeof(float) * params, cudaMemcpyHostToDevice, ctx->stream),
                          "upload model");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "upload model");
    if (s != GC_OK) {
        gc_model_free(m);
        return s;
    }
    *out = m;
    return GC_OK;
}

gc_status gc_model_load(gc_ctx *ctx, const char *path, gc_model **out) {
    if (!ctx || !path || !out) return GC_ERR_INVALID;
    int params = 0, md = 0;
    float *param = nullptr;
    gc_status s = gc_model_read(path, &params, &md, &param);
    if (s != GC_OK) return gc_fail(ctx, s, std::string("cannot read model file ") + path);
    s = gc_model_create(ctx, params, md, param, out);
    free(param);
    return s;
}

void gc_model_free(gc_model *m) {
    if (!m) return;
    gc_ctx *ctx = m->ctx;
    {
        DeviceGuard dg(ctx);
        if (m->d_param) cudaFree(m->d_param);
    }
    free(m->h_param);
    delete m;
    if (ctx) ctx_release(ctx);
}

int gc_model_layers(const gc_model *m) { return m ? m->layers : 0; }

// ---- hot path -------------------------------------------------------------------------------

gc_status gc_priority(gc_ctx *ctx, gc_graph *g, gc_heuristic h, const gc_model *model) {
    if (!ctx || !g || g->ctx != ctx) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s;
    switch (h) {
        case GC_FF:
        case GC_LF:
        case GC_LLF: s = gc_priority_simple(g, h); break;
        case GC_SL:
        case GC_SLL:
            if (g->n_seg > 1) return gc_fail(ctx, GC_ERR_INVALID, "SL / SLL peel each graph on its own: not offered on batches");
            s = gc_priority_peel(g, h == GC_SLL);
            break;
        case GC_GNN:
            if (!model) return gc_fail(ctx, GC_ERR_INVALID, "GNN priorities need a model");
            s = gc_priority_gnn(g, model);
            break;
        default: return gc_fail(ctx, GC_ERR_INVALID, "unknown heuristic");
    }
    if (s != GC_OK) return s;
    g->key_kind = (int)h;
    g->has_keys = true;
    g->has_colors = false;
    return GC_OK;
}

gc_status gc_priority_set(gc_ctx *ctx, gc_graph *g, const double *p) {
    if (!ctx || !g || (g->N && !p)) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    const uint32_t N = g->N;
    std::vector<uint32_t> k(N);
    // Exact order-preserving keys: integers in [0, 2^32) map to themselves; otherwise values are
    // ranked (equal values share a rank).  -0.0 == +0.0 as in the reference's comparisons.
    bool integral = true;
    for (uint32_t u = 0; u < N; u++) {
        double v = p[u];
        if (std::isnan(v)) return gc_fail(ctx, GC_ERR_INVALID, "NaN priority");
        if (!(v >= 0.0 && v <= 4294967295.0 && v == std::floor(v))) integral = false;
    }
    if (integral) {
        for (uint32_t u = 0; u < N; u++) k[u] = (uint32_t)p[u];
    } else {
        std::vector<double> vals(p, p + N);
        for (double &v : vals)
            if (v == 0.0) v = 0.0;
        std::sort(vals.begin(), vals.end());
        vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
        for (uint32_t u = 0; u < N; u++) {
            double v = p[u] == 0.0 ? 0.0 : p[u];
            k[u] = (uint32_t)(std::lower_bound(vals.begin(), vals.end(), v) - vals.begin());
        }
    }
    gc_status s;
    if (N) {
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->key, k.data(), sizeof(uint32_t) * N, cudaMemcpyHostToDevice,
                                                    ctx->stream), "upload priorities")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "upload priorities")) != GC_OK) return s;
    }
    g->user_p.assign(p, p + N);
    g->key_kind = 200;
    g->has_keys = true;
    g->has_colors = false;
    return GC_OK;
}

gc_status gc_color(gc_ctx *ctx, gc_graph *g, int recolor, int *colors_used) {
    if (!ctx || !g || g->ctx != ctx || recolor < 0) return GC_ERR_INVALID;
    if (!g->has_keys) return gc_fail(ctx, GC_ERR_STATE, "no priorities: call gc_priority or gc_priority_set first");
    DeviceGuard dg(ctx);
    gc_status s;
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    if ((s = gc_jp_color(g)) != GC_OK) return s;
    for (int it = 0; it < recolor; it++) {
        if ((s = gc_keys_from_colors(g)) != GC_OK) return s;
        if ((s = gc_jp_color(g)) != GC_OK) return s;
    }
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    if (colors_used) {
        int C = 0;
        if ((s = gc_validate_device(g, &C)) != GC_OK) return s;
        *colors_used = C;
        g->colors_used = C;
    }
    return GC_OK;
}

gc_status gc_recolor(gc_ctx *ctx, gc_graph *g, int iters, int *colors_used) {
    if (!ctx || !g || g->ctx != ctx || iters < 0) return GC_ERR_INVALID;
    if (!g->has_colors) return gc_fail(ctx, GC_ERR_STATE, "no coloring to recolor");
    DeviceGuard dg(ctx);
    gc_status s;
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    for (int it = 0; it < iters; it++) {
        if ((s = gc_keys_from_colors(g)) != GC_OK) return s;
        g->has_keys = true;
        if ((s = gc_jp_color(g)) != GC_OK) return s;
    }
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    if (colors_used) {
        int C = 0;
        if ((s = gc_validate_device(g, &C)) != GC_OK) return s;
        *colors_used = C;
        g->colors_used = C;
    }
    return GC_OK;
}

gc_status gc_validate(gc_ctx *ctx, gc_graph *g, int *max_color) {
    if (!ctx || !g || !max_color) return GC_ERR_INVALID;
    if (!g->has_colors) return gc_fail(ctx, GC_ERR_STATE, "no coloring to validate");
    DeviceGuard dg(ctx);
    return gc_validate_device(g, max_color);
}

gc_status gc_upload_colors(gc_ctx *ctx, gc_graph *g, const int32_t *color) {
    if (!ctx || !g || (g->N && !color)) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_status s;
    if (g->N && (s = gc_check_cuda(ctx, cudaMemcpyAsync(g->color, color, sizeof(int32_t) * g->N, cudaMemcpyHostToDevice,
                                                        ctx->stream), "upload colors")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "upload colors")) != GC_OK) return s;
    g->has_colors = true;
    g->colors_ours = false;
    return GC_OK;
}

gc_status gc_download_colors(gc_ctx *ctx, gc_graph *g, int32_t *color) {
    if (!ctx || !g || (g->N && !color)) return GC_ERR_INVALID;
    if (!g->has_colors) return gc_fail(ctx, GC_ERR_STATE, "no coloring computed");
    DeviceGuard dg(ctx);
    gc_status s;
    if (g->N && (s = gc_check_cuda(ctx, cudaMemcpyAsync(color, g->color, sizeof(int32_t) * g->N, cudaMemcpyDeviceToHost,
                                                        ctx->stream), "download colors")) != GC_OK)
        return s;
    return gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "download colors");
}

gc_status gc_download_priority(gc_ctx *ctx, gc_graph *g, double *p) {
    if (!ctx || !g || (g->N && !p)) return GC_ERR_INVALID;
    if (!g->has_keys) return gc_fail(ctx, GC_ERR_STATE, "no priorities computed");
    DeviceGuard dg(ctx);
    const uint32_t N = g->N;
    if (g->key_kind == 200) {
        memcpy(p, g->user_p.data(), sizeof(double) * N);
        return GC_OK;
    }
    if (N == 0) return GC_OK;
    // widen on the device, then one copy into the caller's buffer
    gc_status s;
    if ((s = gc_alloc(ctx, &g->p64, (size_t)g->cap_N, "priority staging")) != GC_OK) return s;
    k_keys_to_double<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->key, N, g->key_kind == GC_GNN ? 1 : 0, g->p64);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "priority widening")) != GC_OK) return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(p, g->p64, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->stream),
                           "download priorities")) != GC_OK)
        return s;
    return gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "download priorities");
}

gc_status gc_download_priority_begin(gc_ctx *ctx, gc_graph *g, double *p, int *pending) {
    if (!ctx || !g || !pending || (g->N && !p)) return GC_ERR_INVALID;
    *pending = 0;
    if (!g->has_keys) return gc_fail(ctx, GC_ERR_STATE, "no priorities computed");
    if (g->key_kind == 200 || g->N == 0 || ctx->pool || !gc_is_pinned(p)) return gc_download_priority(ctx, g, p);
    DeviceGuard dg(ctx);
    gc_status s;
    if ((s = gc_copy_stream(ctx)) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->p64, (size_t)g->cap_N, "priority staging")) != GC_OK) return s;
    k_keys_to_double<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->key, g->N, g->key_kind == GC_GNN ? 1 : 0, g->p64);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "priority widening")) != GC_OK) return s;
    if ((s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_copy_fence, ctx->stream), "download priorities")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_copy_fence, 0), "download priorities")) !=
        GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(p, g->p64, sizeof(double) * g->N, cudaMemcpyDeviceToHost,
                                                ctx->copy_stream), "download priorities")) != GC_OK)
        return s;
    *pending = 1;
    return GC_OK;
}

gc_status gc_download_priority_wait(gc_ctx *ctx) {
    if (!ctx) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    return ctx->copy_stream ? gc_check_cuda(ctx, cudaStreamSynchronize(ctx->copy_stream), "download priorities")
                            : GC_OK;
}

}  // extern "C"
