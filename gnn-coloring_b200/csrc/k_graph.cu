// Per-graph preparation on the device: maximum degree and the degree classes that the
// split and GNN kernels schedule separately.  Depends only on the CSR, so it runs once per
// upload (the reference likewise prepares its CSR before any timed call, src/main.c:106-133).
#include <algorithm>
#include <vector>

#include "gc_internal.h"

namespace {

__global__ void k_degree_classes(const uint32_t *__restrict__ V, uint32_t N, uint32_t big_deg,
                                 uint32_t chunk, uint32_t hub_deg, uint32_t warp_deg, uint32_t gnn_warp_deg,
                                 uint32_t thin_deg, gc::DevState *st,
                                 uint32_t *__restrict__ tasks, uint32_t task_cap,
                                 uint32_t *__restrict__ hubs, uint32_t hub_cap) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < N; base += stride) {
        uint32_t u = base + threadIdx.x;
        uint32_t beg = 0, d = 0;
        if (u < N) {
            beg = V[u];
            d = V[u + 1] - beg;
        }
        uint32_t wmax = __reduce_max_sync(0xffffffffu, d);
        if ((threadIdx.x & 31) == 0 && wmax) atomicMax(&st->max_color, wmax);
        if (u >= N) continue;
        if (d > big_deg) {
            uint32_t nt = (d + chunk - 1) / chunk;
            uint32_t at = atomicAdd(&st->count, nt);
            if (tasks)
                for (uint32_t k = 0; k < nt; k++)
                    if (at + k < task_cap) {
                        tasks[2 * (at + k)] = u;
                        tasks[2 * (at + k) + 1] = beg + k * chunk;
                    }
        }
        if (d > hub_deg) {
            uint32_t at = atomicAdd(&st->count2, 1u);
            if (hubs && at < hub_cap) hubs[at] = u;
        } else if (d > warp_deg) {
            atomicAdd(&st->min_deg, 1u);  // counts the GNN warp tier
        }
        if (d > gnn_warp_deg && d <= hub_deg) atomicAdd(&st->gnn_wide, 1u);  // counts the GNN warp tier
        if (d <= thin_deg && d <= gnn_warp_deg) atomicAdd(&st->thin, 1u);     // counts the GNN thin tier
        if (d == 0) atomicAdd(&st->isolated, 1u);
    }
}

__global__ void k_degree_keys(const uint32_t *__restrict__ V, uint32_t N, uint32_t *__restrict__ out) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
        out[u] = V[u + 1] - V[u];
}

// Graph-major schedule keys: the warp tier first, then graph by graph (in order), then degree class
// (bit length of the degree) descending.  The sort's ascending-id tie rule keeps each graph's
// vertices of one class in id order.
__global__ void k_segment_keys(const uint32_t *__restrict__ V, uint32_t N, const uint32_t *__restrict__ voff,
                               uint32_t nseg, uint32_t warp_deg, uint32_t *__restrict__ out) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t d = V[u + 1] - V[u];
        const uint32_t s = nseg ? gc::seg_of(voff, nseg, u) : 0u;
        const uint32_t cls = d ? 32u - (uint32_t)__clz(d) : 0u;  // 0 .. 32
        const uint32_t rank = (nseg ? nseg - 1u - s : 0u);      // earlier graphs get larger keys
        out[u] = (d > warp_deg ? 0x80000000u : 0u) | (rank << 6) | cls;
    }
}

int bits_of(uint32_t x) {
    int b = 0;
    while (x) {
        b++;
        x >>= 1;
    }
    return b;
}

__global__ void k_hub_degrees(const uint32_t *__restrict__ V, const uint32_t *__restrict__ hubs, uint32_t n,
                              uint32_t *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t u = hubs[i];
        out[2 * i] = u;
        out[2 * i + 1] = V[u + 1] - V[u];
    }
}

}  // namespace

gc_status gc_graph_prepare(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    g->rows_ready = false;  // the GNN's feature-row order follows the hub list and the degree order
    if (g->N == 0) {
        g->max_deg = 0;
        g->n_big_tasks = 0;
        g->n_hubs = 0;
        g->n_giant = 0;
        g->giant_rows = 0;
        g->n_vorder = 0;
        g->n_thin = 0;
        g->n_iso = 0;
        g->n_wide_gnn = 0;
        return GC_OK;
    }
    int grid = ctx->num_sms * 8;
    // the GNN keeps its own warp tier only with the degree schedule (the graph-major order puts the
    // split's warp tier first, so there the two tiers coincide)
    const uint32_t gnn_wd = g->sched == GC_SCHEDULE_DEGREE ? std::max(g->gnn_warp_deg, g->warp_deg) : g->warp_deg;
    // pass 1: counts
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    k_degree_classes<<<grid, 256, 0, ctx->stream>>>(g->V, g->N, g->hub_deg, GC_SPLIT_CHUNK, g->hub_deg,
                                                    g->warp_deg, gnn_wd, ctx->gnn_thin_deg, ctx->dstate, nullptr, 0, nullptr, 0);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "degree classes")) != GC_OK) return s;
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    g->max_deg = ctx->hstate->max_color;
    uint32_t n_tasks = ctx->hstate->count, n_hubs = ctx->hstate->count2;
    g->n_wide = ctx->hstate->min_deg;
    g->n_thin = g->sched == GC_SCHEDULE_DEGREE ? ctx->hstate->thin : 0u;
    g->n_iso = g->sched == GC_SCHEDULE_DEGREE ? ctx->hstate->isolated : 0u;  // the last entries of the degree order
    g->n_wide_gnn = g->sched == GC_SCHEDULE_DEGREE ? ctx->hstate->gnn_wide : g->n_wide;
    // lists: the hub list and the degree order fit in cap_N; the task list grows when needed
    if (2 * (size_t)n_tasks > g->big_cap) {
        gc_dev_free(ctx, g->big);
        g->big = nullptr;
        if ((s = gc_alloc(ctx, &g->big, 2 * (size_t)n_tasks, "split task list")) != GC_OK) return s;
        g->big_cap = 2 * (size_t)n_tasks;
    }
    if ((s = gc_alloc(ctx, &g->hubs, (size_t)g->cap_N, "hub list")) != GC_OK) return s;
    // pass 2: fill
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    k_degree_classes<<<grid, 256, 0, ctx->stream>>>(g->V, g->N, g->hub_deg, GC_SPLIT_CHUNK, g->hub_deg,
                                                    g->warp_deg, gnn_wd, ctx->gnn_thin_deg, ctx->dstate, g->big, n_tasks,
                                                    g->hubs, n_hubs);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "degree classes")) != GC_OK) return s;
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    g->n_big_tasks = n_tasks;
    g->n_hubs = n_hubs;
    // hubs by descending degree, so the longest FP32 add chains start first
    if (n_hubs > 0) {
        // (vertex, degree) pairs of the hubs, sorted on the host by descending degree
        uint32_t *pairs = nullptr;
        if ((s = gc_alloc(ctx, &pairs, 2 * (size_t)n_hubs, "hub degrees")) != GC_OK) return s;
        k_hub_degrees<<<ctx->num_sms, 256, 0, ctx->stream>>>(g->V, g->hubs, n_hubs, pairs);
        ctx->launches++;
        std::vector<uint32_t> hp(2 * (size_t)n_hubs), h(n_hubs);
        s = gc_check_cuda(ctx, cudaMemcpyAsync(hp.data(), pairs, 8 * (size_t)n_hubs, cudaMemcpyDeviceToHost,
                                               ctx->stream), "hub degrees");
        if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "hub degrees");
        gc_dev_free(ctx, pairs);
        if (s != GC_OK) return s;
        std::vector<uint32_t> idx(n_hubs);
        for (uint32_t i = 0; i < n_hubs; i++) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
            uint32_t da = hp[2 * a + 1], db = hp[2 * b + 1];
            return da != db ? da > db : hp[2 * a] < hp[2 * b];
        });
        for (uint32_t i = 0; i < n_hubs; i++) h[i] = hp[2 * idx[i]];
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->hubs, h.data(), 4 * (size_t)n_hubs,
                                                    cudaMemcpyHostToDevice, ctx->stream), "hub list")) != GC_OK)
            return s;
        // giant hubs: at least GC_GIANT_MIN_DEGREE neighbours and a third of the largest degree.  Their
        // rows are staged by the whole GPU before each GNN layer, and their features split over
        // several SMs (k_hub_stage, k_gnn_hubx)
        const uint32_t top = hp[2 * idx[0] + 1];
        const uint32_t giant_deg = std::max<uint32_t>(GC_GIANT_MIN_DEGREE, top / 3);
        std::vector<uint32_t> off(1, 0);
        uint64_t rows = 0;
        for (uint32_t i = 0; i < n_hubs && hp[2 * idx[i] + 1] >= giant_deg; i++) {
            const uint64_t padded = ((uint64_t)hp[2 * idx[i] + 1] + 1023u) & ~(uint64_t)1023u;
            if (rows + padded > GC_GIANT_MAX_ROWS) break;
            rows += padded;
            off.push_back((uint32_t)rows);
        }
        g->n_giant = (uint32_t)off.size() - 1;
        g->giant_rows = (uint32_t)rows;
        gc_dev_free(ctx, g->giant_off);
        g->giant_off = nullptr;
        if (g->n_giant) {
            if ((s = gc_alloc(ctx, &g->giant_off, off.size(), "giant hub offsets")) != GC_OK) return s;
            if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(g->giant_off, off.data(), 4 * off.size(), cudaMemcpyHostToDevice,
                                                        ctx->stream),
                                   "giant hub offsets")) != GC_OK)
                return s;
        }
        if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "hub list")) != GC_OK) return s;
    } else {
        g->n_giant = 0;
        g->giant_rows = 0;
    }
    // GNN schedule.  By degree: every non-hub vertex by descending degree (ties by id), so that the
    // vertices a warp handles together have nearly equal neighbour counts.  Graph-major (segmented
    // CSRs): the warp tier, then graph by graph, by degree class inside, so that one graph's
    // feature rows stay in L2 while its vertices are processed.  The key buffer is free here (no
    // priorities exist right after an upload).
    if ((s = gc_alloc(ctx, &g->vorder, (size_t)g->cap_N, "degree order")) != GC_OK) return s;
    int key_bits;
    if (g->sched == GC_SCHEDULE_SEGMENT) {
        if (g->n_seg >= (1u << 25)) return gc_fail(ctx, GC_ERR_INVALID, "graph-major schedule: too many graphs");
        k_segment_keys<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, g->seg_voff, g->n_seg, g->warp_deg,
                                                                  g->key);
        key_bits = 32;
    } else {
        k_degree_keys<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, g->key);
        const uint32_t top = g->max_deg < g->hub_deg ? g->max_deg : g->hub_deg;
        key_bits = bits_of(top);
    }
    ctx->launches++;
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    if ((s = gc_sort_vertices(g, g->key, key_bits, SORT_KEEP_DEG_AT_MOST, g->hub_deg, g->vorder,
                              &ctx->dstate->count)) != GC_OK)
        return s;
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    g->n_vorder = ctx->hstate->count;
    if (g->n_vorder + g->n_hubs != g->N) return gc_fail(ctx, GC_ERR_DEVICE, "degree order lost vertices");
    return GC_OK;
}
