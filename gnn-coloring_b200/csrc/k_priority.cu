// Integer priority heuristics on the device.
//
//   FF  key = N - u                      (reference src/first_fit.c:8-12)
//   LF  key = deg(u)                     (src/largest_degree_first.c:12-16)
//   LLF key = 32 - clz(deg), 0 if deg=0  (src/largest_degree_first.c:87-97)
//   SL / SLL  bucket peeling             (src/smallest_degree_last.c:155-246, :359-443)
//
// Keys are uint32; the coloring orders vertices by (key, id) descending, exactly like the
// reference's double comparisons on these integer-valued priorities.
#include "gc_internal.h"

namespace {
using gc::ld_stream;

// FF in a segmented CSR: N - u with the graph's own N and local u, i.e. (end of u's graph) - u.
__global__ void k_simple_keys(const uint32_t *__restrict__ V, uint32_t N, int h, const uint32_t *__restrict__ voff,
                              uint32_t nseg, uint32_t *__restrict__ key) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        uint32_t k;
        if (h == GC_FF) {
            k = (nseg ? __ldg(voff + gc::seg_of(voff, nseg, u) + 1) : N) - u;
        } else {
            uint32_t d = V[u + 1] - V[u];
            k = (h == GC_LF) ? d : (d ? 32u - (uint32_t)__clz(d) : 0u);
        }
        key[u] = k;
    }
}

// ---- bucket peeling -----------------------------------------------------------------------------
//
// Round r removes every remaining vertex whose remaining degree is <= threshold (delta for SL,
// 2^delta for SLL), gives it key = delta, and takes one degree off each remaining neighbour per
// removed neighbour.  SL then sets delta = max(delta + 1, smallest remaining degree); SLL sets
// delta + 1.  Removal within a round depends only on the degrees at the round's start and the
// decrements commute, so the keys equal the reference's at any thread count.
//
// Round state lives on the device so that rounds can be queued without host round trips:
// kernels of a round that finds nothing left to do return immediately.
struct PeelState {
    unsigned int alive;      // vertices still in the graph
    unsigned int next;       // survivors appended this round
    unsigned int removed;    // vertices removed this round
    unsigned int delta;
    unsigned int min_deg;    // smallest survivor degree after this round's decrements
    unsigned int parity;     // which alive buffer is current
    unsigned int rounds;
    unsigned int log_mode;
};

constexpr uint32_t NOT_REMOVED = 0xffffffffu;

__global__ void k_peel_init(const uint32_t *__restrict__ V, uint32_t N, uint32_t *__restrict__ deg,
                            uint32_t *__restrict__ alive, uint32_t *__restrict__ key, PeelState *ps) {
    uint32_t local_min = 0xffffffffu;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        uint32_t d = V[u + 1] - V[u];
        deg[u] = d;
        alive[u] = u;
        key[u] = NOT_REMOVED;
        local_min = min(local_min, d);
    }
    local_min = __reduce_min_sync(0xffffffffu, local_min);
    if ((threadIdx.x & 31) == 0) atomicMin(&ps->min_deg, local_min);
}

__global__ void k_peel_start(PeelState *ps, uint32_t N, int log_mode) {
    // first threshold from the smallest degree
    uint32_t m = ps->min_deg;
    uint32_t delta = 0;
    if (log_mode) {
        while (delta < 32 && (1ull << delta) < (unsigned long long)m) delta++;
    } else {
        delta = m;
    }
    ps->alive = N;
    ps->next = 0;
    ps->removed = 0;
    ps->delta = delta;
    ps->min_deg = 0xffffffffu;
    ps->parity = 0;
    ps->rounds = 0;
    ps->log_mode = log_mode;
}

// Split the alive list into survivors and removed vertices.
__global__ void k_peel_filter(uint32_t *__restrict__ alive0, uint32_t *__restrict__ alive1,
                              uint32_t *__restrict__ removed, const uint32_t *__restrict__ deg,
                              uint32_t *__restrict__ key, PeelState *ps) {
    const uint32_t n = ps->alive;
    if (n == 0) return;
    const uint32_t delta = ps->delta;
    const unsigned long long thr = ps->log_mode ? (1ull << delta) : (unsigned long long)delta;
    const uint32_t *cur = ps->parity ? alive1 : alive0;
    uint32_t *nxt = ps->parity ? alive0 : alive1;
    const int lane = threadIdx.x & 31;
    uint32_t local_min = 0xffffffffu;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        uint32_t i = base + threadIdx.x;
        bool valid = i < n;
        uint32_t u = valid ? cur[i] : 0;
        uint32_t d = valid ? deg[u] : 0;
        bool rm = valid && (unsigned long long)d <= thr;
        bool keep = valid && !rm;
        if (rm) key[u] = delta;
        if (keep) local_min = min(local_min, d);
        // warp-aggregated appends
        unsigned int mrm = __ballot_sync(0xffffffffu, rm), mkeep = __ballot_sync(0xffffffffu, keep);
        unsigned int brm = 0, bkeep = 0;
        if (lane == 0) {
            if (mrm) brm = atomicAdd(&ps->removed, __popc(mrm));
            if (mkeep) bkeep = atomicAdd(&ps->next, __popc(mkeep));
        }
        brm = __shfl_sync(0xffffffffu, brm, 0);
        bkeep = __shfl_sync(0xffffffffu, bkeep, 0);
        unsigned int lt = (1u << lane) - 1u;
        if (rm) removed[brm + __popc(mrm & lt)] = u;
        if (keep) nxt[bkeep + __popc(mkeep & lt)] = u;
    }
    local_min = __reduce_min_sync(0xffffffffu, local_min);
    if (lane == 0 && local_min != 0xffffffffu) atomicMin(&ps->min_deg, local_min);
}

// Each removed vertex takes one degree off every neighbour that is still in the graph.
// One warp per removed vertex; neighbours are read coalesced.
__global__ void k_peel_decrement(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                 const uint32_t *__restrict__ removed, uint32_t *__restrict__ deg,
                                 const uint32_t *__restrict__ key, PeelState *ps) {
    if (ps->alive == 0) return;
    const uint32_t n = ps->removed;
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t local_min = 0xffffffffu;
    for (uint32_t i = warp; i < n; i += nwarps) {
        uint32_t u = removed[i];
        for (uint32_t j = V[u] + lane; j < V[u + 1]; j += 32) {
            uint32_t v = ld_stream(E + j);
            if (key[v] != NOT_REMOVED) continue;  // removed now or earlier
            uint32_t d = atomicSub(&deg[v], 1u) - 1u;
            local_min = min(local_min, d);
        }
    }
    local_min = __reduce_min_sync(0xffffffffu, local_min);
    if (lane == 0 && local_min != 0xffffffffu) atomicMin(&ps->min_deg, local_min);
}

__global__ void k_peel_advance(PeelState *ps) {
    if (ps->alive == 0) return;
    uint32_t delta = ps->delta + 1;
    if (!ps->log_mode && ps->min_deg != 0xffffffffu && ps->min_deg > delta) delta = ps->min_deg;
    ps->delta = delta;
    ps->alive = ps->next;
    ps->next = 0;
    ps->removed = 0;
    ps->min_deg = 0xffffffffu;
    ps->parity ^= 1u;
    ps->rounds++;
}

}  // namespace

gc_status gc_priority_simple(gc_graph *g, gc_heuristic h) {
    gc_ctx *ctx = g->ctx;
    if (g->N == 0) return GC_OK;
    int grid = ctx->num_sms * 4;
    ProfScope ps(ctx, "priority_keys", ctx->stream);
    k_simple_keys<<<grid, 256, 0, ctx->stream>>>(g->V, g->N, (int)h, g->seg_voff, g->n_seg, g->key);
    ctx->launches++;
    return gc_check_launch(ctx, "priority keys");
}

gc_status gc_priority_peel(gc_graph *g, bool log_thresholds) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    const uint32_t N = g->N;
    if (N == 0) return GC_OK;
    if ((s = gc_alloc(ctx, &g->deg_rem, g->cap_N, "peel degrees")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->frontier, g->cap_N, "peel list")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->frontier2, g->cap_N, "peel list")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->removed, g->cap_N + sizeof(PeelState) / 4 + 1, "peel removed list")) != GC_OK)
        return s;
    // the round state sits behind the removed list
    PeelState *ps = reinterpret_cast<PeelState *>(g->removed + g->cap_N);
    PeelState init{};
    init.min_deg = 0xffffffffu;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(ps, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream),
                           "peel state")) != GC_OK)
        return s;
    const int grid = ctx->num_sms * 8;
    k_peel_init<<<grid, 256, 0, ctx->stream>>>(g->V, N, g->deg_rem, g->frontier, g->key, ps);
    k_peel_start<<<1, 1, 0, ctx->stream>>>(ps, N, log_thresholds ? 1 : 0);
    ctx->launches += 2;
    if ((s = gc_check_launch(ctx, "peel init")) != GC_OK) return s;
    // Rounds are queued in batches; a batch past the last round costs only empty launches.
    PeelState host{};
    uint32_t queued = 0;
    uint32_t batch = log_thresholds ? 16 : 32;
    for (;;) {
        ProfScope prof(ctx, "peel_rounds", ctx->stream);
        for (uint32_t r = 0; r < batch; r++) {
            k_peel_filter<<<grid, 256, 0, ctx->stream>>>(g->frontier, g->frontier2, g->removed, g->deg_rem,
                                                        g->key, ps);
            k_peel_decrement<<<grid, 256, 0, ctx->stream>>>(g->V, g->E, g->removed, g->deg_rem, g->key, ps);
            k_peel_advance<<<1, 1, 0, ctx->stream>>>(ps);
            ctx->launches += 3;
        }
        queued += batch;
        if ((s = gc_check_launch(ctx, "peel round")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(&host, ps, sizeof(host), cudaMemcpyDeviceToHost, ctx->stream),
                               "peel state")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "peel rounds")) != GC_OK) return s;
        if (host.alive == 0) break;
        if (queued > 2 * (N + 64)) return gc_fail(ctx, GC_ERR_DEVICE, "peeling did not terminate");
        batch = batch < 256 ? batch * 2 : batch;
    }
    return GC_OK;
}
