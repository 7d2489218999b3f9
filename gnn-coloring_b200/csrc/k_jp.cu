// Jones-Plassmann greedy coloring on the device (reference src/coloring.c:223-330).
//
// The reference peels the priority DAG in rounds: a vertex whose predecessors are all colored
// takes the smallest color >= 1 none of them uses.  The colors are a function of (graph,
// priorities) only: color(u) = mex{color(v) : v precedes u}, evaluated in any topological order.
// This file evaluates that recurrence as a dataflow over the whole GPU:
//
//   1. split   - every vertex packs its predecessors (larger key, or equal key and smaller id)
//                at the front of its CSR segment in P and records their number in pc.  This is
//                the reference's E_split pass (coloring.c:241-264); predecessor order inside
//                the segment is irrelevant to the result.
//   2. order   - vertices by descending key, ascending id on ties: a topological order.
//   3. color   - a persistent kernel hands out tickets in that order, one vertex per warp.  The
//                warp gathers its predecessors' colors, waiting (bounded) on any that are still
//                0, builds a forbidden-color bitmap in shared memory and stores the mex.  A warp
//                only ever waits on vertices with smaller tickets, which are held by running warps
//                or done, so the oldest unfinished ticket always progresses.
//
// Colors are published with relaxed GPU-scope stores and read with relaxed GPU-scope loads: the
// color value is itself the whole message, so no fences are needed.
#include "gc_internal.h"

gc_status gc_sort_order_bits(gc_graph *g, int key_bits);
gc_status gc_order_identity(gc_graph *g);

namespace {
using namespace gc;

// Vertices with at most GC_SPLIT_BIG_DEGREE neighbours: one thread each.  Also resets colors.
__global__ void k_jp_split_small(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                 const uint32_t *__restrict__ key, uint32_t N, uint32_t *__restrict__ P,
                                 uint32_t *__restrict__ pc, int *__restrict__ color) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t beg = V[u], end = V[u + 1];
        color[u] = 0;
        if (end - beg > GC_SPLIT_BIG_DEGREE) {
            pc[u] = 0;  // filled by k_jp_split_big
            continue;
        }
        const uint32_t ku = key[u];
        uint32_t w = beg;
        for (uint32_t i = beg; i < end; i++) {
            uint32_t v = ld_stream(E + i);
            if (precedes(key[v], v, ku, u)) P[w++] = v;
        }
        pc[u] = w - beg;
    }
}

// Larger vertices: one warp per GC_SPLIT_CHUNK-edge chunk, slots reserved with atomics.
__global__ void k_jp_split_big(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                               const uint32_t *__restrict__ key, const uint32_t *__restrict__ tasks,
                               uint32_t n_tasks, uint32_t *__restrict__ P, uint32_t *__restrict__ pc) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    for (uint32_t t = warp; t < n_tasks; t += nwarps) {
        const uint32_t u = tasks[2 * t], e0 = tasks[2 * t + 1];
        const uint32_t end = min(V[u + 1], e0 + GC_SPLIT_CHUNK);
        const uint32_t ku = key[u], beg = V[u];
        for (uint32_t i0 = e0; i0 < end; i0 += 32) {
            const uint32_t i = i0 + lane;
            bool is_pred = false;
            uint32_t v = 0;
            if (i < end) {
                v = ld_stream(E + i);
                is_pred = precedes(key[v], v, ku, u);
            }
            unsigned int m = __ballot_sync(0xffffffffu, is_pred);
            if (!m) continue;
            uint32_t slot = 0;
            if (lane == 0) slot = atomicAdd(&pc[u], (uint32_t)__popc(m));
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (is_pred) P[beg + slot + __popc(m & lt)] = v;
        }
    }
}

constexpr int COLOR_THREADS = 256;
constexpr int COLOR_WARPS = COLOR_THREADS / 32;
constexpr uint32_t WINDOW = 1024;  // colors covered by one pass over the predecessors

__global__ void __launch_bounds__(COLOR_THREADS) k_jp_color(const uint32_t *__restrict__ V, const uint32_t *__restrict__ P,
                                                            const uint32_t *__restrict__ pc,
                                                            const uint32_t *__restrict__ order, uint32_t n,
                                                            int *color, DevState *st, unsigned int spin_limit) {
    __shared__ uint32_t forbid[COLOR_WARPS][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *fb = forbid[warp];
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&st->ticket, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n) break;
        const uint32_t u = order[t];
        const uint32_t base = V[u], cnt = pc[u];
        int result = 1;
        if (cnt) {
            for (uint32_t window = 0;; window++) {
                fb[lane] = 0;
                __syncwarp();
                bool gave_up = false;
                for (uint32_t j = lane; j < cnt; j += 32) {
                    const uint32_t v = P[base + j];
                    int c = ld_relaxed(color + v);
                    uint32_t spins = 0;
                    while (c == 0) {
                        ++spins;
                        if (spins > spin_limit || ((spins & 1023u) == 0 && ld_relaxed_u32(&st->err))) {
                            gave_up = true;
                            break;
                        }
                        if (spins > 256) __nanosleep(128);
                        c = ld_relaxed(color + v);
                    }
                    if (gave_up) break;
                    const uint32_t idx = (uint32_t)(c - 1) - window * WINDOW;
                    if (idx < WINDOW) atomicOr(&fb[idx >> 5], 1u << (idx & 31));
                }
                if (__any_sync(0xffffffffu, gave_up)) {
                    if (lane == 0) raise_error(st, ERR_WAIT_EXPIRED, u);
                    result = -1;  // non-zero, so successors stop waiting; the host reports the error
                    break;
                }
                __syncwarp();
                const uint32_t free_bits = ~fb[lane];
                const unsigned int has = __ballot_sync(0xffffffffu, free_bits != 0);
                if (has) {
                    const int l = __ffs(has) - 1;
                    const uint32_t fw = __shfl_sync(0xffffffffu, free_bits, l);
                    result = (int)(window * WINDOW + (uint32_t)l * 32 + (uint32_t)(__ffs(fw) - 1) + 1);
                    break;
                }
                __syncwarp();
            }
        }
        if (lane == 0) st_relaxed(color + u, result);
        __syncwarp();
    }
}

// One warp per vertex: colors positive and no monochrome edge; largest color.
__global__ void k_validate(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E, uint32_t N,
                           const int *__restrict__ color, DevState *st) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    int cmax = 0;
    bool bad = false;
    for (uint32_t u = warp; u < N; u += nwarps) {
        const int cu = color[u];
        if (cu <= 0) bad = true;
        if (cu > cmax) cmax = cu;
        for (uint32_t j = V[u] + lane; j < V[u + 1]; j += 32)
            if (color[ld_stream(E + j)] == cu) bad = true;
    }
    bad = __any_sync(0xffffffffu, bad);
    cmax = __reduce_max_sync(0xffffffffu, cmax);
    if (lane == 0) {
        if (bad) atomicOr(&st->invalid, 1u);
        atomicMax(&st->max_color, (unsigned int)cmax);
    }
}

__global__ void k_keys_from_colors(const int *__restrict__ color, uint32_t N, uint32_t *__restrict__ key) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
        key[u] = (uint32_t)color[u];
}

__global__ void k_reset_ticket(DevState *st) { st->ticket = 0; }

int bit_length(uint64_t x) {
    int b = 0;
    while (x) {
        b++;
        x >>= 1;
    }
    return b;
}

}  // namespace

gc_status gc_jp_color(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    const uint32_t N = g->N;
    if (N == 0) return GC_OK;
    if ((s = gc_alloc(ctx, &g->P, g->cap_M, "predecessor lists")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->pc, g->cap_N, "predecessor counts")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->order, g->cap_N, "ticket order")) != GC_OK) return s;

    // 1. split
    k_jp_split_small<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->V, g->E, g->key, N, g->P, g->pc, g->color);
    ctx->launches++;
    if (g->n_big_tasks) {
        k_jp_split_big<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->V, g->E, g->key, g->big, g->n_big_tasks, g->P, g->pc);
        ctx->launches++;
    }
    if ((s = gc_check_launch(ctx, "jp split")) != GC_OK) return s;

    // 2. ticket order
    if (g->key_kind == GC_FF) {
        s = gc_order_identity(g);  // key = N - u: descending key is ascending id
    } else {
        int bits = 32;
        if (g->key_kind == GC_LF || g->key_kind == GC_SL) bits = bit_length(g->max_deg);
        else if (g->key_kind == GC_LLF || g->key_kind == GC_SLL) bits = 6;
        else if (g->key_kind == 100) bits = bit_length((uint64_t)g->max_deg + 1);
        s = gc_sort_order_bits(g, bits);
    }
    if (s != GC_OK) return s;

    // 3. ordered coloring
    int &blocks_per_sm = ctx->color_blocks_per_sm;
    if (!blocks_per_sm) {
        if ((s = gc_check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_jp_color,
                                                                                  COLOR_THREADS, 0),
                               "occupancy")) != GC_OK)
            return s;
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    k_reset_ticket<<<1, 1, 0, ctx->stream>>>(ctx->dstate);
    k_jp_color<<<ctx->num_sms * blocks_per_sm, COLOR_THREADS, 0, ctx->stream>>>(g->V, g->P, g->pc, g->order, N, g->color,
                                                                                ctx->dstate, ctx->spin_limit);
    ctx->launches += 2;
    if ((s = gc_check_launch(ctx, "jp color")) != GC_OK) return s;
    g->has_colors = true;
    return GC_OK;
}

gc_status gc_keys_from_colors(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    if (g->N == 0) return GC_OK;
    k_keys_from_colors<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->color, g->N, g->key);
    ctx->launches++;
    g->key_kind = 100;
    return gc_check_launch(ctx, "culberson keys");
}

gc_status gc_validate_device(gc_graph *g, int *max_color) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (g->N == 0) {
        *max_color = 1;  // the reference's validate_coloring_par starts from C = 1
        return GC_OK;
    }
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    k_validate<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->V, g->E, g->N, g->color, ctx->dstate);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "validate")) != GC_OK) return s;
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    int C = (int)ctx->hstate->max_color;
    if (C < 1) C = 1;
    *max_color = ctx->hstate->invalid ? 0 : C;
    return GC_OK;
}
