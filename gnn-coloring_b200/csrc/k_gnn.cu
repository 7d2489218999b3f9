// GraphSAGE-16 priority inference (reference src/fast_gnn.c, src/gnn.c), bit-identical to the
// reference's FP32 results.
//
// Arithmetic contract, per layer and vertex u (fast_gnn.c:13-243):
//   nb_k   = sum over v in CSR order of x[v][k], sequentially from +0 in FP32   (message_kernel)
//   nb_k  /= (float)deg(u) when deg(u) > 0, IEEE division
//   a      = [nb (16), x[u] (16)]
//   c_j    = b_j; c_j = fma(W[i*16+j], a_i, c_j) for i = 0..31 in order          (dense_kernel)
//   y[u][j]= c_j > 0 ? c_j : +0
// Layer 0 builds a from two per-vertex scalars, 8 copies each (message_kernel_input :49-89):
//   deg(v)/md and (float)((double)v/(double)N); md is the model file's normaliser.
// The last layer sums its 16 outputs as t_k = o_k + o_{k+8}, then
//   ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7))                                  (dense_kernel_output)
// and the key is that float's bit pattern (the sum is >= +0, so bit order = value order).
//
// Mapping: lane = feature.  A half-warp owns one regular vertex: it loads 16 neighbour ids at
// a time, then 16 neighbour rows (64 B each, coalesced), then adds them in CSR order.  Vertices
// with more than GC_GNN_HUB_DEGREE neighbours get a whole CTA that streams neighbour rows into
// shared memory with cp.async while one half-warp runs the sequential FP32 chain; those CTAs run
// on a second stream so the long chains overlap the bulk of the layer.
//
// Compiled without fast-math; every add, divide and FMA is an explicit round-to-nearest
// intrinsic so the compiler cannot contract or reassociate them.
#include "gc_internal.h"

namespace {
using namespace gc;

enum : int { MODE_INPUT = 0, MODE_HIDDEN = 1, MODE_OUTPUT = 2 };

__global__ void k_gnn_table0(const uint32_t *__restrict__ V, uint32_t N, float fmd, float2 *__restrict__ t01) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        uint32_t d = V[u + 1] - V[u];
        float deg_feat = __fdiv_rn(__uint2float_rn(d), fmd);
        float id_feat = __double2float_rn(__ddiv_rn((double)u, (double)N));
        t01[u] = make_float2(deg_feat, id_feat);
    }
}

// Dense 32x16 + ReLU for the half-warp's vertex; lane j returns output j.
// nb / self are this lane's feature values (hidden layers) or the four layer-0 scalars.
template <int MODE>
__device__ __forceinline__ float dense_relu(const float (&w)[32], float bias, float nb, float self, float s0,
                                            float s1, float self0, float self1, unsigned int hmask) {
    float c = bias;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        float a;
        if (MODE == MODE_INPUT) {
            a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self0 : self1));
        } else {
            a = __shfl_sync(hmask, i < 16 ? nb : self, i & 15, 16);
        }
        c = __fmaf_rn(w[i], a, c);
    }
    return c > 0.0f ? c : 0.0f;
}

// Fixed-tree sum of the 16 outputs held by lanes 0..15 of a half-warp; valid in lane 0.
__device__ __forceinline__ float output_tree(float o, unsigned int hmask) {
    float t = __fadd_rn(o, __shfl_down_sync(hmask, o, 8, 16));   // t_k = o_k + o_{k+8}, lanes 0..7
    float q = __fadd_rn(t, __shfl_down_sync(hmask, t, 1, 16));   // t0+t1, t2+t3, t4+t5, t6+t7
    float r = __fadd_rn(q, __shfl_down_sync(hmask, q, 2, 16));   // (t0+t1)+(t2+t3), (t4+t5)+(t6+t7)
    return __fadd_rn(r, __shfl_down_sync(hmask, r, 4, 16));      // lane 0: the whole sum
}

template <int MODE>
__global__ void __launch_bounds__(256) k_gnn_layer(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                   uint32_t N, const float2 *__restrict__ t01,
                                                   const float *__restrict__ x, float *__restrict__ y,
                                                   uint32_t *__restrict__ key, const float *__restrict__ Wb,
                                                   uint32_t hub_deg) {
    __shared__ float sW[LAYER_PARAMS];
    for (int i = threadIdx.x; i < LAYER_PARAMS; i += blockDim.x) sW[i] = Wb[i];
    __syncthreads();
    const int lane = threadIdx.x & 15;
    const unsigned int hmask = 0xffffu << (threadIdx.x & 16);
    float w[32];
#pragma unroll
    for (int i = 0; i < 32; i++) w[i] = sW[i * FEAT + lane];
    const float bias = sW[2 * FEAT * FEAT + lane];

    const uint32_t groups = (gridDim.x * blockDim.x) >> 4;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; u < N; u += groups) {
        const uint32_t beg = V[u], end = V[u + 1], d = end - beg;
        if (d > hub_deg) continue;  // hub CTAs own this vertex
        const float fd = __uint2float_rn(d);
        float out;
        if (MODE == MODE_INPUT) {
            float s0 = 0.0f, s1 = 0.0f;
            for (uint32_t b = beg; b < end; b += 16) {
                const uint32_t cnt = min(16u, end - b);
                float2 t = make_float2(0.0f, 0.0f);
                if ((uint32_t)lane < cnt) t = t01[ld_stream(E + b + lane)];
#pragma unroll
                for (uint32_t k = 0; k < 16; k++) {
                    float a0 = __shfl_sync(hmask, t.x, k, 16);
                    float a1 = __shfl_sync(hmask, t.y, k, 16);
                    if (k < cnt) {
                        s0 = __fadd_rn(s0, a0);
                        s1 = __fadd_rn(s1, a1);
                    }
                }
            }
            if (fd > 0.0f) {
                s0 = __fdiv_rn(s0, fd);
                s1 = __fdiv_rn(s1, fd);
            }
            const float2 self = t01[u];
            out = dense_relu<MODE_INPUT>(w, bias, 0.0f, 0.0f, s0, s1, self.x, self.y, hmask);
        } else {
            float s = 0.0f;
            for (uint32_t b = beg; b < end; b += 16) {
                const uint32_t cnt = min(16u, end - b);
                uint32_t e = (uint32_t)lane < cnt ? ld_stream(E + b + lane) : 0u;
                float vals[16];
#pragma unroll
                for (uint32_t k = 0; k < 16; k++) {
                    uint32_t v = __shfl_sync(hmask, e, k, 16);
                    vals[k] = k < cnt ? x[(size_t)v * FEAT + lane] : 0.0f;
                }
#pragma unroll
                for (uint32_t k = 0; k < 16; k++)
                    if (k < cnt) s = __fadd_rn(s, vals[k]);
            }
            if (fd > 0.0f) s = __fdiv_rn(s, fd);
            const float self = x[(size_t)u * FEAT + lane];
            out = dense_relu<MODE>(w, bias, s, self, 0.0f, 0.0f, 0.0f, 0.0f, hmask);
        }
        if (MODE == MODE_OUTPUT) {
            float sum = output_tree(out, hmask);
            if (lane == 0) key[u] = __float_as_uint(sum);
        } else {
            y[(size_t)u * FEAT + lane] = out;
        }
    }
}

// ---- hub vertices: one CTA each --------------------------------------------------------------

constexpr int HUB_THREADS = 256;
constexpr int HUB_ROWS = 256;  // neighbour rows per pipeline stage
constexpr int HUB_STAGES = 4;

__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
    unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
    unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(HUB_THREADS) k_gnn_hub(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                         uint32_t N, const uint32_t *__restrict__ hubs,
                                                         const float2 *__restrict__ t01, const float *__restrict__ x,
                                                         float *__restrict__ y, uint32_t *__restrict__ key,
                                                         const float *__restrict__ Wb) {
    // stage buffers: hidden rows are 16 floats, input rows 2 floats (deg/md, id/N)
    constexpr int ROW = (MODE == MODE_INPUT) ? 2 : FEAT;
    extern __shared__ __align__(16) float smem[];
    float *stage = smem;  // HUB_STAGES * HUB_ROWS * ROW floats
    const uint32_t u = hubs[blockIdx.x];
    const uint32_t beg = V[u], end = V[u + 1], d = end - beg;
    const uint32_t nchunks = (d + HUB_ROWS - 1) / HUB_ROWS;
    const int tid = threadIdx.x;

    auto issue = [&](uint32_t c) {
        if (c < nchunks) {
            uint32_t i = beg + c * HUB_ROWS + tid;
            float *dst = stage + (size_t)(c % HUB_STAGES) * HUB_ROWS * ROW + (size_t)tid * ROW;
            if (i < end) {
                uint32_t v = ld_stream(E + i);
                if (MODE == MODE_INPUT) {
                    cp_async_8(dst, t01 + v);
                } else {
                    const float *src = x + (size_t)v * FEAT;
#pragma unroll
                    for (int q = 0; q < 4; q++) cp_async_16(dst + 4 * q, src + 4 * q);
                }
            }
        }
        cp_async_commit();  // empty groups keep the group count uniform
    };

    for (int c = 0; c < HUB_STAGES - 1; c++) issue(c);
    float s = 0.0f, s1 = 0.0f;  // feature chain (lane), and the second layer-0 chain
    const int lane = tid & 31;
    for (uint32_t c = 0; c < nchunks; c++) {
        issue(c + HUB_STAGES - 1);
        cp_async_wait<HUB_STAGES - 1>();
        __syncthreads();
        if (tid < 16) {
            const float *buf = stage + (size_t)(c % HUB_STAGES) * HUB_ROWS * ROW;
            const uint32_t cnt = min((uint32_t)HUB_ROWS, end - (beg + c * HUB_ROWS));
            if (MODE == MODE_INPUT) {
                // lane 0 sums deg/md, lane 1 sums id/N
                if (lane < 2)
                    for (uint32_t r = 0; r < cnt; r++) s = __fadd_rn(s, buf[2 * r + lane]);
            } else {
                for (uint32_t r = 0; r < cnt; r++) s = __fadd_rn(s, buf[r * FEAT + lane]);
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    if (tid >= 16) return;
    (void)s1;
    const unsigned int hmask = 0xffffu;
    __shared__ float sW[LAYER_PARAMS];
    for (int i = tid; i < LAYER_PARAMS; i += 16) sW[i] = Wb[i];
    __syncwarp(hmask);
    float w[32];
#pragma unroll
    for (int i = 0; i < 32; i++) w[i] = sW[i * FEAT + lane];
    const float bias = sW[2 * FEAT * FEAT + lane];
    const float fd = __uint2float_rn(d);
    float out;
    if (MODE == MODE_INPUT) {
        float s0 = __shfl_sync(hmask, s, 0, 16), sid = __shfl_sync(hmask, s, 1, 16);
        if (fd > 0.0f) {
            s0 = __fdiv_rn(s0, fd);
            sid = __fdiv_rn(sid, fd);
        }
        const float2 self = t01[u];
        out = dense_relu<MODE_INPUT>(w, bias, 0.0f, 0.0f, s0, sid, self.x, self.y, hmask);
    } else {
        if (fd > 0.0f) s = __fdiv_rn(s, fd);
        const float self = x[(size_t)u * FEAT + lane];
        out = dense_relu<MODE>(w, bias, s, self, 0.0f, 0.0f, 0.0f, 0.0f, hmask);
    }
    if (MODE == MODE_OUTPUT) {
        float sum = output_tree(out, hmask);
        if (lane == 0) key[u] = __float_as_uint(sum);
    } else {
        y[(size_t)u * FEAT + lane] = out;
    }
}

template <int MODE>
gc_status launch_layer(gc_graph *g, const float *Wb, const float *x, float *y, cudaStream_t side,
                       cudaEvent_t fork, cudaEvent_t join) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (g->n_hubs) {
        constexpr int ROW = (MODE == MODE_INPUT) ? 2 : FEAT;
        const size_t smem = (size_t)HUB_STAGES * HUB_ROWS * ROW * sizeof(float);
        if ((s = gc_check_cuda(ctx, cudaFuncSetAttribute(k_gnn_hub<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)smem), "hub smem")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventRecord(fork, ctx->stream), "fork")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(side, fork, 0), "fork")) != GC_OK) return s;
        ProfScope ps(ctx, MODE == MODE_INPUT ? "gnn_hub_input" : (MODE == MODE_HIDDEN ? "gnn_hub_hidden" : "gnn_hub_output"),
                     side);
        k_gnn_hub<MODE><<<g->n_hubs, HUB_THREADS, smem, side>>>(g->V, g->E, g->N, g->hubs, g->t01, x, y, g->key, Wb);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "gnn hub layer")) != GC_OK) return s;
    }
    int grid = ctx->num_sms * 8;
    {
        ProfScope ps(ctx, MODE == MODE_INPUT ? "gnn_input" : (MODE == MODE_HIDDEN ? "gnn_hidden" : "gnn_output"),
                     ctx->stream);
        k_gnn_layer<MODE><<<grid, 256, 0, ctx->stream>>>(g->V, g->E, g->N, g->t01, x, y, g->key, Wb, GC_GNN_HUB_DEGREE);
    }
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "gnn layer")) != GC_OK) return s;
    if (g->n_hubs) {
        if ((s = gc_check_cuda(ctx, cudaEventRecord(join, side), "join")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->stream, join, 0), "join")) != GC_OK) return s;
    }
    return GC_OK;
}

}  // namespace

gc_status gc_priority_gnn(gc_graph *g, const gc_model *m) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (!m || m->layers < 2) return gc_fail(ctx, GC_ERR_INVALID, "GNN needs a model with at least 2 layers");
    if (g->N == 0) return GC_OK;
    const size_t rows = (size_t)g->cap_N;
    if ((s = gc_alloc(ctx, &g->x, rows * FEAT, "gnn features")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->y, rows * FEAT, "gnn features")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->t01, rows, "gnn input table")) != GC_OK) return s;
    if (ctx->side_stream == nullptr) {
        if ((s = gc_check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking), "stream")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
    }
    {
        ProfScope ps(ctx, "gnn_table0", ctx->stream);
        k_gnn_table0<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, (float)m->md, g->t01);
    }
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "gnn input table")) != GC_OK) return s;
    const int L = m->layers;
    float *x = g->x, *y = g->y;
    for (int l = 0; l < L; l++) {
        const float *Wb = m->d_param + (size_t)l * LAYER_PARAMS;
        if (l == 0)
            s = launch_layer<MODE_INPUT>(g, Wb, nullptr, y, ctx->side_stream, ctx->ev_fork, ctx->ev_join);
        else if (l < L - 1)
            s = launch_layer<MODE_HIDDEN>(g, Wb, x, y, ctx->side_stream, ctx->ev_fork, ctx->ev_join);
        else
            s = launch_layer<MODE_OUTPUT>(g, Wb, x, nullptr, ctx->side_stream, ctx->ev_fork, ctx->ev_join);
        if (s != GC_OK) return s;
        float *t = x;
        x = y;
        y = t;
    }
    return GC_OK;
}
