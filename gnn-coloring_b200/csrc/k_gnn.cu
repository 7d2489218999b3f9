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
// Mapping, by degree (the degree order built at upload):
//   - thin tier (at most 16 neighbours): one vertex per lane;
//   - quad tier: four lanes per vertex, a float4 of the row each, eight vertices per warp;
//   - warp tier (more than GC_GNN_WIDE_DEGREE neighbours): a warp per vertex, rows staged in
//     shared memory;
//   - hubs (more than GC_GNN_HUB_DEGREE): a CTA per hub that streams neighbour rows into shared
//     memory with cp.async while one thread per feature runs the sequential FP32 chain; the
//     largest hubs read rows that k_gnn_hub_gather first copies into a contiguous buffer.  Hub
//     CTAs run on a second stream, so the long chains overlap the bulk of the layer, and each
//     giant hub's CTA gets an SM of its own (the bulk CTAs leave the first SMs to them).
// Neighbour rows are read with __ldg: a layer never writes the features it reads.  In an A/B on
// R-MAT 22 (GNN3) the explicit read-only load made the bulk hidden and output layers about 6 %
// faster than the plain loads the compiler emits here; the step time did not change, since the
// hub chains bound each layer.
//
// Compiled without fast-math; every add, divide and FMA is an explicit round-to-nearest
// intrinsic so the compiler cannot contract or reassociate them.
#include <algorithm>

#include "gc_internal.h"

namespace {
using namespace gc;

enum : int { MODE_INPUT = 0, MODE_HIDDEN = 1, MODE_OUTPUT = 2 };

// In a segmented CSR the id feature is (local id) / (the graph's own N).
__global__ void k_gnn_table0(const uint32_t *__restrict__ V, uint32_t N, float fmd, const uint32_t *__restrict__ voff,
                             uint32_t nseg, float2 *__restrict__ t01) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        uint32_t d = V[u + 1] - V[u];
        uint32_t base = 0, n = N;
        if (nseg) {
            const uint32_t s = seg_of(voff, nseg, u);
            base = __ldg(voff + s);
            n = __ldg(voff + s + 1) - base;
        }
        float deg_feat = __fdiv_rn(__uint2float_rn(d), fmd);
        float id_feat = __double2float_rn(__ddiv_rn((double)(u - base), (double)n));
        t01[u] = make_float2(deg_feat, id_feat);
    }
}

// ---- shared pieces: four lanes per vertex, lane q owns features 4q..4q+3 ---------------------

constexpr unsigned int FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t sm_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// Bulk work handed out by an atomic counter, n items per warp at a time (used when some SMs are
// left to the giant-hub CTAs, so that the CTAs that do start cover all the work; the sizes are the
// context's gnn_grab and gnn_heavy).
__device__ __forceinline__ uint32_t grab_work(uint32_t *ctr, uint32_t n, int lane) {
    uint32_t b = 0;
    if (lane == 0) b = atomicAdd(ctr, n);
    return __shfl_sync(0xffffffffu, b, 0);
}

__device__ __forceinline__ float4 add4(float4 s, float4 r) {
    return make_float4(__fadd_rn(s.x, r.x), __fadd_rn(s.y, r.y), __fadd_rn(s.z, r.z), __fadd_rn(s.w, r.w));
}
__device__ __forceinline__ float comp(const float4 &v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w)); }
__device__ __forceinline__ float relu(float c) { return c > 0.0f ? c : 0.0f; }

// Dense 32x16 + ReLU for the quad's vertex.  Input feature i is a_i; lane q returns outputs
// 4q..4q+3.  For hidden/output layers a_i (i < 16: neighbour mean, else own row) is held by quad
// lane (i & 15) >> 2 as component i & 3, and is broadcast with a shuffle; for the input layer the
// four scalars are already in every lane.  Each output accumulates i = 0..31 in order with FMA.
template <int MODE>
__device__ __forceinline__ float4 dense_quad(const float4 *__restrict__ W4, float4 b4, int q, int qbase,
                                             unsigned int mask, float4 nb, float4 self, float s0, float s1,
                                             float self0, float self1) {
    float c0 = b4.x, c1 = b4.y, c2 = b4.z, c3 = b4.w;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        float a;
        if (MODE == MODE_INPUT) {
            a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self0 : self1));
        } else {
            const float mine = comp(i < 16 ? nb : self, i & 3);
            a = __shfl_sync(mask, mine, qbase + ((i & 15) >> 2));
        }
        const float4 w = W4[i * 4 + q];
        c0 = __fmaf_rn(w.x, a, c0);
        c1 = __fmaf_rn(w.y, a, c1);
        c2 = __fmaf_rn(w.z, a, c2);
        c3 = __fmaf_rn(w.w, a, c3);
    }
    return make_float4(relu(c0), relu(c1), relu(c2), relu(c3));
}

// The reference's output sum (dense_kernel_output :223-242) over the quad's 16 outputs:
// t_k = o_k + o_{k+8}, then ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7)).  Valid in quad lane 0.
__device__ __forceinline__ float output_sum(float4 o, unsigned int mask) {
    const float p0 = __shfl_down_sync(mask, o.x, 2, 4), p1 = __shfl_down_sync(mask, o.y, 2, 4);
    const float p2 = __shfl_down_sync(mask, o.z, 2, 4), p3 = __shfl_down_sync(mask, o.w, 2, 4);
    // lanes 0 and 1 of the quad now hold t_{4q..4q+3}
    const float t0 = __fadd_rn(o.x, p0), t1 = __fadd_rn(o.y, p1), t2 = __fadd_rn(o.z, p2), t3 = __fadd_rn(o.w, p3);
    const float h = __fadd_rn(__fadd_rn(t0, t1), __fadd_rn(t2, t3));
    return __fadd_rn(h, __shfl_down_sync(mask, h, 1, 4));
}

// ---- regular vertices: 8 per warp, taken from the degree order --------------------------------

constexpr int GNN_THREADS = 256;

// Warp tier: one vertex of up to GC_GNN_HUB_DEGREE neighbours per warp.  All 32 lanes fetch 32
// neighbour rows per step (one id each, then one float4 per lane for 8 rows at a time), stage
// them in the warp's shared-memory slab, and lanes 0..15 add them in CSR order, one feature each.
template <int MODE>
__device__ __forceinline__ void warp_vertex(uint32_t u, const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                            const float2 *__restrict__ t01, const float *__restrict__ x, float *__restrict__ y,
                                            uint32_t *__restrict__ key, const float4 *W4, const float *sW, float *slab,
                                            int lane) {
    const uint32_t beg = V[u], d = V[u + 1] - beg;
    const float fd = __uint2float_rn(d);
    const int q = lane & 3;
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float s = 0.0f, s1 = 0.0f;  // lane l < 16: feature l (input layer: lane 0 sums deg/md, lane 1 id/N)
    uint32_t nxt = lane < d ? ld_stream(E + beg + lane) : 0u;  // ids one step ahead
    for (uint32_t c = 0; c < d; c += 32) {
        const uint32_t e = nxt;
        nxt = c + 32 + lane < d ? ld_stream(E + beg + c + 32 + lane) : 0u;
        if (MODE == MODE_INPUT) {
            const float2 t = c + lane < d ? __ldg(t01 + e) : make_float2(0.0f, 0.0f);
            reinterpret_cast<float2 *>(slab)[lane] = t;
            __syncwarp();
            const uint32_t cnt = min(32u, d - c);
            if (lane < 2)
                for (uint32_t m = 0; m < cnt; m++) s = __fadd_rn(s, slab[2 * m + lane]);
        } else {
            const float4 *X4 = reinterpret_cast<const float4 *>(x);
            float4 r[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int m = j * 8 + (lane >> 2);  // this lane fetches features 4q..4q+3 of row m
                const uint32_t v = __shfl_sync(FULL, e, m);
                r[j] = c + m < d ? __ldg(X4 + (size_t)v * 4 + q) : zero4;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) reinterpret_cast<float4 *>(slab)[(j * 8 + (lane >> 2)) * 4 + q] = r[j];
            __syncwarp();
            const uint32_t cnt = min(32u, d - c);
            if (lane < FEAT) {
                float t[8];
                uint32_t m = 0;
                for (; m + 8 <= cnt; m += 8) {
#pragma unroll
                    for (int k = 0; k < 8; k++) t[k] = slab[(m + k) * FEAT + lane];
#pragma unroll
                    for (int k = 0; k < 8; k++) s = __fadd_rn(s, t[k]);
                }
                for (; m < cnt; m++) s = __fadd_rn(s, slab[m * FEAT + lane]);
            }
        }
        __syncwarp();
    }
    (void)s1;
    // gather the 16 feature sums into float4s for the quad that runs the dense part (lanes 0..3)
    float4 nb;
    nb.x = __shfl_sync(FULL, s, 4 * q + 0);
    nb.y = __shfl_sync(FULL, s, 4 * q + 1);
    nb.z = __shfl_sync(FULL, s, 4 * q + 2);
    nb.w = __shfl_sync(FULL, s, 4 * q + 3);
    const float in0 = __shfl_sync(FULL, s, 0), in1 = __shfl_sync(FULL, s, 1);
    if (lane >= 4) return;
    const unsigned int mask = 0xfu;
    const float4 b4 = reinterpret_cast<const float4 *>(sW + 2 * FEAT * FEAT)[q];
    float4 out;
    if (MODE == MODE_INPUT) {
        float s0 = in0, sid = in1;
        if (fd > 0.0f) {
            s0 = __fdiv_rn(s0, fd);
            sid = __fdiv_rn(sid, fd);
        }
        const float2 self = t01[u];
        out = dense_quad<MODE_INPUT>(W4, b4, q, 0, mask, zero4, zero4, s0, sid, self.x, self.y);
    } else {
        if (fd > 0.0f) nb = make_float4(__fdiv_rn(nb.x, fd), __fdiv_rn(nb.y, fd), __fdiv_rn(nb.z, fd), __fdiv_rn(nb.w, fd));
        const float4 self = reinterpret_cast<const float4 *>(x)[(size_t)u * 4 + q];
        out = dense_quad<MODE>(W4, b4, q, 0, mask, nb, self, 0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (MODE == MODE_OUTPUT) {
        const float sum = output_sum(out, mask);
        if (q == 0) key[u] = __float_as_uint(sum);
    } else {
        reinterpret_cast<float4 *>(y)[(size_t)u * 4 + q] = out;
    }
}

// Degree order split in two tiers: the first n_wide vertices (more than GC_GNN_WARP_DEGREE
// neighbours) one per warp, the rest eight per warp (four lanes each).  Work items are handed out
// by warp index, heaviest first.
template <int MODE>
__global__ void __launch_bounds__(GNN_THREADS, 4) k_gnn_layer(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                              const uint32_t *__restrict__ vorder, uint32_t n_wide,
                                                              uint32_t n_vorder, const float2 *__restrict__ t01,
                                                              const float *__restrict__ x, float *__restrict__ y,
                                                              uint32_t *__restrict__ key, const float *__restrict__ Wb,
                                                              uint32_t *work_ctr, uint32_t reserve, uint32_t grab,
                                                              uint32_t heavy) {
    // an SM left to the giant-hub CTAs: the whole CTA leaves, except the grid's last CTA, which
    // stays wherever it runs, so the counter's work is done whatever the placement
    if (reserve && sm_id() < reserve && blockIdx.x != gridDim.x - 1) return;
    __shared__ __align__(16) float sW[LAYER_PARAMS];
    __shared__ __align__(16) float slabs[GNN_THREADS / 32][32 * FEAT];
    for (int i = threadIdx.x; i < LAYER_PARAMS; i += blockDim.x) sW[i] = Wb[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, q = lane & 3, qbase = lane & ~3;
    const float4 *W4 = reinterpret_cast<const float4 *>(sW);
    const float4 b4 = reinterpret_cast<const float4 *>(sW + 2 * FEAT * FEAT)[q];
    const float4 *X4 = reinterpret_cast<const float4 *>(x);
    float4 *Y4 = reinterpret_cast<float4 *>(y);
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float *slab = slabs[threadIdx.x >> 5];
    const uint32_t n_items = n_wide + (n_vorder - n_wide + 7) / 8;

    auto item = [&](uint32_t it) {
        if (it < n_wide) {
            warp_vertex<MODE>(vorder[it], V, E, t01, x, y, key, W4, sW, slab, lane);
            __syncwarp();
            return;
        }
        const uint32_t g0 = n_wide + (it - n_wide) * 8;
        const uint32_t slot = g0 + (lane >> 2);
        const bool valid = slot < n_vorder;
        const uint32_t u = valid ? vorder[slot] : 0u;
        const uint32_t beg = valid ? V[u] : 0u;
        const uint32_t d = valid ? V[u + 1] - beg : 0u;
        const uint32_t dmax = __reduce_max_sync(FULL, d);  // loop bounds stay warp-uniform
        const float fd = __uint2float_rn(d);
        float4 out;
        if (MODE == MODE_INPUT) {
            float s0 = 0.0f, s1 = 0.0f;
            for (uint32_t c = 0; c < dmax; c += 4) {
                float2 t = make_float2(0.0f, 0.0f);
                if (c + q < d) t = __ldg(t01 + ld_stream(E + beg + c + q));
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float a0 = __shfl_sync(FULL, t.x, qbase + k);
                    const float a1 = __shfl_sync(FULL, t.y, qbase + k);
                    if (c + k < d) {
                        s0 = __fadd_rn(s0, a0);
                        s1 = __fadd_rn(s1, a1);
                    }
                }
            }
            if (fd > 0.0f) {
                s0 = __fdiv_rn(s0, fd);
                s1 = __fdiv_rn(s1, fd);
            }
            const float2 self = valid ? t01[u] : make_float2(0.0f, 0.0f);
            out = dense_quad<MODE_INPUT>(W4, b4, q, qbase, FULL, zero4, zero4, s0, s1, self.x, self.y);
        } else {
            float4 s = zero4;
            // neighbour ids one step ahead, so the row loads never wait for them
            uint32_t n0 = q < d ? ld_stream(E + beg + q) : 0u;
            uint32_t n1 = 4 + q < d ? ld_stream(E + beg + 4 + q) : 0u;
            for (uint32_t c = 0; c < dmax; c += 8) {
                // two groups of four neighbours in flight per quad
                const uint32_t e0 = n0, e1 = n1;
                n0 = c + 8 + q < d ? ld_stream(E + beg + c + 8 + q) : 0u;
                n1 = c + 12 + q < d ? ld_stream(E + beg + c + 12 + q) : 0u;
                float4 r[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint32_t v = __shfl_sync(FULL, k < 4 ? e0 : e1, qbase + (k & 3));
                    r[k] = c + k < d ? __ldg(X4 + (size_t)v * 4 + q) : zero4;
                }
#pragma unroll
                for (int k = 0; k < 8; k++)
                    if (c + k < d) s = add4(s, r[k]);
            }
            if (fd > 0.0f) s = make_float4(__fdiv_rn(s.x, fd), __fdiv_rn(s.y, fd), __fdiv_rn(s.z, fd), __fdiv_rn(s.w, fd));
            const float4 self = valid ? __ldg(X4 + (size_t)u * 4 + q) : zero4;
            out = dense_quad<MODE>(W4, b4, q, qbase, FULL, s, self, 0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (MODE == MODE_OUTPUT) {
            const float sum = output_sum(out, FULL);
            if (valid && q == 0) key[u] = __float_as_uint(sum);
        } else if (valid) {
            Y4[(size_t)u * 4 + q] = out;
        }
    };
    // Dynamic hand-out (work_ctr): items are sorted heaviest first, so the warp-tier vertices
    // (work_ctr[0]) and the leading `heavy` four-lane items (work_ctr[1]) go one at a time and
    // spread over the warps; the rest go `grab` at a time (work_ctr[2]).  Otherwise a fixed
    // stride.  One call site, so the item body is inlined once.
    const uint32_t heavy_end = min(n_items, n_wide + heavy);
    uint32_t phase = 0, cur = 0, end = 0, sit = warp;
    for (;;) {
        uint32_t it;
        if (work_ctr) {
            while (cur == end && phase < 3) {
                if (phase == 0) {
                    const uint32_t x = grab_work(work_ctr, 1u, lane);
                    if (x < n_wide) cur = x, end = x + 1;
                    else phase = 1;
                } else if (phase == 1) {
                    const uint32_t x = n_wide + grab_work(work_ctr + 1, 1u, lane);
                    if (x < heavy_end) cur = x, end = x + 1;
                    else phase = 2;
                } else {
                    const uint32_t x = heavy_end + grab_work(work_ctr + 2, grab, lane);
                    if (x < n_items) cur = x, end = min(x + grab, n_items);
                    else phase = 3;
                }
            }
            if (cur == end) break;
            it = cur++;
        } else {
            if (sit >= n_items) break;
            it = sit;
            sit += nwarps;
        }
        item(it);
    }
}

// ---- thin tier: one vertex per lane --------------------------------------------------------------

// Vertices with at most ctx->gnn_thin_deg neighbours (the tail of the degree order, vorder[first,
// n_vorder)): one per lane, 32 per warp, whose degrees are nearly equal because the order is sorted.
// Each lane adds its vertex's neighbour rows in CSR order (the next row's loads in flight while the
// current one is added; the 16 feature chains interleave) and runs the 32 x 16 dense part alone:
// no lane sits idle on a short neighbour list, and no shuffles are needed.
constexpr int THIN_THREADS = 256;

template <int MODE>
__global__ void __launch_bounds__(THIN_THREADS, 3) k_gnn_thin(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                              const uint32_t *__restrict__ vorder, uint32_t first,
                                                              uint32_t n_vorder, const float2 *__restrict__ t01,
                                                              const float *__restrict__ x, float *__restrict__ y,
                                                              uint32_t *__restrict__ key, const float *__restrict__ Wb,
                                                              uint32_t *work_ctr, uint32_t reserve, uint32_t grab) {
    // an SM left to the giant-hub CTAs: the whole CTA leaves, except the grid's last CTA, which
    // stays wherever it runs, so the counter's work is done whatever the placement
    if (reserve && sm_id() < reserve && blockIdx.x != gridDim.x - 1) return;
    __shared__ __align__(16) float sW[LAYER_PARAMS];
    for (int i = threadIdx.x; i < LAYER_PARAMS; i += blockDim.x) sW[i] = Wb[i];
    __syncthreads();
    const float4 *W4 = reinterpret_cast<const float4 *>(sW);
    const float4 *X4 = reinterpret_cast<const float4 *>(x);
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    auto group = [&](uint32_t base) {  // the 32 vertices vorder[base, base + 32), one per lane
        const uint32_t slot = base + lane;
        const bool valid = slot < n_vorder;
        const uint32_t u = valid ? vorder[slot] : 0u;
        const uint32_t beg = valid ? V[u] : 0u, d = valid ? V[u + 1] - beg : 0u;
        const uint32_t dmax = __reduce_max_sync(FULL, d);
        const float fd = __uint2float_rn(d);
        float c[FEAT];
#pragma unroll
        for (int j = 0; j < FEAT; j++) c[j] = sW[2 * FEAT * FEAT + j];
        if (MODE == MODE_INPUT) {
            float s0 = 0.0f, s1 = 0.0f;
            float2 tn = d ? __ldg(t01 + __ldg(E + beg)) : make_float2(0.0f, 0.0f);
            for (uint32_t k = 0; k < dmax; k++) {
                const float2 t = tn;
                if (k + 1 < d) tn = __ldg(t01 + __ldg(E + beg + k + 1));
                if (k < d) {
                    s0 = __fadd_rn(s0, t.x);
                    s1 = __fadd_rn(s1, t.y);
                }
            }
            if (fd > 0.0f) {
                s0 = __fdiv_rn(s0, fd);
                s1 = __fdiv_rn(s1, fd);
            }
            const float2 self = valid ? t01[u] : make_float2(0.0f, 0.0f);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self.x : self.y));
#pragma unroll
                for (int jq = 0; jq < 4; jq++) {
                    const float4 w = W4[i * 4 + jq];
                    c[4 * jq + 0] = __fmaf_rn(w.x, a, c[4 * jq + 0]);
                    c[4 * jq + 1] = __fmaf_rn(w.y, a, c[4 * jq + 1]);
                    c[4 * jq + 2] = __fmaf_rn(w.z, a, c[4 * jq + 2]);
                    c[4 * jq + 3] = __fmaf_rn(w.w, a, c[4 * jq + 3]);
                }
            }
        } else {
            float acc[FEAT];
#pragma unroll
            for (int f = 0; f < FEAT; f++) acc[f] = 0.0f;
            // ids two ahead, rows one ahead
            uint32_t vnext = d > 1 ? __ldg(E + beg + 1) : 0u;
            float4 rn[4];
            {
                const uint32_t v0 = d ? __ldg(E + beg) : 0u;
#pragma unroll
                for (int p = 0; p < 4; p++) rn[p] = d ? __ldg(X4 + (size_t)v0 * 4 + p) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            for (uint32_t k = 0; k < dmax; k++) {
                float4 r[4];
#pragma unroll
                for (int p = 0; p < 4; p++) r[p] = rn[p];
                if (k + 1 < d) {
                    const uint32_t v = vnext;
                    vnext = k + 2 < d ? __ldg(E + beg + k + 2) : 0u;
#pragma unroll
                    for (int p = 0; p < 4; p++) rn[p] = __ldg(X4 + (size_t)v * 4 + p);
                }
                if (k < d) {
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        acc[4 * p + 0] = __fadd_rn(acc[4 * p + 0], r[p].x);
                        acc[4 * p + 1] = __fadd_rn(acc[4 * p + 1], r[p].y);
                        acc[4 * p + 2] = __fadd_rn(acc[4 * p + 2], r[p].z);
                        acc[4 * p + 3] = __fadd_rn(acc[4 * p + 3], r[p].w);
                    }
                }
            }
            if (fd > 0.0f) {
#pragma unroll
                for (int f = 0; f < FEAT; f++) acc[f] = __fdiv_rn(acc[f], fd);
            }
            float self[FEAT];
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const float4 s4 = valid ? __ldg(X4 + (size_t)u * 4 + p) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                self[4 * p + 0] = s4.x;
                self[4 * p + 1] = s4.y;
                self[4 * p + 2] = s4.z;
                self[4 * p + 3] = s4.w;
            }
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = i < FEAT ? acc[i] : self[i - FEAT];
#pragma unroll
                for (int jq = 0; jq < 4; jq++) {
                    const float4 w = W4[i * 4 + jq];
                    c[4 * jq + 0] = __fmaf_rn(w.x, a, c[4 * jq + 0]);
                    c[4 * jq + 1] = __fmaf_rn(w.y, a, c[4 * jq + 1]);
                    c[4 * jq + 2] = __fmaf_rn(w.z, a, c[4 * jq + 2]);
                    c[4 * jq + 3] = __fmaf_rn(w.w, a, c[4 * jq + 3]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < FEAT; j++) c[j] = relu(c[j]);
        if (!valid) return;
        if (MODE == MODE_OUTPUT) {
            // t_k = o_k + o_{k+8}, then ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7))  (dense_kernel_output)
            float t[8];
#pragma unroll
            for (int k = 0; k < 8; k++) t[k] = __fadd_rn(c[k], c[k + 8]);
            const float sum = __fadd_rn(__fadd_rn(__fadd_rn(t[0], t[1]), __fadd_rn(t[2], t[3])),
                                        __fadd_rn(__fadd_rn(t[4], t[5]), __fadd_rn(t[6], t[7])));
            key[u] = __float_as_uint(sum);
        } else {
            float4 *Y4 = reinterpret_cast<float4 *>(y) + (size_t)u * 4;
#pragma unroll
            for (int p = 0; p < 4; p++) Y4[p] = make_float4(c[4 * p], c[4 * p + 1], c[4 * p + 2], c[4 * p + 3]);
        }
    };
    // one call site, so the group body is inlined once
    const uint32_t n_groups = (n_vorder - first + 31) / 32;
    uint32_t base = first + blockIdx.x * blockDim.x + (threadIdx.x & ~31u), gi = 0, gend = 0;
    for (;;) {
        if (work_ctr) {
            if (gi == gend) {
                gi = grab_work(work_ctr, grab, lane);
                if (gi >= n_groups) break;
                gend = min(gi + grab, n_groups);
            }
            base = first + gi * 32;
            gi++;
        } else if (base >= n_vorder) {
            break;
        }
        group(base);
        if (!work_ctr) base += stride;
    }
}

// ---- hub vertices: one CTA each --------------------------------------------------------------

// Hub CTAs: a producer warp streams the hub's neighbour rows into a shared-memory ring with
// cp.async, each stage completing on its own mbarrier; a consumer quad adds the rows in CSR
// order, four features per lane.  No CTA-wide barrier: the producer runs up to HUB_STAGES stages
// ahead and refills a stage as soon as the consumer releases it.  Every mbarrier wait is bounded:
// on expiry the kernel raises ERR_WAIT_EXPIRED and returns.
constexpr int HUB_THREADS = 64;    // warp 0 adds, warp 1 loads
constexpr int HUB_ROWS = 128;      // rows per stage: 4 per producer lane
#ifndef GC_HUB_STAGES
#define GC_HUB_STAGES 12
#endif
constexpr int HUB_STAGES = GC_HUB_STAGES;
#ifndef GC_HUB_ID_AHEAD
#define GC_HUB_ID_AHEAD 4
#endif
constexpr int HUB_ID_AHEAD = GC_HUB_ID_AHEAD;  // the producer reads neighbour ids this many stages early
constexpr int HUB_BATCH = 16;      // staged values the consumer loads ahead of its add chain
constexpr unsigned int HUB_WAIT_LIMIT = 1u << 20;  // each try_wait may also suspend briefly

__device__ __forceinline__ unsigned int smem_u32(const void *p) { return (unsigned int)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_on_copies(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned int parity) {
    unsigned int ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of `parity` to complete; false if the wait gave up (error raised).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned int parity, DevState *st) {
    for (unsigned int i = 0; i < HUB_WAIT_LIMIT; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023u) == 1023u && ld_relaxed_u32(&st->err)) return false;
    }
    raise_error(st, ERR_WAIT_EXPIRED, 0xffffffffu);
    return false;
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}

// Giant hubs' neighbour rows, in CSR order, into the staging buffer, one column per feature: hub
// slot h owns the block of 16 columns starting at 16 * giant[h], each giant[h + 1] - giant[h] floats
// long (its degree rounded up to 32), so that one warp later streams one feature's column with
// coalesced loads.  All SMs, one warp per task of GC_GIANT_TASK rows.  Hidden and output layers:
// four lanes per 64-byte row (one float4 each), eight rows per instruction; input layer: a lane per
// row and two columns (deg/md, id/N).
template <int MODE>
__global__ void __launch_bounds__(256) k_gnn_hub_gather(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                        const uint32_t *__restrict__ hubs,
                                                        const uint32_t *__restrict__ giant, uint32_t n_giant,
                                                        uint32_t n_tasks, const float2 *__restrict__ t01,
                                                        const float *__restrict__ x, float *__restrict__ stage) {
    const uint32_t *tasks = giant + n_giant + 1;
    const int lane = threadIdx.x & 31, q = lane & 3;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = warp; t < n_tasks; t += nwarps) {
        const uint32_t slot = tasks[2 * t], r0 = tasks[2 * t + 1];
        const uint32_t u = hubs[slot], base = V[u], d = V[u + 1] - base;
        const uint32_t rend = min(d, r0 + GC_GIANT_TASK);
        const size_t dp = giant[slot + 1] - giant[slot];
        float *cols = stage + (size_t)FEAT * giant[slot];
        if (MODE == MODE_INPUT) {
            for (uint32_t r = r0 + lane; r < rend; r += 32) {
                const float2 tv = __ldg(t01 + ld_stream(E + base + r));
                cols[r] = tv.x;
                cols[dp + r] = tv.y;
            }
        } else {
            const float4 *X4 = reinterpret_cast<const float4 *>(x);
            float *c0 = cols + (size_t)(4 * q) * dp;
            for (uint32_t r = r0 + (lane >> 2); r < rend; r += 32) {
                uint32_t v[4];
                float4 val[4];
#pragma unroll
                for (int k = 0; k < 4; k++) v[k] = r + 8 * k < rend ? E[base + r + 8 * k] : 0u;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (r + 8 * k < rend) val[k] = __ldg(X4 + (size_t)v[k] * 4 + q);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (r + 8 * k < rend) {
                        const uint32_t rr = r + 8 * k;
                        c0[rr] = val[k].x;
                        c0[dp + rr] = val[k].y;
                        c0[2 * dp + rr] = val[k].z;
                        c0[3 * dp + rr] = val[k].w;
                    }
            }
        }
    }
}

// The reference's neighbour sum s = (((+0 + a_0) + a_1) + ...) + a_{n-1} in FP32, round to nearest
// even, for a column of n values a_i >= +0 (ReLU outputs, deg/md, id/N: never negative), with the
// whole warp, 1,024 values per step.  Bit-identical to the serial chain, by this argument:
//   While s lies in the binade [2^e, 2^(e+1)), s = m * u with u = 2^(e-23) and an integer m in
//   [2^23, 2^24).  Adding a >= 0 rounds m + a/u to an integer: with a/u = q + r (q integer,
//   0 <= r < 1) the result is m + q for r < 1/2 and m + q + 1 for r > 1/2, whatever m is; only an
//   exact tie (r = 1/2) depends on m (to even).  So as long as every partial sum stays below
//   2^(e+1), i.e. m plus all increments stays below 2^24, the step's result is m + (the integer
//   sum of the increments), and integer addition is associative.  The increments are exact: a/u is
//   a scaling by a power of two.
// A step falls back to the serial chain (shuffles broadcast the values; every lane adds them in
// order, so s stays warp-uniform) when that does not hold: s below 2^-103 (grid or its inverse not
// a normal float, e.g. the first step from +0) or infinite, a value with a/u >= 2^24 (or Inf/NaN), an exact tie
// anywhere in the step, or a step that would carry s into the next binade.  Partial sums are
// clamped at 2^24, which already means "fall back".  Each lane loads its next step's values while
// the current ones are summed.
__device__ __forceinline__ float exact_column_sum(const float *__restrict__ col, uint32_t n, int lane) {
    constexpr uint32_t STEP = 1024, TOP = 1u << 24;
    float s = 0.0f;
    float nx[32];
#pragma unroll
    for (int j = 0; j < 32; j++) {
        const uint32_t i = 32 * j + lane;
        nx[j] = i < n ? __ldcg(col + i) : 0.0f;
    }
    for (uint32_t c0 = 0; c0 < n; c0 += STEP) {
        const uint32_t cn = min(STEP, n - c0);
        float a[32];
#pragma unroll
        for (int j = 0; j < 32; j++) a[j] = nx[j];
        if (c0 + STEP < n) {
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const uint32_t i = c0 + STEP + 32 * j + lane;
                nx[j] = i < n ? __ldcg(col + i) : 0.0f;
            }
        }
        const uint32_t be = (__float_as_uint(s) >> 23) & 0xffu;  // biased exponent of s
        if (be >= 24u && be < 255u) {
            const float scale = __uint_as_float((277u - be) << 23);  // 1/u = 2^(23-e), e = be - 127
            const float unscale = __uint_as_float((be - 23u) << 23);  // u = 2^(e-23)
            const uint32_t m = __float2uint_rz(__fmul_rn(s, scale));
            uint32_t acc = 0;
            bool bad = false;
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const float xv = __fmul_rn(a[j], scale);
                const bool ok = xv < 16777216.0f;  // false for >= 2^24, Inf and NaN
                const float xs = ok ? xv : 0.0f;
                const float qf = floorf(xs);
                const float r = __fsub_rn(xs, qf);  // exact: xs < 2^24
                bad |= !ok || r == 0.5f;
                acc += __float2uint_rz(qf) + (r > 0.5f ? 1u : 0u);  // at most 32 * 2^24
            }
            if (!__any_sync(FULL, bad)) {
                const uint32_t tot = __reduce_add_sync(FULL, min(acc, TOP));
                const uint32_t mend = m + tot;
                if (mend < TOP) {
                    s = __fmul_rn(__uint2float_rn(mend), unscale);
                    continue;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 32; j++) {
            if (32u * j >= cn) break;
#pragma unroll 8
            for (int k = 0; k < 32; k++) {
                const float t = __shfl_sync(FULL, a[j], k);
                if (32u * j + k < cn) s = __fadd_rn(s, t);
            }
        }
    }
    return s;
}

// Giant hubs' layer: one warp per (hub, feature) -- two features in the input layer -- sums the
// hub's staged column with exact_column_sum; the hub's last warp to finish (a counter per hub,
// zeroed before the layer) runs the dense part: mean, 32 x 16 FMA chain in order, ReLU, and in the
// output layer the reference's fixed-tree sum into the key.
template <int MODE>
__global__ void __launch_bounds__(128) k_gnn_giant_chain(const uint32_t *__restrict__ V, const uint32_t *__restrict__ hubs,
                                                         const uint32_t *__restrict__ giant, uint32_t n_giant,
                                                         const float *__restrict__ stage, const float2 *__restrict__ t01,
                                                         const float *__restrict__ x, float *__restrict__ y,
                                                         uint32_t *__restrict__ key, const float *__restrict__ Wb,
                                                         float *__restrict__ sums, uint32_t *__restrict__ done) {
    constexpr int NF = (MODE == MODE_INPUT) ? 2 : FEAT;
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n_giant * NF) return;
    const uint32_t h = w / NF, f = w % NF;
    const uint32_t u = hubs[h], d = V[u + 1] - V[u];
    const size_t dp = giant[h + 1] - giant[h];
    const float sum = exact_column_sum(stage + (size_t)FEAT * giant[h] + f * dp, d, lane);
    uint32_t last = 0;
    if (lane == 0) {
        sums[h * FEAT + f] = sum;
        __threadfence();
        last = atomicAdd(done + h, 1u) == NF - 1;
    }
    if (!__shfl_sync(FULL, last, 0)) return;
    __threadfence();
    const float fd = __uint2float_rn(d);
    const int j = lane & 15;
    float c = __ldg(Wb + 2 * FEAT * FEAT + j);
    if (MODE == MODE_INPUT) {
        float s0 = __ldcg(sums + h * FEAT), s1 = __ldcg(sums + h * FEAT + 1);
        if (fd > 0.0f) {
            s0 = __fdiv_rn(s0, fd);
            s1 = __fdiv_rn(s1, fd);
        }
        const float2 self = t01[u];
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const float a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self.x : self.y));
            c = __fmaf_rn(__ldg(Wb + i * FEAT + j), a, c);
        }
    } else {
        float nb = __ldcg(sums + h * FEAT + j);
        if (fd > 0.0f) nb = __fdiv_rn(nb, fd);
        const float self = x[(size_t)u * FEAT + j];
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const float a = __shfl_sync(FULL, i < FEAT ? nb : self, i & 15);
            c = __fmaf_rn(__ldg(Wb + i * FEAT + j), a, c);
        }
    }
    const float o = relu(c);
    if (MODE == MODE_OUTPUT) {
        // t_k = o_k + o_{k+8}, then ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7))
        const float t = __fadd_rn(o, __shfl_sync(FULL, o, (lane + 8) & 31));
        float tk[8];
#pragma unroll
        for (int k = 0; k < 8; k++) tk[k] = __shfl_sync(FULL, t, k);
        const float p = __fadd_rn(__fadd_rn(__fadd_rn(tk[0], tk[1]), __fadd_rn(tk[2], tk[3])),
                                  __fadd_rn(__fadd_rn(tk[4], tk[5]), __fadd_rn(tk[6], tk[7])));
        if (lane == 0) key[u] = __float_as_uint(p);
    } else if (lane < FEAT) {
        y[(size_t)u * FEAT + lane] = o;
    }
}

// The other hubs (slots n_giant .. n_hubs - 1): one CTA each gathers the rows with cp.async.
template <int MODE>
__global__ void __launch_bounds__(HUB_THREADS) k_gnn_hub(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                         const uint32_t *__restrict__ hubs,
                                                         const float2 *__restrict__ t01, const float *__restrict__ x,
                                                         float *__restrict__ y, uint32_t *__restrict__ key,
                                                         const float *__restrict__ Wb, DevState *st, uint32_t first) {
    constexpr int ROW = (MODE == MODE_INPUT) ? 2 : FEAT;  // floats per staged row
    extern __shared__ __align__(16) float stage[];         // HUB_STAGES * HUB_ROWS * ROW floats
    __shared__ __align__(16) float sW[LAYER_PARAMS];
    __shared__ __align__(8) uint64_t full[HUB_STAGES], empty[HUB_STAGES];
    for (int i = threadIdx.x; i < LAYER_PARAMS; i += blockDim.x) sW[i] = Wb[i];
    if (threadIdx.x == 0) {
        for (int i = 0; i < HUB_STAGES; i++) {
            mbar_init(&full[i], 32);  // one copy-completion arrival per producer lane
            mbar_init(&empty[i], 1);  // the consumer's release
        }
    }
    __syncthreads();
    const uint32_t u = hubs[first + blockIdx.x];
    const uint32_t beg = V[u], end = V[u + 1], d = end - beg;
    const uint32_t nchunks = (d + HUB_ROWS - 1) / HUB_ROWS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) {
        // producer: ids HUB_ID_AHEAD stages ahead in registers, rows via cp.async
        uint32_t ids[HUB_ID_AHEAD][4];
        auto load_ids = [&](uint32_t c, uint32_t (&out)[4]) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t i = beg + c * HUB_ROWS + k * 32 + lane;
                out[k] = (c < nchunks && i < end) ? ld_stream(E + i) : 0xffffffffu;
            }
        };
#pragma unroll
        for (int a = 0; a < HUB_ID_AHEAD; a++) load_ids(a, ids[a]);
        for (uint32_t c = 0; c < nchunks; c++) {
            const uint32_t s = c % HUB_STAGES;
            if (c >= HUB_STAGES && !mbar_wait(&empty[s], ((c / HUB_STAGES) - 1) & 1u, st)) {
                asm volatile("cp.async.wait_all;" ::: "memory");
                return;
            }
            float *buf = stage + (size_t)s * HUB_ROWS * ROW;
            if (MODE == MODE_INPUT) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t v = ids[0][k];
                    if (v != 0xffffffffu) cp_async_8(buf + (size_t)(k * 32 + lane) * ROW, t01 + v);
                }
            } else {
                // four adjacent lanes copy the four 16-byte pieces of one row: each instruction
                // moves eight whole 64-byte rows (two sectors each) rather than 32 scattered pieces
                const int piece = lane & 3;
#pragma unroll
                for (int k = 0; k < 4; k++) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int r = j * 8 + (lane >> 2);  // row k * 32 + r of the stage
                        const uint32_t v = __shfl_sync(0xffffffffu, ids[0][k], r);
                        if (v != 0xffffffffu)
                            cp_async_16(buf + (size_t)(k * 32 + r) * ROW + 4 * piece, x + (size_t)v * FEAT + 4 * piece);
                    }
                }
            }
            mbar_arrive_on_copies(&full[s]);
#pragma unroll
            for (int a = 0; a + 1 < HUB_ID_AHEAD; a++)
#pragma unroll
                for (int k = 0; k < 4; k++) ids[a][k] = ids[a + 1][k];
            load_ids(c + HUB_ID_AHEAD, ids[HUB_ID_AHEAD - 1]);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");  // leave no copy of ours in flight
        return;
    }

    // consumer: warp 0.  Lane l < 16 owns feature l (input layer: lane 0 sums deg/md, lane 1 id/N):
    // one shared-memory load and one add per row per lane, so the chain runs at the add latency.
    float acc = 0.0f;
    for (uint32_t c = 0; c < nchunks; c++) {
        const uint32_t s = c % HUB_STAGES;
        if (!mbar_wait(&full[s], (c / HUB_STAGES) & 1u, st)) return;  // the producer stops at its next wait
        const float *buf = stage + (size_t)s * HUB_ROWS * ROW;
        const uint32_t cnt = min((uint32_t)HUB_ROWS, end - (beg + c * HUB_ROWS));
        if (lane < ROW) {
            if (cnt == HUB_ROWS) {
                // software pipeline: the next HUB_BATCH staged values are loaded while the current
                // ones are added, so the chain runs at the add latency, not the shared-load latency
                float cur[HUB_BATCH], nxt[HUB_BATCH];
#pragma unroll
                for (int k = 0; k < HUB_BATCH; k++) cur[k] = buf[k * ROW + lane];
#pragma unroll
                for (int r = 0; r < HUB_ROWS; r += HUB_BATCH) {
                    if (r + HUB_BATCH < HUB_ROWS) {
#pragma unroll
                        for (int k = 0; k < HUB_BATCH; k++) nxt[k] = buf[(r + HUB_BATCH + k) * ROW + lane];
                    }
#pragma unroll
                    for (int k = 0; k < HUB_BATCH; k++) acc = __fadd_rn(acc, cur[k]);
#pragma unroll
                    for (int k = 0; k < HUB_BATCH; k++) cur[k] = nxt[k];
                }
            } else {
                for (uint32_t r = 0; r < cnt; r++) acc = __fadd_rn(acc, buf[r * ROW + lane]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    // hand the 16 feature sums (or the two input sums) to the quad that runs the dense part
    const int q = lane & 3;
    float4 nb;
    nb.x = __shfl_sync(0xffffffffu, acc, 4 * q + 0);
    nb.y = __shfl_sync(0xffffffffu, acc, 4 * q + 1);
    nb.z = __shfl_sync(0xffffffffu, acc, 4 * q + 2);
    nb.w = __shfl_sync(0xffffffffu, acc, 4 * q + 3);
    const float in0 = __shfl_sync(0xffffffffu, acc, 0), in1 = __shfl_sync(0xffffffffu, acc, 1);
    if (lane >= 4) return;
    const unsigned int mask = 0xfu;
    const float4 *W4 = reinterpret_cast<const float4 *>(sW);
    const float4 b4 = reinterpret_cast<const float4 *>(sW + 2 * FEAT * FEAT)[q];
    const float fd = __uint2float_rn(d);
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float4 out;
    if (MODE == MODE_INPUT) {
        float s0 = in0, s1 = in1;
        if (fd > 0.0f) {
            s0 = __fdiv_rn(s0, fd);
            s1 = __fdiv_rn(s1, fd);
        }
        const float2 self = t01[u];
        out = dense_quad<MODE_INPUT>(W4, b4, q, 0, mask, zero4, zero4, s0, s1, self.x, self.y);
    } else {
        if (fd > 0.0f) nb = make_float4(__fdiv_rn(nb.x, fd), __fdiv_rn(nb.y, fd), __fdiv_rn(nb.z, fd), __fdiv_rn(nb.w, fd));
        const float4 self = reinterpret_cast<const float4 *>(x)[(size_t)u * 4 + q];
        out = dense_quad<MODE>(W4, b4, q, 0, mask, nb, self, 0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (MODE == MODE_OUTPUT) {
        const float sum = output_sum(out, mask);
        if (q == 0) key[u] = __float_as_uint(sum);
    } else {
        reinterpret_cast<float4 *>(y)[(size_t)u * 4 + q] = out;
    }
}

template <int MODE>
gc_status launch_layer(gc_graph *g, const float *Wb, const float *x, float *y, cudaStream_t side,
                       cudaEvent_t fork, cudaEvent_t join, uint32_t reserve) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    // counters, zeroed here for each layer: bulk items (2..4), thin groups (5); with reserve > 0 the
    // bulk CTAs that start on SMs 0..reserve-1 leave those SMs to the giant hubs' chains
    uint32_t *ctr = g->gnn_ctr;
    if ((s = gc_check_cuda(ctx, cudaMemsetAsync(ctr, 0, 8 * sizeof(uint32_t), ctx->stream), "gnn work counters")) !=
        GC_OK)
        return s;
    if (g->n_hubs) {
        constexpr int ROW = (MODE == MODE_INPUT) ? 2 : FEAT;
        constexpr uint32_t NF = (MODE == MODE_INPUT) ? 2 : FEAT;
        const size_t smem = (size_t)HUB_STAGES * HUB_ROWS * ROW * sizeof(float);
        if (!ctx->hub_smem_set[MODE]) {  // once per context: keeps the call out of captured sequences
            if ((s = gc_check_cuda(ctx, cudaFuncSetAttribute(k_gnn_hub<MODE>,
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                   "hub smem")) != GC_OK)
                return s;
            ctx->hub_smem_set[MODE] = true;
        }
        if (ctx->gnn_serial) side = ctx->stream;  // hubs first, then the bulk, on one stream
        if ((s = gc_check_cuda(ctx, cudaEventRecord(fork, ctx->stream), "fork")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(side, fork, 0), "fork")) != GC_OK) return s;
        ProfScope ps(ctx, MODE == MODE_INPUT ? "gnn_hub_input" : (MODE == MODE_HIDDEN ? "gnn_hub_hidden" : "gnn_hub_output"),
                     side);
        if (g->n_giant) {
            float *sums = reinterpret_cast<float *>(g->giant_aux);
            uint32_t *done = g->giant_aux + (size_t)FEAT * g->n_giant;
            if ((s = gc_check_cuda(ctx, cudaMemsetAsync(done, 0, sizeof(uint32_t) * g->n_giant, side),
                                   "giant hub counters")) != GC_OK)
                return s;
            {
                ProfScope pg(ctx, "gnn_giant_gather", side);
                k_gnn_hub_gather<MODE><<<ctx->num_sms * 4, 256, 0, side>>>(g->V, g->E, g->hubs, g->giant, g->n_giant,
                                                                            g->n_giant_tasks, g->t01, x, g->hub_stage);
                ctx->launches++;
            }
            ProfScope pc(ctx, "gnn_giant_chain", side);
            const uint32_t warps = g->n_giant * NF;
            k_gnn_giant_chain<MODE><<<(warps + 3) / 4, 128, 0, side>>>(g->V, g->hubs, g->giant, g->n_giant, g->hub_stage,
                                                                       g->t01, x, y, g->key, Wb, sums, done);
            ctx->launches++;
        }
        if (g->n_hubs > g->n_giant) {
            k_gnn_hub<MODE><<<g->n_hubs - g->n_giant, HUB_THREADS, smem, side>>>(
                g->V, g->E, g->hubs, g->t01, x, y, g->key, Wb, ctx->dstate, g->n_giant);
            ctx->launches++;
        }
        if ((s = gc_check_launch(ctx, "gnn hub layer")) != GC_OK) return s;
    }
    int &blocks = ctx->gnn_blocks_per_sm[MODE];
    if (!blocks) {
        if ((s = gc_check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_gnn_layer<MODE>,
                                                                                  GNN_THREADS, 0),
                               "occupancy")) != GC_OK)
            return s;
        if (blocks < 1) blocks = 1;
    }
    if (g->n_vorder) {
        ProfScope ps(ctx, MODE == MODE_INPUT ? "gnn_input" : (MODE == MODE_HIDDEN ? "gnn_hidden" : "gnn_output"),
                     ctx->stream);
        const uint32_t first_thin = g->n_vorder - g->n_thin;
        if (first_thin) {
            k_gnn_layer<MODE><<<ctx->num_sms * blocks, GNN_THREADS, 0, ctx->stream>>>(
                g->V, g->E, g->vorder, g->n_wide_gnn, first_thin, g->t01, x, y, g->key, Wb, ctr + 2, reserve,
                ctx->gnn_grab, ctx->gnn_heavy);
            ctx->launches++;
        }
        if (g->n_thin) {
            const uint32_t grid = std::min<uint32_t>((uint32_t)ctx->num_sms * 3, (g->n_thin + THIN_THREADS - 1) / THIN_THREADS);
            k_gnn_thin<MODE><<<grid, THIN_THREADS, 0, ctx->stream>>>(g->V, g->E, g->vorder, first_thin, g->n_vorder,
                                                                     g->t01, x, y, g->key, Wb, ctr + 5, reserve,
                                                                     ctx->gnn_grab);
            ctx->launches++;
        }
    }
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
    if (g->n_giant && g->hub_stage_rows < g->giant_rows) {
        gc_dev_free(ctx, g->hub_stage);
        g->hub_stage = nullptr;
        if ((s = gc_alloc(ctx, &g->hub_stage, (size_t)g->giant_rows * FEAT, "giant hub rows")) != GC_OK) return s;
        g->hub_stage_rows = g->giant_rows;
    }
    // giant hubs' feature sums (16 per hub) and completion counters (one per hub)
    if (g->n_giant && g->giant_aux_cap < (size_t)(FEAT + 1) * g->n_giant) {
        gc_dev_free(ctx, g->giant_aux);
        g->giant_aux = nullptr;
        if ((s = gc_alloc(ctx, &g->giant_aux, (size_t)(FEAT + 1) * g->n_giant, "giant hub sums")) != GC_OK) return s;
        g->giant_aux_cap = (size_t)(FEAT + 1) * g->n_giant;
    }
    // SMs left to the giant hubs' chains (ctx->gnn_hub_sms: -1 one per giant hub, 0 none, n: SMs
    // 0..n-1).  The bulk work is handed out by counters either way, so CTAs that start late (behind
    // the hubs' CTAs) take less of it.
    uint32_t reserve = 0;
    if (ctx->gnn_hub_sms != 0 && g->n_giant) {
        reserve = ctx->gnn_hub_sms > 0 ? (uint32_t)ctx->gnn_hub_sms : g->n_giant;
        reserve = std::min<uint32_t>(reserve, (uint32_t)ctx->num_sms / 6);
    }
    if ((s = gc_alloc(ctx, &g->gnn_ctr, 8, "gnn work counters")) != GC_OK) return s;
    if (ctx->side_stream == nullptr) {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        // hub CTAs carry the longest FP32 chains: schedule them ahead of the bulk
        if ((s = gc_check_cuda(ctx, cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, hi),
                               "stream")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
    }
    {
        ProfScope ps(ctx, "gnn_table0", ctx->stream);
        k_gnn_table0<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, (float)m->md, g->seg_voff, g->n_seg,
                                                                 g->t01);
    }
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "gnn input table")) != GC_OK) return s;
    const int L = m->layers;
    float *x = g->x, *y = g->y;
    for (int l = 0; l < L; l++) {
        const float *Wb = m->d_param + (size_t)l * LAYER_PARAMS;
        if (l == 0)
            s = launch_layer<MODE_INPUT>(g, Wb, nullptr, y, ctx->side_stream, ctx->ev_fork, ctx->ev_join, reserve);
        else if (l < L - 1)
            s = launch_layer<MODE_HIDDEN>(g, Wb, x, y, ctx->side_stream, ctx->ev_fork, ctx->ev_join, reserve);
        else
            s = launch_layer<MODE_OUTPUT>(g, Wb, x, nullptr, ctx->side_stream, ctx->ev_fork, ctx->ev_join, reserve);
        if (s != GC_OK) return s;
        float *t = x;
        x = y;
        y = t;
    }
    return GC_OK;
}
