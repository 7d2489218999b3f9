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
//   - hubs (more than GC_GNN_HUB_DEGREE): a persistent kernel on a high-priority side stream; one
//     item per hub gathers its neighbour rows into shared memory, 512 or 1,024 at a time, and one
//     warp per feature evaluates the reference's sequential FP32 chain exactly, a step at a time
//     (exact_step below); the rows of the largest hubs are staged feature-major by the whole GPU
//     first and split into (hub, 4 features) items; the hub's last item runs its dense part.
// Feature rows (x, y and the layer-0 table) are stored in degree order: hub h at row h, vorder[i] at
// row n_hubs + i.  The neighbour lists are read from Er, the CSR with each id replaced by its row
// (entry for entry, so every sum keeps the reference's order), and each row's first CSR entry and
// degree from vrow.  The rows most lists gather then share cache lines, and a warp's own rows,
// offsets and outputs are consecutive: on R-MAT 22 (GNN3) the three layers took 2.97 ms per job
// against 3.33 ms with rows by vertex id.
// Neighbour rows are read with __ldg: a layer never writes the features it reads.  In an A/B on
// R-MAT 22 (GNN3) the explicit read-only load made the bulk hidden and output layers about 6 %
// faster than the plain loads the compiler emits here.
//
// Compiled without fast-math; every add, divide and FMA is an explicit round-to-nearest
// intrinsic so the compiler cannot contract or reassociate them.
#include <algorithm>
#include <cstring>

#include "gc_internal.h"

namespace {
using namespace gc;

enum : int { MODE_INPUT = 0, MODE_HIDDEN = 1, MODE_OUTPUT = 2 };

// In a segmented CSR the id feature is (local id) / (the graph's own N).  Written at the vertex's
// feature row.
__global__ void k_gnn_table0(const uint32_t *__restrict__ V, uint32_t N, float fmd, const uint32_t *__restrict__ voff,
                             uint32_t nseg, const uint32_t *__restrict__ row_of, float2 *__restrict__ t01) {
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
        t01[row_of[u]] = make_float2(deg_feat, id_feat);
    }
}

// Feature rows in degree order: hub h takes row h, vorder[i] row n_hubs + i.  Each row also gets
// its vertex's first CSR entry and degree, so the bulk kernels read them in row order.
__global__ void k_gnn_rows(const uint32_t *__restrict__ V, const uint32_t *__restrict__ hubs, uint32_t n_hubs,
                           const uint32_t *__restrict__ vorder, uint32_t n_vorder, uint32_t *__restrict__ row_of,
                           uint2 *__restrict__ vrow) {
    const uint32_t n = n_hubs + n_vorder;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t u = i < n_hubs ? hubs[i] : vorder[i - n_hubs];
        const uint32_t beg = V[u];
        row_of[u] = i;
        vrow[i] = make_uint2(beg, V[u + 1] - beg);
    }
}

// The CSR's neighbour ids as feature rows, entry for entry: the lists keep their order, so every
// neighbour sum still runs in the reference's CSR order.  Entries [first, first + count); an id of N
// or more (a malformed CSR, when this runs before the upload's own check) raises ERR_BOUND and
// becomes row 0, so nothing is read out of bounds.
__global__ void k_gnn_row_ids(const uint32_t *__restrict__ E, uint32_t first, uint32_t count, uint32_t N,
                              const uint32_t *__restrict__ row_of, uint32_t *__restrict__ Er, DevState *st) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t j = first + k, v = ld_stream(E + j);
        if (v < N) {
            Er[j] = __ldg(row_of + v);
        } else {
            Er[j] = 0u;
            raise_error(st, ERR_BOUND, j);
        }
    }
}

// ---- shared pieces: four lanes per vertex, lane q owns features 4q..4q+3 ---------------------

constexpr unsigned int FULL = 0xffffffffu;

// Bulk work handed out by an atomic counter, n items per warp at a time (the sizes are the context's
// gnn_grab and gnn_heavy), so that the warps that start late take less of it.
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
__device__ __forceinline__ void warp_vertex(uint32_t u, uint32_t r, const uint2 *__restrict__ vrow, const uint32_t *__restrict__ E,
                                            const float2 *__restrict__ t01, const float *__restrict__ x, float *__restrict__ y,
                                            uint32_t *__restrict__ key, const float4 *W4, const float *sW, float *slab,
                                            int lane) {
    const uint2 bd = vrow[r];
    const uint32_t beg = bd.x, d = bd.y;
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
        const float2 self = t01[r];
        out = dense_quad<MODE_INPUT>(W4, b4, q, 0, mask, zero4, zero4, s0, sid, self.x, self.y);
    } else {
        if (fd > 0.0f) nb = make_float4(__fdiv_rn(nb.x, fd), __fdiv_rn(nb.y, fd), __fdiv_rn(nb.z, fd), __fdiv_rn(nb.w, fd));
        const float4 self = reinterpret_cast<const float4 *>(x)[(size_t)r * 4 + q];
        out = dense_quad<MODE>(W4, b4, q, 0, mask, nb, self, 0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (MODE == MODE_OUTPUT) {
        const float sum = output_sum(out, mask);
        if (q == 0) key[u] = __float_as_uint(sum);
    } else {
        reinterpret_cast<float4 *>(y)[(size_t)r * 4 + q] = out;
    }
}

// Work items, heaviest first: the degree order in two tiers, its first n_wide vertices (more than the
// GNN warp degree) one per warp, the rest eight per warp (four lanes each).  Handed out by counters
// (work_ctr).  E holds the neighbours' feature rows; vorder[i]'s own row is row0 + i.
template <int MODE>
__global__ void __launch_bounds__(GNN_THREADS, 4) k_gnn_layer(const uint2 *__restrict__ vrow, const uint32_t *__restrict__ E,
                                                              const uint32_t *__restrict__ vorder, uint32_t row0, uint32_t n_wide,
                                                              uint32_t n_vorder, const float2 *__restrict__ t01,
                                                              const float *__restrict__ x, float *__restrict__ y,
                                                              uint32_t *__restrict__ key, const float *__restrict__ Wb,
                                                              uint32_t *work_ctr, uint32_t grab, uint32_t heavy) {
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
            warp_vertex<MODE>(MODE == MODE_OUTPUT ? vorder[it] : 0u, row0 + it, vrow, E, t01, x, y, key, W4, sW, slab,
                              lane);
            __syncwarp();
            return;
        }
        const uint32_t g0 = n_wide + (it - n_wide) * 8;
        const uint32_t slot = g0 + (lane >> 2);
        const bool valid = slot < n_vorder;
        const uint32_t u = valid && MODE == MODE_OUTPUT ? vorder[slot] : 0u;  // the vertex (for its key)
        const uint32_t r = row0 + slot;                                       // its feature row
        const uint2 bd = valid ? vrow[r] : make_uint2(0u, 0u);
        const uint32_t beg = bd.x, d = bd.y;
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
            const float2 self = valid ? t01[r] : make_float2(0.0f, 0.0f);
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
            const float4 self = valid ? __ldg(X4 + (size_t)r * 4 + q) : zero4;
            out = dense_quad<MODE>(W4, b4, q, qbase, FULL, s, self, 0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (MODE == MODE_OUTPUT) {
            const float sum = output_sum(out, FULL);
            if (valid && q == 0) key[u] = __float_as_uint(sum);
        } else if (valid) {
            Y4[(size_t)r * 4 + q] = out;
        }
    };
    // Dynamic hand-out (work_ctr): items are sorted heaviest first, so the warp-tier vertices
    // (work_ctr[0]) and the leading `heavy` four-lane items (work_ctr[1]) go one at a time
    // and spread over the warps; the rest go `grab` at a time (work_ctr[2]).  Otherwise a fixed
    // stride.  One call site, so the item body is inlined once.
    const uint32_t n_first = n_wide;
    const uint32_t heavy_end = min(n_items, n_first + heavy);
    uint32_t phase = 0, cur = 0, end = 0, sit = warp;
    for (;;) {
        uint32_t it;
        if (work_ctr) {
            while (cur == end && phase < 3) {
                if (phase == 0) {
                    const uint32_t x = grab_work(work_ctr, 1u, lane);
                    if (x < n_first) cur = x, end = x + 1;
                    else phase = 1;
                } else if (phase == 1) {
                    const uint32_t x = n_first + grab_work(work_ctr + 1, 1u, lane);
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

// ---- vertices without neighbours: every layer at once -----------------------------------------
//
// A vertex without neighbours has a neighbour mean of +0 in every layer (no sum, no division), and
// nothing reads its features but itself.  So its whole network runs in one pass, one vertex per lane,
// from its layer-0 inputs to the key, and its rows of x and y are never written.  Each output's FMA
// chain runs over the inputs in the reference's order; the leading inputs are the same for every
// such vertex (the +0 means, and in layer 0 also deg/md = 0/md), so that prefix of each chain is
// evaluated once per CTA, with the same operations, and each vertex continues from it.  These
// vertices are the tail vorder[first, n) of the degree order; vorder[i]'s input row is row0 + i.
constexpr int ISO_THREADS = 256;
constexpr int ISO_MAX_LAYERS = 16;

__global__ void __launch_bounds__(ISO_THREADS) k_gnn_isolated(const uint32_t *__restrict__ vorder, uint32_t row0, uint32_t first,
                                                             uint32_t n, const float2 *__restrict__ t01,
                                                             uint32_t *__restrict__ key, const float *__restrict__ params,
                                                             int layers) {
    extern __shared__ __align__(16) float sP[];  // layers x LAYER_PARAMS
    __shared__ float c0[ISO_MAX_LAYERS][FEAT];   // each output's chain over the common leading inputs
    for (int i = threadIdx.x; i < layers * LAYER_PARAMS; i += blockDim.x) sP[i] = params[i];
    __syncthreads();
    if (threadIdx.x < layers * FEAT) {
        const int l = threadIdx.x / FEAT, j = threadIdx.x % FEAT;
        const float *W = sP + l * LAYER_PARAMS;
        float c = W[2 * FEAT * FEAT + j];
        if (l == 0) {
            const float deg0 = t01[row0 + first].x;  // 0 / md, the same for every vertex here
            for (int i = 0; i < 24; i++) c = __fmaf_rn(W[i * FEAT + j], i < 16 ? 0.0f : deg0, c);
        } else {
            for (int i = 0; i < FEAT; i++) c = __fmaf_rn(W[i * FEAT + j], 0.0f, c);
        }
        c0[l][j] = c;
    }
    __syncthreads();
    for (uint32_t slot = first + blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const uint32_t u = vorder[slot];
        const float id = t01[row0 + slot].y;
        float h[FEAT];
        for (int l = 0; l < layers; l++) {
            const float4 *W4 = reinterpret_cast<const float4 *>(sP + l * LAYER_PARAMS);
            float c[FEAT];
#pragma unroll
            for (int j = 0; j < FEAT; j++) c[j] = c0[l][j];
            // the inputs after the common prefix: layer 0 the id feature (inputs 24..31), later layers
            // the vertex's own previous outputs (inputs 16..31); unrolled so h stays in registers
            auto fma_in = [&](int i, float a) {
#pragma unroll
                for (int jq = 0; jq < 4; jq++) {
                    const float4 w = W4[i * 4 + jq];
                    c[4 * jq + 0] = __fmaf_rn(w.x, a, c[4 * jq + 0]);
                    c[4 * jq + 1] = __fmaf_rn(w.y, a, c[4 * jq + 1]);
                    c[4 * jq + 2] = __fmaf_rn(w.z, a, c[4 * jq + 2]);
                    c[4 * jq + 3] = __fmaf_rn(w.w, a, c[4 * jq + 3]);
                }
            };
            if (l == 0) {
#pragma unroll
                for (int i = 24; i < 32; i++) fma_in(i, id);
            } else {
#pragma unroll
                for (int i = FEAT; i < 32; i++) fma_in(i, h[i - FEAT]);
            }
#pragma unroll
            for (int j = 0; j < FEAT; j++) h[j] = relu(c[j]);
        }
        // t_k = o_k + o_{k+8}, then ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7))  (dense_kernel_output)
        float t[8];
#pragma unroll
        for (int k = 0; k < 8; k++) t[k] = __fadd_rn(h[k], h[k + 8]);
        const float sum = __fadd_rn(__fadd_rn(__fadd_rn(t[0], t[1]), __fadd_rn(t[2], t[3])),
                                    __fadd_rn(__fadd_rn(t[4], t[5]), __fadd_rn(t[6], t[7])));
        key[u] = __float_as_uint(sum);
    }
}

// ---- thin tier: one vertex per lane --------------------------------------------------------------

// Vertices with at most ctx->gnn_thin_deg neighbours (the tail of the degree order, vorder[first,
// n_vorder)): one per lane, 32 per warp, whose degrees are nearly equal because the order is sorted.
// E holds the neighbours' feature rows; vorder[i]'s own row is row0 + i.
// Each lane adds its vertex's neighbour rows in CSR order (the next row's loads in flight while the
// current one is added; the 16 feature chains interleave) and runs the 32 x 16 dense part alone:
// no lane sits idle on a short neighbour list, and no shuffles are needed.
constexpr int THIN_THREADS = 256;

// One layer's 32 x 16 weights and 16 biases as a kernel parameter.  Every lane of the thin tier reads
// the same weight at the same time, with compile-time indices, so each one is a constant-bank
// operand of its FMA: no load through the L1 data pipe, which bounds this kernel (weights in shared
// memory cost it 15 M of 53 M wavefronts per hidden layer on R-MAT 22).
struct LayerArg {
    float w[LAYER_PARAMS];
};

template <int MODE>
__global__ void __launch_bounds__(THIN_THREADS, 3) k_gnn_thin(const uint2 *__restrict__ vrow, const uint32_t *__restrict__ E,
                                                              const uint32_t *__restrict__ vorder, uint32_t row0, uint32_t first,
                                                              uint32_t n_vorder, const float2 *__restrict__ t01,
                                                              const float *__restrict__ x, float *__restrict__ y,
                                                              uint32_t *__restrict__ key, const __grid_constant__ LayerArg P,
                                                              uint32_t *work_ctr, uint32_t grab) {
    const float *W = P.w;  // row i of the weights: W[16 i .. 16 i + 15], biases W[512 ..]
    const float4 *X4 = reinterpret_cast<const float4 *>(x);
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    auto group = [&](uint32_t base) {  // the 32 vertices vorder[base, base + 32), one per lane
        const uint32_t slot = base + lane;
        const bool valid = slot < n_vorder;
        const uint32_t u = valid && MODE == MODE_OUTPUT ? vorder[slot] : 0u;  // the vertex (for its key)
        const uint32_t r = row0 + slot;                                       // its feature row
        const uint2 bd = valid ? vrow[r] : make_uint2(0u, 0u);
        const uint32_t beg = bd.x, d = bd.y;
        const uint32_t dmax = __reduce_max_sync(FULL, d);
        const float fd = __uint2float_rn(d);
        float c[FEAT];
#pragma unroll
        for (int j = 0; j < FEAT; j++) c[j] = W[2 * FEAT * FEAT + j];
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
            const float2 self = valid ? t01[r] : make_float2(0.0f, 0.0f);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self.x : self.y));
#pragma unroll
                for (int j = 0; j < FEAT; j++) c[j] = __fmaf_rn(W[i * FEAT + j], a, c[j]);
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
                const float4 s4 = valid ? __ldg(X4 + (size_t)r * 4 + p) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                self[4 * p + 0] = s4.x;
                self[4 * p + 1] = s4.y;
                self[4 * p + 2] = s4.z;
                self[4 * p + 3] = s4.w;
            }
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = i < FEAT ? acc[i] : self[i - FEAT];
#pragma unroll
                for (int j = 0; j < FEAT; j++) c[j] = __fmaf_rn(W[i * FEAT + j], a, c[j]);
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
            float4 *Y4 = reinterpret_cast<float4 *>(y) + (size_t)r * 4;
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

// ---- hubs: exact neighbour sums by whole warps ----------------------------------------------------
//
// A hub's FP32 neighbour sum s = (((+0 + a_0) + a_1) + ...) + a_{d-1} is a serial chain of d adds in
// the reference (fast_gnn.c:13-47), 4 cycles each on the GPU: 0.65 ms for the largest R-MAT 22 hub
// per layer.  Here a warp evaluates it exactly, 1,024 values per step, from these facts (all values
// are >= +0: ReLU outputs, deg/md, id/N):
//   - While s lies in the binade [2^e, 2^(e+1)), s = m * u with u = 2^(e-23) and an integer m in
//     [2^23, 2^24).  Adding a >= 0 rounds m + a/u to an integer: with a/u = q + r (q integer,
//     0 <= r < 1) the result is m + q for r < 1/2 and m + q + 1 for r > 1/2, whatever m is; an exact
//     tie (r = 1/2) goes to the even result, so it adds q + ((m + q) & 1) and leaves m even.
//   - So while the sum stays in its binade, a run of values adds an integer total that depends only
//     on the parity of m at the run's start: a 2-state transducer (parity in -> total, parity out),
//     and transducers compose associatively.
// Lane l holds values 32l .. 32l+31 of the step and builds its transducer over them for both start
// parities; a 5-round warp scan composes the lanes in order.  The first lane whose run would carry s
// out of the binade, or that holds a value with a/u >= 2^23 (or Inf/NaN), is added with plain FP32
// adds in order (shuffles broadcast its values; every lane adds them, so s stays warp-uniform), and
// the step resumes after it in the new binade.  +0 plus zeros stays +0, and a sum below 2^-103 (grid
// or its inverse not a normal float) is also added lane by lane with FP32 adds.
constexpr uint32_t EXACT_TOP = 1u << 24;
constexpr uint32_t EXACT_SAT = 1u << 25;  // transducer totals are clamped here: >= 2^24 means "leaves"
constexpr uint32_t HX_TILE = 1024;        // values per step

// A transducer as two words, one per start parity P: bits 0..30 the total added, bit 31 the end
// parity (totals are clamped at EXACT_SAT < 2^31).
constexpr uint32_t XD_P = 1u << 31, XD_T = XD_P - 1u;
struct Xd {
    uint32_t w0, w1;  // start parity 0 / 1
};
__device__ __forceinline__ uint32_t xd_then(uint32_t f, const Xd &g) {  // f's total, then g from f's end parity
    const uint32_t gs = (f & XD_P) ? g.w1 : g.w0;
    return min((f & XD_T) + (gs & XD_T), EXACT_SAT) | (gs & XD_P);
}
__device__ __forceinline__ Xd xd_after(const Xd &f, const Xd &g) { return {xd_then(f.w0, g), xd_then(f.w1, g)}; }

// A step's column holds VPL values per lane (32 for a 1,024-value step, 16 for 512): value r = VPL*l + k
// of lane l sits in the lane's VPL-word block, its 16-byte chunk k >> 2 at chunk (k >> 2) ^ sw(l), with
// sw(l) = l & 7 for VPL 32 and (l >> 1) & 3 for VPL 16.  A lane reads its block as float4s, and the
// 8 lanes of each quarter warp then touch 8 distinct 16-byte bank groups (no conflict); the
// producer's stores of 32 consecutive rows hit 32 distinct banks.
template <int VPL>
__device__ __forceinline__ uint32_t hx_sw(uint32_t l) {
    return VPL == 32 ? (l & 7u) : ((l >> 1) & 3u);
}
template <int VPL>
__device__ __forceinline__ uint32_t hx_slot(uint32_t k, uint32_t l) {
    return ((((k >> 2) ^ hx_sw<VPL>(l)) & (VPL / 4 - 1)) << 2) | (k & 3u);
}
template <int VPL>
__device__ __forceinline__ uint32_t hx_pos(uint32_t r) {
    return (r & ~(uint32_t)(VPL - 1)) | hx_slot<VPL>(r & (VPL - 1), r / VPL);
}

// The VPL values of lane c added to s with FP32 adds, in order (every lane reads them: broadcasts).
template <int VPL>
__device__ __forceinline__ void serial_lane(float &s, const float *col, uint32_t c) {
    const float *cp = col + (uint32_t)VPL * c;
#pragma unroll 8
    for (uint32_t k = 0; k < VPL; k++) s = __fadd_rn(s, cp[hx_slot<VPL>(k, c)]);
}

// Parity (0/1) of the increments at the positions of mask m.
__device__ __forceinline__ uint32_t par(uint32_t pm, uint32_t m) { return (uint32_t)__popc(pm & m) & 1u; }

// Increment of one value in units of the binade's grid, ties counted as q (r = 1/2 exactly).
__device__ __forceinline__ uint32_t grid_increment(float xv, bool &tie) {
    const float qf = floorf(xv);
    const float r = __fsub_rn(xv, qf);
    tie = r == 0.5f;
    return __float2uint_rz(qf) + (r > 0.5f ? 1u : 0u);
}

// Adds one step of 32 * VPL values to s, bit-identical to the serial chain.  col is the step's column
// in shared memory, value r at col[hx_pos<VPL>(r)], +0 past the column's end; lane l takes values
// VPL*l .. VPL*l + VPL-1.
//
// A lane's transducer: without ties it adds the total t of its increments (rounded to nearest) and
// flips the parity by t's.  With ties at k_1 < ... < k_n, built from two bit masks, pm (increment odd)
// and tm (value k is a tie, counted as q): the first tie adds one more when P + (increments up to and
// including k_1) is odd (P = the start parity), each later tie k_j adds one when the increments in
// (k_{j-1}, k_j] have odd sum, and after a tie the parity is that of the increments after the last
// one.  The masks are only built (a second pass over the lane's values) when a tie was seen.
template <int VPL>
__device__ __forceinline__ void exact_step(float &s, const float *col, int lane) {
    constexpr uint32_t CH = VPL / 4;  // float4 chunks per lane
    uint32_t start = 0;  // lanes [0, start) are in s (warp-uniform)
    const float4 *colp = reinterpret_cast<const float4 *>(col + (uint32_t)VPL * (uint32_t)lane);
    const uint32_t sw = hx_sw<VPL>((uint32_t)lane);
    while (start < 32) {
        const bool act = (uint32_t)lane >= start;
        if (s == 0.0f) {
            bool nz = false;
#pragma unroll
            for (uint32_t j = 0; j < CH; j++) {
                const float4 v = colp[j ^ sw];
                nz |= (v.x != 0.0f) | (v.y != 0.0f) | (v.z != 0.0f) | (v.w != 0.0f);
            }
            const unsigned int nzm = __ballot_sync(FULL, act && nz);
            if (!nzm) return;
            const uint32_t c = (uint32_t)(__ffs(nzm) - 1);
            serial_lane<VPL>(s, col, c);
            start = c + 1u;
            continue;
        }
        const uint32_t be = (__float_as_uint(s) >> 23) & 0xffu;
        if (be < 24u || be == 255u) {
            serial_lane<VPL>(s, col, start);
            start++;
            continue;
        }
        const float scale = __uint_as_float((277u - be) << 23);  // 1/u = 2^(23-e), e = be - 127
        const uint32_t m = __float2uint_rz(__fmul_rn(s, scale));
        Xd x = {0u, XD_P};  // identity: nothing added, parity kept
        bool bad = false;
        if (act) {
            // Increments rounded to nearest even through the adder, 2^23 + xs: exact for 0 <= xs < 2^23
            // (larger, negative -- -0 included --, Inf and NaN values all have float bits >= those of
            // 2^23 once scaled, so one unsigned maximum flags them, and their lane is added serially).
            // The bits of 2^23 + xs are summed mod 2^32, VPL offsets of 0x4B000000 removed at the end.
            // A tie (xs - RNE(xs) = +-1/2, both exact) sends the lane to the second pass below.
            uint32_t ta = 0, tb = 0, umax = 0;  // two partial sums in flight
            bool anytie = false;
#pragma unroll
            for (uint32_t j = 0; j < CH; j++) {
                const float4 v = colp[j ^ sw];
                const float xs[4] = {__fmul_rn(v.x, scale), __fmul_rn(v.y, scale), __fmul_rn(v.z, scale),
                                     __fmul_rn(v.w, scale)};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    umax = max(umax, __float_as_uint(xs[i]));
                    const float yv = __fadd_rn(xs[i], 8388608.0f);
                    if (i & 1) tb += __float_as_uint(yv);
                    else ta += __float_as_uint(yv);
                    anytie |= fabsf(__fsub_rn(xs[i], __fsub_rn(yv, 8388608.0f))) == 0.5f;
                }
            }
            bad = umax >= 0x4B000000u;  // 2^23
            if (!anytie || bad) {
                const uint32_t t = min(ta + tb - (uint32_t)VPL * 0x4B000000u, EXACT_SAT);
                x.w0 = t | ((t & 1u) << 31);
                x.w1 = t | ((~t & 1u) << 31);
            } else {
                // ties counted as q: totals and the masks pm (increment odd), tm (value k a tie)
                uint32_t tq = 0, pm = 0, tm = 0;
#pragma unroll
                for (uint32_t j = 0; j < CH; j++) {
                    const float4 v = colp[j ^ sw];
                    const float xs[4] = {__fmul_rn(v.x, scale), __fmul_rn(v.y, scale), __fmul_rn(v.z, scale),
                                         __fmul_rn(v.w, scale)};
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        bool tie;
                        const uint32_t nt = grid_increment(xs[i], tie);
                        tq += nt;
                        pm |= (nt & 1u) << (4 * j + i);
                        tm |= (tie ? 1u : 0u) << (4 * j + i);
                    }
                }
                const uint32_t t = min(tq, EXACT_SAT);
                const int k1 = __ffs(tm) - 1;
                const uint32_t first = par(pm, 0xffffffffu >> (31 - k1));  // increments 0 .. k1
                uint32_t extra = 0, rest = tm & (tm - 1u), prev = (uint32_t)k1;
                while (rest) {  // later ties: one more when (prev, k] has odd sum
                    const uint32_t k = (uint32_t)(__ffs(rest) - 1);
                    extra += par(pm, (0xffffffffu >> (31 - k)) & ~(0xffffffffu >> (31 - prev)));
                    prev = k;
                    rest &= rest - 1u;
                }
                const uint32_t pe = prev == 31u ? 0u : par(pm, 0xffffffffu << (prev + 1u));  // end parity
                x.w0 = min(t + extra + first, EXACT_SAT) | (pe << 31);          // P = 0: the first tie adds one when odd
                x.w1 = min(t + extra + (first ^ 1u), EXACT_SAT) | (pe << 31);   // P = 1
            }
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {  // inclusive composition over the lanes, in order
            Xd f;
            f.w0 = __shfl_up_sync(FULL, x.w0, o);
            f.w1 = __shfl_up_sync(FULL, x.w1, o);
            if (lane >= o) x = xd_after(f, x);
        }
        const uint32_t I = ((m & 1u) ? x.w1 : x.w0) & XD_T;  // added through this lane
        const unsigned int cm = __ballot_sync(FULL, act && (bad || m + I >= EXACT_TOP));
        const float unscale = __uint_as_float((be - 23u) << 23);
        if (!cm) {
            s = __fmul_rn(__uint2float_rn(m + __shfl_sync(FULL, I, 31)), unscale);
            return;
        }
        const uint32_t c = (uint32_t)(__ffs(cm) - 1);
        const uint32_t before = __shfl_sync(FULL, I, c > 0 ? (int)c - 1 : 0);
        if (c > start) s = __fmul_rn(__uint2float_rn(m + before), unscale);
        serial_lane<VPL>(s, col, c);
        start = c + 1u;
    }
}

// Hub work comes in two kinds of item, both evaluated with exact_step on feature-major column tiles
// in shared memory (the swizzled layout of hx_pos):
//   - a hub item (kind A): one hub, all its features at once.  Producer warps copy each step's
//     neighbour rows whole -- one 64-byte request per row (the float2 of layer-0 inputs in the input
//     layer) -- by cp.async into a staging ring, and transpose them into the column tiles; one feature
//     warp per feature sums its column.  One request per row, not one per feature group: a single
//     SM issues about one miss request per two cycles, which bounds any per-SM gather of scattered
//     rows;
//   - a staged item (kind B): a giant hub's group of features (4; in the input layer 1).  Before the
//     layer, k_hub_stage gathers the giant hubs' rows with the whole GPU into a feature-major buffer
//     already in the tiles' layout, so a staged item's producer moves each step's columns with one
//     bulk copy per feature, and the giant hub's chain runs on several SMs at its arithmetic speed.
// The hub's last item to finish (a counter per hub) runs the dense part.
template <int MODE>
struct HubCfg {
    static constexpr int NWA = MODE == MODE_INPUT ? 2 : FEAT;  // hub items: feature warps (all features)
    static constexpr int VPLA = MODE == MODE_INPUT ? 32 : 16;  // hub items: values per lane and step
    static constexpr int STEPA = 32 * VPLA;                    // rows per step
    static constexpr int NP = MODE == MODE_INPUT ? 1 : 4;      // producer warps
    static constexpr int ROWB = MODE == MODE_INPUT ? 8 : 64;   // bytes of a staged row
    static constexpr int STA = 3;                              // staging ring depth: 2 steps of rows in flight
    static constexpr int NWB = MODE == MODE_INPUT ? 1 : 4;     // staged items: features per item
    static constexpr int NGB = (MODE == MODE_INPUT ? 2 : FEAT) / NWB;  // staged items per giant hub
    static constexpr int THREADS = 32 * (NWA + NP);
    static constexpr size_t SMEM_A = sizeof(float) * 3 * NWA * STEPA + (size_t)STA * STEPA * ROWB;
    static constexpr size_t SMEM_B = sizeof(float) * 3 * NWB * HX_TILE;
    static constexpr size_t SMEM = SMEM_A > SMEM_B ? SMEM_A : SMEM_B;
};
constexpr int HX_TILES = 3;                       // column tiles ready or being summed
constexpr unsigned int HX_WAIT_LIMIT = 1u << 22;  // polls of one mbarrier phase

__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned int)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned int)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ unsigned int smem_u32(const void *p) { return (unsigned int)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
// One arrival that also announces `bytes` of bulk copies completing on the same phase.
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, unsigned int bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to this CTA's
// shared memory, completing on mbarrier `bar`.
__device__ __forceinline__ void bulk_load(void *smem, const void *gmem, unsigned int bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem)),
                 "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
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
// Waits for the phase of `parity`; false (error raised) when it does not complete in time or another
// wait already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned int parity, DevState *st) {
    for (unsigned int i = 0; i < HX_WAIT_LIMIT; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023u) == 1023u && ld_relaxed_u32(&st->err)) return false;
    }
    raise_error(st, ERR_WAIT_EXPIRED, 0xffffffffu);
    return false;
}

// Giant hubs' rows, feature-major: feature f of a giant hub's row r sits at
// stage[f * R + off + (r & ~1023) + hx_pos<32>(r & 1023)], off its first padded row (a multiple of
// 1,024; rows past the degree are +0) and R all giant hubs' padded rows.  One warp per 32 rows: four
// lanes read a row's four 16-byte pieces together (one request per row), and each store instruction
// fills four features' 8-row runs.
template <int MODE>
__global__ void __launch_bounds__(256) k_hub_stage(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                   const uint32_t *__restrict__ hubs, const uint32_t *__restrict__ off,
                                                   uint32_t n_giant, uint32_t R, const float2 *__restrict__ t01,
                                                   const float *__restrict__ x, float *__restrict__ stage) {
    const int lane = threadIdx.x & 31;
    const uint32_t nchunks = R / 32;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks; c += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t p0 = 32 * c;  // first padded position of the chunk
        uint32_t h = 0;
        while (h + 1 < n_giant && off[h + 1] <= p0) h++;
        const uint32_t u = hubs[h], beg = V[u], d = V[u + 1] - beg;
        const uint32_t r0 = p0 - off[h];  // the chunk's first row (a multiple of 32)
        const uint32_t base = off[h] + (r0 & ~1023u);
        const uint32_t myid = r0 + lane < d ? __ldg(E + beg + r0 + lane) : 0u;
        if (MODE == MODE_INPUT) {
            const uint32_t r = r0 + lane, pos = base + hx_pos<32>(r & 1023u);
            const float2 v = r < d ? __ldg(t01 + myid) : make_float2(0.0f, 0.0f);
            stage[pos] = v.x;
            stage[R + pos] = v.y;
        } else {
            const int q = lane & 3;
            float4 a[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t m = 8 * i + (lane >> 2);  // the row of this lane's piece
                const uint32_t v = __shfl_sync(0xffffffffu, myid, (int)m);
                a[i] = r0 + m < d ? __ldg(reinterpret_cast<const float4 *>(x) + (size_t)v * 4 + q)
                                  : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t m = 8 * i + (lane >> 2);
                const size_t pos = base + hx_pos<32>((r0 + m) & 1023u);
                stage[(size_t)(4 * q + 0) * R + pos] = a[i].x;
                stage[(size_t)(4 * q + 1) * R + pos] = a[i].y;
                stage[(size_t)(4 * q + 2) * R + pos] = a[i].z;
                stage[(size_t)(4 * q + 3) * R + pos] = a[i].w;
            }
        }
    }
}

// A hub item (kind A): hub h, all features.  Producer warp p copies rows [p, p+1) * STEP/NP of each
// step -- four lanes per 64-byte row, one 16-byte piece each, stored at a piece slot XOR-rotated by
// the row so the transpose's loads of 8 consecutive rows hit 8 distinct bank groups -- into a staging
// ring of STA steps (ids read a step ahead), waits for its own copies, writes them as swizzled
// feature columns into the tile ring slot the feature warps released (mbarrier `empty`), and marks
// it full (mbarrier `full`, one arrival per producer warp).  T counts the CTA's kind-A steps over
// all its items, so the barriers' phases continue from item to item.
template <int MODE>
__device__ __forceinline__ bool hub_item(uint32_t h, uint32_t &T, const uint32_t *__restrict__ V,
                                         const uint32_t *__restrict__ E, const uint32_t *__restrict__ hubs,
                                         const float2 *__restrict__ t01, const float *__restrict__ x,
                                         float *__restrict__ sums, unsigned char *smem, uint64_t *full, uint64_t *empty,
                                         DevState *st) {
    using Cfg = HubCfg<MODE>;
    constexpr int NW = Cfg::NWA, VPL = Cfg::VPLA, STEP = Cfg::STEPA, NP = Cfg::NP, ROWB = Cfg::ROWB, STA = Cfg::STA;
    constexpr int LPR = ROWB >= 16 ? ROWB / 16 : 1;  // lanes per row
    constexpr int RPP = STEP / NP;                   // rows per producer warp and step
    constexpr int NI = RPP * LPR / 32;               // copies per lane and step
    constexpr int NID = RPP / 32;                    // row ids per lane and step (lane l: rows l + 32 j)
    float *tiles = reinterpret_cast<float *>(smem);                                 // HX_TILES x NW x STEP
    unsigned char *ring = smem + sizeof(float) * HX_TILES * NW * STEP;               // STA x STEP x ROWB
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t u = hubs[h], beg = V[u], d = V[u + 1] - beg;
    const uint32_t nsteps = (d + STEP - 1) / STEP;
    bool ok = true;
    if (w >= NW) {  // producer
        const uint32_t p = (uint32_t)(w - NW), row0 = p * RPP;
        uint32_t ids[NID];
        auto load_ids = [&](uint32_t t) {
#pragma unroll
            for (int j = 0; j < NID; j++) {
                const uint32_t r = t * STEP + row0 + 32u * j + (uint32_t)lane;
                ids[j] = r < d ? ld_stream(E + beg + r) : 0xffffffffu;
            }
        };
        auto issue = [&](uint32_t t) {  // step t's copies: one commit group, possibly empty
            if (t < nsteps) {
                unsigned char *slot = ring + (size_t)(t % STA) * STEP * ROWB;
#pragma unroll
                for (int i = 0; i < NI; i++) {
                    const uint32_t rel = (uint32_t)(i * 32 + lane) / LPR;  // this lane's row of copy i
                    // its id: held by lane rel % 32 as ids[rel / 32] (rel / 32 is the same in every lane)
                    const uint32_t id = LPR == 1 ? ids[i] : __shfl_sync(0xffffffffu, ids[(i * 32) / LPR / 32], (int)(rel & 31u));
                    const uint32_t row = row0 + rel;
                    if (id != 0xffffffffu) {
                        if (ROWB == 8) {
                            cp_async_8(slot + (size_t)row * 8, t01 + id);
                        } else {
                            const uint32_t q = (uint32_t)lane % LPR, sq = q ^ ((row >> 1) & 3u);
                            cp_async_16(slot + (size_t)row * 64 + 16 * sq, x + (size_t)id * FEAT + 4 * q);
                        }
                    }
                }
            }
            cp_async_commit();
        };
        for (uint32_t t = 0; t + 1 < STA; t++) {
            if (t < nsteps) load_ids(t);
            issue(t);
        }
        if (STA - 1 < nsteps) load_ids(STA - 1);
        for (uint32_t t = 0; t < nsteps; t++, T++) {
            cp_async_wait<STA - 2>();  // step t's copies (this warp's only) have landed
            __syncwarp();
            const uint32_t slot_t = T % HX_TILES;
            if (T >= HX_TILES && !mbar_wait(&empty[slot_t], ((T / HX_TILES) - 1u) & 1u, st)) {
                ok = false;
                break;
            }
            const unsigned char *stg = ring + (size_t)(t % STA) * STEP * ROWB;
            float *tile = tiles + (size_t)slot_t * NW * STEP;
#pragma unroll 2
            for (int i = 0; i < RPP / 32; i++) {  // staged rows -> swizzled columns (rows past the end: +0)
                const uint32_t row = row0 + 32u * i + lane;
                const bool in = t * STEP + row < d;
                const uint32_t pos = hx_pos<VPL>(row);
                if (ROWB == 8) {
                    const float2 v = in ? *reinterpret_cast<const float2 *>(stg + (size_t)row * 8) : make_float2(0.0f, 0.0f);
                    tile[pos] = v.x;
                    tile[STEP + pos] = v.y;
                } else {
#pragma unroll
                    for (uint32_t q = 0; q < 4; q++) {
                        const float4 v = in ? *reinterpret_cast<const float4 *>(stg + (size_t)row * 64 + 16 * (q ^ ((row >> 1) & 3u)))
                                            : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        tile[(4 * q + 0) * STEP + pos] = v.x;
                        tile[(4 * q + 1) * STEP + pos] = v.y;
                        tile[(4 * q + 2) * STEP + pos] = v.z;
                        tile[(4 * q + 3) * STEP + pos] = v.w;
                    }
                }
            }
            __syncwarp();  // the staging slot is read and the tile written by every lane
            if (lane == 0) mbar_arrive(&full[slot_t]);
            const uint32_t tn = t + STA - 1;
            issue(tn);
            if (tn + 1 < nsteps) load_ids(tn + 1);
        }
        cp_async_wait<0>();  // no copy of ours in flight, whatever happened
        __syncwarp();
    } else {  // feature warp w
        float s = 0.0f;
        for (uint32_t t = 0; t < nsteps; t++, T++) {
            const uint32_t slot_t = T % HX_TILES;
            if (!mbar_wait(&full[slot_t], (T / HX_TILES) & 1u, st)) {
                ok = false;
                break;
            }
            exact_step<VPL>(s, tiles + ((size_t)slot_t * NW + w) * STEP, lane);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot_t]);
        }
        if (ok && lane == 0) sums[h * FEAT + (uint32_t)w] = s;
    }
    return ok;
}

// A staged item (kind B): giant hub h, features g*NWB .. g*NWB+NWB-1, from the staging buffer.  Lane 0
// of the first producer warp moves each step's columns with one bulk copy per feature into the tile
// ring (mbarrier `full` carries the byte count); feature warps 0..NWB-1 sum them.  Other warps sit
// the item out.  Before the item ends the producer waits for its copies in flight, so no bulk copy
// outlives the item.  T counts the CTA's kind-B steps (in the warps that take part).
template <int MODE>
__device__ __forceinline__ bool staged_item(uint32_t h, uint32_t g, uint32_t &T, const uint32_t *__restrict__ V,
                                            const uint32_t *__restrict__ hubs, const float *__restrict__ stage,
                                            uint32_t off, uint32_t R, float *__restrict__ sums, unsigned char *smem,
                                            uint64_t *full, uint64_t *empty, DevState *st) {
    using Cfg = HubCfg<MODE>;
    constexpr int NW = Cfg::NWB, NWA = Cfg::NWA;
    constexpr unsigned int COL = sizeof(float) * HX_TILE;
    float *tiles = reinterpret_cast<float *>(smem);  // HX_TILES x NW x HX_TILE
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t u = hubs[h], d = V[u + 1] - V[u];
    const uint32_t nsteps = (d + HX_TILE - 1) / HX_TILE;
    bool ok = true;
    if (w == NWA) {  // the first producer warp
        // the tiles may last have been written through ordinary stores (a hub item): order those
        // before the bulk copies that overwrite them
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        uint32_t t = 0;
        for (; t < nsteps; t++, T++) {
            const uint32_t slot_t = T % HX_TILES;
            if (T >= HX_TILES && !mbar_wait(&empty[slot_t], ((T / HX_TILES) - 1u) & 1u, st)) {
                ok = false;
                break;
            }
            if (lane == 0) {
                mbar_arrive_tx(&full[slot_t], NW * COL);
#pragma unroll
                for (int c = 0; c < NW; c++)
                    bulk_load(tiles + ((size_t)slot_t * NW + c) * HX_TILE,
                              stage + (size_t)(g * NW + c) * R + off + (size_t)t * HX_TILE, COL, &full[slot_t]);
            }
            __syncwarp();
        }
        // the copies of the last (up to HX_TILES) steps issued may still be in flight: wait for them
        for (uint32_t k = 0; k < HX_TILES && k < t; k++) {
            const uint32_t Tk = T - 1u - k;
            mbar_wait(&full[Tk % HX_TILES], (Tk / HX_TILES) & 1u, st);
        }
        __syncwarp();
    } else if (w < NW) {  // feature warp w
        float s = 0.0f;
        for (uint32_t t = 0; t < nsteps; t++, T++) {
            const uint32_t slot_t = T % HX_TILES;
            if (!mbar_wait(&full[slot_t], (T / HX_TILES) & 1u, st)) {
                ok = false;
                break;
            }
            exact_step<32>(s, tiles + ((size_t)slot_t * NW + w) * HX_TILE, lane);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot_t]);
        }
        if (ok && lane == 0) sums[h * FEAT + g * NW + (uint32_t)w] = s;
    }
    return ok;
}

// The dense part of hub h from its 16 feature sums (input layer: the two layer-0 sums), by one warp.
template <int MODE>
__device__ __forceinline__ void hub_dense(uint32_t h, const uint32_t *__restrict__ V, const uint32_t *__restrict__ hubs,
                                          const float2 *__restrict__ t01, const float *__restrict__ x,
                                          float *__restrict__ y, uint32_t *__restrict__ key,
                                          const float *__restrict__ Wb, const float *__restrict__ sums, int lane) {
    const uint32_t u = hubs[h], d = V[u + 1] - V[u];
    const float fd = __uint2float_rn(d);
    const int j = lane & 15;
    float c = __ldg(Wb + 2 * FEAT * FEAT + j);
    if (MODE == MODE_INPUT) {
        float s0 = __ldcg(sums + h * FEAT), s1 = __ldcg(sums + h * FEAT + 1);
        if (fd > 0.0f) {
            s0 = __fdiv_rn(s0, fd);
            s1 = __fdiv_rn(s1, fd);
        }
        const float2 self = t01[h];  // hub h's feature row is h
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const float a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self.x : self.y));
            c = __fmaf_rn(__ldg(Wb + i * FEAT + j), a, c);
        }
    } else {
        float nb = __ldcg(sums + h * FEAT + j);
        if (fd > 0.0f) nb = __fdiv_rn(nb, fd);
        const float self = x[(size_t)h * FEAT + j];
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
        y[(size_t)h * FEAT + lane] = o;
    }
}

// Hubs (more than the hub degree), before each layer kernel: persistent CTAs take items from a
// counter -- the giant hubs' staged items first (heaviest first), then one hub item per other hub,
// by descending degree.  The hub's last item to finish (a counter per hub, zeroed before the layer)
// runs the dense part: mean, 32 x 16 FMA chain in order, ReLU, and in the output layer the
// reference's fixed-tree sum into the key.
template <int MODE>
__global__ void __launch_bounds__(HubCfg<MODE>::THREADS) k_gnn_hubx(
    const uint32_t *__restrict__ V, const uint32_t *__restrict__ E, const uint32_t *__restrict__ hubs,
    const float2 *__restrict__ t01, const float *__restrict__ x, float *__restrict__ y, uint32_t *__restrict__ key,
    const float *__restrict__ Wb, float *__restrict__ sums, uint32_t *__restrict__ done, uint32_t *__restrict__ items,
    uint32_t n_hubs, uint32_t n_giant, const float *__restrict__ stage, const uint32_t *__restrict__ stage_off,
    uint32_t R, DevState *st) {
    using Cfg = HubCfg<MODE>;
    extern __shared__ __align__(16) unsigned char hx_smem[];
    __shared__ __align__(8) uint64_t full_a[HX_TILES], empty_a[HX_TILES], full_b[HX_TILES], empty_b[HX_TILES];
    __shared__ uint32_t item_s, last_s;
    if (threadIdx.x == 0) {
        for (int i = 0; i < HX_TILES; i++) {
            mbar_init(&full_a[i], Cfg::NP);
            mbar_init(&empty_a[i], Cfg::NWA);
            mbar_init(&full_b[i], 1);
            mbar_init(&empty_b[i], Cfg::NWB);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t Ta = 0, Tb = 0;  // this thread's count of the CTA's steps of each kind
    const uint32_t n_staged = n_giant * Cfg::NGB;
    const uint32_t n_items = n_staged + (n_hubs - n_giant);
    for (;;) {
        if (threadIdx.x == 0) item_s = atomicAdd(items, 1u);
        __syncthreads();
        const uint32_t it = item_s;
        if (it >= n_items) return;
        uint32_t h, parts;
        bool ok;
        if (it < n_staged) {
            h = it / Cfg::NGB;
            parts = Cfg::NGB;
            ok = staged_item<MODE>(h, it % Cfg::NGB, Tb, V, hubs, stage, stage_off[h], R, sums, hx_smem, full_b,
                                   empty_b, st);
        } else {
            h = n_giant + (it - n_staged);
            parts = 1;
            ok = hub_item<MODE>(h, Ta, V, E, hubs, t01, x, sums, hx_smem, full_a, empty_a, st);
        }
        if (__syncthreads_or(!ok)) return;  // a wait gave up: the error is raised
        if (threadIdx.x == 0) {
            __threadfence();
            last_s = atomicAdd(done + h, 1u) == parts - 1;
        }
        __syncthreads();
        if (last_s && threadIdx.x < 32) {
            __threadfence();
            hub_dense<MODE>(h, V, hubs, t01, x, y, key, Wb, sums, threadIdx.x);
        }
    }
}

template <int MODE>
gc_status launch_layer(gc_graph *g, const float *Wb, const float *Wh, const float *x, float *y, uint32_t n_iso) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    // counters, zeroed for each layer: warp-tier vertices (0), leading four-lane items (1), the rest
    // (2), thin groups (5)
    uint32_t *ctr = g->gnn_ctr;
    if ((s = gc_check_cuda(ctx, cudaMemsetAsync(ctr, 0, 8 * sizeof(uint32_t), ctx->stream), "gnn work counters")) !=
        GC_OK)
        return s;
    // hubs: persistent CTAs on a high-priority side stream beside the layer kernel, whose grid then
    // leaves one CTA per SM (GC_GNN_HUB_SIDE=0: before it, on the library's stream)
    if (g->n_hubs) {
        using Cfg = HubCfg<MODE>;
        float *sums = reinterpret_cast<float *>(g->hub_aux);
        uint32_t *done = g->hub_aux + (size_t)FEAT * g->n_hubs;  // n_hubs counters, then the item counter
        if ((s = gc_check_cuda(ctx, cudaMemsetAsync(done, 0, sizeof(uint32_t) * (g->n_hubs + 1), ctx->stream),
                               "hub counters")) != GC_OK)
            return s;
        cudaStream_t side = ctx->hub_stream ? ctx->hub_stream : ctx->stream;
        if (side != ctx->stream) {
            if ((s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream), "fork")) != GC_OK) return s;
            if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(side, ctx->ev_fork, 0), "fork")) != GC_OK) return s;
        }
        ProfScope ph(ctx, MODE == MODE_INPUT ? "gnn_hub_input" : (MODE == MODE_HIDDEN ? "gnn_hub_hidden" : "gnn_hub_output"),
                     side);
        if (g->n_giant) {  // the giant hubs' rows, staged by the whole GPU
            k_hub_stage<MODE><<<ctx->num_sms * 8, 256, 0, side>>>(g->V, g->Er, g->hubs, g->giant_off, g->n_giant,
                                                                  g->giant_rows, g->t01, x, g->hub_stage);
            ctx->launches++;
        }
        int &occ = ctx->hub_blocks_per_sm[MODE];
        if (!occ) {  // once per context: keeps these calls out of captured sequences
            if ((s = gc_check_cuda(ctx, cudaFuncSetAttribute(k_gnn_hubx<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             (int)Cfg::SMEM),
                                   "hub smem")) != GC_OK)
                return s;
            if ((s = gc_check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gnn_hubx<MODE>, Cfg::THREADS,
                                                                                      Cfg::SMEM),
                                   "hub occupancy")) != GC_OK)
                return s;
            if (occ < 1) occ = 1;
        }
        // CTAs per SM: as many as fit, at most GC_GNN_HUB_CTAS when set
        const uint32_t per_sm = ctx->gnn_hub_ctas_per_sm ? std::min<uint32_t>(ctx->gnn_hub_ctas_per_sm, (uint32_t)occ)
                                                         : (uint32_t)occ;
        const uint32_t n_items = g->n_giant * Cfg::NGB + (g->n_hubs - g->n_giant);
        const uint32_t grid = std::min<uint32_t>((uint32_t)ctx->num_sms * per_sm, n_items);
        k_gnn_hubx<MODE><<<grid, Cfg::THREADS, Cfg::SMEM, side>>>(g->V, g->Er, g->hubs, g->t01, x, y, g->key, Wb, sums,
                                                                 done, done + g->n_hubs, g->n_hubs, g->n_giant,
                                                                 g->hub_stage, g->giant_off, g->giant_rows, ctx->dstate);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "gnn hubs")) != GC_OK) return s;
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
        const int bb = g->n_hubs && ctx->hub_stream && blocks > 1 ? blocks - 1 : blocks;
        if (first_thin) {
            k_gnn_layer<MODE><<<ctx->num_sms * bb, GNN_THREADS, 0, ctx->stream>>>(
                g->vrow, g->Er, g->vorder, g->n_hubs, g->n_wide_gnn, first_thin, g->t01, x, y, g->key, Wb, ctr,
                ctx->gnn_grab, ctx->gnn_heavy);
            ctx->launches++;
        }
        const uint32_t end_thin = g->n_vorder - n_iso;
        if (end_thin > first_thin) {
            const uint32_t grid = std::min<uint32_t>((uint32_t)ctx->num_sms * 3,
                                                     (end_thin - first_thin + THIN_THREADS - 1) / THIN_THREADS);
            LayerArg la;
            memcpy(la.w, Wh, sizeof(la.w));
            k_gnn_thin<MODE><<<grid, THIN_THREADS, 0, ctx->stream>>>(g->vrow, g->Er, g->vorder, g->n_hubs, first_thin,
                                                                     end_thin, g->t01, x, y, g->key, la, ctr + 5,
                                                                     ctx->gnn_grab);
            ctx->launches++;
        }
    }
    if ((s = gc_check_launch(ctx, "gnn layer")) != GC_OK) return s;
    if (g->n_hubs && ctx->hub_stream) {
        if ((s = gc_check_cuda(ctx, cudaEventRecord(ctx->ev_join, ctx->hub_stream), "join")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0), "join")) != GC_OK) return s;
    }
    return GC_OK;
}

}  // namespace

gc_status gc_gnn_rows_begin(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    const size_t rows = (size_t)g->cap_N;
    if ((s = gc_alloc(ctx, &g->row_of, rows, "feature rows")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->Er, (size_t)g->cap_M, "neighbour rows")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->vrow, rows, "row offsets")) != GC_OK) return s;
    if (g->N == 0) return GC_OK;
    k_gnn_rows<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->hubs, g->n_hubs, g->vorder, g->n_vorder, g->row_of,
                                                           g->vrow);
    ctx->launches++;
    return gc_check_launch(ctx, "gnn feature rows");
}

gc_status gc_gnn_row_ids(gc_graph *g, uint32_t first, uint32_t count) {
    gc_ctx *ctx = g->ctx;
    if (!count) return GC_OK;
    const uint32_t grid = std::min<uint32_t>((uint32_t)ctx->num_sms * 8, (count + 255) / 256);
    k_gnn_row_ids<<<grid, 256, 0, ctx->stream>>>(g->E, first, count, g->N, g->row_of, g->Er, ctx->dstate);
    ctx->launches++;
    return gc_check_launch(ctx, "gnn neighbour rows");
}

gc_status gc_priority_gnn(gc_graph *g, const gc_model *m) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (!m || m->layers < 2) return gc_fail(ctx, GC_ERR_INVALID, "GNN needs a model with at least 2 layers");
    if (g->N == 0) return GC_OK;
    const size_t rows = (size_t)g->cap_N;
    if ((s = gc_alloc(ctx, &g->x, rows * FEAT, "gnn features")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->y, rows * FEAT, "gnn features")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->t01, rows, "gnn input table")) != GC_OK) return s;
    // hubs' feature sums (16 per hub), completion counters (one per hub) and the item counter
    if (g->n_hubs && g->hub_aux_cap < (size_t)(FEAT + 1) * g->n_hubs + 1) {
        gc_dev_free(ctx, g->hub_aux);
        g->hub_aux = nullptr;
        if ((s = gc_alloc(ctx, &g->hub_aux, (size_t)(FEAT + 1) * g->n_hubs + 1, "hub sums")) != GC_OK) return s;
        g->hub_aux_cap = (size_t)(FEAT + 1) * g->n_hubs + 1;
    }
    if (g->n_giant && g->hub_stage_cap < (size_t)FEAT * g->giant_rows) {  // staged rows of the giant hubs
        gc_dev_free(ctx, g->hub_stage);
        g->hub_stage = nullptr;
        if ((s = gc_alloc(ctx, &g->hub_stage, (size_t)FEAT * g->giant_rows, "giant hub rows")) != GC_OK) return s;
        g->hub_stage_cap = (size_t)FEAT * g->giant_rows;
    }
    if (g->n_hubs && ctx->gnn_hub_side && !ctx->hub_stream) {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if ((s = gc_check_cuda(ctx, cudaStreamCreateWithPriority(&ctx->hub_stream, cudaStreamNonBlocking, hi),
                               "hub stream")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
        if ((s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming), "event")) != GC_OK)
            return s;
    }
    if ((s = gc_alloc(ctx, &g->gnn_ctr, 8, "gnn work counters")) != GC_OK) return s;
    if (!g->rows_ready) {  // once per upload: the feature-row order and the neighbour ids as rows
        ProfScope ps(ctx, "gnn_rows", ctx->stream);
        if ((s = gc_gnn_rows_begin(g)) != GC_OK) return s;
        if ((s = gc_gnn_row_ids(g, 0, g->M)) != GC_OK) return s;
        g->rows_ready = true;
    }
    {
        ProfScope ps(ctx, "gnn_table0", ctx->stream);
        k_gnn_table0<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->V, g->N, (float)m->md, g->seg_voff, g->n_seg,
                                                                 g->row_of, g->t01);
    }
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "gnn input table")) != GC_OK) return s;
    const int L = m->layers;
    const uint32_t n_iso = ctx->gnn_fuse_isolated && L <= ISO_MAX_LAYERS ? g->n_iso : 0u;
    if (n_iso) {
        ProfScope ps(ctx, "gnn_isolated", ctx->stream);
        const uint32_t first = g->n_vorder - g->n_iso;
        const uint32_t grid = std::min<uint32_t>((uint32_t)ctx->num_sms * 4, (g->n_iso + ISO_THREADS - 1) / ISO_THREADS);
        const size_t smem = sizeof(float) * LAYER_PARAMS * (size_t)L;
        k_gnn_isolated<<<grid, ISO_THREADS, smem, ctx->stream>>>(g->vorder, g->n_hubs, first, g->n_vorder, g->t01,
                                                                 g->key, m->d_param, L);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "gnn isolated vertices")) != GC_OK) return s;
    }
    float *x = g->x, *y = g->y;
    for (int l = 0; l < L; l++) {
        const float *Wb = m->d_param + (size_t)l * LAYER_PARAMS, *Wh = m->h_param + (size_t)l * LAYER_PARAMS;
        if (l == 0)
            s = launch_layer<MODE_INPUT>(g, Wb, Wh, nullptr, y, n_iso);
        else if (l < L - 1)
            s = launch_layer<MODE_HIDDEN>(g, Wb, Wh, x, y, n_iso);
        else
            s = launch_layer<MODE_OUTPUT>(g, Wb, Wh, x, nullptr, n_iso);
        if (s != GC_OK) return s;
        float *t = x;
        x = y;
        y = t;
    }
    return GC_OK;
}
