// GraphSAGE-16 priorities for callers that must not allocate device memory.
//
// gc_gnn_priority_noalloc computes the same FP32 priorities as gc_priority(GC_GNN) -- the
// reference's fast_gnn.c arithmetic, bit for bit -- for a CSR and a model that the caller already
// holds in device memory, writing one float per vertex into a caller-provided device buffer.  Its
// only scratch (two feature planes and the layer-0 inputs) is the file-scope device array below,
// so the call performs no cudaMalloc, cudaFree or other allocating call.
//
// Who needs this: code that runs where a device allocation is not allowed or not affordable --
// a serving loop that reserved its whole HBM budget up front and may not grow it per request, a
// host framework that owns all device memory and hands plugins only its own buffers, or a
// latency-critical path where cudaMalloc's implicit device synchronisation is unacceptable.
//
// Limits and sharing:
//   - at most GC_NOALLOC_MAX_VERTICES vertices (larger graphs are rejected with GC_ERR_INVALID);
//   - the array lives on every device that loads this library, until the process exits;
//   - every call uses the same array and leaves its last contents there.  Each call writes every
//     element it reads before reading it, so nothing has to start at zero; but two calls whose
//     kernels overlap on a device (different streams, or different host threads) race on it.
//   - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current, and loads every kernel of this entry point (cudaFuncGetAttributes on
//     each), so that under CUDA's lazy module loading a later call -- say a 3-layer model after a
//     2-layer one -- loads no code and allocates nothing; make that first call before any stream
//     capture.
//   - each kernel launch is checked through the status cudaLaunchKernelEx returns for that launch:
//     an error left pending by the caller's earlier work is neither reported as this call's nor
//     cleared.
#include <mutex>

#include "gc_device.cuh"
#include "gnn_coloring.h"

namespace {
using namespace gc;

constexpr uint32_t MAX_V = GC_NOALLOC_MAX_VERTICES;
// x plane, y plane (MAX_V x 16 floats each), then the layer-0 inputs (MAX_V float2)
constexpr size_t SCRATCH_FLOATS = 2 * (size_t)MAX_V * FEAT + 2 * (size_t)MAX_V;
static __device__ __align__(256) float g_noalloc_scratch[SCRATCH_FLOATS];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
float *g_scratch_addr[MAX_DEVICES] = {};
int g_sms[MAX_DEVICES] = {};

enum : int { NA_INPUT = 0, NA_HIDDEN = 1, NA_OUTPUT = 2 };

__global__ void k_na_table0(const uint32_t *__restrict__ V, uint32_t N, float fmd, float2 *__restrict__ t01) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t d = V[u + 1] - V[u];
        t01[u] = make_float2(__fdiv_rn(__uint2float_rn(d), fmd), __double2float_rn(__ddiv_rn((double)u, (double)N)));
    }
}

// Half a warp per vertex, lane = feature: sequential neighbour sums in CSR order, the 32x16 FMA
// chain, ReLU, and for the last layer the reference's fixed-tree output sum.
template <int MODE>
__global__ void __launch_bounds__(256) k_na_layer(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                  uint32_t N, const float2 *__restrict__ t01,
                                                  const float *__restrict__ x, float *__restrict__ y,
                                                  float *__restrict__ p, const float *__restrict__ Wb) {
    __shared__ float sW[LAYER_PARAMS];
    for (int i = threadIdx.x; i < LAYER_PARAMS; i += blockDim.x) sW[i] = Wb[i];
    __syncthreads();
    const int lane = threadIdx.x & 15;
    const unsigned int hmask = 0xffffu << (threadIdx.x & 16);
    const uint32_t groups = (gridDim.x * blockDim.x) >> 4;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; u < N; u += groups) {
        const uint32_t beg = V[u], end = V[u + 1];
        const float fd = __uint2float_rn(end - beg);
        float a_nb = 0.0f, a_self = 0.0f, s0 = 0.0f, s1 = 0.0f, self0 = 0.0f, self1 = 0.0f;
        if (MODE == NA_INPUT) {
            for (uint32_t b = beg; b < end; b += 16) {
                const uint32_t cnt = min(16u, end - b);
                float2 t = make_float2(0.0f, 0.0f);
                if ((uint32_t)lane < cnt) t = t01[E[b + lane]];
                for (uint32_t k = 0; k < 16; k++) {
                    const float a0 = __shfl_sync(hmask, t.x, k, 16), a1 = __shfl_sync(hmask, t.y, k, 16);
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
            self0 = t01[u].x;
            self1 = t01[u].y;
        } else {
            for (uint32_t b = beg; b < end; b += 16) {
                const uint32_t cnt = min(16u, end - b);
                const uint32_t e = (uint32_t)lane < cnt ? E[b + lane] : 0u;
                for (uint32_t k = 0; k < 16; k++) {
                    const uint32_t v = __shfl_sync(hmask, e, k, 16);
                    if (k < cnt) a_nb = __fadd_rn(a_nb, x[(size_t)v * FEAT + lane]);
                }
            }
            if (fd > 0.0f) a_nb = __fdiv_rn(a_nb, fd);
            a_self = x[(size_t)u * FEAT + lane];
        }
        float c = sW[2 * FEAT * FEAT + lane];
        for (int i = 0; i < 2 * FEAT; i++) {
            float a;
            if (MODE == NA_INPUT) a = i < 8 ? s0 : (i < 16 ? s1 : (i < 24 ? self0 : self1));
            else a = __shfl_sync(hmask, i < FEAT ? a_nb : a_self, i & 15, 16);
            c = __fmaf_rn(sW[i * FEAT + lane], a, c);
        }
        const float o = c > 0.0f ? c : 0.0f;
        if (MODE == NA_OUTPUT) {
            const float t = __fadd_rn(o, __shfl_down_sync(hmask, o, 8, 16));  // t_k = o_k + o_{k+8}
            const float q = __fadd_rn(t, __shfl_down_sync(hmask, t, 1, 16));
            const float r = __fadd_rn(q, __shfl_down_sync(hmask, q, 2, 16));
            const float sum = __fadd_rn(r, __shfl_down_sync(hmask, r, 4, 16));
            if (lane == 0) p[u] = sum;
        } else {
            y[(size_t)u * FEAT + lane] = o;
        }
    }
}

// Device address of the scratch array for the current device, looked up once per device; the same
// first call loads this entry point's kernels and reads the SM count.
gc_status scratch_for_current_device(float **out, int *sms_out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return GC_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        cudaFuncAttributes fa;
        int sms = 0;
        bool ok = cudaGetSymbolAddress(&ptr, g_noalloc_scratch) == cudaSuccess && ptr;
        ok = ok && cudaFuncGetAttributes(&fa, k_na_table0) == cudaSuccess;
        ok = ok && cudaFuncGetAttributes(&fa, k_na_layer<NA_INPUT>) == cudaSuccess;
        ok = ok && cudaFuncGetAttributes(&fa, k_na_layer<NA_HIDDEN>) == cudaSuccess;
        ok = ok && cudaFuncGetAttributes(&fa, k_na_layer<NA_OUTPUT>) == cudaSuccess;
        ok = ok && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0;
        if (!ok) {
            cudaGetLastError();  // the failed set-up call's own error
            return GC_ERR_CUDA;
        }
        g_sms[dev] = sms;
        g_scratch_addr[dev] = static_cast<float *>(ptr);
    }
    *out = g_scratch_addr[dev];
    *sms_out = g_sms[dev];
    return GC_OK;
}

// One launch, checked by the status of that launch alone.
template <typename... KArgs, typename... Args>
gc_status launch(void (*kernel)(KArgs...), int grid, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    if (cudaLaunchKernelEx(&cfg, kernel, args...) != cudaSuccess) {
        cudaGetLastError();  // this launch's error, not the caller's
        return GC_ERR_CUDA;
    }
    return GC_OK;
}

}  // namespace

extern "C" gc_status gc_gnn_priority_noalloc(uint32_t N, const uint32_t *dV, const uint32_t *dE, int params, int md,
                                             const float *dparam, float *dp, void *stream) {
    if (N > MAX_V) return GC_ERR_INVALID;  // beyond the fixed scratch: use gc_priority instead
    if (params / LAYER_PARAMS < 2 || !dparam) return GC_ERR_INVALID;
    if (N == 0) return GC_OK;
    if (!dV || !dE || !dp) return GC_ERR_INVALID;
    float *scratch = nullptr;
    int sms = 0;
    gc_status s = scratch_for_current_device(&scratch, &sms);
    if (s != GC_OK) return s;
    float *xa = scratch, *ya = scratch + (size_t)MAX_V * FEAT;
    float2 *t01 = reinterpret_cast<float2 *>(scratch + 2 * (size_t)MAX_V * FEAT);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int L = params / LAYER_PARAMS;
    const int grid = sms * 8;
    if ((s = launch(k_na_table0, grid, st, dV, N, (float)md, t01)) != GC_OK) return s;
    float *x = xa, *y = ya;
    const float2 *t = t01;
    const float *none_in = nullptr;
    float *none_out = nullptr;
    for (int l = 0; l < L && s == GC_OK; l++) {
        const float *Wb = dparam + (size_t)l * LAYER_PARAMS;
        const float *xc = x;
        if (l == 0) s = launch(k_na_layer<NA_INPUT>, grid, st, dV, dE, N, t, none_in, y, none_out, Wb);
        else if (l < L - 1) s = launch(k_na_layer<NA_HIDDEN>, grid, st, dV, dE, N, t, xc, y, none_out, Wb);
        else s = launch(k_na_layer<NA_OUTPUT>, grid, st, dV, dE, N, t, xc, none_out, dp, Wb);
        float *tmp = x;
        x = y;
        y = tmp;
    }
    return s;
}
