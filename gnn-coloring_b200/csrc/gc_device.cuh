// Device-side helpers shared by the coloring kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gc {

constexpr int FEAT = 16;           // GraphSAGE width (reference src/fast_gnn.c:6)
constexpr int LAYER_PARAMS = 528;  // 32x16 weights + 16 biases per layer (src/fast_gnn.c:256)
constexpr int WARP = 32;

// Device-side status block, one per context.  Kernels report problems by OR-ing a code into
// `err` and recording where in `err_info`; the host reads it after a launch sequence.
struct DevState {
    unsigned int ticket;      // next ticket of the ordered coloring kernel
    unsigned int err;         // error bits (DevErr)
    unsigned int err_info;    // vertex (or index) where the first error was seen
    unsigned int invalid;     // validation: non-zero if the coloring is improper
    unsigned int max_color;   // validation / coloring: largest color
    unsigned int count;       // generic counter (frontier sizes, compaction)
    unsigned int count2;      // generic counter
    unsigned int min_deg;     // SL peeling: smallest remaining degree
    unsigned int ordered;     // coloring: vertices that go through the ordered kernel
    unsigned int big_leaves;  // coloring: leaves with too many neighbours for one thread
    unsigned int thin;        // preparation: vertices with at most the GNN thin-tier degree
    unsigned int gnn_wide;    // preparation: vertices in the GNN warp tier
    unsigned int ticket_light;  // coloring: next ticket of the light stream
    unsigned int n_heavy;       // coloring: tickets of the heavy stream (after the core)
    unsigned int n_light;       // coloring: tickets of the light stream (after the core)
    unsigned int isolated;      // preparation: vertices without neighbours (outside the hub list)
};

enum DevErr : unsigned int {
    ERR_WAIT_EXPIRED = 1u,   // a bounded wait for a predecessor's color gave up
    ERR_BOUND = 2u,          // an index or size bound was exceeded
    ERR_ORDER = 4u,          // internal ordering invariant violated
};

// Relaxed GPU-scope accesses: the value itself is the payload, so no fences are needed; these
// bypass L1 so a waiting warp sees another SM's store.
__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(int *p, int v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Streaming load (evict-first): CSR edge arrays are read once per pass.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }

// An L2 policy that keeps the lines it loads (evict-last), for small arrays gathered at random
// beside a large stream (an instruction hint: no device setting changes).
__device__ __forceinline__ uint64_t l2_keep_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Read-only load under that policy.
__device__ __forceinline__ uint32_t ld_keep(const uint32_t *p, uint64_t pol) {
    uint32_t v;
    asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ void raise_error(DevState *st, unsigned int code, unsigned int info) {
    if (atomicOr(&st->err, code) == 0) st->err_info = info;
}

// v precedes u: larger key first, ties to the smaller vertex id (src/coloring.c:249 puts v
// among u's predecessors when p[v] > p[u] || (p[u] == p[v] && u > v)).
__device__ __forceinline__ bool precedes(uint32_t kv, uint32_t v, uint32_t ku, uint32_t u) {
    return kv > ku || (kv == ku && v < u);
}

// Segment of vertex u in a segmented CSR: the s with voff[s] <= u < voff[s + 1] (empty segments
// are skipped).  Requires voff[0] = 0 <= u < voff[nseg].
__device__ __forceinline__ uint32_t seg_of(const uint32_t *__restrict__ voff, uint32_t nseg, uint32_t u) {
    uint32_t lo = 0, hi = nseg;  // voff[lo] <= u < voff[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(voff + mid) <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

}  // namespace gc
