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
//                Early decisions shorten the waits (the critical path is the DAG's depth): a warp
//                with few predecessors left takes the candidate c = mex(colors seen so far) at once
//                when every pending predecessor v provably cannot end up with color c, because
//                pc[v] + 1 < c (v's color is at most its predecessor count + 1) or because one of
//                v's own predecessors already has color c (v's color is the mex of those).  The
//                second fact comes from v's warp, which publishes the colors it has seen
//                (colors 1..256) while it waits.  Every published bit is a final color, so the
//                decision is exact: the final mex is c whatever the pending colors turn out to be.
//
// Colors are published with relaxed GPU-scope stores and read with relaxed GPU-scope loads: the
// color value is itself the whole message, so no fences are needed.
#include <algorithm>
#include <vector>
#include <cstdlib>

#include "gc_internal.h"

gc_status gc_sort_order_bits(gc_graph *g, int key_bits, bool filter, uint32_t *d_count);

namespace {
using namespace gc;

// Split in the GNN's degree order (built at upload): the first n_wide vertices (more than
// GC_GNN_WARP_DEGREE neighbours) one per warp, the rest eight per warp with four lanes each.  A
// vertex is owned by one warp or quad, so its predecessors are packed with ballots alone.  Hubs
// (not in the degree order) are split by k_jp_split_big.
__global__ void __launch_bounds__(256) k_jp_split(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                  const uint32_t *__restrict__ key, const uint32_t *__restrict__ vorder,
                                                  uint32_t n_wide, uint32_t n_vorder, uint32_t *__restrict__ P,
                                                  uint32_t *__restrict__ pc) {
    const int lane = threadIdx.x & 31, q = lane & 3, qbase = lane & ~3;
    const unsigned int lt = (1u << lane) - 1u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n_items = n_wide + (n_vorder - n_wide + 7) / 8;
    for (uint32_t it = warp; it < n_items; it += nwarps) {
        if (it < n_wide) {
            const uint32_t u = vorder[it];
            const uint32_t beg = V[u], d = V[u + 1] - beg, ku = key[u];
            uint32_t cnt = 0;
            for (uint32_t c = 0; c < d; c += 64) {
                const uint32_t ia = c + lane, ib = c + 32 + lane;
                const uint32_t va = ia < d ? ld_stream(E + beg + ia) : 0u, vb = ib < d ? ld_stream(E + beg + ib) : 0u;
                const bool pa = ia < d && precedes(__ldg(key + va), va, ku, u);
                const bool pb = ib < d && precedes(__ldg(key + vb), vb, ku, u);
                const unsigned int ma = __ballot_sync(0xffffffffu, pa);
                if (pa) P[beg + cnt + __popc(ma & lt)] = va;
                cnt += __popc(ma);
                const unsigned int mb = __ballot_sync(0xffffffffu, pb);
                if (pb) P[beg + cnt + __popc(mb & lt)] = vb;
                cnt += __popc(mb);
            }
            if (lane == 0) pc[u] = cnt;
            continue;
        }
        const uint32_t slot = n_wide + (it - n_wide) * 8 + (lane >> 2);
        const bool valid = slot < n_vorder;
        const uint32_t u = valid ? vorder[slot] : 0u;
        const uint32_t beg = valid ? V[u] : 0u, d = valid ? V[u + 1] - beg : 0u;
        const uint32_t ku = valid ? key[u] : 0u;
        const uint32_t dmax = __reduce_max_sync(0xffffffffu, d);
        const unsigned int qlt = (1u << q) - 1u;
        uint32_t cnt = 0;
        for (uint32_t c = 0; c < dmax; c += 4) {
            const uint32_t i = c + q;
            const uint32_t v = i < d ? ld_stream(E + beg + i) : 0u;
            const bool p = i < d && precedes(__ldg(key + v), v, ku, u);
            const unsigned int qm = (__ballot_sync(0xffffffffu, p) >> qbase) & 0xfu;
            if (p) P[beg + cnt + __popc(qm & qlt)] = v;
            cnt += __popc(qm);
        }
        if (valid && q == 0) pc[u] = cnt;
    }
}

__global__ void k_zero_hub_counts(const uint32_t *__restrict__ hubs, uint32_t n, uint32_t *__restrict__ pc) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pc[hubs[i]] = 0;
}

// Hubs: one warp per GC_SPLIT_CHUNK-edge chunk.  The warp gathers its chunk's
// predecessors in shared memory, reserves their slots with one atomic on pc[u], then writes them
// out coalesced (predecessor order within P does not matter).
constexpr int SPLIT_WARPS = 8;
__global__ void __launch_bounds__(SPLIT_WARPS * 32) k_jp_split_big(const uint32_t *__restrict__ V,
                                                                   const uint32_t *__restrict__ E,
                                                                   const uint32_t *__restrict__ key,
                                                                   const uint32_t *__restrict__ tasks, uint32_t n_tasks,
                                                                   uint32_t *__restrict__ P, uint32_t *__restrict__ pc) {
    __shared__ uint32_t buf[SPLIT_WARPS][GC_SPLIT_CHUNK];
    const int lane = threadIdx.x & 31;
    uint32_t *mine = buf[threadIdx.x >> 5];
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned int lt = (1u << lane) - 1u;
    for (uint32_t t = warp; t < n_tasks; t += nwarps) {
        const uint32_t u = tasks[2 * t], e0 = tasks[2 * t + 1];
        const uint32_t end = min(V[u + 1], e0 + GC_SPLIT_CHUNK);
        const uint32_t ku = key[u];
        uint32_t cnt = 0;
        for (uint32_t i0 = e0; i0 < end; i0 += 64) {
            const uint32_t ia = i0 + lane, ib = i0 + 32 + lane;
            const uint32_t va = ia < end ? ld_stream(E + ia) : 0u, vb = ib < end ? ld_stream(E + ib) : 0u;
            const bool pa = ia < end && precedes(__ldg(key + va), va, ku, u);
            const bool pb = ib < end && precedes(__ldg(key + vb), vb, ku, u);
            const unsigned int ma = __ballot_sync(0xffffffffu, pa);
            if (pa) mine[cnt + __popc(ma & lt)] = va;
            cnt += __popc(ma);
            const unsigned int mb = __ballot_sync(0xffffffffu, pb);
            if (pb) mine[cnt + __popc(mb & lt)] = vb;
            cnt += __popc(mb);
        }
        __syncwarp();
        uint32_t slot = 0;
        if (lane == 0 && cnt) slot = atomicAdd(&pc[u], cnt);
        slot = __shfl_sync(0xffffffffu, slot, 0);
        uint32_t *out = P + V[u] + slot;
        for (uint32_t j = lane; j < cnt; j += 32) out[j] = mine[j];
        __syncwarp();
    }
}

// Sources (no predecessor) take color 1 now; everything else starts uncolored.
__global__ void k_jp_init_colors(const uint32_t *__restrict__ pc, uint32_t N, int *__restrict__ color) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
        color[u] = pc[u] == 0 ? 1 : 0;
}

constexpr int COLOR_THREADS = 256;
constexpr int COLOR_WARPS = COLOR_THREADS / 32;
constexpr uint32_t WINDOW = 1024;   // colors covered by one pass over the predecessors
constexpr int TRACK = 64;           // per lane: predecessors whose wait is tracked in a bitmask
constexpr int LOADS = 4;            // predecessor colors in flight per lane

__device__ __forceinline__ void mark(uint32_t *fb, int c, uint32_t window) {
    const uint32_t idx = (uint32_t)(c - 1) - window * WINDOW;
    if (idx < WINDOW) atomicOr(&fb[idx >> 5], 1u << (idx & 31));
}

// Smallest free color of the window from the warp's shared bitmap; 0 if the window is full.
__device__ __forceinline__ int window_mex(const uint32_t *fb, int lane, uint32_t window) {
    const uint32_t free_bits = ~fb[lane];
    const unsigned int has = __ballot_sync(0xffffffffu, free_bits != 0);
    if (!has) return 0;
    const int l = __ffs(has) - 1;
    const uint32_t fw = __shfl_sync(0xffffffffu, free_bits, l);
    return (int)(window * WINDOW + (uint32_t)l * 32 + (uint32_t)(__ffs(fw) - 1) + 1);
}

// Colors one vertex whose predecessors are list[0..cnt): the smallest color >= 1 none of them
// has.  Predecessor colors are loaded without waiting first (LOADS per lane in flight); lane
// entries found uncolored are remembered in a bitmask (the first TRACK entries of each lane) and
// polled until they are colored, so a warp waiting on its last predecessor re-reads one word, not
// the whole list.  Entries beyond TRACK per lane (lists longer than 32 * TRACK) are waited on in
// place.  Returns -1 when a wait exceeded spin_limit polls or another warp raised the error flag.
__device__ int color_one(const uint32_t *__restrict__ list, uint32_t cnt, const int *color, uint32_t *fb, int lane,
                         DevState *st, unsigned int spin_limit) {
    for (uint32_t window = 0;; window++) {
        fb[lane] = 0;
        __syncwarp();
        unsigned long long waiting = 0;  // bit k: entry lane + 32k still uncolored
        bool gave_up = false;
        for (uint32_t j0 = 0; j0 < cnt && !gave_up; j0 += 32 * LOADS) {
            uint32_t v[LOADS];
            int c[LOADS];
#pragma unroll
            for (int q = 0; q < LOADS; q++) {
                const uint32_t j = j0 + q * 32 + lane;
                v[q] = j < cnt ? __ldg(list + j) : 0xffffffffu;
            }
#pragma unroll
            for (int q = 0; q < LOADS; q++) c[q] = v[q] != 0xffffffffu ? ld_relaxed(color + v[q]) : -1;
#pragma unroll
            for (int q = 0; q < LOADS; q++) {
                if (c[q] > 0) {
                    mark(fb, c[q], window);
                } else if (c[q] == 0) {
                    const uint32_t k = (j0 >> 5) + q;  // entry index within the lane
                    if (k < TRACK) {
                        waiting |= 1ull << k;
                    } else {  // untracked: wait in place
                        unsigned int spins = 0;
                        int cc;
                        while ((cc = ld_relaxed(color + v[q])) == 0) {
                            if (++spins > spin_limit || ((spins & 255u) == 0 && ld_relaxed_u32(&st->err))) {
                                gave_up = true;
                                break;
                            }
                            __nanosleep(64);
                        }
                        if (!gave_up) mark(fb, cc, window);
                    }
                }
            }
        }
        // poll the tracked entries until every one is colored
        unsigned int spins = 0;
        while (__any_sync(0xffffffffu, waiting != 0 && !gave_up)) {
            bool progress = false;
            unsigned long long w = waiting;
            while (w && !gave_up) {
                const int k = __ffsll((long long)w) - 1;
                w &= w - 1;
                const int cc = ld_relaxed(color + __ldg(list + (uint32_t)k * 32 + lane));
                if (cc) {
                    mark(fb, cc, window);
                    waiting &= ~(1ull << k);
                    progress = true;
                }
            }
            if (waiting && !progress) {
                if (++spins > spin_limit || ((spins & 255u) == 0 && ld_relaxed_u32(&st->err))) gave_up = true;
                else if (spins > 32) __nanosleep(spins > 512 ? 256 : 32);
            }
        }
        if (__any_sync(0xffffffffu, gave_up)) return -1;
        __syncwarp();
        const int m = window_mex(fb, lane, window);
        __syncwarp();
        if (m) return m;
    }
}

constexpr int COLOR_WARPS_PER_CTA = 8;
constexpr int PENDING = 128;  // per warp: uncolored predecessors remembered for polling
constexpr uint32_t DECIDE_MAX = 32;  // early decisions are tried with at most this many predecessors pending

// Publishes the warp's forbidden colors 1..256 (window 0 of its bitmap) for vertex `self`, tagged
// with the run's epoch.  Lanes 0..7, one 64-bit word each.
__device__ __forceinline__ void publish_mask(unsigned long long *fmask, uint32_t self, unsigned long long tag,
                                             const uint32_t *fb, int lane) {
    if (lane < GC_JP_MASK_WORDS) st_relaxed_u64(fmask + (size_t)self * GC_JP_MASK_WORDS + lane, tag | fb[lane]);
}

// Colors one ordered vertex whose predecessors are list[0..cnt): the smallest color >= 1 none of
// them has.  Every predecessor color is read first without waiting (LOADS per lane in flight);
// the ids of uncolored ones go to the warp's pending list in shared memory, and only those are
// re-read (one global load each) until colored: back to back at first, then with growing sleeps.
// Pending-list overflow (more than PENDING uncolored predecessors) waits in place.  Returns -1
// when a wait exceeded spin_limit rounds or another warp raised the error flag.
// With `fmask` set, the warp also publishes the colors it has seen (for vertex `self`) while it
// waits, and tries early decisions once at most DECIDE_MAX predecessors are pending.
__device__ int color_one_v(const uint32_t *__restrict__ list, uint32_t cnt, const int *color, uint32_t *fb,
                           uint32_t *pend, int lane, DevState *st, unsigned int spin_limit, unsigned int tight,
                           unsigned int nap, const uint32_t *__restrict__ pc, unsigned long long *fmask,
                           uint32_t epoch, uint32_t self) {
    const unsigned long long tag = (unsigned long long)epoch << 32;
    for (uint32_t window = 0;; window++) {
        fb[lane] = 0;
        __syncwarp();
        uint32_t npend = 0;  // warp-uniform
        bool gave_up = false;
        for (uint32_t j0 = 0; j0 < cnt; j0 += 32 * LOADS) {
            uint32_t v[LOADS];
            int c[LOADS];
#pragma unroll
            for (int q = 0; q < LOADS; q++) {
                const uint32_t j = j0 + q * 32 + lane;
                v[q] = j < cnt ? __ldg(list + j) : 0xffffffffu;
            }
#pragma unroll
            for (int q = 0; q < LOADS; q++) c[q] = v[q] != 0xffffffffu ? ld_relaxed(color + v[q]) : -1;
#pragma unroll
            for (int q = 0; q < LOADS; q++) {
                if (c[q] > 0) mark(fb, c[q], window);
                const unsigned int zero = __ballot_sync(0xffffffffu, c[q] == 0);
                if (zero) {
                    const uint32_t slot = npend + __popc(zero & ((1u << lane) - 1u));
                    if (c[q] == 0) {
                        if (slot < PENDING) {
                            pend[slot] = v[q];
                        } else {  // list full: wait in place
                            unsigned int spins = 0;
                            int cc;
                            while ((cc = ld_relaxed(color + v[q])) == 0) {
                                if (++spins > spin_limit || ((spins & 255u) == 0 && ld_relaxed_u32(&st->err))) {
                                    gave_up = true;
                                    break;
                                }
                                __nanosleep(64);
                            }
                            if (!gave_up) mark(fb, cc, window);
                        }
                    }
                    npend = min((uint32_t)PENDING, npend + __popc(zero));
                }
            }
        }
        __syncwarp();
        const bool publish = fmask && window == 0 && npend > 0;
        if (publish) publish_mask(fmask, self, tag, fb, lane);
        // poll the pending list: lane l re-reads entries l, l + 32, ...
        uint32_t nleft = npend;  // pending entries after the last round (warp-uniform)
        unsigned int spins = 0;
        for (;;) {
            // the candidate of an early decision: the mex of the colors seen so far
            int cand = 0;
            if (fmask && nleft <= DECIDE_MAX) {
                __syncwarp();
                cand = window_mex(fb, lane, window);
            }
            bool progress = false, undecided = false;
            uint32_t mine = 0;
            for (uint32_t i = lane; i < npend && !gave_up; i += 32) {
                const uint32_t v = pend[i];
                if (v == 0xffffffffu) continue;
                const int cc = ld_relaxed(color + v);
                bool excluded = false;  // v cannot end up with color cand
                if (cand > 0 && cc == 0) {
                    excluded = __ldg(pc + v) + 1u < (uint32_t)cand;
                    if (!excluded && cand <= 32 * GC_JP_MASK_WORDS) {
                        const unsigned long long w =
                            ld_relaxed_u64(fmask + (size_t)v * GC_JP_MASK_WORDS + ((uint32_t)(cand - 1) >> 5));
                        excluded = (uint32_t)(w >> 32) == epoch && ((w >> ((uint32_t)(cand - 1) & 31u)) & 1ull);
                    }
                }
                if (cc) {
                    mark(fb, cc, window);
                    pend[i] = 0xffffffffu;
                    progress = true;
                    if (cc == cand) undecided = true;  // the candidate is taken
                } else {
                    mine++;
                    if (!excluded) undecided = true;
                }
            }
            if (cand > 0 && !__any_sync(0xffffffffu, undecided || gave_up)) {
                __syncwarp();
                return cand;  // every pending predecessor is excluded from cand: the mex is cand
            }
            nleft = __reduce_add_sync(0xffffffffu, mine);
            if (nleft == 0 || __any_sync(0xffffffffu, gave_up)) break;
            if (__any_sync(0xffffffffu, progress)) {
                if (publish) {
                    __syncwarp();
                    publish_mask(fmask, self, tag, fb, lane);
                }
            } else {
                if (++spins > spin_limit || ((spins & 255u) == 0 && ld_relaxed_u32(&st->err))) gave_up = true;
                else if (spins > tight) __nanosleep(spins > 16 * tight + 64 ? 4 * nap : nap);
            }
        }
        if (__any_sync(0xffffffffu, gave_up)) return -1;
        __syncwarp();
        const int m = window_mex(fb, lane, window);
        __syncwarp();
        if (m) return m;
    }
}

// The ordered vertices (neither sources nor leaves), one warp each, tickets taken one at a time
// in order.  A warp waits only on vertices with smaller tickets, which are held by running warps
// or done, so the oldest unfinished ticket always progresses.
// Ticket records: rec[t] = (vertex, first CSR entry, predecessor count) of ticket t, so that a
// warp needs one 16-byte load per ticket instead of the order -> V, pc chain.
__global__ void k_jp_records(const uint32_t *__restrict__ order, const uint32_t *__restrict__ V,
                             const uint32_t *__restrict__ pc, const DevState *st, uint4 *__restrict__ rec) {
    const uint32_t n = st->ordered;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t u = order[t];
        rec[t] = make_uint4(u, V[u], pc[u], 0u);
    }
}

// A warp takes its next ticket only when it is free: a ticket held ahead by a warp still waiting on
// its current vertex would stall every vertex that waits on the held one (measured several times
// slower on R-MAT 22).
__global__ void __launch_bounds__(COLOR_WARPS_PER_CTA * 32, 2) k_jp_color(const uint4 *__restrict__ rec,
                                                                       const uint32_t *__restrict__ P,
                                                                       const uint32_t *__restrict__ pc, int *color,
                                                                       DevState *st, unsigned int spin_limit,
                                                                       unsigned int tight, unsigned int nap,
                                                                       unsigned long long *fmask,
                                                                       const unsigned long long *epoch_word) {
    __shared__ uint32_t forbid[COLOR_WARPS_PER_CTA][32];
    __shared__ uint32_t pending[COLOR_WARPS_PER_CTA][PENDING];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n = ld_relaxed_u32(&st->ordered);
    const uint32_t epoch = fmask ? (uint32_t)*epoch_word : 0u;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&st->ticket, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n) break;
        const uint4 r = rec[t];
        const uint32_t u = r.x;
        const int c = color_one_v(P + r.y, r.z, color, forbid[warp], pending[warp], lane, st, spin_limit, tight, nap,
                                  pc, fmask, epoch, u);
        if (lane == 0) {
            if (c < 0) raise_error(st, ERR_WAIT_EXPIRED, u);
            // -1 on error is non-zero, so successors stop waiting; the host reports the error
            st_relaxed(color + u, c);
        }
        __syncwarp();
    }
}

// Culberson rounds (keys = the previous colors): the ticket order sorts the inner vertices by key, so
// each color class is a contiguous run of it.  first[k] = the first position of key k (runs of absent
// keys keep the fill value).
__global__ void k_jp_class_bounds(const uint32_t *__restrict__ order, const uint32_t *__restrict__ key,
                                  DevState *st, uint32_t *__restrict__ first, uint32_t words) {
    const uint32_t n = st->ordered;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = key[order[i]];
        if (k >= words) raise_error(st, ERR_BOUND, order[i]);
        else if (i == 0 || key[order[i - 1]] != k) first[k] = i;
    }
}

// One class of a Culberson round: the inner vertices order[a, b), whose key (old color) is the same.
// A class is an independent set and its predecessors (larger old colors) are sources or vertices of
// classes colored before it, so nothing waits: one thread per vertex with at most 62 predecessors
// (the mex, at most 63, is a bit of a 64-bit mask); the warp colors the larger ones together.
__global__ void __launch_bounds__(COLOR_THREADS) k_jp_class(const uint32_t *__restrict__ order, uint32_t a, uint32_t b,
                                                           const uint32_t *__restrict__ V, const uint32_t *__restrict__ P,
                                                           const uint32_t *__restrict__ pc, int *color, DevState *st,
                                                           unsigned int spin_limit) {
    __shared__ uint32_t forbid[COLOR_WARPS][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = a + blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < b; base += stride) {
        const uint32_t i = base + lane;
        const bool valid = i < b;
        const uint32_t u = valid ? order[i] : 0u;
        const uint32_t cnt = valid ? pc[u] : 0u;
        const bool big = valid && cnt > 62;
        if (valid && !big) {
            const uint32_t *list = P + V[u];
            unsigned long long used = 1;  // bit 0 stands for "color 0", never free
            for (uint32_t j = 0; j < cnt; j++) {
                const int c = color[list[j]];
                if (c > 0 && c < 64) used |= 1ull << c;
            }
            color[u] = __ffsll((long long)~used) - 1;
        }
        unsigned int bigs = __ballot_sync(0xffffffffu, big);
        while (bigs) {
            const int l = __ffs(bigs) - 1;
            bigs &= bigs - 1;
            const uint32_t ub = __shfl_sync(0xffffffffu, u, l), cb = __shfl_sync(0xffffffffu, cnt, l);
            // every predecessor is colored: the bounded wait inside never runs
            const int c = color_one(P + V[ub], cb, color, forbid[warp], lane, st, spin_limit);
            if (lane == 0) {
                if (c < 0) raise_error(st, ERR_WAIT_EXPIRED, ub);
                color[ub] = c;
            }
            __syncwarp();
        }
    }
}

// Leaves (every neighbour is a predecessor) are colored after all other vertices, in parallel:
// nothing waits on them.  One thread per leaf with a 64-bit mask for degrees up to 62 (so the mex,
// at most degree + 1, is a bit of the mask); larger leaves are listed for the warp kernel.
__global__ void k_jp_leaves(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E, const uint32_t *__restrict__ pc,
                            uint32_t N, int *__restrict__ color, uint32_t *__restrict__ big, DevState *st) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        const uint32_t beg = V[u], d = V[u + 1] - beg;
        if (d == 0 || pc[u] != d) continue;
        if (d > 62) {
            big[atomicAdd(&st->big_leaves, 1u)] = u;
            continue;
        }
        unsigned long long used = 1;  // bit 0 stands for "color 0", never free
        for (uint32_t i = beg; i < beg + d; i++) {
            const int c = color[ld_stream(E + i)];
            if (c > 0 && c < 64) used |= 1ull << c;
        }
        color[u] = __ffsll((long long)~used) - 1;
    }
}

__global__ void __launch_bounds__(COLOR_THREADS, 6) k_jp_big_leaves(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                                 const uint32_t *__restrict__ big, int *color,
                                                                 DevState *st, unsigned int spin_limit) {
    __shared__ uint32_t forbid[COLOR_WARPS][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n = st->big_leaves;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
        const uint32_t u = big[i];
        // every neighbour is colored already, so color_one does not wait here; its waits stay bounded
        // all the same, and an expiry is reported rather than stored as a color
        const int c = color_one(E + V[u], V[u + 1] - V[u], color, forbid[warp], lane, st, spin_limit);
        if (lane == 0) {
            if (c < 0) raise_error(st, ERR_WAIT_EXPIRED, u);
            color[u] = c;
        }
        __syncwarp();
    }
}

// Coloring statistics: every color positive, no monochrome edge, largest color -- per segment of
// a segmented CSR (stat[2s] largest color, stat[2s + 1] improper flag), or for the whole graph
// into DevState when nseg = 0.  Work items, heaviest first, one warp each: the hubs' split tasks
// (GC_SPLIT_CHUNK edges), the warp-tier vertices (vorder[0, n_wide)), then blocks of 32
// consecutive vertices, which a warp takes 8 at a time with 4 lanes per vertex.  Vertices above
// warp_deg have their edges checked by the first two kinds of item only.
__device__ __forceinline__ void stats_record(int *stat, DevState *st, uint32_t nseg, uint32_t s, int cmax, bool bad) {
    if (nseg) {
        atomicMax(stat + 2 * s, cmax);
        if (bad) atomicOr(stat + 2 * s + 1, 1);
    } else {
        atomicMax(&st->max_color, (unsigned int)max(cmax, 0));
        if (bad) atomicOr(&st->invalid, 1u);
    }
}

__global__ void __launch_bounds__(256) k_color_stats(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                     const int *__restrict__ color, const uint32_t *__restrict__ vorder,
                                                     uint32_t n_wide, const uint32_t *__restrict__ tasks,
                                                     uint32_t n_tasks, const uint32_t *__restrict__ voff,
                                                     uint32_t nseg, uint32_t N, uint32_t warp_deg, int *stat,
                                                     DevState *st) {
    const int lane = threadIdx.x & 31, q = lane & 3;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n_blocks = (N + 31) / 32;
    const uint32_t n_items = n_tasks + n_wide + n_blocks;
    for (uint32_t it = warp; it < n_items; it += nwarps) {
        if (it < n_tasks + n_wide) {
            uint32_t u, b, e;
            if (it < n_tasks) {
                u = tasks[2 * it];
                b = tasks[2 * it + 1];
                e = min(V[u + 1], b + GC_SPLIT_CHUNK);
            } else {
                u = vorder[it - n_tasks];
                b = V[u];
                e = V[u + 1];
            }
            const int cu = color[u];
            bool hit = false;
            for (uint32_t j = b + lane; j < e; j += 32) hit |= color[ld_stream(E + j)] == cu;
            if (__any_sync(0xffffffffu, hit) && lane == 0)
                stats_record(stat, st, nseg, nseg ? seg_of(voff, nseg, u) : 0u, 0, true);
            continue;
        }
        const uint32_t base = (it - n_tasks - n_wide) * 32;
        const uint32_t last = min(base + 31, N - 1);
        const uint32_t s0 = nseg ? seg_of(voff, nseg, base) : 0u;
        const bool uniform = !nseg || last < __ldg(voff + s0 + 1);
        int bmax = 0;
        bool bbad = false;
#pragma unroll 1
        for (int sub = 0; sub < 4; sub++) {
            const uint32_t u = base + 8 * sub + (lane >> 2);
            const bool valid = u < N;
            const uint32_t b = valid ? V[u] : 0u, e = valid ? V[u + 1] : 0u;
            const int cu = valid ? color[u] : 0;
            bool bad = valid && cu <= 0;
            if (valid && e - b <= warp_deg) {
                uint32_t j = b + q;
                for (; j + 12 < e; j += 16) {
                    const uint32_t v0 = ld_stream(E + j), v1 = ld_stream(E + j + 4);
                    const uint32_t v2 = ld_stream(E + j + 8), v3 = ld_stream(E + j + 12);
                    bad |= (color[v0] == cu) | (color[v1] == cu) | (color[v2] == cu) | (color[v3] == cu);
                }
                for (; j < e; j += 4) bad |= color[ld_stream(E + j)] == cu;
            }
            if (uniform) {
                bmax = max(bmax, cu);
                bbad |= bad;
            } else {
                const uint32_t s = valid ? seg_of(voff, nseg, u) : 0xffffffffu;
                const unsigned int peers = __match_any_sync(0xffffffffu, s);
                const int m = __reduce_max_sync(peers, cu);
                const unsigned int anybad = __reduce_or_sync(peers, bad ? 1u : 0u);
                if (valid && lane == __ffs(peers) - 1) stats_record(stat, st, nseg, s, m, anybad != 0);
            }
        }
        if (uniform) {
            const int m = __reduce_max_sync(0xffffffffu, bmax);
            const unsigned int anybad = __reduce_or_sync(0xffffffffu, bbad ? 1u : 0u);
            if (lane == 0) stats_record(stat, st, nseg, s0, m, anybad != 0);
        }
    }
}

__global__ void k_keys_from_colors(const int *__restrict__ color, uint32_t N, uint32_t *__restrict__ key) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
        key[u] = (uint32_t)color[u];
}

// Also advances the epoch of the published forbidden colors (never 0: the buffer starts zeroed).
__global__ void k_reset_ticket(DevState *st, unsigned long long *epoch_word) {
    st->ticket = 0;
    st->big_leaves = 0;
    if (epoch_word) {
        const unsigned long long e = (*epoch_word + 1) & 0xffffffffull;
        *epoch_word = e ? e : 1;
    }
}

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
    if (N == 0) {
        g->has_colors = true;
        return GC_OK;
    }
    if ((s = gc_alloc(ctx, &g->P, g->cap_M, "predecessor lists")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->pc, g->cap_N, "predecessor counts")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->order, g->cap_N, "ticket order")) != GC_OK) return s;
    if ((s = gc_alloc(ctx, &g->leaf_list, g->cap_N, "leaf list")) != GC_OK) return s;
    const bool decide = ctx->jp_decide;
    if (decide && !g->fmask) {
        const size_t words = (size_t)g->cap_N * GC_JP_MASK_WORDS + 1;
        if ((s = gc_alloc(ctx, &g->fmask, words, "published forbidden colors")) != GC_OK) return s;
        if ((s = gc_check_cuda(ctx, cudaMemsetAsync(g->fmask, 0, sizeof(unsigned long long) * words, ctx->stream),
                               "published forbidden colors")) != GC_OK)
            return s;
    }
    unsigned long long *fmask = decide ? g->fmask : nullptr;
    unsigned long long *epoch_word = decide ? g->fmask + (size_t)g->cap_N * GC_JP_MASK_WORDS : nullptr;
    const int grid = ctx->num_sms * 8;

    // 1. split, and color the sources
    {
        ProfScope ps(ctx, "jp_split", ctx->stream);
        if (g->n_vorder) {
            k_jp_split<<<grid, 256, 0, ctx->stream>>>(g->V, g->E, g->key, g->vorder, g->n_wide, g->n_vorder, g->P, g->pc);
            ctx->launches++;
        }
        if (g->n_big_tasks) {
            k_zero_hub_counts<<<ctx->num_sms, 256, 0, ctx->stream>>>(g->hubs, g->n_hubs, g->pc);
            k_jp_split_big<<<grid, SPLIT_WARPS * 32, 0, ctx->stream>>>(g->V, g->E, g->key, g->big, g->n_big_tasks, g->P,
                                                                      g->pc);
            ctx->launches += 2;
        }
        k_jp_init_colors<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->pc, N, g->color);
        ctx->launches++;
    }
    if ((s = gc_check_launch(ctx, "jp split")) != GC_OK) return s;

    // 2. ticket order of the inner vertices (0 < predecessors < degree)
    int bits = 32;
    if (g->key_kind == GC_FF) bits = 0;  // key = N - u: descending key is ascending id
    else if (g->key_kind == GC_LF || g->key_kind == GC_SL) bits = bit_length(g->max_deg);
    else if (g->key_kind == GC_LLF || g->key_kind == GC_SLL) bits = 6;
    else if (g->key_kind == 100) bits = bit_length((uint64_t)g->max_deg + 1);
    if ((s = gc_sort_order_bits(g, bits, true, &ctx->dstate->ordered)) != GC_OK) return s;

    // 3a. Culberson rounds: class by class, outside stream capture (it reads the class bounds back)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cap);
    if (g->key_kind == 100 && ctx->jp_classes && cap == cudaStreamCaptureStatusNone) {
        const size_t words = (size_t)g->max_deg + 2;  // keys (old colors) are at most max_deg + 1
        if (words > g->class_cap) {
            gc_dev_free(ctx, g->class_first);
            g->class_first = nullptr;
            if ((s = gc_alloc(ctx, &g->class_first, words, "class bounds")) != GC_OK) return s;
            g->class_cap = words;
        }
        if ((s = gc_check_cuda(ctx, cudaMemsetAsync(g->class_first, 0xff, 4 * words, ctx->stream), "class bounds")) !=
            GC_OK)
            return s;
        k_jp_class_bounds<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->order, g->key, ctx->dstate, g->class_first,
                                                                     (uint32_t)words);
        ctx->launches++;
        std::vector<uint32_t> first(words);
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(first.data(), g->class_first, 4 * words, cudaMemcpyDeviceToHost,
                                                    ctx->stream), "class bounds")) != GC_OK)
            return s;
        if ((s = gc_read_state(ctx)) != GC_OK) return s;  // syncs; also brings the ordered count
        const uint32_t n_ordered = ctx->hstate->ordered;
        {
            ProfScope ps(ctx, "jp_classes", ctx->stream);
            uint32_t end = n_ordered;
            // positions grow as keys fall: walk the keys upwards, each class ending where the next
            // larger key's class begins, and launch in descending key order
            std::vector<std::pair<uint32_t, uint32_t>> runs;
            for (size_t k = 0; k < words; k++)
                if (first[k] != 0xffffffffu) {
                    runs.push_back({first[k], end});
                    end = first[k];
                }
            for (auto it = runs.rbegin(); it != runs.rend(); ++it) {
                const uint32_t a = it->first, b = it->second;
                const uint32_t blocks = std::min<uint32_t>((b - a + COLOR_THREADS - 1) / COLOR_THREADS, ctx->num_sms * 8);
                k_jp_class<<<blocks, COLOR_THREADS, 0, ctx->stream>>>(g->order, a, b, g->V, g->P, g->pc, g->color,
                                                                     ctx->dstate, ctx->spin_limit);
                ctx->launches++;
            }
        }
        if ((s = gc_check_launch(ctx, "jp classes")) != GC_OK) return s;
        // the leaf kernels append to the big-leaf list from a zero count, as after the ticket kernel
        k_reset_ticket<<<1, 1, 0, ctx->stream>>>(ctx->dstate, nullptr);
        ctx->launches++;
        {
            ProfScope ps(ctx, "jp_leaves", ctx->stream);
            k_jp_leaves<<<grid, 256, 0, ctx->stream>>>(g->V, g->E, g->pc, N, g->color, g->leaf_list, ctx->dstate);
            k_jp_big_leaves<<<ctx->num_sms * 2, COLOR_THREADS, 0, ctx->stream>>>(g->V, g->E, g->leaf_list, g->color,
                                                                                  ctx->dstate, ctx->spin_limit);
            ctx->launches += 2;
        }
        if ((s = gc_check_launch(ctx, "jp color")) != GC_OK) return s;
        g->has_colors = true;
        g->colors_ours = true;
        return GC_OK;
    }

    if ((s = gc_alloc(ctx, &g->jprec, g->cap_N, "ticket records")) != GC_OK) return s;
    k_jp_records<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->order, g->V, g->pc, ctx->dstate, g->jprec);
    ctx->launches++;

    // 3. ordered coloring
    int &occupancy = ctx->color_blocks_per_sm;
    if (!occupancy) {
        if ((s = gc_check_cuda(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, k_jp_color,
                                                                                  COLOR_WARPS_PER_CTA * 32, 0),
                               "occupancy")) != GC_OK)
            return s;
        if (occupancy < 1) occupancy = 1;
    }
    const int want = g->jp_ctas > 0 ? g->jp_ctas : ctx->jp_ctas_per_sm;
    const int blocks = (want > 0 && want < occupancy) ? want : occupancy;
    const unsigned int tight = g->jp_ctas > 0 ? g->jp_tight : ctx->jp_tight;
    const unsigned int nap = g->jp_ctas > 0 ? g->jp_nap : ctx->jp_nap;
    k_reset_ticket<<<1, 1, 0, ctx->stream>>>(ctx->dstate, epoch_word);
    ctx->launches++;
    {
        ProfScope ps(ctx, "jp_color", ctx->stream);
        k_jp_color<<<ctx->num_sms * blocks, COLOR_WARPS_PER_CTA * 32, 0, ctx->stream>>>(
            g->jprec, g->P, g->pc, g->color, ctx->dstate, ctx->spin_limit, tight, nap, fmask, epoch_word);
        ctx->launches++;
    }
    // 4. leaves
    {
        ProfScope ps(ctx, "jp_leaves", ctx->stream);
        k_jp_leaves<<<grid, 256, 0, ctx->stream>>>(g->V, g->E, g->pc, N, g->color, g->leaf_list, ctx->dstate);
        k_jp_big_leaves<<<ctx->num_sms * 2, COLOR_THREADS, 0, ctx->stream>>>(g->V, g->E, g->leaf_list, g->color,
                                                                              ctx->dstate, ctx->spin_limit);
        ctx->launches += 2;
    }
    if ((s = gc_check_launch(ctx, "jp color")) != GC_OK) return s;
    g->has_colors = true;
    g->colors_ours = true;
    return GC_OK;
}

gc_status gc_keys_from_colors(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    if (g->N == 0) return GC_OK;
    ProfScope ps(ctx, "culberson_keys", ctx->stream);
    k_keys_from_colors<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->color, g->N, g->key);
    ctx->launches++;
    // the library's own colors are at most max degree + 1 (narrow sort, class rounds); caller colors
    // may be anything (full-width keys, tickets)
    g->key_kind = g->colors_ours ? 100 : 101;
    return gc_check_launch(ctx, "culberson keys");
}

namespace {

gc_status launch_color_stats(gc_graph *g, int *stat, uint32_t nseg) {
    gc_ctx *ctx = g->ctx;
    ProfScope ps(ctx, "color_stats", ctx->stream);
    k_color_stats<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->V, g->E, g->color, g->vorder, g->n_wide, g->big,
                                                             g->n_big_tasks, g->seg_voff, nseg, g->N, g->warp_deg,
                                                             stat, ctx->dstate);
    ctx->launches++;
    return gc_check_launch(ctx, "color statistics");
}

}  // namespace

gc_status gc_validate_device(gc_graph *g, int *max_color) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (g->N == 0) {
        *max_color = 1;  // the reference's validate_coloring_par starts from C = 1
        return GC_OK;
    }
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    if ((s = launch_color_stats(g, nullptr, 0)) != GC_OK) return s;
    if ((s = gc_read_state(ctx)) != GC_OK) return s;
    int C = (int)ctx->hstate->max_color;
    if (C < 1) C = 1;
    *max_color = ctx->hstate->invalid ? 0 : C;
    return GC_OK;
}

gc_status gc_segment_stats(gc_graph *g) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    if (!g->n_seg) return GC_OK;
    if ((s = gc_check_cuda(ctx, cudaMemsetAsync(g->seg_stat, 0, sizeof(int32_t) * 2 * g->n_seg, ctx->stream),
                           "segment statistics")) != GC_OK)
        return s;
    if (g->N == 0) return GC_OK;
    return launch_color_stats(g, g->seg_stat, g->n_seg);
}
