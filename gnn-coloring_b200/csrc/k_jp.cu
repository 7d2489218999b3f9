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
constexpr int SPLIT_LOADS = 4;  // per lane and step of the split: neighbour ids (then their keys) in flight

__global__ void __launch_bounds__(256) k_jp_split(const uint32_t *__restrict__ V, const uint32_t *__restrict__ E,
                                                  const uint32_t *__restrict__ key, const uint32_t *__restrict__ vorder,
                                                  uint32_t n_wide, uint32_t n_vorder, uint32_t *__restrict__ P,
                                                  uint32_t *__restrict__ pc) {
    const int lane = threadIdx.x & 31, q = lane & 3, qbase = lane & ~3;
    const unsigned int lt = (1u << lane) - 1u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n_items = n_wide + (n_vorder - n_wide + 7) / 8;
    const uint64_t keep = l2_keep_policy();  // the keys (4N bytes) stay in L2 while E streams past
    for (uint32_t it = warp; it < n_items; it += nwarps) {
        if (it < n_wide) {
            const uint32_t u = vorder[it];
            const uint32_t beg = V[u], d = V[u + 1] - beg, ku = key[u];
            uint32_t cnt = 0;
            for (uint32_t c = 0; c < d; c += 32 * SPLIT_LOADS) {
                // SPLIT_LOADS ids and then their keys in flight per lane
                uint32_t v[SPLIT_LOADS], kv[SPLIT_LOADS];
#pragma unroll
                for (int k = 0; k < SPLIT_LOADS; k++) {
                    const uint32_t i = c + 32 * k + lane;
                    v[k] = i < d ? ld_stream(E + beg + i) : 0u;
                }
#pragma unroll
                for (int k = 0; k < SPLIT_LOADS; k++) kv[k] = c + 32 * k + lane < d ? ld_keep(key + v[k], keep) : 0u;
#pragma unroll
                for (int k = 0; k < SPLIT_LOADS; k++) {
                    const bool pk = c + 32 * k + lane < d && precedes(kv[k], v[k], ku, u);
                    const unsigned int mk = __ballot_sync(0xffffffffu, pk);
                    if (pk) P[beg + cnt + __popc(mk & lt)] = v[k];
                    cnt += __popc(mk);
                }
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
        for (uint32_t c = 0; c < dmax; c += 4 * SPLIT_LOADS) {
            // SPLIT_LOADS ids and then their keys in flight per lane (entries c + 4k + q)
            uint32_t v[SPLIT_LOADS], kv[SPLIT_LOADS];
#pragma unroll
            for (int k = 0; k < SPLIT_LOADS; k++) {
                const uint32_t i = c + 4 * k + q;
                v[k] = i < d ? ld_stream(E + beg + i) : 0u;
            }
#pragma unroll
            for (int k = 0; k < SPLIT_LOADS; k++) kv[k] = c + 4 * k + q < d ? ld_keep(key + v[k], keep) : 0u;
#pragma unroll
            for (int k = 0; k < SPLIT_LOADS; k++) {
                const bool pk = c + 4 * k + q < d && precedes(kv[k], v[k], ku, u);
                const unsigned int qm = (__ballot_sync(0xffffffffu, pk) >> qbase) & 0xfu;
                if (pk) P[beg + cnt + __popc(qm & qlt)] = v[k];
                cnt += __popc(qm);
            }
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

// The smallest free color of the window other than c (a free color of the window); 0 if none.
__device__ __forceinline__ int window_mex_after(const uint32_t *fb, int lane, uint32_t window, int c) {
    const uint32_t idx = (uint32_t)(c - 1) - window * WINDOW;
    uint32_t free_bits = ~fb[lane];
    if ((uint32_t)lane == idx >> 5) free_bits &= ~(1u << (idx & 31u));
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
// With `rank` set, the tickets below kmax (the cluster-colored core) also record rank[u] = t.
__global__ void k_jp_records(const uint32_t *__restrict__ order, const uint32_t *__restrict__ V,
                             const uint32_t *__restrict__ pc, const DevState *st, uint4 *__restrict__ rec,
                             uint32_t *__restrict__ rank, uint32_t kmax) {
    const uint32_t n = st->ordered;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t u = order[t];
        rec[t] = make_uint4(u, V[u], pc[u], 0u);
        if (rank && t < kmax) rank[u] = t;
    }
}

// ---- the dense core: the first tickets, colored inside one thread-block cluster --------------------
//
// On power-law graphs the priority DAG's long chains lie almost all among the highest-priority inner
// vertices (R-MAT 22, GNN3 keys: depth 2,683 in all, yet depth 2,000 is reached by ticket 8,422, and
// with the first 32,768 tickets colored the rest is only 214 deep).  Through global memory every
// link of a chain costs a store-to-poll round trip in L2 (about 1 us), so these tickets bound the
// whole kernel.  Here one cluster colors tickets [0, K) with every color exchanged through
// distributed shared memory instead:
//   - each CTA holds a replica of the K core colors (16 bits each) in its shared memory;
//   - tickets go to the CTAs in blocks of B consecutive ones (block k to CTA k % C), so a short link
//     of a chain often stays inside one SM; a CTA hands its tickets out in order to whichever warp
//     is free (a counter in shared memory).  A warp waits only on smaller tickets, and the oldest
//     unfinished ticket is always held by a warp (all of its CTA's warps would otherwise hold older
//     ones), so it always progresses;
//   - the owner writes a color into all C replicas (lane i stores into CTA i) and to global memory;
//     waiting warps poll their own replica;
//   - a core vertex's predecessors are sources (color 1, known before) or inner vertices with smaller
//     tickets (core vertices): leaves precede nothing.  A pre-pass rewrites each core ticket's
//     predecessor list in place as ticket ranks and records whether a source is among them;
//   - early decisions: a vertex's color is the mex c of the colors seen so far as soon as no pending
//     predecessor can take c.  A vertex with p predecessors ends with a color <= p + 1, and one whose
//     seen colors hold c cannot take c.  So every CTA keeps all core predecessor counts, and a
//     waiting warp publishes the colors 1..256 it has seen in its CTA's shared memory, where the
//     warps of every CTA read them.  Bits are only ever set, so a stale read only delays a decision.
// Waits are bounded (spin_limit polls; on expiry the error is raised and the warp publishes
// 0xffff, which releases its successors).  A cluster barrier before exit keeps every CTA's shared
// memory alive while others may still store into it.
constexpr int CORE_WARPS = 32;                 // most warps per CTA (the launch takes ctx->jp_core_warps)
constexpr int CORE_PEND = 256;                 // per warp: uncolored predecessors remembered for polling
constexpr uint32_t CORE_MAX = 32768;           // most core tickets (16-bit ranks, 64 KB replica)
constexpr int CORE_LOADS = 8;                  // per lane: predecessor ranks in flight in the first pass
constexpr int CORE_PUB = 8;                    // published seen colors per core ticket: 8 words, colors 1..256
constexpr uint32_t CORE_DECIDE = 32;           // at most this many pending: one per lane, early decisions tried
static_assert(CORE_DECIDE <= 32, "one pending predecessor per lane");

// Tickets one CTA of a C-CTA cluster owns, for K core tickets in blocks of B (an upper bound).
__host__ __device__ __forceinline__ uint32_t core_owned(uint32_t K, uint32_t B, uint32_t C) {
    return ((K + B * C - 1) / (B * C)) * B;
}

__device__ __forceinline__ unsigned int cluster_rank() {
    unsigned int r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned int cluster_size() {
    unsigned int r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned int core_ld(const unsigned short *p) {
    unsigned short v;
    asm volatile("ld.relaxed.cluster.shared::cta.u16 %0, [%1];"
                 : "=h"(v)
                 : "r"((unsigned int)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
// Loads the word at p in CTA `rank`'s shared memory.
__device__ __forceinline__ uint32_t core_ld_remote(const uint32_t *p, unsigned int rank) {
    unsigned int remote;
    uint32_t v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(remote)
                 : "r"((unsigned int)__cvta_generic_to_shared(p)), "r"(rank));
    asm volatile("ld.relaxed.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(remote) : "memory");
    return v;
}
// Stores the word v at p in this CTA's shared memory, for loads from the whole cluster.
__device__ __forceinline__ void core_st_local(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.cluster.shared::cta.u32 [%0], %1;" ::"r"((unsigned int)__cvta_generic_to_shared(p)), "r"(v)
                 : "memory");
}
// Stores v into CTA `rank`'s copy of the replica element p.
__device__ __forceinline__ void core_st_remote(const unsigned short *p, unsigned int rank, unsigned short v) {
    unsigned int remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(remote)
                 : "r"((unsigned int)__cvta_generic_to_shared(p)), "r"(rank));
    asm volatile("st.relaxed.cluster.shared::cluster.u16 [%0], %1;" ::"r"(remote), "h"(v) : "memory");
}

// Pre-pass, one warp per core ticket t < K: the predecessor list P[first, first + count) becomes the
// ranks of its inner predecessors (compacted in place, CSR order kept), rec[t].z their number and
// rec[t].w = (all predecessors, at most 65,535) << 1 | (1 when a source, color 1 from the split, is
// among them).
__global__ void __launch_bounds__(256) k_jp_core_lists(uint4 *__restrict__ rec, uint32_t *__restrict__ P,
                                                       const uint32_t *__restrict__ rank, const int *__restrict__ color,
                                                       const DevState *st, uint32_t kmax) {
    const uint32_t K = min(st->ordered, kmax);
    const int lane = threadIdx.x & 31;
    const unsigned int lt = (1u << lane) - 1u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < K; t += nwarps) {
        const uint4 r = rec[t];
        uint32_t cnt = 0;
        bool source = false;
        for (uint32_t j0 = 0; j0 < r.z; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t rk = 0;
            bool inner = false;
            if (j < r.z) {
                const uint32_t v = P[r.y + j];
                if (color[v] == 1) source = true;
                else inner = true, rk = rank[v];
            }
            const unsigned int m = __ballot_sync(0xffffffffu, inner);
            __syncwarp();  // every lane has read its entry before any is overwritten
            if (inner) P[r.y + cnt + __popc(m & lt)] = rk;
            cnt += __popc(m);
        }
        const bool any_source = __any_sync(0xffffffffu, source);
        if (lane == 0) rec[t] = make_uint4(r.x, r.y, cnt, (min(r.z, 65535u) << 1) | (any_source ? 1u : 0u));
    }
}

// Marks color c (>= 1) in the warp's 1,024-color window bitmap.
__device__ __forceinline__ void core_mark(uint32_t *fb, unsigned int c, uint32_t window) {
    const uint32_t idx = c - 1u - window * WINDOW;
    if (idx < WINDOW) atomicOr(&fb[idx >> 5], 1u << (idx & 31));
}

__global__ void __launch_bounds__(CORE_WARPS * 32, 1) k_jp_core(const uint4 *__restrict__ rec,
                                                                const uint32_t *__restrict__ P, int *color,
                                                                DevState *st, unsigned int spin_limit,
                                                                uint32_t kmax, uint32_t B, unsigned int nap,
                                                                bool decide) {
    extern __shared__ __align__(16) unsigned char core_smem[];
    __shared__ uint32_t next_local;  // this CTA's next ticket (its index among the CTA's tickets)
    const unsigned int C = cluster_size(), me = cluster_rank();
    const uint32_t kr = (kmax + 7u) & ~7u;
    unsigned short *replica = reinterpret_cast<unsigned short *>(core_smem);  // colors, kr
    unsigned short *cpc = replica + kr;                                       // predecessor counts, kr
    uint32_t *pub = reinterpret_cast<uint32_t *>(cpc + kr);                   // this CTA's tickets' seen colors
    const uint32_t npub = core_owned(kmax, B, C);
    uint32_t *fb_all = pub + (size_t)npub * CORE_PUB;                         // W x 32
    unsigned short *pend_all = reinterpret_cast<unsigned short *>(fb_all + CORE_WARPS * 32);  // W x CORE_PEND
    const uint32_t K = min(ld_relaxed_u32(&st->ordered), kmax);
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
        replica[i] = 0;
        cpc[i] = (unsigned short)(rec[i].w >> 1);
    }
    for (uint32_t i = threadIdx.x; i < npub * CORE_PUB; i += blockDim.x) pub[i] = 0;
    if (threadIdx.x == 0) next_local = 0;
    cluster_sync_all();  // every replica is zeroed before any remote store
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *fb = fb_all + warp * 32;
    unsigned short *pend = pend_all + warp * CORE_PEND;
    for (;;) {
        // a free warp takes the CTA's next ticket: tickets start in order, and none waits for a
        // particular busy warp
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(&next_local, 1u);
        i = __shfl_sync(0xffffffffu, i, 0);
        const uint32_t t = ((i / B) * C + me) * B + i % B;  // this CTA's i-th ticket
        if (t >= K) break;
        uint32_t *mypub = pub + (size_t)i * CORE_PUB;  // i = the ticket's index among this CTA's
        const uint4 r = rec[t];
        const uint32_t *list = P + r.y;
        const uint32_t cnt = r.z;
        int result = -1;
        bool gave_up = false;
        for (uint32_t window = 0; result < 0 && !gave_up; window++) {
            fb[lane] = 0;
            __syncwarp();
            if ((r.w & 1u) && window == 0 && lane == 0) core_mark(fb, 1u, 0);
            uint32_t npend = 0;  // warp-uniform
            for (uint32_t j0 = 0; j0 < cnt; j0 += 32 * CORE_LOADS) {
                // CORE_LOADS list entries per lane in flight, then their colors from the replica
                uint32_t rks[CORE_LOADS];
                unsigned int cs[CORE_LOADS];
#pragma unroll
                for (int q = 0; q < CORE_LOADS; q++) {
                    const uint32_t j = j0 + 32 * q + lane;
                    rks[q] = j < cnt ? __ldg(list + j) : 0xffffffffu;
                }
#pragma unroll
                for (int q = 0; q < CORE_LOADS; q++) cs[q] = rks[q] != 0xffffffffu ? core_ld(replica + rks[q]) : 0xffffffffu;
#pragma unroll
                for (int q = 0; q < CORE_LOADS; q++) {
                    const uint32_t rk = rks[q];
                    const unsigned int c = cs[q];
                    if (c != 0 && c != 0xffffffffu) core_mark(fb, c, window);
                    const unsigned int zero = __ballot_sync(0xffffffffu, c == 0);
                    if (zero) {
                        const uint32_t slot = npend + __popc(zero & ((1u << lane) - 1u));
                        if (c == 0) {
                            if (slot < CORE_PEND) {
                                pend[slot] = (unsigned short)rk;
                            } else {  // list full: wait in place
                                unsigned int spins = 0, cc;
                                while ((cc = core_ld(replica + rk)) == 0) {
                                    if (++spins > spin_limit || ((spins & 1023u) == 0 && ld_relaxed_u32(&st->err))) {
                                        gave_up = true;
                                        break;
                                    }
                                }
                                if (!gave_up) core_mark(fb, cc, window);
                            }
                        }
                        npend = min((uint32_t)CORE_PEND, npend + __popc(zero));
                    }
                }
            }
            __syncwarp();
            const bool publish = decide && window == 0 && npend > 0;
            if (publish && lane < CORE_PUB) core_st_local(mypub + lane, fb[lane]);
            // Polling.  With more than CORE_DECIDE pending, rounds over the shared list, moving the entries
            // still uncolored to its front.  Then each lane holds at most one pending rank in a
            // register and polls it in the local replica, and the warp acts only when a color
            // arrives.  With one left, both outcomes are precomputed (below).  Early decisions (at
            // most CORE_DECIDE pending): the candidate c = mex(colors seen) is the color when no
            // pending predecessor v can take c -- count(v) + 1 < c, or c among the colors v has seen
            // (v's published set, read from its CTA's shared memory; the lanes' loads in flight
            // together) -- tried after each arrival and every 64 polls.
            unsigned int spins = 0;
            while (npend > CORE_DECIDE && !gave_up) {
                bool progress = false;
                uint32_t kept = 0;
                for (uint32_t c0 = 0; c0 < npend; c0 += 32) {
                    const uint32_t i2 = c0 + (uint32_t)lane;
                    unsigned short rk = 0;
                    bool keep = false;
                    if (i2 < npend) {
                        rk = pend[i2];
                        const unsigned int cc = core_ld(replica + rk);
                        if (cc) {
                            core_mark(fb, cc, window);
                            progress = true;
                        } else {
                            keep = true;
                        }
                    }
                    const unsigned int km = __ballot_sync(0xffffffffu, keep);
                    __syncwarp();  // every lane has read its entry before any is moved
                    if (keep) pend[kept + __popc(km & ((1u << lane) - 1u))] = rk;
                    kept += __popc(km);
                }
                npend = kept;
                __syncwarp();
                const bool prog = __any_sync(0xffffffffu, progress);
                if (publish && prog && lane < CORE_PUB) core_st_local(mypub + lane, fb[lane]);
                bool stop = ++spins > spin_limit;
                if ((spins & 1023u) == 0) stop |= __shfl_sync(0xffffffffu, lane == 0 ? ld_relaxed_u32(&st->err) : 0u, 0) != 0;
                if (stop) gave_up = true;
                else if (nap && !prog) __nanosleep(nap);
            }
            if (!gave_up && npend > 0) {
                uint32_t rk_l = (uint32_t)lane < npend ? pend[lane] : 0u;
                bool fresh = true;  // try a decision at once
                for (;;) {
                    if (npend == 1) {
                        // one predecessor left: both outcomes are known in advance -- c1 = mex(colors
                        // seen), or the next free color c2 if the predecessor takes c1 -- so the warp
                        // polls that one entry alone and answers the moment its color lands (early
                        // decisions re-tried every 64 polls)
                        __syncwarp();
                        const int c1 = window_mex(fb, lane, window);
                        const int c2 = c1 > 0 ? window_mex_after(fb, lane, window, c1) : 0;
                        const unsigned int rk0 = pend[0];
                        unsigned int cc = 0;
                        for (;;) {  // lane 0 reads, the warp follows its values
                            cc = __shfl_sync(0xffffffffu, lane == 0 ? core_ld(replica + rk0) : 0u, 0);
                            if (cc) break;
                            bool stop = ++spins > spin_limit;
                            if ((spins & 1023u) == 0) stop |= __shfl_sync(0xffffffffu, lane == 0 ? ld_relaxed_u32(&st->err) : 0u, 0) != 0;
                            if (stop) {
                                gave_up = true;
                                break;
                            }
                            if (publish && c1 > 0 && (spins & 63u) == 1u) {
                                bool excluded = (unsigned int)cpc[rk0] + 1u < (unsigned int)c1;
                                if (!excluded && c1 <= 32 * CORE_PUB) {
                                    const unsigned int owner = (rk0 / B) % C;
                                    const uint32_t li = (rk0 / (B * C)) * B + rk0 % B;
                                    const uint32_t word = __shfl_sync(
                                        0xffffffffu,
                                        lane == 0 ? core_ld_remote(pub + (size_t)li * CORE_PUB + ((uint32_t)(c1 - 1) >> 5), owner)
                                                  : 0u,
                                        0);
                                    excluded = (word >> ((uint32_t)(c1 - 1) & 31u)) & 1u;
                                }
                                if (excluded) {
                                    result = c1;
                                    break;
                                }
                            }
                            if (nap) __nanosleep(nap);
                        }
                        if (gave_up || result > 0) break;
                        if (c1 > 0 && (cc != (unsigned int)c1 || c2 > 0)) {
                            result = cc == (unsigned int)c1 ? c2 : c1;
                            break;
                        }
                        // the window holds no answer: record the color and go on to the next window
                        if (lane == 0) core_mark(fb, cc, window);
                        npend = 0;
                        __syncwarp();
                        break;
                    }
                    const unsigned int cc = (uint32_t)lane < npend ? core_ld(replica + rk_l) : 0u;
                    if (__ballot_sync(0xffffffffu, cc != 0u)) {
                        if (cc) core_mark(fb, cc, window);
                        const bool keep = (uint32_t)lane < npend && cc == 0u;
                        const unsigned int remain = __ballot_sync(0xffffffffu, keep);
                        if (keep) pend[__popc(remain & ((1u << lane) - 1u))] = (unsigned short)rk_l;
                        npend = (uint32_t)__popc(remain);
                        __syncwarp();  // marks and the compacted list are visible
                        rk_l = (uint32_t)lane < npend ? pend[lane] : 0u;
                        if (publish && lane < CORE_PUB) core_st_local(mypub + lane, fb[lane]);
                        if (npend == 0) break;
                        fresh = true;
                        continue;
                    }
                    if (publish && (fresh || (spins & 63u) == 0u)) {
                        fresh = false;
                        const int cand = window_mex(fb, lane, 0);
                        if (cand > 0) {
                            bool undecided = false;
                            if ((uint32_t)lane < npend) {
                                bool excluded = (unsigned int)cpc[rk_l] + 1u < (unsigned int)cand;
                                if (!excluded && cand <= 32 * CORE_PUB) {
                                    const unsigned int owner = (rk_l / B) % C;
                                    const uint32_t li = (rk_l / (B * C)) * B + rk_l % B;
                                    const uint32_t word =
                                        core_ld_remote(pub + (size_t)li * CORE_PUB + ((uint32_t)(cand - 1) >> 5), owner);
                                    excluded = (word >> ((uint32_t)(cand - 1) & 31u)) & 1u;
                                }
                                undecided = !excluded;
                            }
                            if (!__any_sync(0xffffffffu, undecided)) {
                                result = cand;
                                break;
                            }
                        }
                    }
                    bool stop = ++spins > spin_limit;
                    if ((spins & 1023u) == 0) stop |= __shfl_sync(0xffffffffu, lane == 0 ? ld_relaxed_u32(&st->err) : 0u, 0) != 0;
                    if (stop) {
                        gave_up = true;
                        break;
                    }
                    if (nap) __nanosleep(nap);
                }
            }
            if (result > 0) break;  // decided early
            gave_up = __any_sync(0xffffffffu, gave_up);
            if (gave_up) break;
            __syncwarp();
            const int m = window_mex(fb, lane, window);
            __syncwarp();
            if (m) result = m;
        }
        const unsigned short val = gave_up ? (unsigned short)0xffffu : (unsigned short)result;
        if ((unsigned int)lane < C) core_st_remote(replica + t, (unsigned int)lane, val);
        if (lane == 0) {
            if (gave_up) raise_error(st, ERR_WAIT_EXPIRED, r.x);
            st_relaxed(color + r.x, gave_up ? -1 : result);
        }
        __syncwarp();
    }
    cluster_sync_all();  // no CTA leaves while another may still store into its replica
}

// ---- after the core: a heavy and a light stream --------------------------------------------------
//
// Past the core the DAG is shallow and the ticket kernel is bound by how many vertices are in flight
// (about 1.7 us from ticket to color, most of it three dependent loads).  Most of these vertices
// have few predecessors, so they are split off: tickets with at most LIGHT_MAX predecessors form the
// light stream, colored one vertex per lane (32 per warp), the others the heavy stream, one vertex
// per warp as before.  Both streams keep the priority order, and each has warps of its own, so the
// oldest unfinished vertex of either stream is always held by a running warp and all its
// predecessors are done: the kernel always progresses.
constexpr uint32_t LIGHT_MAX = 63;   // a light vertex's color is at most 64: one 64-bit mask
constexpr uint32_t PART_TILE = 1024;

// Heavy tickets per tile of the tickets after the core, [first, n).
__global__ void __launch_bounds__(PART_TILE) k_jp_part_count(const uint4 *__restrict__ rec, const DevState *st,
                                                             uint32_t core, uint32_t *__restrict__ tile_heavy) {
    __shared__ uint32_t warp_cnt[PART_TILE / 32];
    const uint32_t n = st->ordered, first = min(n, core);
    const uint32_t t = first + blockIdx.x * PART_TILE + threadIdx.x;
    const bool heavy = t < n && rec[t].z > LIGHT_MAX;
    const unsigned int m = __ballot_sync(0xffffffffu, heavy);
    if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x < 32) {
        const uint32_t c = warp_cnt[threadIdx.x];
        const uint32_t tot = __reduce_add_sync(0xffffffffu, c);
        if (threadIdx.x == 0) tile_heavy[blockIdx.x] = tot;
    }
}

// Exclusive prefix of the tiles' heavy counts (in place), one CTA; the stream sizes into the state.
__global__ void __launch_bounds__(1024) k_jp_part_scan(uint32_t *__restrict__ tile_heavy, uint32_t ntiles, DevState *st,
                                                       uint32_t core) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < ntiles; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < ntiles ? tile_heavy[i] : 0u;
        uint32_t x = v;  // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sum[lane], wx = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, wx, o);
                if (lane >= o) wx += y;
            }
            warp_sum[lane] = wx - w;  // exclusive
        }
        __syncthreads();
        const uint32_t c = carry;
        if (i < ntiles) tile_heavy[i] = c + warp_sum[warp] + x - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = c + warp_sum[31] + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint32_t n = st->ordered, first = min(n, core);
        st->n_heavy = carry;
        st->n_light = n - first - carry;
        st->ticket_light = 0;
    }
}

// Stable split: heavy tickets to out[0, n_heavy) in order, light tickets to out[cap - 1 - i] for the
// i-th light ticket (the light stream is read from the top down).
__global__ void __launch_bounds__(PART_TILE) k_jp_part_scatter(const uint4 *__restrict__ rec, const DevState *st,
                                                               uint32_t core, const uint32_t *__restrict__ tile_heavy,
                                                               uint4 *__restrict__ out, uint32_t cap) {
    __shared__ uint32_t warp_off[PART_TILE / 32];
    const uint32_t n = st->ordered, first = min(n, core);
    const uint32_t tile0 = first + blockIdx.x * PART_TILE;
    const uint32_t t = tile0 + threadIdx.x;
    const bool valid = t < n;
    const uint4 r = valid ? rec[t] : make_uint4(0u, 0u, 0u, 0u);
    const bool heavy = valid && r.z > LIGHT_MAX;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned int m = __ballot_sync(0xffffffffu, heavy);
    if (lane == 0) warp_off[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_off[lane];
        uint32_t x = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        warp_off[lane] = x - w;
    }
    __syncthreads();
    if (!valid) return;
    const uint32_t heavy_before = tile_heavy[blockIdx.x] + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
    if (heavy) out[heavy_before] = r;
    else out[cap - 1u - ((t - first) - heavy_before)] = r;
}

// Light stream, one vertex per lane: the predecessors' colors go into a 64-bit mask (a light vertex
// has at most 63 predecessors, so its color is at most 64); uncolored ones are remembered by their
// list position and re-read until colored (bounded; growing sleeps).  Returns -1 on expiry.
__device__ __forceinline__ int color_light(const uint32_t *__restrict__ list, uint32_t cnt, const int *color,
                                           DevState *st, unsigned int spin_limit, unsigned int nap) {
    unsigned long long used = 0, pend = 0;  // colors 1..64 taken; list positions still uncolored
    constexpr int GROUP = 8;                // ids, then colors, GROUP at a time in flight
    for (uint32_t j0 = 0; j0 < cnt; j0 += GROUP) {
        uint32_t v[GROUP];
        int c[GROUP];
#pragma unroll
        for (int k = 0; k < GROUP; k++) v[k] = j0 + k < cnt ? __ldg(list + j0 + k) : 0xffffffffu;
#pragma unroll
        for (int k = 0; k < GROUP; k++) c[k] = v[k] != 0xffffffffu ? ld_relaxed(color + v[k]) : -2;
#pragma unroll
        for (int k = 0; k < GROUP; k++) {
            if (c[k] > 0 && c[k] <= 64) used |= 1ull << (c[k] - 1);
            else if (c[k] == 0) pend |= 1ull << (j0 + k);  // (-1: a predecessor whose wait failed; raised)
        }
    }
    unsigned int spins = 0;
    while (pend) {
        bool progress = false;
        unsigned long long w = pend;
        while (w) {
            const int j = __ffsll((long long)w) - 1;
            w &= w - 1;
            const int c = ld_relaxed(color + __ldg(list + j));
            if (c) {
                if (c > 0 && c <= 64) used |= 1ull << (c - 1);
                pend &= ~(1ull << j);
                progress = true;
            }
        }
        if (pend && !progress) {
            if (++spins > spin_limit || ((spins & 255u) == 0 && ld_relaxed_u32(&st->err))) return -1;
            if (spins > 32) __nanosleep(spins > 512 ? 4 * nap : nap);
        }
    }
    return __ffsll((long long)~used);  // at most 63 bits are set: a free color <= 64 exists
}

// A warp takes its next ticket only when it is free: a ticket held ahead by a warp still waiting on
// its current vertex would stall every vertex that waits on the held one (measured several times
// slower on R-MAT 22).
// Without a split (split == nullptr) every warp takes tickets of rec in order.  With a split, the
// CTA's first COLOR_WARPS_PER_CTA - light_warps warps take the heavy stream split[0, n_heavy) one
// vertex each (ticket counter st->ticket, from 0), the others the light stream -- split[cap - 1 - i],
// i < n_light -- 32 vertices at a time, one per lane (counter st->ticket_light).
__global__ void __launch_bounds__(COLOR_WARPS_PER_CTA * 32, 2) k_jp_color(const uint4 *__restrict__ rec,
                                                                       const uint32_t *__restrict__ P,
                                                                       const uint32_t *__restrict__ pc, int *color,
                                                                       DevState *st, unsigned int spin_limit,
                                                                       unsigned int tight, unsigned int nap,
                                                                       unsigned long long *fmask,
                                                                       const unsigned long long *epoch_word,
                                                                       const uint4 *__restrict__ split, uint32_t cap,
                                                                       int light_warps) {
    __shared__ uint32_t forbid[COLOR_WARPS_PER_CTA][32];
    __shared__ uint32_t pending[COLOR_WARPS_PER_CTA][PENDING];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t epoch = fmask ? (uint32_t)*epoch_word : 0u;
    if (split && warp >= COLOR_WARPS_PER_CTA - light_warps) {
        const uint32_t nl = ld_relaxed_u32(&st->n_light);
        for (;;) {
            uint32_t t0 = 0;
            if (lane == 0) t0 = atomicAdd(&st->ticket_light, 32u);
            t0 = __shfl_sync(0xffffffffu, t0, 0);
            if (t0 >= nl) break;
            const uint32_t i = t0 + lane;
            if (i < nl) {
                const uint4 r = split[cap - 1u - i];
                const int c = color_light(P + r.y, r.z, color, st, spin_limit, nap);
                if (c < 0) raise_error(st, ERR_WAIT_EXPIRED, r.x);
                st_relaxed(color + r.x, c);  // -1 on error is non-zero: successors stop waiting
            }
            __syncwarp();
        }
        return;
    }
    const uint4 *src = split ? split : rec;
    const uint32_t n = split ? ld_relaxed_u32(&st->n_heavy) : ld_relaxed_u32(&st->ordered);
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&st->ticket, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n) break;
        const uint4 r = src[t];
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
// The ordered kernel's first ticket: past the core tickets the cluster colored (first_cap of them
// at most), else 0.
__global__ void k_reset_ticket(DevState *st, unsigned long long *epoch_word, uint32_t first_cap = 0) {
    st->ticket = min(st->ordered, first_cap);
    st->big_leaves = 0;
    if (epoch_word) {
        const unsigned long long e = (*epoch_word + 1) & 0xffffffffull;
        *epoch_word = e ? e : 1;
    }
}

size_t core_smem_bytes(uint32_t kmax, uint32_t B, uint32_t C) {
    return 4 * (size_t)((kmax + 7u) & ~7u) + sizeof(uint32_t) * CORE_PUB * core_owned(kmax, B, C) +
           sizeof(uint32_t) * CORE_WARPS * 32 + sizeof(unsigned short) * CORE_WARPS * CORE_PEND;
}

// Once per context: the core kernel's cluster size -- 16 CTAs (a non-portable size) when the device
// can place such a cluster with the most shared memory a CTA may have, else 8, else 0 (no core phase).
gc_status core_cluster_config(gc_ctx *ctx) {
    if (ctx->jp_core_cluster >= 0) return GC_OK;
    ctx->jp_core_cluster = 0;
    int optin = 0;
    gc_status s = gc_check_cuda(ctx, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device),
                                "smem per block");
    if (s != GC_OK) return s;
    cudaFuncAttributes fa{};
    s = gc_check_cuda(ctx, cudaFuncGetAttributes(&fa, k_jp_core), "core attributes");
    if (s != GC_OK) return s;
    const size_t smem = (size_t)optin - fa.sharedSizeBytes;  // the dynamic part: the rest is static
    ctx->jp_core_smem = smem;
    s = gc_check_cuda(ctx, cudaFuncSetAttribute(k_jp_core, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                "core smem");
    if (s != GC_OK) return s;
    if (cudaFuncSetAttribute(k_jp_core, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        cudaGetLastError();
    for (int C : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(CORE_WARPS * 32);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_jp_core, &cfg) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (n >= 1) {
            ctx->jp_core_cluster = C;
            break;
        }
    }
    return GC_OK;
}

// The most core tickets, up to kmax, whose replicas and published sets fit the core kernel's shared
// memory on a cluster of the configured size.
uint32_t core_fit(const gc_ctx *ctx, uint32_t kmax) {
    const uint32_t B = ctx->jp_core_block ? ctx->jp_core_block : 1u, C = (uint32_t)ctx->jp_core_cluster;
    uint32_t k = std::min(kmax, CORE_MAX) & ~7u;
    while (k && core_smem_bytes(k, B, C) > ctx->jp_core_smem) k -= 8;
    return k;
}

gc_status launch_core(gc_ctx *ctx, gc_graph *g, uint32_t kmax) {
    const int C = ctx->jp_core_cluster;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(32 * std::min(std::max(ctx->jp_core_warps, 1), CORE_WARPS));
    const uint32_t B = ctx->jp_core_block ? ctx->jp_core_block : 1u;
    cfg.dynamicSmemBytes = core_smem_bytes(kmax, B, (uint32_t)C);
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const uint4 *rec = g->jprec;
    const uint32_t *P = g->P;
    int *color = g->color;
    DevState *st = ctx->dstate;
    const unsigned int spin = ctx->spin_limit;
    const unsigned int nap = ctx->jp_core_nap;
    const bool decide = ctx->jp_core_decide;
    gc_status s = gc_check_cuda(ctx, cudaLaunchKernelEx(&cfg, k_jp_core, rec, P, color, st, spin, kmax, B, nap, decide),
                                "jp core");
    ctx->launches++;
    return s;
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
    uint32_t core = 0;  // core tickets colored in one cluster (at most)
    if (ctx->jp_core_max && (s = core_cluster_config(ctx)) == GC_OK && ctx->jp_core_cluster > 0) core = core_fit(ctx, ctx->jp_core_max);
    if (s != GC_OK) return s;
    if (core && (s = gc_alloc(ctx, &g->rank, g->cap_N, "core ranks")) != GC_OK) return s;
    k_jp_records<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(g->order, g->V, g->pc, ctx->dstate, g->jprec,
                                                            core ? g->rank : nullptr, core);
    ctx->launches++;
    if (core) {
        ProfScope ps(ctx, "jp_core", ctx->stream);
        k_jp_core_lists<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(g->jprec, g->P, g->rank, g->color, ctx->dstate,
                                                                   core);
        ctx->launches++;
        if ((s = launch_core(ctx, g, core)) != GC_OK) return s;
    }

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
    // the tickets after the core as a heavy and a light stream (light_warps warps per CTA take the light one)
    const int light_warps = ctx->jp_light_warps;
    uint4 *split = nullptr;
    if (light_warps > 0 && light_warps < COLOR_WARPS_PER_CTA) {
        const uint32_t ntiles = (N + PART_TILE - 1) / PART_TILE;
        if ((s = gc_alloc(ctx, &g->jpsplit, g->cap_N, "ticket streams")) != GC_OK) return s;
        if ((s = gc_alloc(ctx, &g->part_tiles, (g->cap_N + PART_TILE - 1) / PART_TILE, "ticket stream tiles")) != GC_OK)
            return s;
        ProfScope ps(ctx, "jp_streams", ctx->stream);
        k_jp_part_count<<<ntiles, PART_TILE, 0, ctx->stream>>>(g->jprec, ctx->dstate, core, g->part_tiles);
        k_jp_part_scan<<<1, 1024, 0, ctx->stream>>>(g->part_tiles, ntiles, ctx->dstate, core);
        k_jp_part_scatter<<<ntiles, PART_TILE, 0, ctx->stream>>>(g->jprec, ctx->dstate, core, g->part_tiles, g->jpsplit,
                                                                 g->cap_N);
        ctx->launches += 3;
        split = g->jpsplit;
    }
    k_reset_ticket<<<1, 1, 0, ctx->stream>>>(ctx->dstate, epoch_word, split ? 0u : core);
    ctx->launches++;
    {
        ProfScope ps(ctx, "jp_color", ctx->stream);
        k_jp_color<<<ctx->num_sms * blocks, COLOR_WARPS_PER_CTA * 32, 0, ctx->stream>>>(
            g->jprec, g->P, g->pc, g->color, ctx->dstate, ctx->spin_limit, tight, nap, fmask, epoch_word, split,
            g->cap_N, light_warps);
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
