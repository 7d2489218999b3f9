// Ticket order for the coloring kernel: all vertices by descending key, ties by ascending id,
// i.e. a topological order of the reference's priority DAG (src/coloring.c:72 and :249: v
// precedes u when p[v] > p[u], or p[v] == p[u] and v < u).  Any topological order would do; this
// is the one every heuristic shares.
//
// LSD radix sort with 8-bit digits over the complemented key (ascending ~key = descending key).
// The input sequence lists vertices by ascending id and every pass is stable, so equal keys end
// up by ascending id.  Passes over digits that no key can have set are skipped: the caller
// passes the key's bit width (known per heuristic: degree bound, color bound, 32 for floats).
//
// Per pass: tile histograms (and digit totals) -> scan of the digit totals -> one CTA per digit
// scans that digit's tile counts -> stable scatter.
// Stability inside a tile: each warp walks its own contiguous run of the tile in order, ranking
// equal digits with __match_any_sync; per-digit warp totals are then prefixed across warps.
#include "gc_internal.h"

namespace {
using namespace gc;

constexpr int SORT_WARPS = 8;
constexpr int SORT_THREADS = SORT_WARPS * 32;
constexpr int SORT_ITEMS = 32;                               // per lane
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;          // 8192 elements per CTA
constexpr int RADIX = 256;

// Element j of a pass: the first pass reads the heuristic's keys directly (optionally keeping
// only vertices the filter selects); later passes read the previous pass's output, whose length
// the first pass's scan left in device memory.
struct SortIn {
    const uint32_t *kin, *vin;  // previous pass (later passes)
    const uint32_t *key;        // keys by vertex (first pass)
    const uint32_t *V, *pc;     // filter inputs
    const uint32_t *d_n;        // element count of later passes
    uint32_t N;
    uint32_t max_deg;           // SORT_KEEP_DEG_AT_MOST: largest degree kept
    int first, filter;
};

__device__ __forceinline__ bool sort_elem(const SortIn &in, uint32_t j, uint32_t n, uint32_t &k, uint32_t &v) {
    if (in.first) {
        if (j >= in.N) return false;
        if (in.filter == SORT_KEEP_INNER) {
            const uint32_t p = in.pc[j], d = in.V[j + 1] - in.V[j];
            if (p == 0 || p >= d) return false;
        } else if (in.filter == SORT_KEEP_DEG_AT_MOST) {
            if (in.V[j + 1] - in.V[j] > in.max_deg) return false;
        }
        k = in.key[j];
        v = j;
        return true;
    }
    if (j >= n) return false;
    k = in.kin[j];
    v = in.vin[j];
    return true;
}

__device__ __forceinline__ uint32_t digit_of(uint32_t k, int shift, uint32_t mask) { return ((~k) >> shift) & mask; }

__device__ __forceinline__ uint32_t pass_len(const SortIn &in) { return in.first ? in.N : min(in.N, *in.d_n); }

__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(SortIn in, int shift, uint32_t mask,
                                                            uint32_t *__restrict__ counts, uint32_t ntiles,
                                                            uint32_t *__restrict__ digit_total) {
    __shared__ uint32_t hist[RADIX];
    for (int i = threadIdx.x; i < RADIX; i += SORT_THREADS) hist[i] = 0;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * SORT_TILE;
    const uint32_t n = pass_len(in);
    const int lane = threadIdx.x & 31;
    if (base < n) {
        for (int s = 0; s < SORT_ITEMS; s++) {
            uint32_t j = base + s * SORT_THREADS + threadIdx.x, k, v;
            bool valid = sort_elem(in, j, n, k, v);
            uint32_t d = valid ? digit_of(k, shift, mask) : 0xffffffffu;
            unsigned int peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&hist[d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) {
        counts[(size_t)d * ntiles + tile] = hist[d];
        if (hist[d]) atomicAdd(&digit_total[d], hist[d]);
    }
}

// Exclusive scan of the 256 digit totals (one CTA); the grand total -- the number of sorted
// elements -- goes to *d_total when given.
__global__ void __launch_bounds__(RADIX) k_sort_scan_digits(const uint32_t *__restrict__ digit_total,
                                                            uint32_t *__restrict__ digit_base, uint32_t *d_total) {
    __shared__ uint32_t part[RADIX];
    part[threadIdx.x] = digit_total[threadIdx.x];
    __syncthreads();
    for (int off = 1; off < RADIX; off <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    digit_base[threadIdx.x] = threadIdx.x ? part[threadIdx.x - 1] : 0;
    if (d_total && threadIdx.x == RADIX - 1) *d_total = part[RADIX - 1];
}

// One CTA per digit: exclusive scan of that digit's tile counts, offset by the digit's base, so
// counts[d][t] becomes the first output position of digit d in tile t.
constexpr int SCAN_THREADS = 512;
__global__ void __launch_bounds__(SCAN_THREADS) k_sort_scan_tiles(uint32_t *__restrict__ counts, uint32_t ntiles,
                                                                  const uint32_t *__restrict__ digit_base) {
    __shared__ uint32_t part[SCAN_THREADS];
    uint32_t *row = counts + (size_t)blockIdx.x * ntiles;
    const uint32_t per = (ntiles + SCAN_THREADS - 1) / SCAN_THREADS;
    const uint32_t b = threadIdx.x * per, e = min(ntiles, b + per);
    uint32_t sum = 0;
    for (uint32_t i = b; i < e; i++) sum += row[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < SCAN_THREADS; off <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = digit_base[blockIdx.x] + (threadIdx.x ? part[threadIdx.x - 1] : 0);
    for (uint32_t i = b; i < e; i++) {
        const uint32_t c = row[i];
        row[i] = run;
        run += c;
    }
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(SortIn in, int shift, uint32_t mask,
                                                               const uint32_t *__restrict__ offsets, uint32_t ntiles,
                                                               uint32_t *__restrict__ kout, uint32_t *__restrict__ vout) {
    __shared__ uint32_t wcnt[SORT_WARPS][RADIX];
    __shared__ uint32_t gbase[RADIX];
    const uint32_t n = pass_len(in);
    if (blockIdx.x * SORT_TILE >= n) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = lane; d < RADIX; d += 32) wcnt[warp][d] = 0;
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) gbase[d] = offsets[(size_t)d * ntiles + blockIdx.x];
    __syncwarp();
    const uint32_t wbase = blockIdx.x * SORT_TILE + warp * (32 * SORT_ITEMS);
    uint32_t k[SORT_ITEMS], v[SORT_ITEMS], pos[SORT_ITEMS];
    uint32_t valid_mask = 0;
    const unsigned int lt = (1u << lane) - 1u;
#pragma unroll
    for (int s = 0; s < SORT_ITEMS; s++) {
        uint32_t j = wbase + s * 32 + lane;
        bool valid = sort_elem(in, j, n, k[s], v[s]);
        if (valid) valid_mask |= 1u << s;
        uint32_t d = valid ? digit_of(k[s], shift, mask) : 0xffffffffu;
        unsigned int peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = valid ? wcnt[warp][d] : 0;
        pos[s] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix across warps, then add the tile's global offset
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) {
        uint32_t run = gbase[d];
        for (int w = 0; w < SORT_WARPS; w++) {
            uint32_t c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < SORT_ITEMS; s++) {
        if (valid_mask & (1u << s)) {
            uint32_t dst = wcnt[warp][digit_of(k[s], shift, mask)] + pos[s];
            kout[dst] = k[s];
            vout[dst] = v[s];
        }
    }
}

// ---- single-sweep passes (vertex sorts) ----------------------------------------------------------
//
// The vertex sorts run every digit pass as one kernel: a histogram kernel first counts the digits of
// all passes at once (the first pass's filter decides which vertices take part), one CTA scans those
// totals into each digit's first output position per pass, and then each pass is a single kernel in
// which a CTA takes the next tile from a counter, ranks it (stable, as above), publishes its digit
// counts and finds the counts of all earlier tiles by decoupled look-back: tile k's status word per
// digit holds its own count (flag AGG) and, once known, the count of tiles 0..k (flag INC); a tile
// walks back from k-1, adding AGG counts, until it meets an INC.  Tiles are taken in order, so every
// tile looked at is running or done; each wait is bounded (SW_WAIT_LIMIT polls, then ERR_WAIT_EXPIRED:
// a fixed bound, since these waits only end a pass, unlike the coloring's configurable ones).
constexpr uint32_t SW_AGG = 1u << 30, SW_INC = 2u << 30, SW_VAL = SW_AGG - 1u;
constexpr int SW_WINDOW = 4;  // predecessor status words in flight per look-back step
constexpr unsigned int SW_WAIT_LIMIT = 1u << 22;

__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist_all(SortIn in, int passes, uint32_t mask,
                                                                uint32_t *__restrict__ totals) {
    __shared__ uint32_t hist[4][RADIX];
    for (int i = threadIdx.x; i < 4 * RADIX; i += SORT_THREADS) (&hist[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t n = in.N;  // the first pass's input: every vertex
    constexpr int H = 8;      // elements per thread and round, their loads in flight together
    for (uint32_t base = blockIdx.x * SORT_THREADS * H; base < n; base += gridDim.x * SORT_THREADS * H) {
        uint32_t k[H], v[H], valid = 0;
#pragma unroll
        for (int h = 0; h < H; h++)
            if (sort_elem(in, base + h * SORT_THREADS + threadIdx.x, n, k[h], v[h])) valid |= 1u << h;
#pragma unroll
        for (int h = 0; h < H; h++) {
            const bool ok = (valid >> h) & 1u;
            const unsigned int okm = __ballot_sync(0xffffffffu, ok);
            if (!okm) continue;
            const int leader = __ffs(okm) - 1;
            for (int p = 0; p < passes; p++) {
                // one atomic for the warp when its valid elements share the digit (the high digits of
                // clustered keys), else one per element (spread digits rarely collide)
                const uint32_t d = ok ? digit_of(k[h], 8 * p, mask) : 0u;
                const uint32_t d0 = __shfl_sync(0xffffffffu, d, leader);
                if (__all_sync(0xffffffffu, !ok || d == d0)) {
                    if (lane == leader) atomicAdd(&hist[p][d0], (uint32_t)__popc(okm));
                } else if (ok) {
                    atomicAdd(&hist[p][d], 1u);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RADIX; i += SORT_THREADS) {
        const uint32_t c = (&hist[0][0])[i];
        if (c) atomicAdd(&totals[i], c);
    }
}

// Per pass: exclusive scan of the digit totals into the digits' first output positions (one CTA of
// RADIX threads); the element count goes to *d_count.
__global__ void __launch_bounds__(RADIX) k_sort_scan_all(const uint32_t *__restrict__ totals, int passes,
                                                         uint32_t *__restrict__ bases, uint32_t *d_count) {
    __shared__ uint32_t part[RADIX];
    for (int p = 0; p < passes; p++) {
        part[threadIdx.x] = totals[p * RADIX + threadIdx.x];
        __syncthreads();
        for (int off = 1; off < RADIX; off <<= 1) {
            const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
            __syncthreads();
            part[threadIdx.x] += v;
            __syncthreads();
        }
        bases[p * RADIX + threadIdx.x] = threadIdx.x ? part[threadIdx.x - 1] : 0;
        if (p == 0 && d_count && threadIdx.x == RADIX - 1) *d_count = part[RADIX - 1];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_sweep(SortIn in, int shift, uint32_t mask,
                                                             const uint32_t *__restrict__ bases,
                                                             uint32_t *__restrict__ status, uint32_t *tile_ctr,
                                                             uint32_t *__restrict__ kout, uint32_t *__restrict__ vout,
                                                             DevState *st) {
    __shared__ uint32_t wcnt[SORT_WARPS][RADIX];
    __shared__ uint32_t gbase[RADIX];
    __shared__ uint32_t tile_s;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = tile_s;
    const uint32_t n = pass_len(in);
    if (tile * SORT_TILE >= n) return;  // later tiles are empty too: nobody looks at this one
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = lane; d < RADIX; d += 32) wcnt[warp][d] = 0;
    __syncwarp();
    const uint32_t wbase = tile * SORT_TILE + warp * (32 * SORT_ITEMS);
    uint32_t k[SORT_ITEMS], v[SORT_ITEMS], pos[SORT_ITEMS];
    uint32_t valid_mask = 0;
    const unsigned int lt = (1u << lane) - 1u;
#pragma unroll
    for (int s = 0; s < SORT_ITEMS; s++) {  // every load in flight before the ranking
        if (sort_elem(in, wbase + s * 32 + lane, n, k[s], v[s])) valid_mask |= 1u << s;
    }
#pragma unroll
    for (int s = 0; s < SORT_ITEMS; s++) {
        const bool valid = (valid_mask >> s) & 1u;
        const uint32_t d = valid ? digit_of(k[s], shift, mask) : 0xffffffffu;
        const unsigned int peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = valid ? wcnt[warp][d] : 0;
        pos[s] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix across warps, the tile's count, its status, then the look-back
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) {
        uint32_t run = 0;
        for (int w = 0; w < SORT_WARPS; w++) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
        uint32_t *mine = status + (size_t)tile * RADIX + d;
        uint32_t excl = 0;
        if (tile == 0) {
            st_relaxed_u32(mine, SW_INC | run);
        } else {
            st_relaxed_u32(mine, SW_AGG | run);
            int32_t j = (int32_t)tile - 1;
            unsigned int spins = 0;
            bool done = false;
            while (!done) {
                uint32_t w[SW_WINDOW];
#pragma unroll
                for (int q = 0; q < SW_WINDOW; q++)
                    w[q] = j - q >= 0 ? ld_relaxed_u32(status + (size_t)(j - q) * RADIX + d) : SW_INC;
                int q = 0;
                for (; q < SW_WINDOW; q++) {
                    if (!(w[q] & (SW_AGG | SW_INC))) break;  // not published yet: reload from here
                    excl += w[q] & SW_VAL;
                    if (w[q] & SW_INC) {
                        done = true;
                        break;
                    }
                }
                j -= q;
                if (!done && q < SW_WINDOW && ++spins > SW_WAIT_LIMIT) {
                    raise_error(st, ERR_WAIT_EXPIRED, tile);
                    break;
                }
            }
            st_relaxed_u32(mine, SW_INC | (excl + run));
        }
        gbase[d] = bases[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < SORT_ITEMS; s++) {
        if (valid_mask & (1u << s)) {
            const uint32_t d = digit_of(k[s], shift, mask);
            const uint32_t dst = gbase[d] + wcnt[warp][d] + pos[s];
            if (dst < in.N) {
                kout[dst] = k[s];
                vout[dst] = v[s];
            } else {
                raise_error(st, ERR_BOUND, dst);
            }
        }
    }
}

}  // namespace

// Sorts vertex ids by descending key (ascending id on ties) into `out`.  key_bits: number of low
// key bits that may be non-zero; 0 means "all keys equal" (a stable compaction by id).  `filter`
// selects which vertices take part (SORT_KEEP_*); their number is left in *d_count.
gc_status gc_sort_vertices(gc_graph *g, const uint32_t *keys, int key_bits, int filter, uint32_t max_deg,
                           uint32_t *out, uint32_t *d_count) {
    gc_ctx *ctx = g->ctx;
    gc_status s;
    const uint32_t N = g->N;
    if (N == 0) return GC_OK;
    if ((s = gc_alloc(ctx, &g->sort_buf, 4 * (size_t)g->cap_N, "sort buffers")) != GC_OK) return s;
    const int passes = key_bits <= 0 ? 1 : (key_bits + 7) / 8;
    const uint32_t ntiles = (N + SORT_TILE - 1) / SORT_TILE;
    // digit totals and bases (4 passes at most), tile counters, then the tiles' status words per pass
    const size_t head = 2 * 4 * RADIX + 4;
    const size_t words = head + (size_t)passes * ntiles * RADIX;
    if (g->sort_hist_cap < words) {
        gc_dev_free(ctx, g->sort_hist);
        g->sort_hist = nullptr;
        if ((s = gc_alloc(ctx, &g->sort_hist, words, "sort histogram")) != GC_OK) return s;
        g->sort_hist_cap = (uint32_t)words;
    }
    uint32_t *totals = g->sort_hist, *bases = totals + 4 * RADIX, *tile_ctr = bases + 4 * RADIX;
    uint32_t *status = g->sort_hist + head;
    ProfScope ps(ctx, "sort", ctx->stream);
    if ((s = gc_check_cuda(ctx, cudaMemsetAsync(g->sort_hist, 0, sizeof(uint32_t) * words, ctx->stream),
                           "sort state")) != GC_OK)
        return s;
    uint32_t *k0 = g->sort_buf, *v0 = g->sort_buf + g->cap_N;
    uint32_t *k1 = g->sort_buf + 2 * (size_t)g->cap_N, *v1 = g->sort_buf + 3 * (size_t)g->cap_N;
    SortIn in{};
    in.key = keys;
    in.V = g->V;
    in.pc = g->pc;
    in.d_n = d_count;
    in.N = N;
    in.max_deg = max_deg;
    in.filter = filter;
    in.first = 1;
    const uint32_t mask = key_bits <= 0 ? 0u : (uint32_t)(RADIX - 1);
    k_sort_hist_all<<<std::min<uint32_t>(ntiles, (uint32_t)ctx->num_sms * 4), SORT_THREADS, 0, ctx->stream>>>(
        in, passes, mask, totals);
    k_sort_scan_all<<<1, RADIX, 0, ctx->stream>>>(totals, passes, bases, d_count);
    ctx->launches += 2;
    for (int p = 0; p < passes; p++) {
        in.first = (p == 0);
        uint32_t *kout = (p & 1) ? k1 : k0, *vout = (p & 1) ? v1 : v0;
        if (p == passes - 1) vout = out;  // last pass writes the result directly
        k_sort_sweep<<<ntiles, SORT_THREADS, 0, ctx->stream>>>(in, 8 * p, mask, bases + p * RADIX,
                                                                status + (size_t)p * ntiles * RADIX, tile_ctr + p,
                                                                kout, vout, ctx->dstate);
        ctx->launches++;
        if ((s = gc_check_launch(ctx, "radix sort")) != GC_OK) return s;
        in.kin = kout;
        in.vin = vout;
    }
    return GC_OK;
}

gc_status gc_sort_order_bits(gc_graph *g, int key_bits, bool filter, uint32_t *d_count) {
    return gc_sort_vertices(g, g->key, key_bits, filter ? SORT_KEEP_INNER : SORT_KEEP_ALL, 0, g->order, d_count);
}

// Stable sort of n (key, value) pairs by ascending key into (kout, vout), reusing the passes above:
// they order by the complemented key, so the keys are complemented on the way in and out.  kbuf and
// vbuf are ping-pong buffers of n words; hist needs ntiles * 256 + 2 * 256 * 4 words and d_n one
// device word.  key_bits: bit width of the largest key.
namespace {
__global__ void k_complement_into(const uint32_t *__restrict__ kin, uint32_t n, uint32_t *__restrict__ kout) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) kout[i] = ~kin[i];
}
}  // namespace

size_t gc_sort_pairs_hist_words(uint32_t n) {
    const uint32_t ntiles = (n + SORT_TILE - 1) / SORT_TILE;
    return (size_t)RADIX * (ntiles ? ntiles : 1) + 4 * 2 * RADIX + 1;
}

gc_status gc_sort_pairs(gc_ctx *ctx, uint32_t n, const uint32_t *kin, const uint32_t *vin, int key_bits,
                        uint32_t *kbuf, uint32_t *vbuf, uint32_t *kout, uint32_t *vout, uint32_t *hist) {
    gc_status s;
    if (n == 0) return GC_OK;
    const uint32_t ntiles = (n + SORT_TILE - 1) / SORT_TILE;
    const int passes = key_bits <= 0 ? 0 : (key_bits + 7) / 8;
    uint32_t *digit_words = hist + (size_t)RADIX * ntiles;
    uint32_t *d_n = digit_words + 4 * 2 * RADIX;
    if (passes > 4) return gc_fail(ctx, GC_ERR_INVALID, "sort keys wider than 32 bits");
    if ((s = gc_check_cuda(ctx, cudaMemsetAsync(digit_words, 0, sizeof(uint32_t) * 4 * 2 * RADIX, ctx->stream),
                           "sort digit totals")) != GC_OK)
        return s;
    if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(d_n, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream),
                           "sort length")) != GC_OK)
        return s;
    // complemented keys into the first buffer of the chain that ends in kout
    uint32_t *kb[2] = {kbuf, kout}, *vb[2] = {vbuf, vout};
    const int first = passes % 2 == 0 ? 1 : 0;  // buffer the complemented keys start in
    k_complement_into<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(kin, n, kb[first]);
    ctx->launches++;
    if (passes == 0) {
        if ((s = gc_check_cuda(ctx, cudaMemcpyAsync(vb[first], vin, 4ull * n, cudaMemcpyDeviceToDevice, ctx->stream),
                               "sort values")) != GC_OK)
            return s;
    }
    SortIn in{};
    in.kin = kb[first];
    in.vin = passes == 0 ? vb[first] : vin;
    in.d_n = d_n;
    in.N = n;
    in.first = 0;
    int cur = first;
    for (int p = 0; p < passes; p++) {
        const int nxt = cur ^ 1;
        uint32_t *digit_total = digit_words + 2 * RADIX * p, *digit_base = digit_total + RADIX;
        k_sort_hist<<<ntiles, SORT_THREADS, 0, ctx->stream>>>(in, 8 * p, RADIX - 1, hist, ntiles, digit_total);
        k_sort_scan_digits<<<1, RADIX, 0, ctx->stream>>>(digit_total, digit_base, nullptr);
        k_sort_scan_tiles<<<RADIX, SCAN_THREADS, 0, ctx->stream>>>(hist, ntiles, digit_base);
        k_sort_scatter<<<ntiles, SORT_THREADS, 0, ctx->stream>>>(in, 8 * p, RADIX - 1, hist, ntiles, kb[nxt], vb[nxt]);
        ctx->launches += 4;
        if ((s = gc_check_launch(ctx, "pair sort")) != GC_OK) return s;
        in.kin = kb[nxt];
        in.vin = vb[nxt];
        cur = nxt;
    }
    // the chain ends in (kout, vout); undo the complement
    k_complement_into<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(kout, n, kout);
    ctx->launches++;
    return gc_check_launch(ctx, "pair sort");
}
