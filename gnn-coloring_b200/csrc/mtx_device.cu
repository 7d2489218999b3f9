// Matrix Market to CSR on the GPU: the reference's loader rules (src/fast_io.c:33-222, 450-477) --
// N = max(rows, cols), every entry in both directions, self-loops and duplicates dropped, each
// adjacency list sorted ascending -- with the text parsed and the pairs sorted on the device.
// The host reads the file and its header only.
//
//   1. line starts: per block of text, the count of line starts (a host scan of the block sums
//      gives each block its base), then each block writes its positions in order;
//   2. parse: one thread per line; '%' lines are comments; a data line gives its first two numbers
//      (1-based; digits only, as the reference's scanner); the first L such lines are the entries;
//   3. symmetrise: entry k becomes the directed pairs 2k and 2k + 1 (a self-loop becomes two
//      sentinel pairs that sort last and are dropped);
//   4. two stable LSD sorts -- by column, then by row -- order the pairs by (row, column);
//   5. dedupe: the first of each run of equal pairs is kept (block counts, host scan, compaction),
//      and the row offsets are filled from the rows of the kept pairs, empty rows included.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gc_internal.h"

namespace {

constexpr int MTX_THREADS = 256;
constexpr uint32_t TEXT_PER_THREAD = 64;  // bytes of text per thread when finding line starts
constexpr uint64_t TEXT_PER_BLOCK = (uint64_t)MTX_THREADS * TEXT_PER_THREAD;
constexpr uint32_t ITEMS_PER_BLOCK = 4096;  // lines or pairs per block in the counting passes

__device__ __forceinline__ bool line_start(const char *T, uint64_t p) { return p == 0 || T[p - 1] == '\n'; }

// Block-wide exclusive scan of one value per thread; returns the thread's prefix.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < MTX_THREADS; off <<= 1) {
        const uint32_t x = threadIdx.x >= (unsigned)off ? sh[threadIdx.x - off] : 0;
        __syncthreads();
        sh[threadIdx.x] += x;
        __syncthreads();
    }
    const uint32_t incl = sh[threadIdx.x];
    __syncthreads();
    return incl - v;
}

__global__ void k_count_lines(const char *__restrict__ T, uint64_t S, uint32_t *__restrict__ block_count) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint64_t a = blockIdx.x * TEXT_PER_BLOCK + (uint64_t)threadIdx.x * TEXT_PER_THREAD;
    uint32_t c = 0;
    for (uint64_t p = a; p < a + TEXT_PER_THREAD && p < S; p++) c += line_start(T, p);
    const uint32_t before = block_exclusive(c, sh);
    if (threadIdx.x == MTX_THREADS - 1) block_count[blockIdx.x] = before + c;
}

__global__ void k_write_lines(const char *__restrict__ T, uint64_t S, const uint32_t *__restrict__ block_base,
                              uint64_t *__restrict__ starts) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint64_t a = blockIdx.x * TEXT_PER_BLOCK + (uint64_t)threadIdx.x * TEXT_PER_THREAD;
    uint32_t c = 0;
    for (uint64_t p = a; p < a + TEXT_PER_THREAD && p < S; p++) c += line_start(T, p);
    uint32_t at = block_base[blockIdx.x] + block_exclusive(c, sh);
    for (uint64_t p = a; p < a + TEXT_PER_THREAD && p < S; p++)
        if (line_start(T, p)) starts[at++] = p;
}

// Line k: its first two numbers, or not a data line (comment, fewer than two numbers).
__global__ void k_parse_lines(const char *__restrict__ T, uint64_t S, const uint64_t *__restrict__ starts,
                              uint32_t n_lines, uint32_t *__restrict__ A, uint32_t *__restrict__ B,
                              uint8_t *__restrict__ is_data) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_lines; k += gridDim.x * blockDim.x) {
        uint64_t p = starts[k];
        bool ok = p < S && T[p] != '%';
        uint32_t v[2] = {0, 0};
        for (int f = 0; f < 2 && ok; f++) {
            while (p < S && T[p] != '\n' && (T[p] < '0' || T[p] > '9')) p++;
            if (p >= S || T[p] == '\n') {
                ok = false;
                break;
            }
            uint64_t x = 0;
            while (p < S && T[p] >= '0' && T[p] <= '9') x = x * 10 + (uint64_t)(T[p++] - '0');
            v[f] = x > 0xffffffffull ? 0xffffffffu : (uint32_t)x;
        }
        is_data[k] = ok;
        A[k] = v[0];
        B[k] = v[1];
    }
}

__global__ void k_count_flags(const uint8_t *__restrict__ flag, uint32_t n, uint32_t *__restrict__ block_count) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint32_t a = blockIdx.x * ITEMS_PER_BLOCK + threadIdx.x * (ITEMS_PER_BLOCK / MTX_THREADS);
    uint32_t c = 0;
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n; i++) c += flag[i];
    const uint32_t before = block_exclusive(c, sh);
    if (threadIdx.x == MTX_THREADS - 1) block_count[blockIdx.x] = before + c;
}

// The first L data lines, each as two directed pairs (row, col) in 0-based ids; self-loops as
// sentinel pairs (N, N).  An id outside 1..N raises ERR_BOUND.
__global__ void k_emit_pairs(const uint8_t *__restrict__ is_data, const uint32_t *__restrict__ A,
                             const uint32_t *__restrict__ B, uint32_t n_lines, const uint32_t *__restrict__ block_base,
                             uint32_t L, uint32_t N, uint32_t *__restrict__ row, uint32_t *__restrict__ col,
                             gc::DevState *st) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint32_t a = blockIdx.x * ITEMS_PER_BLOCK + threadIdx.x * (ITEMS_PER_BLOCK / MTX_THREADS);
    uint32_t c = 0;
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n_lines; i++) c += is_data[i];
    uint32_t rank = block_base[blockIdx.x] + block_exclusive(c, sh);
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n_lines; i++) {
        if (!is_data[i]) continue;
        if (rank < L) {
            const uint32_t x = A[i], y = B[i];
            if (x < 1 || y < 1 || x > N || y > N) {
                gc::raise_error(st, gc::ERR_BOUND, i);
            } else if (x == y) {
                row[2 * rank] = row[2 * rank + 1] = col[2 * rank] = col[2 * rank + 1] = N;
            } else {
                row[2 * rank] = x - 1;
                col[2 * rank] = y - 1;
                row[2 * rank + 1] = y - 1;
                col[2 * rank + 1] = x - 1;
            }
        }
        rank++;
    }
}

// After the sorts: pair q is (row[q], col[q]); keep it when it is a real pair and differs from
// pair q - 1.
__device__ __forceinline__ bool keep_pair(const uint32_t *row, const uint32_t *col, uint32_t q, uint32_t N) {
    return row[q] < N && (q == 0 || row[q] != row[q - 1] || col[q] != col[q - 1]);
}

__global__ void k_count_kept(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col, uint32_t n, uint32_t N,
                             uint32_t *__restrict__ block_count) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint32_t a = blockIdx.x * ITEMS_PER_BLOCK + threadIdx.x * (ITEMS_PER_BLOCK / MTX_THREADS);
    uint32_t c = 0;
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n; i++) c += keep_pair(row, col, i, N);
    const uint32_t before = block_exclusive(c, sh);
    if (threadIdx.x == MTX_THREADS - 1) block_count[blockIdx.x] = before + c;
}

// Kept pairs into E (and their rows into rows_out), in order.
__global__ void k_compact_pairs(const uint32_t *__restrict__ row, const uint32_t *__restrict__ col, uint32_t n,
                                uint32_t N, const uint32_t *__restrict__ block_base, uint32_t *__restrict__ E,
                                uint32_t *__restrict__ rows_out) {
    __shared__ uint32_t sh[MTX_THREADS];
    const uint32_t a = blockIdx.x * ITEMS_PER_BLOCK + threadIdx.x * (ITEMS_PER_BLOCK / MTX_THREADS);
    uint32_t c = 0;
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n; i++) c += keep_pair(row, col, i, N);
    uint32_t at = block_base[blockIdx.x] + block_exclusive(c, sh);
    for (uint32_t i = a; i < a + ITEMS_PER_BLOCK / MTX_THREADS && i < n; i++)
        if (keep_pair(row, col, i, N)) {
            E[at] = col[i];
            rows_out[at] = row[i];
            at++;
        }
}

// Row offsets from the sorted rows of the M kept pairs: V[r] = the first q with rows[q] >= r.
__global__ void k_row_offsets(const uint32_t *__restrict__ rows, uint32_t M, uint32_t N, uint32_t *__restrict__ V) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= N; r += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = M;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (rows[mid] < r) lo = mid + 1;
            else hi = mid;
        }
        V[r] = lo;
    }
}

int bit_width(uint64_t x) {
    int b = 0;
    while (x) {
        b++;
        x >>= 1;
    }
    return b;
}

// Exclusive scan of block counts on the host (a few thousand words): the bases back to the device.
gc_status scan_blocks(gc_ctx *ctx, uint32_t *d_counts, uint32_t nblocks, uint64_t *total) {
    std::vector<uint32_t> h(nblocks);
    gc_status s = gc_check_cuda(ctx, cudaMemcpyAsync(h.data(), d_counts, 4ull * nblocks, cudaMemcpyDeviceToHost,
                                                     ctx->stream), "block counts");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "block counts");
    if (s != GC_OK) return s;
    uint64_t run = 0;
    for (uint32_t b = 0; b < nblocks; b++) {
        const uint32_t c = h[b];
        h[b] = (uint32_t)run;
        run += c;
    }
    *total = run;
    if (run > 0xffffffffull) return gc_fail(ctx, GC_ERR_INVALID, "more than 2^32 items");
    s = gc_check_cuda(ctx, cudaMemcpyAsync(d_counts, h.data(), 4ull * nblocks, cudaMemcpyHostToDevice, ctx->stream),
                      "block bases");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "block bases");
    return s;
}

// Device buffers of one load, freed on every exit.
struct Scratch {
    gc_ctx *ctx;
    std::vector<void *> bufs;
    explicit Scratch(gc_ctx *c) : ctx(c) {}
    template <typename T>
    gc_status get(T **p, size_t count, const char *what) {
        *p = nullptr;
        gc_status s = gc_alloc(ctx, p, count, what);
        if (s == GC_OK) bufs.push_back(*p);
        return s;
    }
    ~Scratch() {
        for (void *p : bufs) gc_dev_free(ctx, p);
    }
};

// The header by the reference's rules ('%' lines, then rows, columns and entries; the rest of that
// line is skipped): N = max(rows, cols), L, and the offset of the first data line.
gc_status read_header(gc_ctx *ctx, FILE *f, uint32_t *N, uint32_t *L, uint64_t *data0) {
    uint64_t off = 0;
    int c = fgetc(f);
    while (c == '%') {  // comment lines
        while (c != EOF && c != '\n') {
            c = fgetc(f);
            off++;
        }
        if (c == EOF) break;
        c = fgetc(f);
        off++;
    }
    uint32_t hdr[3];
    for (int k = 0; k < 3; k++) {
        while (c != EOF && (c < '0' || c > '9')) {
            c = fgetc(f);
            off++;
        }
        if (c == EOF) return gc_fail(ctx, GC_ERR_FORMAT, "Matrix Market header needs rows, columns and entries");
        uint64_t x = 0;
        while (c >= '0' && c <= '9') {
            x = x * 10 + (uint64_t)(c - '0');
            if (x > 0xffffffffull) return gc_fail(ctx, GC_ERR_FORMAT, "header value out of range");
            c = fgetc(f);
            off++;
        }
        hdr[k] = (uint32_t)x;
    }
    while (c != EOF && c != '\n') {  // the rest of the header line
        c = fgetc(f);
        off++;
    }
    *data0 = off + 1;
    *N = hdr[0] > hdr[1] ? hdr[0] : hdr[1];
    *L = hdr[2];
    return GC_OK;
}

// Bytes [data0, size) of the file into T on the device, then a final newline: file reads into one
// pinned chunk overlap the copy of the other.
gc_status upload_text(gc_ctx *ctx, FILE *f, uint64_t data0, uint64_t S, char *T) {
    constexpr size_t CHUNK = 16u << 20;
    char *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    gc_status s = GC_OK;
    for (int b = 0; b < 2 && s == GC_OK; b++) {
        s = gc_check_cuda(ctx, cudaMallocHost((void **)&stage[b], CHUNK), "pinned text chunk");
        if (s == GC_OK) s = gc_check_cuda(ctx, cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "chunk event");
    }
    if (s == GC_OK && fseeko(f, (off_t)data0, SEEK_SET) != 0) s = gc_fail(ctx, GC_ERR_IO, "cannot seek to the data lines");
    const uint64_t body = S - 1;  // file bytes; the last byte of T is the added newline
    uint64_t at = 0;
    for (int b = 0; s == GC_OK && at < body; b ^= 1) {
        const size_t n = (size_t)std::min<uint64_t>(CHUNK, body - at);
        s = gc_check_cuda(ctx, cudaEventSynchronize(done[b]), "text chunk");  // the chunk's last copy is done
        if (s != GC_OK) break;
        if (fread(stage[b], 1, n, f) != n) {
            s = gc_fail(ctx, GC_ERR_IO, "short read");
            break;
        }
        s = gc_check_cuda(ctx, cudaMemcpyAsync(T + at, stage[b], n, cudaMemcpyHostToDevice, ctx->stream), "upload text");
        if (s == GC_OK) s = gc_check_cuda(ctx, cudaEventRecord(done[b], ctx->stream), "text chunk");
        at += n;
    }
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaMemsetAsync(T + body, '\n', 1, ctx->stream), "final newline");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "upload text");
    for (int b = 0; b < 2; b++) {
        if (done[b]) cudaEventDestroy(done[b]);
        if (stage[b]) cudaFreeHost(stage[b]);
    }
    return s;
}

// The whole pipeline into a new device graph.
gc_status load(gc_ctx *ctx, const char *path, gc_graph **out) {
    struct File {
        FILE *f;
        ~File() {
            if (f) fclose(f);
        }
    } file{fopen(path, "rb")};
    if (!file.f) return gc_fail(ctx, GC_ERR_IO, std::string("cannot open ") + path);
    if (fseeko(file.f, 0, SEEK_END) != 0) return gc_fail(ctx, GC_ERR_IO, "cannot size the file");
    const off_t fsize = ftello(file.f);
    if (fsize < 0 || fseeko(file.f, 0, SEEK_SET) != 0) return gc_fail(ctx, GC_ERR_IO, "cannot size the file");
    uint64_t data0 = 0;
    uint32_t N = 0, L = 0;
    gc_status s = read_header(ctx, file.f, &N, &L, &data0);
    if (s != GC_OK) return s;
    if ((uint64_t)L * 2 > 0xffffffffull) return gc_fail(ctx, GC_ERR_INVALID, "more than 2^31 entries");
    Scratch sc(ctx);
    // 1. the data lines on the device, with a final newline; line starts
    const uint64_t S = (data0 < (uint64_t)fsize ? (uint64_t)fsize - data0 : 0) + 1;
    char *T = nullptr;
    uint32_t *blk = nullptr;
    const uint64_t nb_text = (S + TEXT_PER_BLOCK - 1) / TEXT_PER_BLOCK;
    if (S >= (1ull << 40)) return gc_fail(ctx, GC_ERR_INVALID, "file too large");
    if ((s = sc.get(&T, S, "mtx text")) != GC_OK) return s;
    if ((s = upload_text(ctx, file.f, data0, S, T)) != GC_OK) return s;
    const uint32_t nbt = (uint32_t)nb_text;
    // block counts of every counting pass: text blocks, line blocks (at most one line per byte) and
    // pair blocks
    const size_t blk_words = std::max<size_t>(nbt, std::max<uint64_t>(S, 2ull * L) / ITEMS_PER_BLOCK + 2);
    if ((s = sc.get(&blk, blk_words, "block counts")) != GC_OK) return s;
    uint64_t n_lines64 = 0;
    k_count_lines<<<nbt, MTX_THREADS, 0, ctx->stream>>>(T, S, blk);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "count lines")) != GC_OK) return s;
    if ((s = scan_blocks(ctx, blk, nbt, &n_lines64)) != GC_OK) return s;
    const uint32_t n_lines = (uint32_t)n_lines64;
    uint64_t *starts = nullptr;
    uint32_t *A = nullptr, *B = nullptr;
    uint8_t *is_data = nullptr;
    if ((s = sc.get(&starts, n_lines, "line starts")) != GC_OK) return s;
    if ((s = sc.get(&A, n_lines, "entries")) != GC_OK) return s;
    if ((s = sc.get(&B, n_lines, "entries")) != GC_OK) return s;
    if ((s = sc.get(&is_data, n_lines, "entry flags")) != GC_OK) return s;
    if (n_lines) {
        k_write_lines<<<nbt, MTX_THREADS, 0, ctx->stream>>>(T, S, blk, starts);
        // 2. parse
        k_parse_lines<<<ctx->num_sms * 8, MTX_THREADS, 0, ctx->stream>>>(T, S, starts, n_lines, A, B, is_data);
        ctx->launches += 2;
        if ((s = gc_check_launch(ctx, "parse lines")) != GC_OK) return s;
    }
    // 3. the first L data lines as directed pairs
    const uint32_t nbl = (n_lines + ITEMS_PER_BLOCK - 1) / ITEMS_PER_BLOCK;
    uint64_t n_data = 0;
    if (nbl) {
        k_count_flags<<<nbl, MTX_THREADS, 0, ctx->stream>>>(is_data, n_lines, blk);
        ctx->launches++;
        if ((s = scan_blocks(ctx, blk, nbl, &n_data)) != GC_OK) return s;
    }
    if (n_data < L) return gc_fail(ctx, GC_ERR_FORMAT, "fewer entries than the header announces");
    const uint32_t P = 2 * L;
    uint32_t *row = nullptr, *col = nullptr, *k2 = nullptr, *v2 = nullptr, *kb = nullptr, *vb = nullptr,
             *hist = nullptr;
    if ((s = sc.get(&row, P, "pairs")) != GC_OK) return s;
    if ((s = sc.get(&col, P, "pairs")) != GC_OK) return s;
    if ((s = sc.get(&k2, P, "pairs")) != GC_OK) return s;
    if ((s = sc.get(&v2, P, "pairs")) != GC_OK) return s;
    if ((s = sc.get(&kb, P, "sort buffers")) != GC_OK) return s;
    if ((s = sc.get(&vb, P, "sort buffers")) != GC_OK) return s;
    if ((s = sc.get(&hist, gc_sort_pairs_hist_words(P), "sort histogram")) != GC_OK) return s;
    if ((s = gc_reset_state(ctx)) != GC_OK) return s;
    if (nbl) {
        k_emit_pairs<<<nbl, MTX_THREADS, 0, ctx->stream>>>(is_data, A, B, n_lines, blk, L, N, row, col, ctx->dstate);
        ctx->launches++;
    }
    if ((s = gc_read_state(ctx)) != GC_OK)
        return s == GC_ERR_DEVICE ? gc_fail(ctx, GC_ERR_FORMAT, "Matrix Market entry outside 1..N") : s;
    // 4. by column (value: row), then stably by row (value: column): (row, col) in (row, col) order
    const int bits = bit_width(N);  // ids and the sentinel N
    if ((s = gc_sort_pairs(ctx, P, col, row, bits, kb, vb, k2, v2, hist)) != GC_OK) return s;
    if ((s = gc_sort_pairs(ctx, P, v2, k2, bits, kb, vb, row, col, hist)) != GC_OK) return s;
    // 5. dedupe, compact, row offsets
    const uint32_t nbp = (P + ITEMS_PER_BLOCK - 1) / ITEMS_PER_BLOCK;
    uint64_t M64 = 0;
    if (nbp) {
        k_count_kept<<<nbp, MTX_THREADS, 0, ctx->stream>>>(row, col, P, N, blk);
        ctx->launches++;
        if ((s = scan_blocks(ctx, blk, nbp, &M64)) != GC_OK) return s;
    }
    const uint32_t M = (uint32_t)M64;
    gc_graph *g = nullptr;
    if ((s = gc_graph_create(ctx, N, M, &g)) != GC_OK) return s;
    uint32_t *rows_out = k2;  // free again after the sorts
    if (nbp) {
        k_compact_pairs<<<nbp, MTX_THREADS, 0, ctx->stream>>>(row, col, P, N, blk, g->E, rows_out);
        ctx->launches++;
    }
    k_row_offsets<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(rows_out, M, N, g->V);
    ctx->launches++;
    if ((s = gc_check_launch(ctx, "csr from pairs")) != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    g->N = N;
    g->M = M;
    if ((s = gc_graph_finish_upload(g)) != GC_OK) {
        gc_graph_free(g);
        return s;
    }
    *out = g;
    return GC_OK;
}

}  // namespace

extern "C" {

gc_status gc_graph_load_mtx(gc_ctx *ctx, const char *path, gc_graph **g) {
    if (!ctx || !path || !g) return GC_ERR_INVALID;
    *g = nullptr;
    DeviceGuard dg(ctx);
    return load(ctx, path, g);
}

gc_status gc_mtx_read_device(gc_ctx *ctx, const char *path, uint32_t *N, uint32_t **V, uint32_t **E) {
    if (!ctx || !path || !N || !V || !E) return GC_ERR_INVALID;
    DeviceGuard dg(ctx);
    gc_graph *g = nullptr;
    gc_status s = load(ctx, path, &g);
    if (s != GC_OK) return s;
    const uint32_t n = g->N, m = g->M;
    uint32_t *v = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    uint32_t *e = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    if (!v || !e) {
        free(v);
        free(e);
        gc_graph_free(g);
        return gc_fail(ctx, GC_ERR_NOMEM, "host CSR");
    }
    s = gc_check_cuda(ctx, cudaMemcpyAsync(v, g->V, 4ull * (n + 1), cudaMemcpyDeviceToHost, ctx->stream), "download V");
    if (s == GC_OK && m)
        s = gc_check_cuda(ctx, cudaMemcpyAsync(e, g->E, 4ull * m, cudaMemcpyDeviceToHost, ctx->stream), "download E");
    if (s == GC_OK) s = gc_check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "download CSR");
    gc_graph_free(g);
    if (s != GC_OK) {
        free(v);
        free(e);
        return s;
    }
    *N = n;
    *V = v;
    *E = e;
    return GC_OK;
}

}  // extern "C"
