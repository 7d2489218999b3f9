// Host-side graph preparation: CSR construction with the reference's simplification rules,
// Matrix Market and .gnn readers, and seeded synthetic graph generators.
//
// CSR rules follow the reference's loader (src/fast_io.c): every Matrix Market entry (i, j) is
// added in both directions (mtx_to_graph_par, fast_io.c:171-202), N = max(rows, cols)
// (fast_io.c:86-87), adjacency lists are sorted ascending (graph_sort_edges_par,
// fast_io.c:450-455) and self-loops and repeated neighbours are dropped (graph_make_simple,
// fast_io.c:457-477).  The result is independent of the thread count.
#include <omp.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gnn_coloring.h"
#include "fast_io.h"
#include "host_graph.h"

namespace {

inline uint64_t splitmix64_next(uint64_t &s) {
    // SplitMix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number generators", 2014).
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// A stream keyed by (seed, index): independent of the order in which indices are visited.
inline uint64_t stream_state(uint64_t seed, uint64_t index) {
    uint64_t s = seed * 0xd1b54a32d192ed03ULL + 0x2545f4914f6cdd1dULL;
    uint64_t a = splitmix64_next(s);
    s = a ^ (index * 0x9e3779b97f4a7c15ULL);
    splitmix64_next(s);
    return s;
}

inline double uniform01(uint64_t &s) { return (double)(splitmix64_next(s) >> 11) * 0x1.0p-53; }

}  // namespace

// Counting-sort the 2L directed entries by source, then sort and simplify each list.
gc_status gc_csr_build(uint32_t N, uint64_t L, const uint32_t *I, const uint32_t *J,
                       uint32_t **V_out, uint32_t **E_out) {
    if (!V_out || !E_out || (L > 0 && (!I || !J))) return GC_ERR_INVALID;
    if (2 * L > 0xffffffffULL) return GC_ERR_INVALID;
    int out_of_range = 0;
#pragma omp parallel for schedule(static) reduction(| : out_of_range)
    for (uint64_t k = 0; k < L; k++) out_of_range |= (I[k] >= N) | (J[k] >= N);
    if (out_of_range) return GC_ERR_INVALID;

    uint64_t *off = (uint64_t *)calloc((size_t)N + 1, sizeof(uint64_t));
    uint32_t *V = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)N + 1));
    if (!off || !V) {
        free(off);
        free(V);
        return GC_ERR_NOMEM;
    }
    // Inside an enclosing parallel region (many graphs built at once) or for small inputs the
    // passes run on this thread alone, without atomics.
    const bool par = !omp_in_parallel() && L >= (1u << 16);
    // degree count
    if (par) {
#pragma omp parallel for schedule(static)
        for (uint64_t k = 0; k < L; k++) {
            __atomic_add_fetch(&off[I[k] + 1], 1, __ATOMIC_RELAXED);
            __atomic_add_fetch(&off[J[k] + 1], 1, __ATOMIC_RELAXED);
        }
    } else {
        for (uint64_t k = 0; k < L; k++) {
            off[I[k] + 1]++;
            off[J[k] + 1]++;
        }
    }
    for (uint32_t u = 0; u < N; u++) off[u + 1] += off[u];
    uint64_t M2 = off[N];
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (M2 ? M2 : 1));
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)N + 1));
    if (!tmp || !cur) {
        free(off);
        free(V);
        free(tmp);
        free(cur);
        return GC_ERR_NOMEM;
    }
    memcpy(cur, off, sizeof(uint64_t) * ((size_t)N + 1));
    if (par) {
#pragma omp parallel for schedule(static)
        for (uint64_t k = 0; k < L; k++) {
            uint64_t a = __atomic_fetch_add(&cur[I[k]], 1, __ATOMIC_RELAXED);
            tmp[a] = J[k];
            uint64_t b = __atomic_fetch_add(&cur[J[k]], 1, __ATOMIC_RELAXED);
            tmp[b] = I[k];
        }
    } else {
        for (uint64_t k = 0; k < L; k++) {
            tmp[cur[I[k]]++] = J[k];
            tmp[cur[J[k]]++] = I[k];
        }
    }
    free(cur);
    // sort + simplify each list in place; record the kept count
    uint32_t *kept = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)N + 1));
    if (!kept) {
        free(off);
        free(V);
        free(tmp);
        return GC_ERR_NOMEM;
    }
#pragma omp parallel for schedule(dynamic, 1024) if (par)
    for (uint32_t u = 0; u < N; u++) {
        uint32_t *a = tmp + off[u];
        uint64_t d = off[u + 1] - off[u];
        if (d <= 24) {  // short lists: insertion sort
            for (uint64_t i = 1; i < d; i++) {
                const uint32_t x = a[i];
                uint64_t j = i;
                for (; j > 0 && a[j - 1] > x; j--) a[j] = a[j - 1];
                a[j] = x;
            }
        } else {
            std::sort(a, a + d);
        }
        uint64_t w = 0;
        for (uint64_t i = 0; i < d; i++) {
            uint32_t v = a[i];
            if (v == u || (i > 0 && v == a[i - 1])) continue;
            a[w++] = v;
        }
        kept[u] = (uint32_t)w;
    }
    V[0] = 0;
    for (uint32_t u = 0; u < N; u++) V[u + 1] = V[u] + kept[u];
    free(kept);
    uint32_t M = V[N];
    uint32_t *E = (uint32_t *)malloc(sizeof(uint32_t) * (M ? M : 1));
    if (!E) {
        free(off);
        free(V);
        free(tmp);
        return GC_ERR_NOMEM;
    }
#pragma omp parallel for schedule(dynamic, 1024) if (par)
    for (uint32_t u = 0; u < N; u++)
        memcpy(E + V[u], tmp + off[u], sizeof(uint32_t) * (V[u + 1] - V[u]));
    free(tmp);
    free(off);
    *V_out = V;
    *E_out = E;
    return GC_OK;
}

extern "C" {

gc_status gc_csr_from_pairs(uint32_t N, uint64_t L, const uint32_t *I, const uint32_t *J,
                            uint32_t **V, uint32_t **E) {
    return gc_csr_build(N, L, I, J, V, E);
}

void gc_host_free(void *p) { free(p); }

// ---- Matrix Market ----------------------------------------------------------------------------

// Reads the raw entry list: header comments, "rows cols nnz", then nnz lines "i j [value]".
// Indices are 1-based; 0 or > max(rows, cols) is a format error (the reference would index out
// of bounds there).  Comment lines between entries are skipped, as in mtx_parse_raw
// (fast_io.c:54-59).
// Parses a whole Matrix Market text held in memory.
static gc_status parse_mtx(const char *data, size_t n, uint32_t *N_out, uint64_t *L_out, uint32_t **I_out,
                           uint32_t **J_out) {
    size_t p = 0;
    auto skip_line = [&](size_t &q) {
        while (q < n && data[q] != '\n') q++;
        if (q < n) q++;
    };
    auto parse_uint = [&](size_t &q, uint64_t &v) -> bool {
        while (q < n && (data[q] == ' ' || data[q] == '\t' || data[q] == '\r')) q++;
        if (q >= n || data[q] < '0' || data[q] > '9') return false;
        v = 0;
        while (q < n && data[q] >= '0' && data[q] <= '9') {
            v = v * 10 + (uint64_t)(data[q++] - '0');
            if (v > 0xffffffffULL) return false;
        }
        return true;
    };

    while (p < n && data[p] == '%') skip_line(p);
    while (p < n && (data[p] == '\n' || data[p] == '\r')) p++;
    uint64_t rows, cols, nnz;
    if (!parse_uint(p, rows) || !parse_uint(p, cols) || !parse_uint(p, nnz)) return GC_ERR_FORMAT;
    skip_line(p);
    uint64_t N = rows > cols ? rows : cols;
    uint32_t *I = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    uint32_t *J = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    if (!I || !J) {
        free(I);
        free(J);
        return GC_ERR_NOMEM;
    }
    for (uint64_t k = 0; k < nnz; k++) {
        while (p < n && (data[p] == '%' || data[p] == '\n' || data[p] == '\r')) skip_line(p);
        uint64_t a, b;
        if (!parse_uint(p, a) || !parse_uint(p, b) || a == 0 || b == 0 || a > N || b > N) {
            free(I);
            free(J);
            return GC_ERR_FORMAT;
        }
        I[k] = (uint32_t)(a - 1);
        J[k] = (uint32_t)(b - 1);
        skip_line(p);
    }
    *N_out = (uint32_t)N;
    *L_out = nnz;
    *I_out = I;
    *J_out = J;
    return GC_OK;
}

static gc_status read_all(FILE *f, char **data, size_t *n) {
    size_t cap = 1 << 20, len = 0;
    char *buf = (char *)malloc(cap);
    if (!buf) return GC_ERR_NOMEM;
    for (;;) {
        if (len == cap) {
            char *nb = (char *)realloc(buf, cap * 2);
            if (!nb) {
                free(buf);
                return GC_ERR_NOMEM;
            }
            buf = nb;
            cap *= 2;
        }
        size_t got = fread(buf + len, 1, cap - len, f);
        len += got;
        if (got == 0) break;
    }
    if (ferror(f)) {
        free(buf);
        return GC_ERR_IO;
    }
    *data = buf;
    *n = len;
    return GC_OK;
}

gc_status gc_mtx_read_pairs_file(FILE *f, uint32_t *N, uint64_t *L, uint32_t **I, uint32_t **J) {
    char *data;
    size_t n;
    gc_status s = read_all(f, &data, &n);
    if (s != GC_OK) return s;
    s = parse_mtx(data, n, N, L, I, J);
    free(data);
    return s;
}

gc_status gc_mtx_read_pairs(const char *path, uint32_t *N, uint64_t *L, uint32_t **I, uint32_t **J) {
    FILE *f = fopen(path, "rb");
    if (!f) return GC_ERR_IO;
    gc_status s = gc_mtx_read_pairs_file(f, N, L, I, J);
    fclose(f);
    return s;
}

gc_status gc_mtx_read(const char *path, uint32_t *N, uint32_t **V, uint32_t **E) {
    if (!path || !N || !V || !E) return GC_ERR_INVALID;
    uint32_t n, *I, *J;
    uint64_t L;
    gc_status s = gc_mtx_read_pairs(path, &n, &L, &I, &J);
    if (s != GC_OK) return s;
    s = gc_csr_build(n, L, I, J, V, E);
    free(I);
    free(J);
    if (s == GC_OK) *N = n;
    return s;
}

gc_status gc_mtx_write(const char *path, uint32_t N, const uint32_t *V, const uint32_t *E) {
    FILE *f = fopen(path, "w");
    if (!f) return GC_ERR_IO;
    uint64_t L = 0;
    for (uint32_t u = 0; u < N; u++)
        for (uint32_t i = V[u]; i < V[u + 1]; i++)
            if (E[i] < u) L++;
    fprintf(f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n");
    fprintf(f, "%u %u %llu\n", N, N, (unsigned long long)L);
    for (uint32_t u = 0; u < N; u++)
        for (uint32_t i = V[u]; i < V[u + 1]; i++)
            if (E[i] < u) fprintf(f, "%u %u\n", u + 1, E[i] + 1);
    int bad = ferror(f);
    fclose(f);
    return bad ? GC_ERR_IO : GC_OK;
}

// ---- .gnn model files ------------------------------------------------------------------------

// Format of src/gnn.c:33-40: "params md" then params whitespace-separated floats, parsed like
// fscanf("%f") (strtof, round to nearest).
gc_status gc_model_read(const char *path, int *params, int *md, float **param) {
    if (!path || !params || !md || !param) return GC_ERR_INVALID;
    FILE *f = fopen(path, "r");
    if (!f) return GC_ERR_IO;
    int np = 0, m = 0;
    if (fscanf(f, "%d %d", &np, &m) != 2 || np <= 0 || np % 528 != 0 || np / 528 < 2) {
        fclose(f);
        return GC_ERR_FORMAT;
    }
    float *w = (float *)malloc(sizeof(float) * (size_t)np);
    if (!w) {
        fclose(f);
        return GC_ERR_NOMEM;
    }
    for (int i = 0; i < np; i++) {
        if (fscanf(f, "%f", w + i) != 1) {
            free(w);
            fclose(f);
            return GC_ERR_FORMAT;
        }
    }
    fclose(f);
    *params = np;
    *md = m;
    *param = w;
    return GC_OK;
}

// ---- generators -------------------------------------------------------------------------------

gc_status gc_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t **V, uint32_t **E) {
    if (!V || !E) return GC_ERR_INVALID;
    if (n < 2 && m > 0) return GC_ERR_INVALID;
    if (m > (uint64_t)n * (n - 1) / 2) return GC_ERR_INVALID;
    // Open-addressing set of accepted pairs; the accepted sequence is the stream order.
    uint64_t cap = 16;
    while (cap < 2 * m + 16) cap <<= 1;
    std::vector<uint64_t> table(cap, 0);
    std::vector<uint32_t> I, J;
    I.reserve(m);
    J.reserve(m);
    uint64_t s = stream_state(seed, 0x45525f6772617068ULL);
    while (I.size() < m) {
        uint64_t r = splitmix64_next(s);
        uint32_t a = (uint32_t)(((r & 0xffffffffULL) * n) >> 32);
        uint32_t b = (uint32_t)(((r >> 32) * n) >> 32);
        if (a == b) continue;
        uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
        uint64_t key = ((uint64_t)hi << 32 | lo) + 1;
        uint64_t h = (key * 0x9e3779b97f4a7c15ULL) & (cap - 1);
        bool fresh = true;
        while (table[h]) {
            if (table[h] == key) {
                fresh = false;
                break;
            }
            h = (h + 1) & (cap - 1);
        }
        if (!fresh) continue;
        table[h] = key;
        I.push_back(hi);
        J.push_back(lo);
    }
    return gc_csr_build(n, m, I.data(), J.data(), V, E);
}

gc_status gc_gen_rmat(uint32_t n, double ef, double a, double b, double c, uint64_t seed,
                      uint32_t **V, uint32_t **E) {
    if (!V || !E || n == 0 || ef < 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
        return GC_ERR_INVALID;
    uint32_t scale = 0;
    while (scale < 32 && (1ULL << scale) < n) scale++;
    uint64_t samples = (uint64_t)llround(ef * (double)n);
    if (2 * samples > 0xffffffffULL) return GC_ERR_INVALID;
    uint32_t *I = (uint32_t *)malloc(sizeof(uint32_t) * (samples ? samples : 1));
    uint32_t *J = (uint32_t *)malloc(sizeof(uint32_t) * (samples ? samples : 1));
    uint8_t *keep = (uint8_t *)malloc(samples ? samples : 1);
    if (!I || !J || !keep) {
        free(I);
        free(J);
        free(keep);
        return GC_ERR_NOMEM;
    }
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (uint64_t k = 0; k < samples; k++) {
        uint64_t s = stream_state(seed, k);
        uint64_t u = 0, v = 0;
        for (uint32_t bit = 0; bit < scale; bit++) {
            double r = uniform01(s);
            uint64_t ub = r >= ab, vb = (r >= a && r < ab) || r >= abc;
            u |= ub << bit;
            v |= vb << bit;
        }
        keep[k] = (u < n && v < n);
        I[k] = (uint32_t)u;
        J[k] = (uint32_t)v;
    }
    uint64_t w = 0;
    for (uint64_t k = 0; k < samples; k++)
        if (keep[k]) {
            I[w] = I[k];
            J[w] = J[k];
            w++;
        }
    free(keep);
    gc_status st = gc_csr_build(n, w, I, J, V, E);
    free(I);
    free(J);
    return st;
}

gc_status gc_gen_rgg2d(uint32_t n, double radius, uint64_t seed, uint32_t **V, uint32_t **E) {
    if (!V || !E || n == 0 || !(radius > 0)) return GC_ERR_INVALID;
    std::vector<double> x(n), y(n);
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < n; i++) {
        uint64_t s = stream_state(seed, i);
        x[i] = uniform01(s);
        y[i] = uniform01(s);
    }
    // bucket grid with cell side >= radius
    uint32_t g = (uint32_t)std::max(1.0, std::floor(1.0 / radius));
    if (g > 65536) g = 65536;
    std::vector<uint32_t> cell_of(n), cell_start((size_t)g * g + 1, 0), order(n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t cx = std::min(g - 1, (uint32_t)(x[i] * g));
        uint32_t cy = std::min(g - 1, (uint32_t)(y[i] * g));
        cell_of[i] = cy * g + cx;
        cell_start[cell_of[i] + 1]++;
    }
    for (size_t c = 0; c < (size_t)g * g; c++) cell_start[c + 1] += cell_start[c];
    {
        std::vector<uint32_t> fill(cell_start.begin(), cell_start.end() - 1);
        for (uint32_t i = 0; i < n; i++) order[fill[cell_of[i]]++] = i;
    }
    const double r2 = radius * radius;
    int nt = omp_get_max_threads();
    std::vector<std::vector<uint32_t>> PI(nt), PJ(nt);
#pragma omp parallel
    {
        int t = omp_get_thread_num();
#pragma omp for schedule(dynamic, 4096)
        for (uint32_t i = 0; i < n; i++) {
            int cx = (int)(cell_of[i] % g), cy = (int)(cell_of[i] / g);
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    int nx = cx + dx, ny = cy + dy;
                    if (nx < 0 || ny < 0 || nx >= (int)g || ny >= (int)g) continue;
                    size_t c = (size_t)ny * g + nx;
                    for (uint32_t q = cell_start[c]; q < cell_start[c + 1]; q++) {
                        uint32_t j = order[q];
                        if (j <= i) continue;
                        double ddx = x[i] - x[j], ddy = y[i] - y[j];
                        if (ddx * ddx + ddy * ddy < r2) {
                            PI[t].push_back(i);
                            PJ[t].push_back(j);
                        }
                    }
                }
        }
    }
    size_t L = 0;
    for (int t = 0; t < nt; t++) L += PI[t].size();
    std::vector<uint32_t> I, J;
    I.reserve(L);
    J.reserve(L);
    for (int t = 0; t < nt; t++) {
        I.insert(I.end(), PI[t].begin(), PI[t].end());
        J.insert(J.end(), PJ[t].begin(), PJ[t].end());
    }
    return gc_csr_build(n, L, I.data(), J.data(), V, E);
}

gc_status gc_gen_stencil27(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t **V_out, uint32_t **E_out) {
    if (!V_out || !E_out || nx == 0 || ny == 0 || nz == 0) return GC_ERR_INVALID;
    uint64_t N64 = (uint64_t)nx * ny * nz;
    if (N64 >= 0xffffffffULL) return GC_ERR_INVALID;
    uint32_t N = (uint32_t)N64;
    auto span = [](uint32_t c, uint32_t n) -> uint64_t { return (c > 0) + 1 + (c + 1 < n); };
    uint32_t *V = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)N + 1));
    if (!V) return GC_ERR_NOMEM;
    V[0] = 0;
    uint64_t acc = 0;
    for (uint32_t z = 0; z < nz; z++)
        for (uint32_t y = 0; y < ny; y++)
            for (uint32_t x = 0; x < nx; x++) {
                acc += span(x, nx) * span(y, ny) * span(z, nz) - 1;
                if (acc > 0xffffffffULL) {
                    free(V);
                    return GC_ERR_INVALID;
                }
                V[((size_t)z * ny + y) * nx + x + 1] = (uint32_t)acc;
            }
    uint32_t *E = (uint32_t *)malloc(sizeof(uint32_t) * (acc ? acc : 1));
    if (!E) {
        free(V);
        return GC_ERR_NOMEM;
    }
#pragma omp parallel for schedule(static) collapse(2)
    for (uint32_t z = 0; z < nz; z++)
        for (uint32_t y = 0; y < ny; y++)
            for (uint32_t x = 0; x < nx; x++) {
                uint32_t u = (uint32_t)(((size_t)z * ny + y) * nx + x);
                uint32_t w = V[u];
                // ascending ids: z-major, then y, then x
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dx = -1; dx <= 1; dx++) {
                            if (!dx && !dy && !dz) continue;
                            int64_t X = (int64_t)x + dx, Y = (int64_t)y + dy, Z = (int64_t)z + dz;
                            if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                            E[w++] = (uint32_t)((Z * ny + Y) * nx + X);
                        }
            }
    *V_out = V;
    *E_out = E;
    return GC_OK;
}

gc_status gc_gen_mixed(uint64_t seed, uint32_t n_min, uint32_t n_max, uint32_t *n_out, int *kind_out,
                       double *param_out, uint32_t **V, uint32_t **E) {
    if (!V || !E || n_min < 2 || n_max < n_min) return GC_ERR_INVALID;
    uint64_t s = stream_state(seed, 0x6d69786564ULL);
    const double lo = std::log((double)n_min), hi = std::log((double)n_max);
    double nf = std::exp(lo + uniform01(s) * (hi - lo));
    uint32_t n = (uint32_t)std::llround(nf);
    n = std::min(std::max(n, n_min), n_max);
    const int kind = (int)(seed & 1);
    double param;
    gc_status st;
    if (kind == 0) {
        param = 8.0 + 24.0 * uniform01(s);
        uint64_t m = (uint64_t)std::llround((double)n * param / 2.0);
        m = std::min<uint64_t>(m, (uint64_t)n * (n - 1) / 2);
        st = gc_gen_er(n, m, seed, V, E);
    } else {
        param = 8.0;
        st = gc_gen_rmat(n, param, 0.57, 0.19, 0.19, seed, V, E);
    }
    if (st != GC_OK) return st;
    if (n_out) *n_out = n;
    if (kind_out) *kind_out = kind;
    if (param_out) *param_out = param;
    return GC_OK;
}

gc_status gc_gen_mixed_batch(uint32_t G, uint64_t seed0, uint32_t n_min, uint32_t n_max, uint32_t **voff_out,
                             uint32_t **V_out, uint32_t **E_out) {
    if (!voff_out || !V_out || !E_out || n_min < 2 || n_max < n_min) return GC_ERR_INVALID;
    std::vector<uint32_t *> Vs(G, nullptr), Es(G, nullptr);
    std::vector<uint32_t> ns(G, 0);
    int failed = 0;
    // graphs in parallel; each generator's own parallel loops run single-threaded inside
#pragma omp parallel for schedule(dynamic, 1) reduction(| : failed)
    for (uint32_t i = 0; i < G; i++)
        if (gc_gen_mixed(seed0 + i, n_min, n_max, &ns[i], nullptr, nullptr, &Vs[i], &Es[i]) != GC_OK) failed = 1;
    auto release = [&]() {
        for (uint32_t i = 0; i < G; i++) {
            free(Vs[i]);
            free(Es[i]);
        }
    };
    if (failed) {
        release();
        return GC_ERR_NOMEM;
    }
    uint32_t *voff = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)G + 1));
    std::vector<uint64_t> eoff((size_t)G + 1, 0);
    if (!voff) {
        release();
        return GC_ERR_NOMEM;
    }
    uint64_t nv = 0;
    voff[0] = 0;
    for (uint32_t i = 0; i < G; i++) {
        nv += ns[i];
        eoff[i + 1] = eoff[i] + Vs[i][ns[i]];
        if (nv >= 0xffffffffULL || eoff[i + 1] > 0xffffffffULL) {
            release();
            free(voff);
            return GC_ERR_INVALID;
        }
        voff[i + 1] = (uint32_t)nv;
    }
    uint32_t *V = (uint32_t *)malloc(sizeof(uint32_t) * (nv + 1));
    uint32_t *E = (uint32_t *)malloc(sizeof(uint32_t) * (eoff[G] ? eoff[G] : 1));
    if (!V || !E) {
        release();
        free(voff);
        free(V);
        free(E);
        return GC_ERR_NOMEM;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t i = 0; i < G; i++) {
        for (uint32_t r = 0; r < ns[i]; r++) V[voff[i] + r] = (uint32_t)eoff[i] + Vs[i][r];
        memcpy(E + eoff[i], Es[i], sizeof(uint32_t) * (eoff[i + 1] - eoff[i]));
        free(Vs[i]);
        free(Es[i]);
        Vs[i] = Es[i] = nullptr;
    }
    V[nv] = (uint32_t)eoff[G];
    *voff_out = voff;
    *V_out = V;
    *E_out = E;
    return GC_OK;
}

// ---- the reference's fast_io.h entry points (host side) --------------------------------------

static void mtx_parse_or_die(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E) {
    uint32_t n, *I, *J;
    uint64_t L;
    gc_status s = gc_mtx_read_pairs_file(f, &n, &L, &I, &J);
    if (s == GC_OK) {
        s = gc_csr_build(n, L, I, J, V, E);
        free(I);
        free(J);
    }
    if (s != GC_OK) {
        fprintf(stderr, "gnn-coloring: cannot parse Matrix Market input: %s\n", gc_status_string(s));
        exit(1);
    }
    *N = n;
}

void mtx_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E) { mtx_parse_or_die(f, N, V, E); }
void mtx_parse_par(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E) { mtx_parse_or_die(f, N, V, E); }

void graph_sort_edges_par(uint32_t N, const uint32_t *V, uint32_t *E) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (uint32_t u = 0; u < N; u++) std::sort(E + V[u], E + V[u + 1]);
}
void graph_sort_edges(uint32_t N, const uint32_t *V, uint32_t *E) {
    for (uint32_t u = 0; u < N; u++) std::sort(E + V[u], E + V[u + 1]);
}

void graph_make_simple(uint32_t N, uint32_t *V, uint32_t **E) {
    uint32_t *e = *E, w = 0, start = 0;
    for (uint32_t u = 0; u < N; u++) {
        uint32_t b = V[u], end = V[u + 1];
        V[u] = start;
        for (uint32_t i = b; i < end; i++) {
            uint32_t v = e[i];
            if (v == u || (i > b && v == e[i - 1])) continue;
            e[w++] = v;
        }
        start = w;
    }
    uint32_t old = V[N];
    V[N] = w;
    if (w < old && w > 0) {
        uint32_t *ne = (uint32_t *)realloc(e, sizeof(uint32_t) * w);
        if (ne) *E = ne;
    }
}

static int in_sorted(const uint32_t *a, uint32_t n, uint32_t x) { return std::binary_search(a, a + n, x); }

uint32_t graph_validate_par(uint32_t N, const uint32_t *V, const uint32_t *E) {
    if (V[0] != 0) return 0;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (uint32_t u = 0; u < N; u++) {
        if (V[u + 1] < V[u]) {
            bad = 1;
            continue;
        }
        for (uint32_t i = V[u]; i < V[u + 1]; i++) {
            uint32_t v = E[i];
            if (v >= N || v == u || (i > V[u] && v <= E[i - 1])) {
                bad = 1;
                break;
            }
            if (V[v + 1] < V[v] || !in_sorted(E + V[v], V[v + 1] - V[v], u)) {
                bad = 1;
                break;
            }
        }
    }
    return bad ? 0 : 1;
}
uint32_t graph_validate(uint32_t N, const uint32_t *V, const uint32_t *E) { return graph_validate_par(N, V, E); }

}  // extern "C"
