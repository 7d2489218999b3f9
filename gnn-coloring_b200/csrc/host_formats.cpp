// The reference's other graph formats (src/fast_io.c:224-437): GBBS adjacency graphs, PACE .gr and
// METIS .graph readers and writers, and the Matrix Market writer.  The readers return the CSR each
// of the reference's readers returns -- not yet symmetric, sorted or simple -- so that callers that
// run the reference's own clean-up steps afterwards get the reference's V and E; gc_read_graph does
// the whole pipeline and returns the simple, sorted CSR the coloring path expects.
//
// Number scanning follows the reference's parser (fast_io.c:7-15): skip every byte that is not a
// decimal digit, then read the digits.  Files are read whole, with a newline and a NUL appended, so
// a missing final newline never reads past the buffer.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fast_io.h"
#include "gnn_coloring.h"
#include "host_graph.h"

namespace {

struct Text {
    std::vector<char> d;
    size_t i = 0;
    bool ok = false;
    explicit Text(FILE *f) {
        if (!f) return;
        if (fseek(f, 0, SEEK_END) != 0) return;
        const long size = ftell(f);
        if (size < 0 || fseek(f, 0, SEEK_SET) != 0) return;
        d.resize((size_t)size + 2);
        if (size && fread(d.data(), 1, (size_t)size, f) != (size_t)size) return;
        d[(size_t)size] = '\n';
        d[(size_t)size + 1] = '\0';
        ok = true;
    }
    bool end() const { return i + 1 >= d.size(); }
    // the next decimal number; false at the end of the text
    bool number(uint32_t *v) {
        while (!end() && (d[i] < '0' || d[i] > '9')) i++;
        if (end()) return false;
        uint32_t x = 0;
        while (d[i] >= '0' && d[i] <= '9') x = x * 10 + (uint32_t)(d[i++] - '0');
        *v = x;
        return true;
    }
    void skip_line() {
        while (!end() && d[i] != '\n') i++;
        if (!end()) i++;
    }
    void skip_comments(char c) {
        while (!end() && d[i] == c) skip_line();
    }
};

[[noreturn]] void die(const char *what) {
    fprintf(stderr, "%s\n", what);
    exit(1);
}

template <class T>
T *alloc_or_die(size_t n) {
    T *p = (T *)malloc(sizeof(T) * (n ? n : 1));
    if (!p) die("out of memory");
    return p;
}

// PACE .gr edges into the reference's CSR: both directions, each row filled from its end in edge
// order (fast_io.c:322-350), so a row lists its neighbours in reverse order of appearance.
void pairs_to_csr_reversed(uint32_t N, const std::vector<uint32_t> &I, const std::vector<uint32_t> &J, uint32_t **V,
                           uint32_t **E) {
    uint32_t *v = alloc_or_die<uint32_t>((size_t)N + 1);
    std::fill(v, v + N + 1, 0u);
    for (size_t k = 0; k < I.size(); k++) {
        v[I[k]]++;
        v[J[k]]++;
    }
    for (uint32_t u = 1; u <= N; u++) v[u] += v[u - 1];
    uint32_t *e = alloc_or_die<uint32_t>(2 * I.size());
    for (size_t k = 0; k < I.size(); k++) {
        e[--v[I[k]]] = J[k];
        e[--v[J[k]]] = I[k];
    }
    *V = v;
    *E = e;
}

}  // namespace

extern "C" {

void adj_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E) {
    Text t(f);
    if (!t.ok) die("adj_parse: unreadable file");
    uint32_t n = 0, m = 0;
    if (!t.number(&n) || !t.number(&m)) die("adj_parse: missing header");
    uint32_t *v = alloc_or_die<uint32_t>((size_t)n + 1);
    for (uint32_t j = 0; j < n; j++)
        if (!t.number(v + j)) die("adj_parse: truncated offsets");
    v[n] = m;
    uint32_t *e = alloc_or_die<uint32_t>(m);
    for (uint32_t j = 0; j < m; j++)
        if (!t.number(e + j)) die("adj_parse: truncated edges");
    *N = n;
    *V = v;
    *E = e;
}

void adj_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E) {
    fprintf(f, "AdjacencyGraph\n%u\n%u\n", N, V[N]);
    for (uint32_t u = 0; u < N; u++) fprintf(f, "%u\n", V[u]);
    for (uint32_t i = 0; i < V[N]; i++) fprintf(f, "%u\n", E[i]);
}

void gr_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E) {
    Text t(f);
    if (!t.ok) die("gr_parse: unreadable file");
    t.skip_comments('c');
    uint32_t n = 0, m = 0;
    if (!t.number(&n) || !t.number(&m)) die("gr_parse: missing p line");
    std::vector<uint32_t> I(m), J(m);
    for (uint32_t k = 0; k < m; k++) {
        t.skip_line();
        t.skip_comments('c');
        uint32_t x = 0, y = 0;
        if (!t.number(&x) || !t.number(&y)) die("gr_parse: truncated edge list");
        if (x < 1 || y < 1 || x > n || y > n) die("gr_parse: vertex out of range");
        I[k] = x - 1;
        J[k] = y - 1;
    }
    *N = n;
    pairs_to_csr_reversed(n, I, J, V, E);
}

void gr_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E) {
    fprintf(f, "p td %u %u\n", N, V[N] / 2);
    for (uint32_t u = 0; u < N; u++)
        for (uint32_t i = V[u]; i < V[u + 1]; i++)
            if (E[i] > u) fprintf(f, "%u %u\n", u + 1, E[i] + 1);
}

void metis_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E, uint32_t **W) {
    Text t(f);
    if (!t.ok) die("metis_parse: unreadable file");
    t.skip_comments('%');
    uint32_t n = 0, m = 0, fmt = 0;
    if (!t.number(&n) || !t.number(&m) || !t.number(&fmt)) die("metis_parse: missing header");
    const bool vweights = fmt == 10 || fmt == 11, eweights = fmt == 1 || fmt == 11;
    const size_t cap = 2 * (size_t)m;
    uint32_t *v = alloc_or_die<uint32_t>((size_t)n + 1);
    uint32_t *e = alloc_or_die<uint32_t>(cap);
    uint32_t *w = vweights ? alloc_or_die<uint32_t>(n) : nullptr;
    v[0] = 0;
    for (uint32_t u = 0; u < n; u++) {
        t.skip_line();
        t.skip_comments('%');
        if (vweights && !t.number(w + u)) die("metis_parse: truncated vertex weights");
        size_t s = v[u];
        // neighbours (1-based) up to the end of the line; spaces after the last one are skipped
        while (!t.end() && t.d[t.i] != '\n' && s < cap) {
            uint32_t x = 0, ew = 0;
            if (!t.number(&x)) break;
            if (x < 1 || x > n) die("metis_parse: vertex out of range");
            e[s++] = x - 1;
            if (eweights) t.number(&ew);
            while (t.d[t.i] == ' ' && s < cap) t.i++;
        }
        v[u + 1] = (uint32_t)s;
    }
    *N = n;
    *V = v;
    *E = e;
    *W = w;
}

void metis_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E, const uint32_t *W) {
    fprintf(f, "%u %u %u\n", N, V[N] / 2, W == nullptr ? 0u : 10u);
    for (uint32_t u = 0; u < N; u++) {
        if (W) fprintf(f, "%u ", W[u]);
        for (uint32_t i = V[u]; i < V[u + 1]; i++) fprintf(f, "%u ", E[i] + 1);
        fprintf(f, "\n");
    }
}

void mtx_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E) {
    // the reference writes its banner through a format string, so one '%' appears (fast_io.c:226)
    fprintf(f, "%%MatrixMarket matrix coordinate patter symmetric\n%u %u %u\n", N, N, V[N] / 2);
    for (uint32_t u = 0; u < N; u++)
        for (uint32_t i = V[u]; i < V[u + 1]; i++)
            if (E[i] > u) fprintf(f, "%u %u\n", u + 1, E[i] + 1);
}

gc_status gc_read_graph(const char *path, uint32_t *N, uint32_t **V, uint32_t **E) {
    if (!path || !N || !V || !E) return GC_ERR_INVALID;
    const std::string p(path);
    auto ends = [&](const char *x) {
        const size_t n = strlen(x);
        return p.size() >= n && p.compare(p.size() - n, n, x) == 0;
    };
    if (ends(".mtx")) return gc_mtx_read(path, N, V, E);
    FILE *f = fopen(path, "rb");
    if (!f) return GC_ERR_IO;
    uint32_t n = 0, *v = nullptr, *e = nullptr, *w = nullptr;
    if (ends(".gr")) gr_parse(f, &n, &v, &e);
    else if (ends(".graph")) metis_parse(f, &n, &v, &e, &w);
    else if (ends(".adj")) adj_parse(f, &n, &v, &e);
    else {
        fclose(f);
        return GC_ERR_FORMAT;
    }
    fclose(f);
    free(w);
    // every entry in both directions, then sorted and simple: the rules of the Matrix Market path
    const uint64_t L = v[n];
    std::vector<uint32_t> I(L), J(L);
    for (uint32_t u = 0; u < n; u++)
        for (uint32_t i = v[u]; i < v[u + 1]; i++) {
            if (e[i] >= n) {
                free(v);
                free(e);
                return GC_ERR_FORMAT;
            }
            I[i] = u;
            J[i] = e[i];
        }
    free(v);
    free(e);
    *N = n;
    return gc_csr_from_pairs(n, L, I.data(), J.data(), V, E);
}

}  // extern "C"
