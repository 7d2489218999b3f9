// The reference's host functions (include/coloring.h, first_fit.h, largest_degree_first.h,
// smallest_degree_last.h, gnn.h, fast_gnn.h, runner.h of KennethLangedal/GNN-COLORING) with the
// same names, signatures and results, running on the GPU through the native API.
//
// Conventions kept from the reference: void functions, host buffers owned by the caller,
// malloc'd results from *_coloring, opaque setup states, fatal errors print and exit(1)
// (src/gnn.c:28-32).  All calls share one process-wide context (device $GC_DEVICE, default 0),
// guarded by a mutex.
#include <omp.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "coloring.h"
#include "fast_gnn.h"
#include "first_fit.h"
#include "gnn.h"
#include "gnn_coloring.h"
#include "overlap.h"
#include "largest_degree_first.h"
#include "runner.h"
#include "smallest_degree_last.h"

namespace {

std::recursive_mutex g_mu;
gc_ctx *g_ctx = nullptr;

[[noreturn]] void die(const char *what, gc_status s) {
    fprintf(stderr, "gnn-coloring: %s failed: %s%s%s\n", what, gc_status_string(s), g_ctx ? ": " : "",
            g_ctx ? gc_last_error(g_ctx) : "");
    exit(1);
}

void check(gc_status s, const char *what) {
    if (s != GC_OK) die(what, s);
}

gc_ctx *ctx() {
    if (!g_ctx) {
        const char *d = getenv("GC_DEVICE");
        check(gc_ctx_create(d ? atoi(d) : 0, &g_ctx), "GPU context creation");
    }
    return g_ctx;
}

// Coloring state (greedy_setup / jones_plassmann_setup): device memory for one graph.  While a
// runner owns the state, the uploaded graph is bound to the runner's V/E (which the runner
// protocol never changes) and is not re-uploaded per call.
struct ColorState {
    gc_graph *g = nullptr;
    uint32_t cap_N = 0, cap_M = 0;
    const uint32_t *bound_V = nullptr, *bound_E = nullptr;
    uint32_t bound_N = 0;
    bool bind = false;
};

// Heuristic state (X_setup): which heuristic, and the model for GNN.
struct HeurState {
    gc_heuristic h = GC_FF;
    gc_model *model = nullptr;
};

ColorState *new_color_state(uint32_t N, uint32_t M) {
    ColorState *cs = new ColorState();
    cs->cap_N = N;
    cs->cap_M = M;
    check(gc_graph_create(ctx(), N, M, &cs->g), "device allocation");
    return cs;
}

void free_color_state(ColorState *cs) {
    if (!cs) return;
    gc_graph_free(cs->g);
    delete cs;
}

// Puts (N, V, E) into the state's device graph, growing it when needed.
void load_graph(ColorState *cs, uint32_t N, const uint32_t *V, const uint32_t *E, bool gnn = false) {
    if (cs->bind && cs->bound_V == V && cs->bound_E == E && cs->bound_N == N) return;
    std::vector<uint32_t> zeros;
    if (!V) {  // orderings that ignore the graph may be called without one
        zeros.assign((size_t)N + 1, 0);
        V = zeros.data();
    }
    const uint32_t M = V[N];
    if (N > cs->cap_N || M > cs->cap_M) {
        gc_graph_free(cs->g);
        cs->g = nullptr;
        cs->cap_N = N > cs->cap_N ? N : cs->cap_N;
        cs->cap_M = M > cs->cap_M ? M : cs->cap_M;
        check(gc_graph_create(ctx(), cs->cap_N, cs->cap_M, &cs->g), "device allocation");
    }
    gc_graph_gnn_hint(cs->g, gnn);  // GNN priorities follow: E becomes feature rows while it arrives
    check(gc_graph_reupload(ctx(), cs->g, N, V, E), "graph upload");
    if (cs->bind && V != zeros.data()) {
        cs->bound_V = V;
        cs->bound_E = E;
        cs->bound_N = N;
    }
}

// Process-wide scratch state for the stateless entry points.
ColorState *scratch() {
    static ColorState *s = nullptr;
    if (!s) s = new_color_state(0, 0);
    return s;
}

std::string model_path(int l) {
    char buf[512];
    const char *dir = getenv("GC_MODEL_DIR");
    if (dir)
        snprintf(buf, sizeof buf, "%s/m%d.gnn", dir, l);
    else
        snprintf(buf, sizeof buf, "models/m%d.gnn", l);
    return buf;
}

gc_model *load_model_or_die(int l) {
    gc_model *m = nullptr;
    if (gc_model_load(ctx(), model_path(l).c_str(), &m) != GC_OK) {
        fprintf(stderr, "Failed to open model file (%d layers)\n", l);
        exit(1);
    }
    return m;
}

void priority_into(ColorState *cs, uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h,
                   const gc_model *m, double *p) {
    load_graph(cs, N, V, E, h == GC_GNN);
    check(gc_priority(ctx(), cs->g, h, m), "priority");
    if (p) check(gc_download_priority(ctx(), cs->g, p), "priority download");
}

void color_into(ColorState *cs, int *color) {
    check(gc_color(ctx(), cs->g, 0, nullptr), "coloring");
    check(gc_download_colors(ctx(), cs->g, color), "color download");
}

void ordering(uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h, double *p) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    priority_into(scratch(), N, V, E, h, nullptr, p);
}

int *coloring_of(uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int *color = (int *)malloc(sizeof(int) * (N ? N : 1));
    ColorState *cs = scratch();
    priority_into(cs, N, V, E, h, nullptr, nullptr);
    color_into(cs, color);
    return color;
}

// X_internal / X_internal_par: priorities of `h` into p, then the coloring into color.
void heuristic_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *hs, void *cs, double *p,
                        int *color) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    HeurState *H = (HeurState *)hs;
    ColorState *C = (ColorState *)cs;
    priority_into(C, N, V, E, H->h, H->model, nullptr);
    // the priorities come down while the coloring runs (page-locked p; otherwise before it)
    int pending = 0;
    if (p) check(gc_download_priority_begin(ctx(), C->g, p, &pending), "priority download");
    color_into(C, color);
    if (pending) check(gc_download_priority_wait(ctx()), "priority download");
}

void *heuristic_setup(gc_heuristic h, int l) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    HeurState *H = new HeurState();
    H->h = h;
    if (h == GC_GNN) H->model = load_model_or_die(l);
    return H;
}

void heuristic_cleanup(void *hs) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    HeurState *H = (HeurState *)hs;
    if (!H) return;
    gc_model_free(H->model);
    delete H;
}

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace

extern "C" {

int layers = 2;  // model depth read by gnn_setup (src/gnn.c:18)

// ---- coloring.h ------------------------------------------------------------------------------

void *greedy_setup(uint32_t N, uint32_t M) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    return new_color_state(N, M);
}
void greedy_cleanup(void *gd) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    free_color_state((ColorState *)gd);
}
void greedy_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *gd, const double *p, int *color) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    ColorState *cs = (ColorState *)gd;
    load_graph(cs, N, V, E);
    check(gc_priority_set(ctx(), cs->g, p), "priority upload");
    color_into(cs, color);
}
int *greedy_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const double *p) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int *color = (int *)malloc(sizeof(int) * (N ? N : 1));
    greedy_internal(N, V, E, scratch(), p, color);
    return color;
}
int validate_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const int *color) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    ColorState *cs = scratch();
    load_graph(cs, N, V, E);
    check(gc_upload_colors(ctx(), cs->g, color), "color upload");
    int C = 0;
    check(gc_validate(ctx(), cs->g, &C), "validation");
    return C;
}

void *jones_plassmann_setup(uint32_t N, uint32_t M) { return greedy_setup(N, M); }
void jones_plassmann_cleanup(void *jp) { greedy_cleanup(jp); }
void jones_plassmann_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *jp, const double *p,
                              int *color) {
    greedy_internal(N, V, E, jp, p, color);
}
int *jones_plassmann_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const double *p) {
    return greedy_coloring(N, V, E, p);
}
int validate_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E, const int *color) {
    return validate_coloring(N, V, E, color);
}

// ---- fast_gnn.h ------------------------------------------------------------------------------

void cgnn_graph_sage_16_par(int params, const float *param, uint32_t N, const uint32_t *V, const uint32_t *E,
                            int md, float *x, float *y, double *p) {
    (void)x;
    (void)y;
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    gc_model *m = nullptr;
    check(gc_model_create(ctx(), params, md, param, &m), "model upload");
    priority_into(scratch(), N, V, E, GC_GNN, m, p);
    gc_model_free(m);
}
void cgnn_graph_sage_16(int params, const float *param, uint32_t N, const uint32_t *V, const uint32_t *E, int md,
                        float *x, float *y, double *p) {
    cgnn_graph_sage_16_par(params, param, N, V, E, md, x, y, p);
}

// ---- orderings -------------------------------------------------------------------------------

void first_fit_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) { ordering(N, V, E, GC_FF, p); }
void first_fit_ordering_par(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) { ordering(N, V, E, GC_FF, p); }
void largest_degree_first_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    ordering(N, V, E, GC_LF, p);
}
void largest_log_degree_first_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    ordering(N, V, E, GC_LLF, p);
}
void largest_log_degree_first_ordering_par(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    ordering(N, V, E, GC_LLF, p);
}
void smallest_degree_last_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    ordering(N, V, E, GC_SL, p);
}
void smallest_log_degree_last_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) {
    ordering(N, V, E, GC_SLL, p);
}
void gnn_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p, int l) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    layers = l;
    gc_model *m = load_model_or_die(l);
    priority_into(scratch(), N, V, E, GC_GNN, m, p);
    gc_model_free(m);
}

// ---- *_coloring -------------------------------------------------------------------------------

int *first_fit_coloring(uint32_t N, const uint32_t *V, const uint32_t *E) { return coloring_of(N, V, E, GC_FF); }
int *first_fit_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E) { return coloring_of(N, V, E, GC_FF); }
int *largest_degree_first_coloring(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_LF);
}
int *largest_degree_first_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_LF);
}
int *largest_log_degree_first_coloring(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_LLF);
}
int *largest_log_degree_first_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_LLF);
}
int *smallest_degree_last_coloring(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_SL);
}
int *smallest_degree_last_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_SL);
}
int *smallest_log_degree_last_coloring(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_SLL);
}
int *smallest_log_degree_last_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E) {
    return coloring_of(N, V, E, GC_SLL);
}

// ---- runner vtables ---------------------------------------------------------------------------

#define GC_VTABLE(prefix, H)                                                                                    \
    void *prefix##_setup(uint32_t N, uint32_t M) {                                                              \
        (void)N;                                                                                                \
        (void)M;                                                                                                \
        return heuristic_setup(H, 0);                                                                           \
    }                                                                                                           \
    void prefix##_cleanup(void *s) { heuristic_cleanup(s); }                                                    \
    void prefix##_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *hs, void *gd, double *p,     \
                           int *color) {                                                                        \
        heuristic_internal(N, V, E, hs, gd, p, color);                                                          \
    }                                                                                                           \
    void prefix##_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *hs, void *jp, double *p, \
                               int *color) {                                                                    \
        heuristic_internal(N, V, E, hs, jp, p, color);                                                          \
    }

GC_VTABLE(first_fit, GC_FF)
GC_VTABLE(largest_degree_first, GC_LF)
GC_VTABLE(smallest_degree_last, GC_SL)
#undef GC_VTABLE

// LLF and SLL share their setup with LF and SL in the reference (src/largest_degree_first.c:165,
// src/smallest_degree_last.c:463); the heuristic is picked by the internal function instead.
static void internal_as(gc_heuristic h, uint32_t N, const uint32_t *V, const uint32_t *E, void *cs, double *p,
                        int *color) {
    HeurState H;
    H.h = h;
    heuristic_internal(N, V, E, &H, cs, p, color);
}
void largest_log_degree_first_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *gd,
                                       double *p, int *color) {
    (void)lf;
    internal_as(GC_LLF, N, V, E, gd, p, color);
}
void largest_log_degree_first_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *jp,
                                           double *p, int *color) {
    (void)lf;
    internal_as(GC_LLF, N, V, E, jp, p, color);
}
void smallest_log_degree_last_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *gd,
                                       double *p, int *color) {
    (void)sl;
    internal_as(GC_SLL, N, V, E, gd, p, color);
}
void smallest_log_degree_last_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *jp,
                                           double *p, int *color) {
    (void)sl;
    internal_as(GC_SLL, N, V, E, jp, p, color);
}

void *gnn_setup(uint32_t N, uint32_t M) {
    (void)N;
    (void)M;
    return heuristic_setup(GC_GNN, layers);
}
void gnn_cleanup(void *ad) { heuristic_cleanup(ad); }
void gnn_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *ad, void *gd, double *p, int *color) {
    heuristic_internal(N, V, E, ad, gd, p, color);
}
void gnn_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *ad, void *jp, double *p, int *color) {
    heuristic_internal(N, V, E, ad, jp, p, color);
}

// ---- runner -----------------------------------------------------------------------------------

// The reference's protocol (src/runner.c:85-176): `it` repetitions of the sequential column and
// of each thread-count column, k-1 Culberson recolorings after each, validation of every coloring,
// then one line per Culberson index with the best time of each column.  The device graph is
// uploaded once and bound to (V, E) for the whole run; the Culberson step (p := color, recolor)
// runs on the device.  -c 0 is treated as -c 1 (the reference's zero-length arrays crash).
void runner_test_full(uint32_t N, const uint32_t *V, const uint32_t *E, void *(*setup)(uint32_t, uint32_t),
                      void (*cleanup)(void *),
                      void (*f_seq)(uint32_t, const uint32_t *, const uint32_t *, void *, void *, double *, int *),
                      void (*f_par)(uint32_t, const uint32_t *, const uint32_t *, void *, void *, double *, int *),
                      const char *s, int it, int k, int t_tot, int ntc, const int *nt) {
    (void)t_tot;
    (void)nt;
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (k < 1) k = 1;
    if (it < 1) it = 1;
    if (ntc < 0) ntc = 0;
    const uint32_t M = N ? V[N] : 0;
    const int cols = ntc + 1;
    std::vector<int> n_colors(k, -1);
    std::vector<double> times((size_t)it * k * cols, 0.0);
    auto T = [&](int t, int i, int j) -> double & { return times[((size_t)t * k + i) * cols + j]; };
    int *colors = (int *)malloc(sizeof(int) * (N ? N : 1));
    double *p = (double *)malloc(sizeof(double) * ((size_t)N + 8));
    void *fd = setup(N, M);
    ColorState *cs = new_color_state(N, M);
    cs->bind = true;
    load_graph(cs, N, V, E);

    auto validate_into = [&](int i) {
        int c = 0;
        check(gc_validate(ctx(), cs->g, &c), "validation");
        if (c == 0)
            printf("Invalid coloring\n");
        else if (n_colors[i] < 0)
            n_colors[i] = c;
        else if (n_colors[i] != c)
            printf("Unexpected number of colors (%d %d)\n", n_colors[i], c);
    };
    auto culberson = [&](int i, int col, int t) {
        double t0 = now();
        check(gc_recolor(ctx(), cs->g, 1, nullptr), "recoloring");  // keys := colors, recolor
        check(gc_download_colors(ctx(), cs->g, colors), "color download");
        T(t, i, col) = (now() - t0) + T(t, i - 1, col);
        validate_into(i);
    };
    for (int t = 0; t < it; t++) {
        double t0 = now();
        f_seq(N, V, E, fd, cs, p, colors);
        T(t, 0, 0) = now() - t0;
        validate_into(0);
        for (int i = 1; i < k; i++) culberson(i, 0, t);
        for (int c = 0; c < ntc; c++) {
            t0 = now();
            f_par(N, V, E, fd, cs, p, colors);
            T(t, 0, c + 1) = now() - t0;
            validate_into(0);
            for (int i = 1; i < k; i++) culberson(i, c + 1, t);
        }
    }
    for (int i = 0; i < k; i++) {
        printf("%s_%d %d ", s, i, n_colors[i]);
        for (int j = 0; j < cols; j++) {
            double best = 9999.9;
            for (int t = 0; t < it; t++)
                if (T(t, i, j) < best) best = T(t, i, j);
            printf("%.6lf ", best);
        }
        printf("\n");
    }
    fflush(stdout);
    free(colors);
    free(p);
    cleanup(fd);
    free_color_state(cs);
}

void first_fit_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot, int ntc,
                      const int *nt) {
    runner_test_full(N, V, E, first_fit_setup, first_fit_cleanup, first_fit_internal, first_fit_internal_par, "FF", it,
                     k, t_tot, ntc, nt);
}
void largest_degree_first_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot, int ntc,
                                 const int *nt) {
    runner_test_full(N, V, E, largest_degree_first_setup, largest_degree_first_cleanup, largest_degree_first_internal,
                     largest_degree_first_internal_par, "LF", it, k, t_tot, ntc, nt);
}
void largest_log_degree_first_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                     int ntc, const int *nt) {
    runner_test_full(N, V, E, largest_degree_first_setup, largest_degree_first_cleanup,
                     largest_log_degree_first_internal, largest_log_degree_first_internal_par, "LLF", it, k, t_tot,
                     ntc, nt);
}
void smallest_degree_last_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot, int ntc,
                                 const int *nt) {
    runner_test_full(N, V, E, smallest_degree_last_setup, smallest_degree_last_cleanup, smallest_degree_last_internal,
                     smallest_degree_last_internal_par, "SL", it, k, t_tot, ntc, nt);
}
void smallest_log_degree_last_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                     int ntc, const int *nt) {
    runner_test_full(N, V, E, smallest_degree_last_setup, smallest_degree_last_cleanup,
                     smallest_log_degree_last_internal, smallest_log_degree_last_internal_par, "SLL", it, k, t_tot,
                     ntc, nt);
}
void gnn_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int l, int it, int k, int t_tot, int ntc,
                const int *nt) {
    layers = l;
    char name[32];
    snprintf(name, sizeof name, "GNN%d", l);
    runner_test_full(N, V, E, gnn_setup, gnn_cleanup, gnn_internal, gnn_internal_par, name, it, k, t_tot, ntc, nt);
}

}  // extern "C"
