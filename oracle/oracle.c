/*
 * oracle.c -- CPU restatement of the reference's coloring hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, never the library.
 *
 * Each function restates one reference routine (KennethLangedal/GNN-COLORING, cited file:line)
 * as plain scalar C.  The restatement is pinned against the reference's own compiled code
 * (oracle/_ref, built by oracle/Makefile) and against the committed golden vectors in
 * tests/golden/ that the reference produced.
 *
 * Priorities are doubles, exactly as the reference's `double *p`; colors are 1-based ints.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FEAT 16          /* GraphSAGE width (fast_gnn.c:6)                   */
#define LAYER_PARAMS 528 /* 32x16 weights + 16 biases per layer (fast_gnn.c:256) */

/* p[i] = N - i (first_fit.c:8-12). */
void oracle_ff_ordering(uint32_t N, const uint32_t *V, double *p) {
    (void)V;
    for (uint32_t i = 0; i < N; i++) p[i] = (double)(N - i);
}

/* p[u] = deg(u) (largest_degree_first.c:12-16). */
void oracle_lf_ordering(uint32_t N, const uint32_t *V, double *p) {
    for (uint32_t u = 0; u < N; u++) p[u] = (double)(V[u + 1] - V[u]);
}

/* p[u] = bit length of deg(u), 0 for isolated vertices (largest_degree_first.c:87-97). */
void oracle_llf_ordering(uint32_t N, const uint32_t *V, double *p) {
    for (uint32_t u = 0; u < N; u++) {
        uint32_t d = V[u + 1] - V[u], b = 0;
        while (d) {
            b++;
            d >>= 1;
        }
        p[u] = (double)b;
    }
}

/*
 * Smallest-degree-last bucket peeling (smallest_degree_last.c:155-246, same result as the
 * sequential :62-124).  Each round removes every remaining vertex whose remaining degree is
 * <= delta and gives it p = delta; remaining neighbours of removed vertices lose one degree per
 * removed neighbour; then delta = max(delta + 1, smallest remaining degree).
 * log_thresholds selects the SLL variant (:359-443): threshold 2^delta, delta starts at the
 * smallest d with 2^d >= min degree and grows by one per round.
 */
static void peel(uint32_t N, const uint32_t *V, const uint32_t *E, double *p, int log_thresholds) {
    uint32_t *deg = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t *alive = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t *keep = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t *gone = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t min_deg = N;
    for (uint32_t u = 0; u < N; u++) {
        deg[u] = V[u + 1] - V[u];
        alive[u] = u;
        p[u] = -1.0;
        if (deg[u] < min_deg) min_deg = deg[u];
    }
    uint32_t delta = 0;
    if (log_thresholds) {
        while ((1ull << delta) < (uint64_t)min_deg) delta++;
    } else {
        delta = min_deg;
    }
    uint32_t n_alive = N;
    while (n_alive > 0) {
        uint64_t thr = log_thresholds ? (1ull << delta) : (uint64_t)delta;
        uint32_t n_keep = 0, n_gone = 0;
        min_deg = N;
        for (uint32_t i = 0; i < n_alive; i++) {
            uint32_t u = alive[i];
            if ((uint64_t)deg[u] <= thr) {
                gone[n_gone++] = u;
                p[u] = (double)delta;
            } else {
                keep[n_keep++] = u;
                if (deg[u] < min_deg) min_deg = deg[u];
            }
        }
        for (uint32_t i = 0; i < n_gone; i++) {
            uint32_t u = gone[i];
            for (uint32_t j = V[u]; j < V[u + 1]; j++) {
                uint32_t v = E[j];
                if (p[v] >= 0.0) continue;
                deg[v]--;
                if (deg[v] < min_deg) min_deg = deg[v];
            }
        }
        delta++;
        if (!log_thresholds && min_deg > delta) delta = min_deg;
        memcpy(alive, keep, sizeof(uint32_t) * n_keep);
        n_alive = n_keep;
    }
    free(deg);
    free(alive);
    free(keep);
    free(gone);
}

void oracle_sl_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) { peel(N, V, E, p, 0); }
void oracle_sll_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p) { peel(N, V, E, p, 1); }

/*
 * GraphSAGE-16 inference with the reference's FP32 operation order (fast_gnn.c:13-243, 252-295):
 *  - neighbour sums run sequentially over the CSR list from +0 (message_kernel :22-33);
 *  - the mean divides by (float)deg only when deg > 0 (:35-41);
 *  - layer-0 features are (float)deg/(float)md and (float)((double)v/(double)N), 8 copies each,
 *    for the neighbour mean and for the vertex itself (message_kernel_input :49-89);
 *  - the dense part is c_j = b_j, then c_j = fmaf(W[i*16+j], a_i, c_j) for i = 0..31 in order,
 *    and ReLU keeps c only when c > 0 (dense_kernel :91-162);
 *  - the output layer sums the 16 ReLU outputs as t_k = s_k + s_{k+8}, then
 *    ((t0+t1)+(t2+t3)) + ((t4+t5)+(t6+t7)), widened to double (dense_kernel_output :164-243).
 * x and y are scratch of N*16 floats each.
 */
void oracle_gnn_ordering(int params, const float *param, int md, uint32_t N, const uint32_t *V,
                         const uint32_t *E, double *p) {
    int L = params / LAYER_PARAMS;
    float *x = malloc(sizeof(float) * FEAT * (N ? N : 1));
    float *y = malloc(sizeof(float) * FEAT * (N ? N : 1));
    float a[2 * FEAT], o[FEAT];
    const float fmd = (float)md;
    for (int l = 0; l < L; l++) {
        const float *W = param + (size_t)l * LAYER_PARAMS, *b = W + 2 * FEAT * FEAT;
        for (uint32_t u = 0; u < N; u++) {
            uint32_t d = V[u + 1] - V[u];
            float fd = (float)d;
            if (l == 0) {
                float s0 = 0.0f, s1 = 0.0f;
                for (uint32_t i = V[u]; i < V[u + 1]; i++) {
                    uint32_t v = E[i];
                    s0 = s0 + (float)(V[v + 1] - V[v]) / fmd;
                    s1 = s1 + (float)((double)v / (double)N);
                }
                if (fd > 0.0f) {
                    s0 = s0 / fd;
                    s1 = s1 / fd;
                }
                float self_deg = fd / fmd, self_id = (float)((double)u / (double)N);
                for (int k = 0; k < 8; k++) {
                    a[k] = s0;
                    a[8 + k] = s1;
                    a[16 + k] = self_deg;
                    a[24 + k] = self_id;
                }
            } else {
                for (int k = 0; k < FEAT; k++) {
                    float s = 0.0f;
                    for (uint32_t i = V[u]; i < V[u + 1]; i++) s = s + x[(size_t)E[i] * FEAT + k];
                    if (fd > 0.0f) s = s / fd;
                    a[k] = s;
                    a[FEAT + k] = x[(size_t)u * FEAT + k];
                }
            }
            for (int j = 0; j < FEAT; j++) {
                float c = b[j];
                for (int i = 0; i < 2 * FEAT; i++) c = fmaf(W[i * FEAT + j], a[i], c);
                o[j] = c > 0.0f ? c : 0.0f;
            }
            if (l < L - 1) {
                memcpy(y + (size_t)u * FEAT, o, sizeof(o));
            } else {
                float t[8];
                for (int k = 0; k < 8; k++) t[k] = o[k] + o[k + 8];
                float s = ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
                p[u] = (double)s;
            }
        }
        float *tmp = x;
        x = y;
        y = tmp;
    }
    free(x);
    free(y);
}

/* The same network in FP64 throughout (for stating the FP32 error); not a parity target. */
void oracle_gnn_ordering_f64(int params, const float *param, int md, uint32_t N, const uint32_t *V,
                             const uint32_t *E, double *p) {
    int L = params / LAYER_PARAMS;
    double *x = malloc(sizeof(double) * FEAT * (N ? N : 1));
    double *y = malloc(sizeof(double) * FEAT * (N ? N : 1));
    double a[2 * FEAT], o[FEAT];
    for (int l = 0; l < L; l++) {
        const float *W = param + (size_t)l * LAYER_PARAMS, *b = W + 2 * FEAT * FEAT;
        for (uint32_t u = 0; u < N; u++) {
            uint32_t d = V[u + 1] - V[u];
            if (l == 0) {
                double s0 = 0, s1 = 0;
                for (uint32_t i = V[u]; i < V[u + 1]; i++) {
                    uint32_t v = E[i];
                    s0 += (double)(V[v + 1] - V[v]) / md;
                    s1 += (double)v / (double)N;
                }
                if (d) {
                    s0 /= d;
                    s1 /= d;
                }
                for (int k = 0; k < 8; k++) {
                    a[k] = s0;
                    a[8 + k] = s1;
                    a[16 + k] = (double)d / md;
                    a[24 + k] = (double)u / (double)N;
                }
            } else {
                for (int k = 0; k < FEAT; k++) {
                    double s = 0;
                    for (uint32_t i = V[u]; i < V[u + 1]; i++) s += x[(size_t)E[i] * FEAT + k];
                    if (d) s /= d;
                    a[k] = s;
                    a[FEAT + k] = x[(size_t)u * FEAT + k];
                }
            }
            for (int j = 0; j < FEAT; j++) {
                double c = b[j];
                for (int i = 0; i < 2 * FEAT; i++) c += (double)W[i * FEAT + j] * a[i];
                o[j] = c > 0 ? c : 0;
            }
            if (l < L - 1) {
                memcpy(y + (size_t)u * FEAT, o, sizeof(o));
            } else {
                double s = 0;
                for (int k = 0; k < FEAT; k++) s += o[k];
                p[u] = s;
            }
        }
        double *tmp = x;
        x = y;
        y = tmp;
    }
    free(x);
    free(y);
}

/* v precedes u (coloring.c:72 and :249). */
static inline int precedes(const double *p, uint32_t v, uint32_t u) {
    return p[v] > p[u] || (p[u] == p[v] && v < u);
}

/*
 * Greedy coloring in priority order by DAG peeling (coloring.c:60-125): a vertex is colored once
 * all its predecessors are, with the smallest color >= 1 none of them uses.  The result equals
 * jones_plassmann_internal (coloring.c:223-330) on any thread count.
 * Returns the number of peeling rounds (the longest predecessor chain).
 */
uint32_t oracle_greedy_color(uint32_t N, const uint32_t *V, const uint32_t *E, const double *p, int *color) {
    uint32_t *count = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t *cur = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t *nxt = malloc(sizeof(uint32_t) * (N ? N : 1));
    uint32_t max_deg = 0, n_cur = 0, rounds = 0;
    for (uint32_t u = 0; u < N; u++) {
        uint32_t c = 0;
        for (uint32_t i = V[u]; i < V[u + 1]; i++) c += precedes(p, E[i], u);
        count[u] = c;
        color[u] = 0;
        if (!c) cur[n_cur++] = u;
        if (V[u + 1] - V[u] > max_deg) max_deg = V[u + 1] - V[u];
    }
    uint32_t *mark = malloc(sizeof(uint32_t) * (max_deg + 2));
    for (uint32_t i = 0; i < max_deg + 2; i++) mark[i] = UINT32_MAX;
    while (n_cur) {
        rounds++;
        uint32_t n_nxt = 0;
        for (uint32_t k = 0; k < n_cur; k++) {
            uint32_t u = cur[k];
            for (uint32_t i = V[u]; i < V[u + 1]; i++) {
                uint32_t v = E[i];
                if (precedes(p, v, u)) mark[color[v]] = u;
            }
            int c = 1;
            while (mark[c] == u) c++;
            color[u] = c;
            for (uint32_t i = V[u]; i < V[u + 1]; i++) {
                uint32_t v = E[i];
                if (precedes(p, u, v) && --count[v] == 0) nxt[n_nxt++] = v;
            }
        }
        uint32_t *t = cur;
        cur = nxt;
        nxt = t;
        n_cur = n_nxt;
    }
    free(mark);
    free(count);
    free(cur);
    free(nxt);
    return rounds;
}

/* Culberson recoloring (runner.c:139-152): p := color, recolor; repeated `iters` times. */
void oracle_culberson(uint32_t N, const uint32_t *V, const uint32_t *E, double *p, int *color, int iters) {
    for (int it = 0; it < iters; it++) {
        for (uint32_t u = 0; u < N; u++) p[u] = (double)color[u];
        oracle_greedy_color(N, V, E, p, color);
    }
}

/* Number of colors if every color is >= 1 and no edge is monochrome, else 0 (coloring.c:127-146). */
int oracle_validate(uint32_t N, const uint32_t *V, const uint32_t *E, const int *color) {
    int bad = 0, C = 1;
    for (uint32_t u = 0; u < N; u++) {
        if (color[u] <= 0) bad = 1;
        for (uint32_t i = V[u]; i < V[u + 1]; i++)
            if (color[E[i]] == color[u]) bad = 1;
        if (color[u] > C) C = color[u];
    }
    return bad ? 0 : C;
}
