/*
 * coloring -- command-line drop-in for the reference's ./coloring (src/main.c), running on the GPU.
 *
 *   coloring -g graph.mtx [-h -v -q -f -c K -t T] tc1 tc2 ... tcn
 *
 * Output (runner mode), one line per heuristic and Culberson index, as src/runner.c:156-169:
 *   NAME_i colors seconds_seq seconds_tc1 ... seconds_tcn
 * Heuristic order FF, LF, LLF, SL, SLL, GNN2, GNN3, GNN4 (LLF and SLL skipped with -f).
 * Quick mode (-q) prints "FF LF LLF SL SLL ID SDA SD GNN2 GNN3 GNN4" color counts after K-1
 * recolorings (src/main.c:135-188).  ID, SDA and SD are the reference's sequential orderings, run
 * on the host (include/incidence_degree.h); with -f they print 0, as in the reference.
 *
 * -c 0 behaves like -c 1 (a single coloring, reported as NAME_0); the reference crashes there.
 * -t and the thread counts are accepted for compatibility; every column times the GPU path.
 * GNN models are read from models/m<l>.gnn (or $GC_MODEL_DIR/m<l>.gnn).
 * Matrix Market (.mtx) files are parsed on the GPU (gc_mtx_read_device: the CSR of the reference's
 * mtx_parse_par + graph_sort_edges_par + graph_make_simple, src/main.c:106-127).  Besides .mtx, -g
 * reads the reference's other formats by extension: PACE .gr, METIS .graph and GBBS .adj
 * (src/fast_io.c:224-437), made simple and sorted like the .mtx path.
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "incidence_degree.h"
#include "coloring.h"
#include "fast_io.h"
#include "first_fit.h"
#include "gnn.h"
#include "gnn_coloring.h"
#include "largest_degree_first.h"
#include "smallest_degree_last.h"

static const char *usage =
    "Greedy graph coloring on the GPU (FF, LF, LLF, SL, SLL and GraphSAGE GNN2/3/4 priorities,\n"
    "Jones-Plassmann coloring, optional Culberson recoloring).\n"
    "\nUsage: coloring -g <graph.mtx> [options] tc1 tc2 ... tcn\n"
    "\nOutput: one line per heuristic and recoloring round:\n"
    "  <heuristic>_<round> <colors> <seconds seq> <seconds tc1> ... <seconds tcn>\n"
    "\nOptions:\n"
    "  -h        this message\n"
    "  -v        verbose progress\n"
    "  -g path   Matrix Market graph (required)\n"
    "  -q        quick mode: only color counts of every heuristic\n"
    "  -f        only FF, LF, SL and GNN (skip LLF and SLL)\n"
    "  -c K      K colorings: the first, then K-1 Culberson recolorings\n"
    "  -t T      accepted for compatibility (setup threads)\n";

static double wall(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* JP by p, then K-1 rounds of p := color and recolor; returns the validated color count. */
static int quick_count(uint32_t N, const uint32_t *V, const uint32_t *E, void *jp, double *p, int *color, int K) {
    jones_plassmann_internal(N, V, E, jp, p, color);
    for (int i = 1; i < K; i++) {
        for (uint32_t u = 0; u < N; u++) p[u] = color[u];
        jones_plassmann_internal(N, V, E, jp, p, color);
    }
    return validate_coloring_par(N, V, E, color);
}

int main(int argc, char **argv) {
    const char *graph_path = NULL;
    int quick = 0, fast = 0, K = 1, threads = 1, verbose = 0, opt;
    opterr = 0;
    while ((opt = getopt(argc, argv, "hvfqg:c:t:")) != -1) {
        switch (opt) {
            case 'g': graph_path = optarg; break;
            case 'q': quick = 1; break;
            case 'f': fast = 1; break;
            case 'c': K = atoi(optarg); break;
            case 't': threads = atoi(optarg); break;
            case 'v': verbose = 1; break;
            case 'h': printf("%s\n", usage); return 0;
            case '?':
                if (optopt == 'c' || optopt == 'g' || optopt == 't')
                    fprintf(stderr, "Option -%c requires an argument.\n", optopt);
                else if (isprint(optopt))
                    fprintf(stderr, "Unknown option `-%c'.\n", optopt);
                else
                    fprintf(stderr, "Unknown option character `\\x%x'.\n", optopt);
                return 1;
            default: return 1;
        }
    }
    if (K < 1) K = 1;
    int ntc = argc - optind;
    int *nt = malloc(sizeof(int) * (ntc > 0 ? ntc : 1));
    for (int i = 0; i < ntc; i++) {
        nt[i] = atoi(argv[optind + i]);
        if (nt[i] > threads) threads = nt[i];
    }

    FILE *fp = graph_path ? fopen(graph_path, "r") : NULL;
    if (!fp) {
        printf("Unable to open file %s\n", graph_path ? graph_path : "");
        return 1;
    }
    uint32_t N, *V, *E;
    double t0 = wall();
    const size_t plen = strlen(graph_path);
    if (plen >= 4 && strcmp(graph_path + plen - 4, ".mtx") == 0) {
        /* Matrix Market: parsed and turned into the sorted, simple CSR on the GPU */
        fclose(fp);
        gc_ctx *io = NULL;
        const char *dev = getenv("GC_DEVICE");
        gc_status st = gc_ctx_create(dev ? atoi(dev) : 0, &io);
        if (st == GC_OK) st = gc_mtx_read_device(io, graph_path, &N, &V, &E);
        if (st != GC_OK) {
            printf("Unable to read graph %s: %s%s%s\n", graph_path, gc_status_string(st), io ? ": " : "",
                   io ? gc_last_error(io) : "");
            return 1;
        }
        gc_ctx_destroy(io);
    } else {
        /* .gr, .graph or .adj: the library's readers, already sorted and simple */
        fclose(fp);
        if (gc_read_graph(graph_path, &N, &V, &E) != GC_OK) {
            printf("Unable to read graph %s (expected .mtx, .gr, .graph or .adj)\n", graph_path);
            return 1;
        }
    }
    if (verbose) printf("Parsing took: %.4lfs, |V|=%u, |E|=%u\n", wall() - t0, N, V[N]);
    t0 = wall();
    graph_sort_edges_par(N, V, E);
    if (verbose) printf("Sorting edges took: %.4lfs\n", wall() - t0);
    t0 = wall();
    graph_make_simple(N, V, &E);
    if (verbose) printf("Making the graph simple took %.4lfs, new size |V|=%u, |E|=%u\n", wall() - t0, N, V[N]);

    if (quick) {
        void *jp = jones_plassmann_setup(N, V[N]);
        double *p = malloc(sizeof(double) * ((size_t)N + 8));
        int *color = malloc(sizeof(int) * (N ? N : 1));
        int ff, lf, llf = 0, sl, sll = 0, id = 0, sda = 0, sd = 0, gnn2, gnn3, gnn4;
        first_fit_ordering_par(N, V, E, p);
        ff = quick_count(N, V, E, jp, p, color, K);
        largest_degree_first_ordering(N, V, E, p);
        lf = quick_count(N, V, E, jp, p, color, K);
        smallest_degree_last_ordering(N, V, E, p);
        sl = quick_count(N, V, E, jp, p, color, K);
        gnn_ordering(N, V, E, p, 2);
        gnn2 = quick_count(N, V, E, jp, p, color, K);
        gnn_ordering(N, V, E, p, 3);
        gnn3 = quick_count(N, V, E, jp, p, color, K);
        gnn_ordering(N, V, E, p, 4);
        gnn4 = quick_count(N, V, E, jp, p, color, K);
        if (!fast) {
            largest_log_degree_first_ordering(N, V, E, p);
            llf = quick_count(N, V, E, jp, p, color, K);
            smallest_log_degree_last_ordering(N, V, E, p);
            sll = quick_count(N, V, E, jp, p, color, K);
            incidence_degree_ordering(N, V, E, p);
            id = quick_count(N, V, E, jp, p, color, K);
            saturation_degree_ordering_alt(N, V, E, p);
            sda = quick_count(N, V, E, jp, p, color, K);
            saturation_degree_ordering(N, V, E, p);
            sd = quick_count(N, V, E, jp, p, color, K);
        }
        if (verbose) printf("FF LF LLF SL SLL ID SDA SD GNN2 GNN3 GNN4\n");
        printf("%d %d %d %d %d %d %d %d %d %d %d\n", ff, lf, llf, sl, sll, id, sda, sd, gnn2, gnn3, gnn4);
        jones_plassmann_cleanup(jp);
        free(p);
        free(color);
    } else {
        if (verbose) {
            printf("name colors seq ");
            for (int i = 0; i < ntc; i++) printf("%d ", nt[i]);
            printf("\n");
        }
        first_fit_runner(N, V, E, 5, K, threads, ntc, nt);
        largest_degree_first_runner(N, V, E, 5, K, threads, ntc, nt);
        if (!fast) largest_log_degree_first_runner(N, V, E, 5, K, threads, ntc, nt);
        smallest_degree_last_runner(N, V, E, 5, K, threads, ntc, nt);
        if (!fast) smallest_log_degree_last_runner(N, V, E, 5, K, threads, ntc, nt);
        gnn_runner(N, V, E, 2, 5, K, threads, ntc, nt);
        gnn_runner(N, V, E, 3, 5, K, threads, ntc, nt);
        gnn_runner(N, V, E, 4, 5, K, threads, ntc, nt);
    }
    free(V);
    free(E);
    free(nt);
    return 0;
}
