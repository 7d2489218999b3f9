/*
 * fast_io.h -- the reference's Matrix Market loader and CSR utilities (include/fast_io.h), host
 * side.  mtx_parse already returns the sorted, simple CSR; graph_sort_edges and
 * graph_make_simple are then no-ops, so the three-step pipeline of src/main.c:114-129 yields
 * exactly the reference's V and E.  Arrays are malloc'd; the caller frees them.
 * The GBBS adjacency, PACE .gr and METIS .graph readers return the CSR the reference's readers
 * return (not yet sorted or simple; .adj not symmetrised); the writers print the reference's text.
 * Malformed input ends the process with a message on stderr, as the reference's fatal errors do.
 */
#pragma once
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/fast_io.h:35 */
void mtx_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E);
/* include/fast_io.h:37 */
void mtx_parse_par(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E);
/* include/fast_io.h:39 -- writes each undirected edge once, 1-based */
void mtx_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/fast_io.h:69 -- "AdjacencyGraph", N, M, N offsets, M edges (0-based) */
void adj_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E);
/* include/fast_io.h:71 */
void adj_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/fast_io.h:98 -- 'c' comments, "p td N M", M edges (1-based), added in both directions */
void gr_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E);
/* include/fast_io.h:100 */
void gr_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/fast_io.h:119 -- '%' comments, "N M fmt", one neighbour line per vertex (1-based); fmt 10/11
 * carry a vertex weight first (W, else W = NULL), fmt 1/11 an edge weight after each neighbour */
void metis_parse(FILE *f, uint32_t *N, uint32_t **V, uint32_t **E, uint32_t **W);
/* include/fast_io.h:121 */
void metis_store(FILE *f, uint32_t N, const uint32_t *V, const uint32_t *E, const uint32_t *W);
/* include/fast_io.h:128 */
void graph_sort_edges(uint32_t N, const uint32_t *V, uint32_t *E);
/* include/fast_io.h:130 */
void graph_sort_edges_par(uint32_t N, const uint32_t *V, uint32_t *E);
/* include/fast_io.h:133 -- drops self-loops and repeated neighbours of sorted lists */
void graph_make_simple(uint32_t N, uint32_t *V, uint32_t **E);
/* include/fast_io.h:146 -- 1 if simple, sorted, symmetric and consistent, else 0 */
uint32_t graph_validate(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/fast_io.h:148 */
uint32_t graph_validate_par(uint32_t N, const uint32_t *V, const uint32_t *E);

#ifdef __cplusplus
}
#endif
