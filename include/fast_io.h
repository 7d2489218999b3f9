/*
 * fast_io.h -- the reference's Matrix Market loader and CSR utilities (include/fast_io.h), host
 * side.  mtx_parse already returns the sorted, simple CSR; graph_sort_edges and
 * graph_make_simple are then no-ops, so the three-step pipeline of src/main.c:114-129 yields
 * exactly the reference's V and E.  Arrays are malloc'd; the caller frees them.
 * The adjacency-list, PACE and METIS formats (fast_io.h:49-132) are not provided.
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
