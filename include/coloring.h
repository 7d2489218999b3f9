/*
 * coloring.h -- drop-in for the reference's include/coloring.h (KennethLangedal/GNN-COLORING).
 * Same names, signatures and result semantics; the work runs on the GPU (one process-wide
 * context on device $GC_DEVICE, default 0).  Host buffers in, host buffers out.
 * A device failure prints a message and exits, as the reference does on fatal errors.
 *
 * "greedy" and "Jones-Plassmann" give identical colors in the reference (both color each vertex
 * with the smallest color its higher-priority neighbours leave free); both run the GPU coloring.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/coloring.h:6 -- malloc'd int[N] the caller frees. */
int *greedy_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const double *p);
/* include/coloring.h:8 -- reserves device memory for graphs of up to N vertices, M edges. */
void *greedy_setup(uint32_t N, uint32_t M);
/* include/coloring.h:10 */
void greedy_cleanup(void *gd);
/* include/coloring.h:12-13 -- colors by p into color[N] (1-based). */
void greedy_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *gd, const double *p, int *color);
/* include/coloring.h:15 -- number of colors if proper and all colors > 0, else 0. */
int validate_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const int *color);

/* include/coloring.h:19 */
int *jones_plassmann_coloring(uint32_t N, const uint32_t *V, const uint32_t *E, const double *p);
/* include/coloring.h:22 */
void *jones_plassmann_setup(uint32_t N, uint32_t M);
/* include/coloring.h:24 */
void jones_plassmann_cleanup(void *jp);
/* include/coloring.h:26-27 */
void jones_plassmann_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *jp, const double *p,
                              int *color);
/* include/coloring.h:29 */
int validate_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E, const int *color);

#ifdef __cplusplus
}
#endif
