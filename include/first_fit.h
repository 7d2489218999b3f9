/* first_fit.h -- drop-in for the reference's include/first_fit.h (GPU-backed, host buffers). */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/first_fit.h:4 -- p[i] = N - i */
void first_fit_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/first_fit.h:6 */
void first_fit_ordering_par(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/first_fit.h:8 -- malloc'd colors of the natural-order greedy */
int *first_fit_coloring(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/first_fit.h:10 */
int *first_fit_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/first_fit.h:12-13 -- prints FF_i lines (runner protocol, see runner.h) */
void first_fit_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot, int ntc,
                      const int *nt);

/* Runner vtable entries (src/first_fit.c:39-87; not in the reference's header). */
void *first_fit_setup(uint32_t N, uint32_t M);
void first_fit_cleanup(void *ff);
void first_fit_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *ff, void *gd, double *p, int *color);
void first_fit_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *ff, void *jp, double *p,
                            int *color);

#ifdef __cplusplus
}
#endif
