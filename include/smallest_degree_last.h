/* smallest_degree_last.h -- drop-in for the reference's include/smallest_degree_last.h. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/smallest_degree_last.h:4 -- bucket-peeling priorities (p = peel threshold) */
void smallest_degree_last_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/smallest_degree_last.h:6 */
int *smallest_degree_last_coloring(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/smallest_degree_last.h:8 */
int *smallest_degree_last_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/smallest_degree_last.h:10-11 */
void smallest_degree_last_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                 int ntc, const int *nt);

/* include/smallest_degree_last.h:13 -- thresholds 2^delta */
void smallest_log_degree_last_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/smallest_degree_last.h:15 */
int *smallest_log_degree_last_coloring(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/smallest_degree_last.h:17 */
int *smallest_log_degree_last_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/smallest_degree_last.h:19-20 */
void smallest_log_degree_last_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                     int ntc, const int *nt);

/* Runner vtable entries (src/smallest_degree_last.c:15-60, 133-138, 155-246, 337-443). */
void *smallest_degree_last_setup(uint32_t N, uint32_t M);
void smallest_degree_last_cleanup(void *sl);
void smallest_degree_last_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *gd, double *p,
                                   int *color);
void smallest_degree_last_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *jp,
                                       double *p, int *color);
void smallest_log_degree_last_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *gd,
                                       double *p, int *color);
void smallest_log_degree_last_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *sl, void *jp,
                                           double *p, int *color);

#ifdef __cplusplus
}
#endif
