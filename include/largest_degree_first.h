/* largest_degree_first.h -- drop-in for the reference's include/largest_degree_first.h. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/largest_degree_first.h:4 -- p = deg */
void largest_degree_first_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/largest_degree_first.h:6 */
int *largest_degree_first_coloring(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/largest_degree_first.h:8 */
int *largest_degree_first_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/largest_degree_first.h:10-11 */
void largest_degree_first_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                 int ntc, const int *nt);

/* include/largest_degree_first.h:13 -- p = 32 - clz(deg), 0 for isolated vertices */
void largest_log_degree_first_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
/* include/largest_degree_first.h:15 */
int *largest_log_degree_first_coloring(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/largest_degree_first.h:17.  The reference's version passes its JP state to the
 * sequential greedy (src/largest_degree_first.c:146); here it simply returns the LLF coloring. */
int *largest_log_degree_first_coloring_par(uint32_t N, const uint32_t *V, const uint32_t *E);
/* include/largest_degree_first.h:19-20 */
void largest_log_degree_first_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int it, int k, int t_tot,
                                     int ntc, const int *nt);

/* Runner vtable entries (src/largest_degree_first.c:18-57, 99-138). */
void *largest_degree_first_setup(uint32_t N, uint32_t M);
void largest_degree_first_cleanup(void *lf);
void largest_degree_first_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *gd, double *p,
                                   int *color);
void largest_degree_first_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *jp,
                                       double *p, int *color);
void largest_log_degree_first_ordering_par(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);
void largest_log_degree_first_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *gd,
                                       double *p, int *color);
void largest_log_degree_first_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *lf, void *jp,
                                           double *p, int *color);

#ifdef __cplusplus
}
#endif
