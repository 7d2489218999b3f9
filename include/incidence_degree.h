/*
 * incidence_degree.h -- the reference's sequential orderings, exported by libgnncolor.so under the
 * reference's names (KennethLangedal/GNN-COLORING include/incidence_degree.h).
 *
 * Each vertex is picked by a count that depends on every earlier pick, so these run on the host.
 * They are used by quick mode (-q, src/main.c:135-188) and give p[u] = N - (pick index): the first
 * vertex picked has the largest priority; vertices never picked keep p = -1, as in the reference.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Incidence degree: the next vertex has the most already-picked neighbours, then the largest
 * degree, then the largest id (src/incidence_degree.c:107-164). */
void incidence_degree_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);

/* Saturation degree: the next vertex has the most distinct colors among its neighbours (each
 * picked vertex takes the first free color), then the largest degree, then the largest id
 * (src/incidence_degree.c:166-255). */
void saturation_degree_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);

/* Batched saturation degree: starts from every maximum-degree vertex of each component and picks
 * all vertices tied on (saturation, degree) at once, with one shared priority
 * (src/incidence_degree.c:257-361). */
void saturation_degree_ordering_alt(uint32_t N, const uint32_t *V, const uint32_t *E, double *p);

#ifdef __cplusplus
}
#endif
