/*
 * fast_gnn.h -- drop-in for the reference's include/fast_gnn.h: GraphSAGE with 16 features,
 * inputs built from degree and id, output = sum of the last layer's features per vertex.
 * The FP32 results are bit-identical to the reference's.  x and y are accepted for signature
 * compatibility (the reference uses them as layer scratch); the GPU keeps its own scratch and
 * leaves them untouched.  p needs N entries (the reference asks for 8 extra rows; they are not
 * written here).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/fast_gnn.h:13-15 */
void cgnn_graph_sage_16(int params, const float *param, uint32_t N, const uint32_t *V, const uint32_t *E, int md,
                        float *x, float *y, double *p);
/* include/fast_gnn.h:17-19 */
void cgnn_graph_sage_16_par(int params, const float *param, uint32_t N, const uint32_t *V, const uint32_t *E,
                            int md, float *x, float *y, double *p);

#ifdef __cplusplus
}
#endif
