/*
 * gnn.h -- drop-in for the reference's include/gnn.h.
 * Model files are read from models/m<l>.gnn relative to the working directory, as in the
 * reference (src/gnn.c:24-25), or from $GC_MODEL_DIR/m<l>.gnn when that variable is set.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/gnn.h:4 -- GraphSAGE-16 priorities with an l-layer model */
void gnn_ordering(uint32_t N, const uint32_t *V, const uint32_t *E, double *p, int l);
/* include/gnn.h:6-7 -- prints GNN<l>_i lines */
void gnn_runner(uint32_t N, const uint32_t *V, const uint32_t *E, int l, int it, int k, int t_tot, int ntc,
                const int *nt);

/* Runner vtable entries (src/gnn.c:18-91); gnn_setup reads the model named by `layers`. */
extern int layers;
void *gnn_setup(uint32_t N, uint32_t M);
void gnn_cleanup(void *ad);
void gnn_internal(uint32_t N, const uint32_t *V, const uint32_t *E, void *ad, void *gd, double *p, int *color);
void gnn_internal_par(uint32_t N, const uint32_t *V, const uint32_t *E, void *ad, void *jp, double *p, int *color);

#ifdef __cplusplus
}
#endif
