// Library-internal entry points that let the reference-facing calls overlap host copies with
// device work (not part of the public ABI).
#pragma once
#include "gnn_coloring.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Starts the download of g's priorities (as doubles) into p on the context's copy stream, after
 * the priority kernels and beside whatever the caller launches next; *pending = 1 then, and
 * gc_download_priority_wait must be called before p is read or g's priorities change.  When p is
 * not page-locked host memory the download is the synchronous gc_download_priority (*pending = 0). */
gc_status gc_download_priority_begin(gc_ctx *ctx, gc_graph *g, double *p, int *pending);
gc_status gc_download_priority_wait(gc_ctx *ctx);

/* Announces that GNN priorities follow g's next upload.  With a page-locked E that upload then
 * converts E to the GNN's feature rows piece by piece as it arrives, beside the copy, instead of in
 * the first GNN call; the id check is part of that conversion. */
void gc_graph_gnn_hint(gc_graph *g, int on);

#ifdef __cplusplus
}
#endif
