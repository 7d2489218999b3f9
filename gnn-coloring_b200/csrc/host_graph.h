// Internal declarations shared by the host-side graph code and the C ABI layer.
#pragma once
#include <stdint.h>
#include <stdio.h>

#include "gnn_coloring.h"

// Simple, symmetric, sorted CSR from L 0-based pairs (both directions added); malloc'd outputs.
gc_status gc_csr_build(uint32_t N, uint64_t L, const uint32_t *I, const uint32_t *J,
                       uint32_t **V_out, uint32_t **E_out);

#ifdef __cplusplus
extern "C" {
#endif
// Raw Matrix Market entries as 0-based pairs plus N = max(rows, cols); malloc'd outputs.
gc_status gc_mtx_read_pairs(const char *path, uint32_t *N, uint64_t *L, uint32_t **I, uint32_t **J);
gc_status gc_mtx_read_pairs_file(FILE *f, uint32_t *N, uint64_t *L, uint32_t **I, uint32_t **J);
#ifdef __cplusplus
}
#endif
