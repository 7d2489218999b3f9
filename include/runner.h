/*
 * runner.h -- drop-in for the reference's include/runner.h benchmark protocol.
 *
 * runner_test_full runs `it` repetitions of: f_seq (+ k-1 Culberson recolorings with
 * greedy_internal), then f_par for each thread count (+ k-1 recolorings with
 * jones_plassmann_internal); every coloring is validated; then it prints, per Culberson index i,
 *     "<s>_<i> <colors> <best seconds seq> <best seconds tc1> ... \n"
 * with "%.6lf " per column (src/runner.c:85-176).  Thread counts do not apply to the GPU: each
 * f_par column times the same GPU path, which is what the column means here.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/runner.h:12-17 */
void runner_test_full(uint32_t N, const uint32_t *V, const uint32_t *E, void *(*setup)(uint32_t, uint32_t),
                      void (*cleanup)(void *),
                      void (*f_seq)(uint32_t, const uint32_t *, const uint32_t *, void *, void *, double *, int *),
                      void (*f_par)(uint32_t, const uint32_t *, const uint32_t *, void *, void *, double *, int *),
                      const char *s, int it, int k, int t_tot, int ntc, const int *nt);

#ifdef __cplusplus
}
#endif
