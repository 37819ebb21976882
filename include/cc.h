/*
 * cc.h - local connected components.
 *
 * Drop-in for the reference's include/cc.h.  Every call runs on the current
 * CUDA device (sm_100a) through libccb200.so; labels[v] is the minimum
 * vertex id of v's component, which is what the reference's label
 * propagation produces (src/cc_pthreads.c:32-73,169-170).
 */
#ifndef CC_H
#define CC_H

#include <stdint.h>

#include "graph.h"

/* Reference include/cc.h:7: chunk used when chunk_size <= 0. */
#define DEFAULT_CHUNK_SIZE 4096

/* The reference declares these four variants without defining them
 * (include/cc.h:11,15,19,23).  Here they are all the GPU solver; the
 * chunk_size of _omp/_cilk means what it means for _pthreads. */
void compute_connected_components(const CSRGraph *restrict G, uint32_t *restrict labels);
void compute_connected_components_bfs(const CSRGraph *restrict G, uint32_t *restrict labels);
void compute_connected_components_omp(const CSRGraph *restrict G, uint32_t *restrict labels,
                                      int chunk_size);
void compute_connected_components_cilk(const CSRGraph *restrict G, uint32_t *restrict labels,
                                       int chunk_size);

/* Reference include/cc.h:27-28.  G and labels are host memory; the graph is
 * copied to HBM, solved, and the labels copied back.  num_threads is the
 * reference's pthread count and only a hint here.  chunk_size: 1 = static
 * blocks, > 1 = vertices per dynamic work grab, <= 0 = DEFAULT_CHUNK_SIZE
 * (the reference's meaning, src/cc_pthreads.c:156-157); it changes the
 * schedule, never the labels.  On a failure the message goes to stderr and,
 * as in the reference (src/cc_pthreads.c:163-167), the process exits unless
 * ccb200_set_exit_on_error(0) was called; ccgpu_local_cc_host (ccgpu.h) is
 * the status-returning twin. */
void compute_connected_components_pthreads(const CSRGraph *restrict G, uint32_t *restrict labels,
                                           int num_threads, int chunk_size);

/* Reference include/cc.h:32 (declared, never defined there): number of
 * distinct values in labels[0..n) that are < n. */
uint32_t count_unique_labels(const uint32_t *restrict labels, uint32_t n);

/* 1 (default): a failing void call prints its message and exits, as the
 * reference does.  0: it prints and returns, leaving outputs unspecified;
 * ccgpu_last_error() holds the message.  Returns the previous mode. */
int ccb200_set_exit_on_error(int on);

#endif /* CC_H */
