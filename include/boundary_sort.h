/*
 * boundary_sort.h - boundary edge sort and dedup.
 *
 * Drop-in for the reference's include/boundary_sort.h:8-9.  The arrays are
 * host memory, sorted in place; the sort runs on the current CUDA device as
 * an LSD radix sort over only the digits the values use (the reference sorts
 * with an in-place MSD radix sort on the host, src/boundary_sort.c:34-98).
 * Order: ascending on remote << 32 | rep.
 */
#ifndef BOUNDARY_SORT_H
#define BOUNDARY_SORT_H

#include <stdint.h>

#include "vec_helpers.h"

void boundary_edges_sort(BoundaryEdge *edges, uint64_t count);
/* Removes adjacent duplicates; returns the new count. */
uint64_t boundary_edges_dedup(BoundaryEdge *edges, uint64_t count);

#endif /* BOUNDARY_SORT_H */
