/*
 * graph.h - CSR graph storage and loaders.
 *
 * Drop-in for the reference's include/graph.h:8-33: the CSRGraph layout and
 * the four loader/free prototypes are unchanged, so code compiled against
 * the reference links against libccb200.so as is.
 */
#ifndef GRAPH_H
#define GRAPH_H

#include <stddef.h>
#include <stdint.h>

/* Compressed sparse row graph: the neighbours of v are
 * col_idx[row_ptr[v] .. row_ptr[v+1]).  Same layout as the reference
 * (include/graph.h:8-14). */
typedef struct
{
    uint32_t n;
    uint64_t m;
    uint64_t *row_ptr;
    uint32_t *col_idx;
} CSRGraph;

/* Matrix Market reader (reference include/graph.h:19, declared there but
 * never defined).  symmetrize adds reverse edges, drop_self_loops skips
 * (i,i); duplicates are removed.  Returns 0 on success. */
int load_csr_from_mtx(const char *path, int symmetrize, int drop_self_loops, CSRGraph *out);

/* MATLAB level-5 .mat reader (reference include/graph.h:23, src/graph.c:38-128):
 * takes field A of a struct named Problem, else the first sparse variable,
 * and turns its CSC arrays into CSR with the column index as the neighbour.
 * Return codes follow the reference: 0 ok, 1 cannot open, 2 no sparse
 * matrix, 3 out of memory; 4 = a MAT feature this reader does not handle. */
int load_csr_from_mat(const char *path, CSRGraph *out);

/* Dispatch on the extension (reference src/graph.c:14-35): ".mat" ->
 * load_csr_from_mat, ".mtx"/".txt" -> -1 (as the reference), ".csrbin" ->
 * load_csr_from_csrbin, anything else -> 99.  symmetrize and
 * drop_self_loops are ignored, as in the reference. */
int load_csr_from_file(const char *path, int symmetrize, int drop_self_loops, CSRGraph *out);

/* Frees row_ptr/col_idx and zeroes the struct (reference src/graph.c:130-141). */
void free_csr(CSRGraph *g);

/* ---- additions (no counterpart in the reference) ---------------------- */

/* Raw binary CSR ("CSRB" magic, u32 version, u32 n, u64 m, row_ptr, col_idx)
 * for graphs a MAT v5 file cannot hold (3.6e9 nonzeros overflow its 32-bit
 * element sizes).  Returns 0, 1 cannot open, 3 OOM, 5 bad format. */
int load_csr_from_csrbin(const char *path, CSRGraph *out);
int save_csr_to_csrbin(const char *path, const CSRGraph *g);
/* Writes g as a logical sparse matrix inside struct Problem (field A),
 * uncompressed MAT level 5.  Returns 0, 1 cannot open, 4 too large. */
int save_csr_to_mat(const char *path, const CSRGraph *g);

#endif /* GRAPH_H */
