/* Helpers shared by the host C sources of libccb200. */
#ifndef CCB200_HOST_COMMON_H
#define CCB200_HOST_COMMON_H

#include "cc_comm.h"

/* Prints "<where>: <ccgpu_last_error()>" to stderr and, unless
 * ccb200_set_exit_on_error(0) was called, exits as the reference does on
 * failures (src/runtime_utils.c:9-14, src/cc_pthreads.c:163-167). */
void ccb200_fail(const char *where, int status);
int ccb200_exit_on_error(void);
/* Sets this thread's ccgpu_last_error() message; returns status. */
int ccb200_set_error(int status, const char *fmt, ...);

/* Per-rank pointer table of a group (one slot per rank), for the
 * rendezvous collectives of the per-rank calls. */
void **cc_group_slots(cc_group *view);
void cc_group_store_stats(cc_group *g, const ccgpu_dist_stats *s);

/* Pairwise mailboxes of the neighbourhood exchanges.  post: this rank
 * offers buf, with element offset off[q] and count cnt[q] for each reader
 * rank q, to `readers` readers (waits first until its previous post has
 * been read by all of its readers).  take: waits for src's next post and
 * calls copy(arg, buf, off[me], cnt[me]).  drain: waits until this rank's
 * post has been read by all of its readers.  Waits are bounded
 * (CCB200_GROUP_TIMEOUT_S, default 600 s); a timeout returns
 * CCGPU_ERR_TIMEOUT. */
int cc_group_post(cc_group *view, const void *buf, const int *off, const int *cnt, int readers);
int cc_group_take(cc_group *view, int src,
                  void (*copy)(void *arg, const void *buf, int off, int cnt), void *arg);
int cc_group_drain(cc_group *view);

/* The CSC arrays of a .mat sparse matrix (struct Problem's field A, or the
 * first sparse variable), as stored: column starts jc[ncols+1], row indices
 * ir[nnz].  Return codes as load_csr_from_mat. */
typedef struct {
    uint32_t nrows, ncols;
    uint64_t nnz;
    uint64_t *jc;
    uint32_t *ir;
} mat_csc;
int load_csc_from_mat(const char *path, mat_csc *out);
void free_mat_csc(mat_csc *c);

#endif
