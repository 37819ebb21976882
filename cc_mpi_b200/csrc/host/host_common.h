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

#endif
