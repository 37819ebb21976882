/*
 * runtime_utils.h - error exit and host thread count.
 *
 * Drop-in for the reference's include/runtime_utils.h: mpi_die_abort prints
 * the message to stderr and ends the process (the reference calls
 * MPI_Abort, src/runtime_utils.c:9-14); runtime_default_threads returns the
 * online host cores (src/runtime_utils.c:16-24).
 */
#ifndef RUNTIME_UTILS_H
#define RUNTIME_UTILS_H

#include "cc_comm.h"

void mpi_die_abort(MPI_Comm comm, const char *msg);
int runtime_default_threads(void);

#endif /* RUNTIME_UTILS_H */
