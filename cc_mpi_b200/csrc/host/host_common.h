/* Helpers shared by the host C sources of libccb200. */
#ifndef CCB200_HOST_COMMON_H
#define CCB200_HOST_COMMON_H

/* Prints "<where>: <ccgpu_last_error()>" to stderr and, unless
 * ccb200_set_exit_on_error(0) was called, exits as the reference does on
 * failures (src/runtime_utils.c:9-14, src/cc_pthreads.c:163-167). */
void ccb200_fail(const char *where, int status);

#endif
