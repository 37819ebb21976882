/* Build shim for compiling the reference's MPI-free sources (cc_pthreads.c,
 * boundary_sort.c, opt_parser.c, results_writer.c) into oracle/_ref/.  Their
 * headers only name the MPI_Comm type in prototypes they never call. */
#ifndef CCB200_REF_SHIM_MPI_H
#define CCB200_REF_SHIM_MPI_H
typedef int MPI_Comm;
#endif
