/*
 * vec_helpers.h - boundary edge types and growable host vectors.
 *
 * Drop-in for the reference's include/vec_helpers.h: same struct layouts
 * (BoundaryEdge {rep, remote} is the 8-byte record the boundary sort orders
 * by remote << 32 | rep) and the same vector helpers, which abort through
 * mpi_die_abort on allocation failure as in the reference.
 */
#ifndef VEC_HELPERS_H
#define VEC_HELPERS_H

#include <stdint.h>

#include "cc_comm.h"

typedef struct
{
    uint32_t *data;
    uint64_t size;
    uint64_t cap;
} U32Vec;

void u32vec_init(U32Vec *v);
void u32vec_free(U32Vec *v);
void u32vec_reserve(U32Vec *v, uint64_t new_cap, MPI_Comm comm);
void u32vec_push(U32Vec *v, uint32_t x, MPI_Comm comm);

typedef struct
{
    uint32_t *data;
    int size;
    int cap;
} U32VecI;

void u32veci_init(U32VecI *v);
void u32veci_free(U32VecI *v);
void u32veci_reserve(U32VecI *v, int new_cap, MPI_Comm comm);
void u32veci_push(U32VecI *v, uint32_t x, MPI_Comm comm);

/* Local representative and remote vertex of a cut edge. */
typedef struct
{
    uint32_t rep;
    uint32_t remote;
} BoundaryEdge;

typedef struct
{
    BoundaryEdge *data;
    uint64_t size;
    uint64_t cap;
} BEVec;

void bevec_init(BEVec *v);
void bevec_free(BEVec *v);
void bevec_reserve(BEVec *v, uint64_t new_cap, MPI_Comm comm);
void bevec_push(BEVec *v, BoundaryEdge e, MPI_Comm comm);

/* Local representative and ghost index. */
typedef struct
{
    uint32_t rep;
    uint32_t gidx;
} BoundaryPair;

typedef struct
{
    BoundaryPair *data;
    uint64_t size;
    uint64_t cap;
} BPVec;

void bpvec_init(BPVec *v);
void bpvec_free(BPVec *v);
void bpvec_reserve(BPVec *v, uint64_t new_cap, MPI_Comm comm);
void bpvec_push(BPVec *v, BoundaryPair x, MPI_Comm comm);

#endif /* VEC_HELPERS_H */
