/* The subset of libmatio that the reference's loader (src/graph.c) calls,
 * for compiling it unmodified without libmatio.  TEST INFRASTRUCTURE ONLY:
 * it builds the checker in oracle/_ref, never the product.  fakematio.c
 * reads little-endian MAT level-5 files (plain and zlib-compressed elements,
 * sparse, struct and other classes) and, for graphs too large for MAT v5,
 * the CSR binary format (magic "CSRB") served as one sparse variable. */
#ifndef FAKEMATIO_MATIO_H
#define FAKEMATIO_MATIO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint32_t mat_uint32_t;

enum mat_acc { MAT_ACC_RDONLY = 0, MAT_ACC_RDWR = 1 };

enum matio_types {
    MAT_T_UNKNOWN = 0, MAT_T_INT8 = 1, MAT_T_UINT8 = 2, MAT_T_INT16 = 3, MAT_T_UINT16 = 4,
    MAT_T_INT32 = 5, MAT_T_UINT32 = 6, MAT_T_SINGLE = 7, MAT_T_DOUBLE = 9, MAT_T_INT64 = 12,
    MAT_T_UINT64 = 13, MAT_T_MATRIX = 14, MAT_T_COMPRESSED = 15, MAT_T_UTF8 = 16,
    MAT_T_UTF16 = 17, MAT_T_UTF32 = 18, MAT_T_STRING = 20, MAT_T_CELL = 21, MAT_T_STRUCT = 22,
    MAT_T_ARRAY = 23, MAT_T_FUNCTION = 24
};

enum matio_classes {
    MAT_C_EMPTY = 0, MAT_C_CELL = 1, MAT_C_STRUCT = 2, MAT_C_OBJECT = 3, MAT_C_CHAR = 4,
    MAT_C_SPARSE = 5, MAT_C_DOUBLE = 6, MAT_C_SINGLE = 7, MAT_C_INT8 = 8, MAT_C_UINT8 = 9,
    MAT_C_INT16 = 10, MAT_C_UINT16 = 11, MAT_C_INT32 = 12, MAT_C_UINT32 = 13, MAT_C_INT64 = 14,
    MAT_C_UINT64 = 15, MAT_C_FUNCTION = 16, MAT_C_OPAQUE = 17
};

typedef struct mat_t mat_t;

typedef struct mat_sparse_t {
    size_t nzmax;
    mat_uint32_t *ir; /* row index of each stored entry */
    size_t nir;
    mat_uint32_t *jc; /* column starts, ncols + 1 entries */
    size_t njc;
    size_t ndata;
    void *data;
} mat_sparse_t;

typedef struct matvar_t {
    size_t nbytes;
    int rank;
    enum matio_types data_type;
    int data_size;
    enum matio_classes class_type;
    int isComplex;
    int isGlobal;
    int isLogical;
    size_t *dims;
    char *name;
    void *data;
    int mem_conserve;
    void *internal;
} matvar_t;

mat_t *Mat_Open(const char *matname, int mode);
int Mat_Close(mat_t *mat);
matvar_t *Mat_VarReadNext(mat_t *mat);
matvar_t *Mat_VarGetStructFieldByName(matvar_t *matvar, const char *field_name, size_t index);
void Mat_VarFree(matvar_t *matvar);

#ifdef __cplusplus
}
#endif

#endif /* FAKEMATIO_MATIO_H */
