/* The subset of HYPRE's declarations that the hook code in INTEGRATION.md
 * uses, shaped like AmgT's HYPRE 2.31 headers (AmgT_HYPRE/src/seq_mv/
 * seq_mv.h:154-199 for hypre_CSRMatrix and its AmgT fields and accessors,
 * :359-377 for hypre_Vector; _hypre_utilities.h for the allocator and the
 * error macros; _hypre_parcsr_mv.h for the ParCSR accessors).  Test
 * infrastructure: tests/test_integration_shim.py compiles the document's
 * code against it so that the shim text keeps compiling. */
#ifndef AMGT_TEST_HYPRE_SUBSET_H
#define AMGT_TEST_HYPRE_SUBSET_H

#include <stddef.h>
#include <stdlib.h>

#include "amgt_b200.h"

typedef int HYPRE_Int;
typedef int HYPRE_BigInt;
typedef int hypre_int;
typedef double HYPRE_Real;
typedef double HYPRE_Complex;
typedef enum { HYPRE_MEMORY_UNDEFINED = -1, HYPRE_MEMORY_HOST = 0, HYPRE_MEMORY_DEVICE = 1 } HYPRE_MemoryLocation;

typedef amgt_bsr bsrMAT; /* as INTEGRATION.md section 1 has seq_mv.h do */

typedef struct {
    int coasen_level;
    char bsr_spmv_balanced_tag;
    char bsr_tag;
    char vector_space_flag;
    char mixed_precision_flag;
    char tag_mid_matrix;
    bsrMAT *bsr_mat;
    HYPRE_Int *i;
    HYPRE_Int *j;
    HYPRE_BigInt *big_j;
    HYPRE_Int num_rows;
    HYPRE_Int num_cols;
    HYPRE_Int num_nonzeros;
    hypre_int *i_short;
    hypre_int *j_short;
    HYPRE_Int owns_data;
    HYPRE_Int pattern_only;
    HYPRE_Complex *data;
    HYPRE_Int *rownnz;
    HYPRE_Int num_rownnz;
    HYPRE_MemoryLocation memory_location;
} hypre_CSRMatrix;

#define hypre_CSRMatrixI(m) ((m)->i)
#define hypre_CSRMatrixJ(m) ((m)->j)
#define hypre_CSRMatrixData(m) ((m)->data)
#define hypre_CSRMatrixNumRows(m) ((m)->num_rows)
#define hypre_CSRMatrixNumCols(m) ((m)->num_cols)
#define hypre_CSRMatrixNumNonzeros(m) ((m)->num_nonzeros)
#define hypre_CSRMatrixMemoryLocation(m) ((m)->memory_location)
#define hypre_BSRBALANCEDTAG(m) ((m)->bsr_spmv_balanced_tag)
#define hypre_BSRTAG(m) ((m)->bsr_tag)
#define hypre_BSR(m) ((m)->bsr_mat)
#define hypre_Level(m) ((m)->coasen_level)

typedef struct {
    HYPRE_Complex *data;
    HYPRE_Int size;
    HYPRE_Int owns_data;
    HYPRE_MemoryLocation memory_location;
    HYPRE_Int num_vectors;
    HYPRE_Int multivec_storage_method;
    HYPRE_Int vecstride;
    HYPRE_Int idxstride;
} hypre_Vector;

#define hypre_VectorData(v) ((v)->data)
#define hypre_VectorNumVectors(v) ((v)->num_vectors)
#define hypre_VectorVectorStride(v) ((v)->vecstride)

typedef struct { hypre_CSRMatrix *diag; } hypre_ParCSRMatrix;
typedef struct { hypre_Vector *local_vector; } hypre_ParVector;
#define hypre_ParCSRMatrixDiag(A) ((A)->diag)
#define hypre_ParVectorLocalVector(v) ((v)->local_vector)

void *hypre_MAlloc_device(size_t bytes, HYPRE_MemoryLocation where);
void hypre_Free_device(void *p, HYPRE_MemoryLocation where);
#define hypre_TAlloc(type, count, where) ((type *)hypre_MAlloc_device(sizeof(type) * (size_t)(count), (where)))
#define hypre_TFree(p, where) hypre_Free_device((p), (where))

extern HYPRE_Int hypre_error_flag;
#define HYPRE_ERROR_GENERIC 1
void hypre_error_handler(const char *file, HYPRE_Int line, HYPRE_Int ierr, const char *msg);
#define hypre_error_w_msg(IERR, msg) hypre_error_handler(__FILE__, __LINE__, IERR, msg)

hypre_CSRMatrix *hypre_CSRMatrixCreate(HYPRE_Int num_rows, HYPRE_Int num_cols, HYPRE_Int num_nonzeros);

typedef struct hypre_Handle_struct hypre_Handle;
hypre_Handle *hypre_handle(void);
void *hypre_HandleComputeStream(hypre_Handle *h);

/* the shim's own lookup of 1 ./ l1 norms kept beside HYPRE's l1_norms */
const double *amgt_inv_l1_of(const HYPRE_Real *l1_norms);

#endif
