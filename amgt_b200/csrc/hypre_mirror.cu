// HYPRE-facing mirror layer: the two hooks AmgT puts into HYPRE, with
// HYPRE's argument meaning and error behaviour, over a struct that carries
// the hypre_CSRMatrix fields the AmgT path uses.
//
//   amgt_CSRSpGemm        <- hypreDevice_CSRSpGemm
//                            (AmgT_HYPRE/src/seq_mv/csr_spgemm_device.c:2579-2608)
//   amgt_CSRMatrixMatvec  <- hypre_CSRMatrixMatvecCusparseNewAPI
//                            (AmgT_HYPRE/src/seq_mv/csr_matvec_device.c:2397-2437)
//
// Caching follows the reference: the mBSR form is built on first use and
// kept on the matrix (bsr_tag, CSR2BSR_GPU :1201-1205), the long-row segment
// table is built when the spread of block-row lengths is >= 12
// (BSR_BALANCED_PREPROCESS_GPU with ADAPTIVE_AMGT_SPMV, :1269-1275), value
// shadows are built once per precision (mixed_precision_flag), and an
// SpGEMM result carries its mBSR with bsr_tag = 1 (:1834-1842).  Unlike the
// reference, trans = 1 is honoured (through a cached block transpose) and
// multivectors go through the mBSR SpMM.
#include <cstdlib>
#include <cstring>

#include "amgt_internal.cuh"

using namespace amgt;

static cudaStream_t g_stream = nullptr;

static int ensure_bsr(amgt_CSRMatrix *A)
{
    if (A->bsr_tag && A->bsr_mat) return AMGT_OK;
    if (!A->bsr_mat) {
        A->bsr_mat = (amgt_bsr *)calloc(1, sizeof(amgt_bsr));
        if (!A->bsr_mat) return AMGT_ERR_ALLOC;
    }
    AMGT_TRY(amgt_csr_to_bsr(&A->csr, A->bsr_mat, (amgt_stream_t)g_stream));
    A->bsr_tag = 1;
    return AMGT_OK;
}

static int ensure_shadow(amgt_bsr *M, int prec)
{
    if (prec == AMGT_DOUBLE) return AMGT_OK;
    return amgt_bsr_make_shadow(M, prec, (amgt_stream_t)g_stream);
}

extern "C" {

int amgt_set_stream(amgt_stream_t stream)
{
    g_stream = (cudaStream_t)stream;
    return AMGT_OK;
}

amgt_CSRMatrix *amgt_CSRMatrixCreate(int num_rows, int num_cols, int num_nonzeros, int *i, int *j, double *data,
                                     int level)
{
    if (num_rows < 0 || num_cols < 0 || num_nonzeros < 0) return nullptr;
    amgt_CSRMatrix *A = (amgt_CSRMatrix *)calloc(1, sizeof(amgt_CSRMatrix));
    if (!A) return nullptr;
    A->csr.num_rows = num_rows;
    A->csr.num_cols = num_cols;
    A->csr.num_nonzeros = num_nonzeros;
    A->csr.i = i;
    A->csr.j = j;
    A->csr.data = data;
    A->coasen_level = level;
    return A;
}

int amgt_CSRMatrixDestroy(amgt_CSRMatrix *A)
{
    if (!A) return AMGT_OK;
    if (A->bsr_mat) {
        amgt_bsr_free(A->bsr_mat, (amgt_stream_t)g_stream);
        free(A->bsr_mat);
    }
    if (A->bsr_mat_T) {
        amgt_bsr_free(A->bsr_mat_T, (amgt_stream_t)g_stream);
        free(A->bsr_mat_T);
    }
    if (A->owns_data) amgt_csr_free(&A->csr, (amgt_stream_t)g_stream);
    free(A);
    return AMGT_OK;
}

int amgt_CSRSpGemm(amgt_CSRMatrix *A, amgt_CSRMatrix *B, amgt_CSRMatrix **C_ptr)
{
    if (!A || !B || !C_ptr) return AMGT_ERR_INVALID;
    if (A->csr.num_cols != B->csr.num_rows) return AMGT_ERR_INVALID;
    *C_ptr = nullptr;
    AMGT_TRY(ensure_bsr(A));
    AMGT_TRY(ensure_bsr(B));
    const int prec = amgt_precision_for_level(A->coasen_level);
    AMGT_TRY(ensure_shadow(A->bsr_mat, prec));
    AMGT_TRY(ensure_shadow(B->bsr_mat, prec));
    if (prec != AMGT_DOUBLE) A->mixed_precision_flag = B->mixed_precision_flag = 1;
    amgt_CSRMatrix *C = (amgt_CSRMatrix *)calloc(1, sizeof(amgt_CSRMatrix));
    if (!C) return AMGT_ERR_ALLOC;
    C->bsr_mat = (amgt_bsr *)calloc(1, sizeof(amgt_bsr));
    if (!C->bsr_mat) {
        free(C);
        return AMGT_ERR_ALLOC;
    }
    const int rc = amgt_spgemm(prec, A->bsr_mat, B->bsr_mat, C->bsr_mat, &C->csr, (amgt_stream_t)g_stream);
    if (rc != AMGT_OK) {
        free(C->bsr_mat);
        free(C);
        return rc;
    }
    C->bsr_tag = 1;
    C->owns_data = 1;
    C->coasen_level = A->coasen_level;
    C->mixed_precision_flag = prec != AMGT_DOUBLE;
    *C_ptr = C;
    return AMGT_OK;
}

int amgt_CSRMatrixMatvec(int trans, double alpha, amgt_CSRMatrix *A, const amgt_vector *x, double beta,
                         amgt_vector *y, int offset)
{
    if (!A || !x || !y) return AMGT_ERR_INVALID;
    if (offset != 0) return AMGT_ERR_INVALID;
    const int nrow = trans ? A->csr.num_cols : A->csr.num_rows;
    const int ncol = trans ? A->csr.num_rows : A->csr.num_cols;
    const int nvec = x->num_vectors > 1 ? x->num_vectors : 1;
    if (x->size != ncol || y->size != nrow) return AMGT_ERR_INVALID;
    if ((y->num_vectors > 1 ? y->num_vectors : 1) != nvec) return AMGT_ERR_INVALID;
    AMGT_TRY(ensure_bsr(A));
    amgt_bsr *M = A->bsr_mat;
    if (trans) {
        if (!A->bsr_mat_T) {
            A->bsr_mat_T = (amgt_bsr *)calloc(1, sizeof(amgt_bsr));
            if (!A->bsr_mat_T) return AMGT_ERR_ALLOC;
            const int rc = amgt_bsr_transpose(A->bsr_mat, A->bsr_mat_T, (amgt_stream_t)g_stream);
            if (rc != AMGT_OK) {
                free(A->bsr_mat_T);
                A->bsr_mat_T = nullptr;
                return rc;
            }
        }
        M = A->bsr_mat_T;
    }
    const int prec = amgt_precision_for_level(A->coasen_level);
    AMGT_TRY(ensure_shadow(M, prec));
    if (prec != AMGT_DOUBLE) A->mixed_precision_flag = 1;
    if (!M->rowPtrbyWarp && M->stand >= 12.0) {
        AMGT_TRY(amgt_bsr_balance(M, (amgt_stream_t)g_stream));
        if (!trans) A->bsr_spmv_balanced_tag = 1;
    }
    if (nvec == 1) return amgt_spmv(prec, alpha, M, x->data, beta, y->data, (amgt_stream_t)g_stream);
    const int ldx = x->vecstride > 0 ? x->vecstride : x->size;
    const int ldy = y->vecstride > 0 ? y->vecstride : y->size;
    return amgt_spmm(prec, alpha, M, nvec, x->data, ldx, beta, y->data, ldy, (amgt_stream_t)g_stream);
}

}  // extern "C"
