/*
 * amgt_b200.h - C ABI of the B200 (sm_100a) mBSR kernels behind HYPRE's
 * device SpGEMM and SpMV hooks.
 *
 * Plain C: no CUDA, C++ or torch types cross this boundary.  Every pointer
 * inside amgt_csr / amgt_bsr / amgt_vector is DEVICE memory unless stated
 * otherwise.  Every entry point returns an amgt_status (0 = success) and is
 * stream-ordered on the stream it is given (NULL = the legacy default
 * stream); an entry point only blocks the host where it must learn a size
 * that decides an allocation (noted per function).  Host threads may call
 * the library at the same time on one device (each thread stages its
 * read-backs in its own pinned buffer; the device error word is shared, so
 * AMGT_ERR_DEVICE may reach the thread that reads back first); one handle
 * (amgt_amg) belongs to one thread at a time.
 *
 * Reference interfaces replaced (paths inside the AmgT repository,
 * R = AmgT_HYPRE/src):
 *   hypreDevice_CSRSpGemm                 R/seq_mv/csr_spgemm_device.c:2579-2608
 *   hypre_CSRMatrixMatvecCusparseNewAPI   R/seq_mv/csr_matvec_device.c:2397-2437
 *   bsrMAT                                R/seq_mv/seq_mv.h:105-129
 *   AmgT fields of hypre_CSRMatrix        R/seq_mv/seq_mv.h:154-199
 */
#ifndef AMGT_B200_H
#define AMGT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define AMGT_API __attribute__((visibility("default")))
#else
#define AMGT_API
#endif

/* Opaque CUDA stream handle (binary-identical to cudaStream_t). */
typedef struct CUstream_st *amgt_stream_t;

/* ---------------------------------------------------------------- status */
typedef enum {
    AMGT_OK = 0,
    AMGT_ERR_INVALID = 1,     /* bad argument (NULL, negative size, mismatch) */
    AMGT_ERR_ALLOC = 2,       /* the allocator returned NULL */
    AMGT_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    AMGT_ERR_DEVICE = 4,      /* a kernel raised its device error word
                                 (bounded hash probe exhausted, bad index) */
    AMGT_ERR_UNSUPPORTED = 5, /* precision / shape not built */
    AMGT_ERR_NO_DEVICE = 6,   /* no CUDA device visible to the library */
    AMGT_ERR_TOO_LARGE = 7    /* a size exceeds a fixed maximum of the call */
} amgt_status;

AMGT_API const char *amgt_status_string(int status);

/* Library + device sanity: returns AMGT_OK when an sm_100 device is current
 * and the kernels of this library can launch on it. */
AMGT_API int amgt_init(void);

/* Number of kernels this library has launched since load (all entry points,
 * all streams).  Used to prove that a measured region ran native kernels. */
AMGT_API uint64_t amgt_kernel_launch_count(void);

/* Architecture of the device code the current device runs for this library
 * (cudaFuncGetAttributes().binaryVersion of one of its kernels: 100 for the
 * sm_100a build).  AMGT_ERR_NO_DEVICE without a device. */
AMGT_API int amgt_kernel_arch(int *binary_version);

/* ---------------------------------------------------------- allocation */
/* Every DEVICE array the library returns or uses as scratch comes from this
 * allocator.  HYPRE plugs hypre_TAlloc/hypre_TFree here so that
 * hypre_CSRMatrixDestroy can free an SpGEMM result (the reference allocates C
 * with hypre_TAlloc, R/seq_mv/csr_spgemm_device.c:1808-1839).  Exceptions,
 * all small and all pinned HOST memory from cudaMallocHost: each host
 * thread's 512-byte read-back staging per device (freed when the thread
 * exits), an AMG handle's read-back slots (8 * (max_iter + 170) bytes) and
 * a batch's (8 * (3 * nsys + 4) bytes), each one block from a library cache
 * of pinned blocks (taken by the setup, given back by amgt_amg_destroy,
 * reused by later setups, freed by amgt_trim_pool); the per-device
 * error word (16 bytes, cudaMalloc, held until exit); and the fixed array of
 * amgt_spmv_segmented_noalloc.
 * Install or remove an allocator only while no other library call runs and
 * no array the library allocated is still live: a block is always freed
 * through the allocator installed when the free happens. */
/* Default: a stream-ordered memory pool owned by the library (one per
 * device) that keeps freed memory for reuse; amgt_trim_pool(keep) returns
 * all but `keep` bytes of it to the driver (synchronises the device). */
AMGT_API int amgt_trim_pool(size_t keep_bytes);
typedef void *(*amgt_alloc_fn)(size_t bytes, amgt_stream_t stream, void *ctx);
typedef void (*amgt_free_fn)(void *ptr, amgt_stream_t stream, void *ctx);
AMGT_API int amgt_set_allocator(amgt_alloc_fn alloc_fn, amgt_free_fn free_fn, void *ctx);

/* ----------------------------------------------------------- precision */
/* AMGT_PRECISION of R/seq_mv/seq_mv.h:139-144, plus BF16. */
typedef enum {
    AMGT_DOUBLE = 0, /* fp64 values, fp64 arithmetic                      */
    AMGT_FLOAT = 1,  /* fp32 value shadow, fp32 arithmetic                */
    AMGT_HALF = 2,   /* fp16 value shadow, fp32 arithmetic (accumulate)   */
    AMGT_BF16 = 3    /* bf16 value shadow, fp32 arithmetic (accumulate)   */
} amgt_precision;

/* get_calculationPrecison, R/seq_mv/csr_spgemm_device.c:1847-1862:
 * level 0 -> DOUBLE, 1 -> FLOAT, >=2 -> HALF under the default policy.
 * amgt_set_level_policy replaces the table: prec[l] for level l < n, and
 * prec[n-1] for every deeper level.  n = 0 restores the default. */
AMGT_API int amgt_precision_for_level(int level);
AMGT_API int amgt_set_level_policy(const int *prec, int n);

/* ------------------------------------------------------------- formats */
/* CSR, 0-based, HYPRE_Int = int32 indices, HYPRE_Complex = double values.
 * Column order inside a row is free (HYPRE stores the diagonal first,
 * R/parcsr_mv/par_csr_triplemat_device.c:896); duplicates are not allowed. */
typedef struct {
    int num_rows;
    int num_cols;
    int num_nonzeros;
    int *i;       /* [num_rows + 1] */
    int *j;       /* [num_nonzeros] */
    double *data; /* [num_nonzeros] */
} amgt_csr;

/* mBSR: 4x4 blocks, bitmap per block.  Mirrors bsrMAT
 * (R/seq_mv/seq_mv.h:105-129) field for field; the fp16 shadow is stored as
 * uint16 halves instead of uint32-packed half2, and a bf16 shadow and the
 * longest block-row length are added.  Block values are row-major, 16 per
 * block, zero-padded; bit (r*4 + c) of blcMap is set iff the CSR source had
 * an entry at (4*brow + r, 4*bcol + c).  Block columns ascend within a
 * block row. */
typedef struct {
    int row, col;        /* scalar dimensions                       */
    int nnz;             /* 16 * blc_num (stored values), saturates at INT_MAX */
    int blc_row, blc_col;/* ceil(row/4), ceil(col/4)                */
    int blc_num;         /* number of stored 4x4 blocks             */
    double stand;        /* std-dev of blocks per block row          */
    double avg_nnz;      /* CSR nonzeros per stored block            */
    int *blcPtr;         /* [blc_row + 1]                           */
    int *blcIdx;         /* [blc_num] block column                  */
    double *blcVal;      /* [16 * blc_num]                          */
    uint16_t *blcMap;    /* [blc_num]                               */
    int warpnum;         /* load-balanced segments (see amgt_bsr_balance) */
    int *rowPtrbyWarp;   /* [blc_row + 1] segments per block row, scanned */
    int *rowIdxbyWarp;   /* [warpnum] block row of each segment      */
    float *blcVal_fp32;  /* [16 * blc_num] or NULL                  */
    uint16_t *blcVal_fp16; /* [16 * blc_num] IEEE half bits or NULL  */
    uint16_t *blcVal_bf16; /* [16 * blc_num] bfloat16 bits or NULL   */
    int max_blc_per_row; /* longest block row                        */
    int csr_nnz;         /* number of set bitmap bits (CSR nonzeros) */
    int exact_prec;      /* AMGT_HALF / AMGT_FLOAT: that shadow holds every
                            value exactly (amgt_bsr_make_exact), and fp64
                            products read it with unchanged results;
                            AMGT_DOUBLE (0): none                     */
} amgt_bsr;

/* Dense vector / column-major multivector, mirrors the fields of
 * hypre_Vector the matvec hook reads (data, size, num_vectors, vecstride). */
typedef struct {
    double *data;
    int size;
    int num_vectors;
    int vecstride;       /* distance between vectors, >= size */
} amgt_vector;

/* -------------------------------------------------------- conversions */
/* CSR -> mBSR.  Replaces CSR2BSR_GPU (R/seq_mv/csr_matvec_device.c:1201-1267)
 * with its kernels csr2bsr_get_ptr / _compute_bin / _set_bin / _getidx /
 * _getidx_large / getStand (:638-1092).  Fills every field of *out except the
 * shadows and the balanced-segment arrays (NULL / 0).  Host-blocking once (to
 * size the block arrays). */
AMGT_API int amgt_csr_to_bsr(const amgt_csr *A, amgt_bsr *out, amgt_stream_t stream);

/* mBSR -> CSR (set bitmap bits, ascending columns per row).  Replaces
 * BSR2CSR_step1-3 / bsr2csr_get_ptr / bsr2csr_get_idx_val
 * (R/seq_mv/csr_spgemm_device.c:1344-1440, 1501-1525).  Host-blocking once. */
AMGT_API int amgt_bsr_to_csr(const amgt_bsr *A, amgt_csr *out, amgt_stream_t stream);

/* Segments of <= 64 blocks for long block rows.  Replaces
 * BSR_BALANCED_PREPROCESS_GPU + get_rowPtrbyWarp / get_rowIdxbyWarp
 * (R/seq_mv/csr_matvec_device.c:615-637, 1269-1300); fills warpnum,
 * rowPtrbyWarp, rowIdxbyWarp.  Host-blocking once. */
AMGT_API int amgt_bsr_balance(amgt_bsr *A, amgt_stream_t stream);

/* Builds the value shadow for prec (FLOAT / HALF / BF16) from blcVal,
 * round-to-nearest-even.  Replaces bsr_val_fp64_to_32 / _to_16
 * (R/seq_mv/csr_spgemm_device.c:1467-1499).  No-op for DOUBLE or when the
 * shadow exists. */
AMGT_API int amgt_bsr_make_shadow(amgt_bsr *A, int prec, amgt_stream_t stream);

/* Block transpose: out = A^T in mBSR (values and bitmaps transposed per
 * block, block columns ascending).  No reference counterpart inside AmgT:
 * HYPRE builds R = P^T in CSR (keepT, R/parcsr_ls/par_amg.c:307-315); this
 * keeps it in mBSR.  Host-blocking once. */
AMGT_API int amgt_bsr_transpose(const amgt_bsr *A, amgt_bsr *out, amgt_stream_t stream);

/* Exact narrow storage (no counterpart in the reference): checks whether
 * every value of A is an fp16 value (else an fp32 value); if so builds that
 * shadow and sets A->exact_prec, after which fp64 products (amgt_spmv,
 * amgt_bsr_residual / _jacobi at AMGT_DOUBLE) read 2 or 4 bytes per value
 * instead of 8 with bit-identical results.  Stencil operators with
 * dyadic-rational coefficients and their interpolation / Galerkin
 * products qualify.  One host read-back.  Call again after changing the
 * values (or set exact_prec to AMGT_DOUBLE). */
AMGT_API int amgt_bsr_make_exact(amgt_bsr *A, amgt_stream_t stream);
/* Frees every array of *A (through the allocator) and zeroes the struct. */
AMGT_API int amgt_bsr_free(amgt_bsr *A, amgt_stream_t stream);
AMGT_API int amgt_csr_free(amgt_csr *A, amgt_stream_t stream);

/* ---------------------------------------------------------------- SpMV */
/* y <- alpha * A * x + beta * y, A in mBSR, x and y fp64.  Replaces
 * spmv_amgT_fp64 / _fp32 / _fp16 and their bsr_spmv_* kernels
 * (R/seq_mv/csr_matvec_device.c:319-613, 1302-1542, 1654-2309).
 * prec selects the value array (DOUBLE: blcVal, FLOAT: blcVal_fp32, HALF:
 * blcVal_fp16, BF16: blcVal_bf16; the shadow must exist).  Reduced
 * precisions convert x to fp32 in registers, accumulate in fp32 and combine
 * with beta*y in fp64.  beta == 0 does not read y.  Deterministic: no
 * atomics; the sum order depends only on the block-row length.
 * Never blocks the host. */
AMGT_API int amgt_spmv(int prec, double alpha, const amgt_bsr *A, const double *x,
              double beta, double *y, amgt_stream_t stream);

/* Same for nvec column-major vectors (x[v*ldx + i], y[v*ldy + i]); the block
 * values are read once for all vectors (mBSR SpMM). */
AMGT_API int amgt_spmm(int prec, double alpha, const amgt_bsr *A, int nvec,
              const double *x, int ldx, double beta, double *y, int ldy,
              amgt_stream_t stream);

/* Row-major multivector SpMM for the batching form (many right-hand sides
 * at once): Y[i*nvec + v] <- alpha * (A X)[i][v] + beta * Y[i*nvec + v],
 * X[j*nvec + v], 1 <= nvec <= 32, X and Y fp64.  The reference's matvec
 * hook ignores num_vectors (R/seq_mv/csr_matvec_device.c:2409-2437); its
 * multivector storage is column-wise (:139-170), this one interleaves the
 * vectors so that a block column's x rows are contiguous.
 * prec FLOAT / HALF / BF16 on the tensor cores (engine TENSOR_CORE): two
 * block rows per mma.m16n8k8 (tf32 in, fp32 accumulate), values and x split
 * into tf32 high and low parts so that the products carry fp32 accuracy;
 * the result is combined with beta * Y in fp64 (so Y = B, alpha = -1,
 * beta = 1 gives an fp64 residual of products computed on the tensor
 * cores).  prec DOUBLE: fp64 on the CUDA cores.  engine CUDA_CORE: a warp
 * per block row, a lane per right-hand side.  engine AUTO: amgt_autotune's
 * choice for (A, prec, nvec), else the tensor cores with 8 warps per CTA.
 * An fp32 request on a matrix whose exact fp16 shadow holds every value
 * reads that shadow.  Never blocks the host. */
#define AMGT_ENGINE_AUTO 0
#define AMGT_ENGINE_CUDA_CORE 1
#define AMGT_ENGINE_TENSOR_CORE 2
AMGT_API int amgt_spmm_rm(int prec, int engine, double alpha, const amgt_bsr *A, int nvec, const double *X,
                          double beta, double *Y, amgt_stream_t stream);

/* Autotuner (no reference counterpart: the reference's launch shape is
 * fixed, WARP_NUM_SPMV = 4, R/seq_mv/seq_mv.h:84-99).  Times every
 * candidate launch shape on A (3 warm-up + 10 timed launches each, CUDA
 * events on `stream`; blocks the host) and keeps the fastest for A:
 *   nvec == 1: lanes per block row of amgt_spmv and the fused forms,
 *              candidates 4, 8, 16, 32 (the choice changes the order of a
 *              row's sums, not its terms);
 *   nvec > 1:  amgt_spmm_rm's engine and warps per CTA, candidate code
 *              10 * engine + warps (engine 0 CUDA cores, 1 tensor cores).
 * The choice is dropped when A is freed (amgt_bsr_free) or by
 * amgt_autotune_clear. */
typedef struct {
    int count;          /* candidates timed                 */
    int candidate[8];   /* their codes                       */
    float ms[8];        /* mean time per launch              */
    int choice;         /* the fastest code, now in use      */
} amgt_tune_result;
AMGT_API int amgt_autotune(const amgt_bsr *A, int prec, int nvec, amgt_tune_result *out, amgt_stream_t stream);
AMGT_API int amgt_autotune_clear(void);

/* ------------------------------------------------ smoother / residual */
/* l1 row norms l1[i] = sum_j |a_ij| of the fp64 values: the norms HYPRE's
 * l1-Jacobi (relax 18) divides by, hypre_ParCSRComputeL1Norms option 1
 * (R/parcsr_ls/ams.c:627-636). */
AMGT_API int amgt_bsr_l1_norms(const amgt_bsr *A, double *l1, amgt_stream_t stream);

/* r = f - A u in one pass (the residual of hypre_BoomerAMGCycle,
 * R/parcsr_ls/par_cycle.c:678, MatvecOutOfPlace(-1, A, u, 1, f, r)). */
AMGT_API int amgt_bsr_residual(int prec, const amgt_bsr *A, const double *f,
                               const double *u, double *r, amgt_stream_t stream);

/* One l1-Jacobi sweep in one pass: u_out = u + weight * (f - A u) ./ l1,
 * inv_l1 = 1 ./ l1 (relax 18, hypre_BoomerAMGRelax18WeightedL1Jacobi /
 * Relax7Jacobi, R/parcsr_ls/par_relax.c:1178-1260, which needs a copy of f,
 * a matvec and a vector update).  u_out must not alias u. */
AMGT_API int amgt_bsr_jacobi(int prec, const amgt_bsr *A, const double *inv_l1,
                             double weight, const double *f, const double *u,
                             double *u_out, amgt_stream_t stream);

/* ------------------------------------------------- bitmap-packed values */
/* mBSR with only the values of set bitmap bits stored, block after block in
 * bitmap (row-major) order.  The block
 * structure (blcPtr, blcIdx, blcMap) is borrowed from the amgt_bsr it was
 * packed from, which must outlive it.  At the fill of AMG operators (about
 * 4 of 16) an SpMV reads ~3x fewer bytes than on the 16-value blocks.  No
 * counterpart in the reference (it keeps 16 values per block).  Each block
 * row's values are contiguous, starting at rowVoff[b]; block k's start at
 * blcVoff[k]. */
typedef struct {
    int row, col, blc_row, blc_col, blc_num;
    int nnz;                  /* stored values (= set bits)            */
    int prec;                 /* amgt_precision of val                 */
    const int *blcPtr;        /* borrowed                              */
    const int *blcIdx;        /* borrowed                              */
    const uint16_t *blcMap;   /* borrowed                              */
    int *rowVoff;             /* [blc_row + 1] offset of each block
                                 row's first value                      */
    void *val;                /* [nnz] double / float / half / bf16    */
    int max_blc_per_row;
    int *blcVoff;             /* [blc_num + 1] offset of each block's
                                 first value                            */
} amgt_pbsr;

AMGT_API int amgt_bsr_pack(const amgt_bsr *A, int prec, amgt_pbsr *out, amgt_stream_t stream);
AMGT_API int amgt_pbsr_free(amgt_pbsr *A, amgt_stream_t stream);
/* y <- alpha A x + beta y; r = f - A u; u_out = u + w (f - A u) ./ l1: the
 * same forms as amgt_spmv / amgt_bsr_residual / amgt_bsr_jacobi, in the
 * packed matrix's precision (fp32 accumulation below fp64). */
AMGT_API int amgt_pbsr_spmv(double alpha, const amgt_pbsr *A, const double *x, double beta,
                            double *y, amgt_stream_t stream);
AMGT_API int amgt_pbsr_residual(const amgt_pbsr *A, const double *f, const double *u,
                                double *r, amgt_stream_t stream);
AMGT_API int amgt_pbsr_jacobi(const amgt_pbsr *A, const double *inv_l1, double weight,
                              const double *f, const double *u, double *u_out,
                              amgt_stream_t stream);

/* Segmented SpMV that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they run a matvec:
 * a solver whose device memory went, whole, to a pool sized at set-up and
 * not allowed to grow; a caller whose allocator hook may not be called from
 * the thread issuing the solve; a caller that cannot pay for cudaMalloc /
 * cudaFree, which can synchronise the whole device.  Computes y <- alpha*A*x
 * + beta*y exactly as amgt_spmv does on its long-row (segmented) path, same
 * kernels and summation order, but takes the partial-sum scratch from a
 * fixed device array of AMGT_NOALLOC_MAX_SEGMENTS * 4 doubles (8 MiB, held
 * by every GPU that loads the library until the process exits) instead of
 * the allocator.  A must carry the segment table (amgt_bsr_balance, called
 * during set-up); A->warpnum > AMGT_NOALLOC_MAX_SEGMENTS returns
 * AMGT_ERR_TOO_LARGE.  The first call on a device, with that device
 * current, looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  All calls share the array:
 * calls whose kernels overlap on the GPU race and must be ordered by the
 * caller.  Never blocks the host. */
#define AMGT_NOALLOC_MAX_SEGMENTS (1 << 18)
AMGT_API int amgt_spmv_segmented_noalloc(int prec, double alpha, const amgt_bsr *A,
                                         const double *x, double beta, double *y,
                                         amgt_stream_t stream);

/* -------------------------------------------------------------- SpGEMM */
/* C = A * B on mBSR.  Replaces spgemm_amgT_fp64 / _fp32 / _fp16
 * (R/seq_mv/csr_spgemm_device.c:1527-2578) and its kernels compute_Cub_bin,
 * set_bin, symbolic_spgemm_step1/2(+_large, _gl), numeric_spgemm_hybrid
 * (_tf32, _f16) (:82-1342).  The C block pattern is exactly the set of block
 * columns with a non-zero bitmap product OR-ed over A's row; C's bitmap is
 * that OR.  prec DOUBLE: fp64 products, each 4x4 product summed in k order
 * and added to C in A-row order.  FLOAT / HALF / BF16: A and B shadows
 * (built on demand), fp32 arithmetic, C values rounded to fp64 and a C
 * shadow of the same precision.  If Ccsr != NULL the CSR form of C
 * (BSR2CSR) is also written, by the numeric pass itself (rows of few C
 * blocks) or by a pass right after it.
 * Host-blocking twice (upper bound and C size). */
AMGT_API int amgt_spgemm(int prec, const amgt_bsr *A, const amgt_bsr *B, amgt_bsr *C,
                amgt_csr *Ccsr, amgt_stream_t stream);
/* Engine of the HALF / BF16 block products of later amgt_spgemm calls (all
 * threads; the reference multiplies dense A blocks on the tensor cores,
 * numeric_spgemm_hybrid_f16, R/seq_mv/csr_spgemm_device.c:753-937):
 * AMGT_ENGINE_AUTO / AMGT_ENGINE_CUDA_CORE (default): fp32 multiply and add
 * in the sequential order, the same C bit for bit as the oracle;
 * AMGT_ENGINE_TENSOR_CORE: mma.m16n8k16 with fp32 accumulation, four C
 * blocks' 4x4 products per MMA (block-diagonal in the tile), sums in the
 * tensor core's order (within about 1e-6 of |A||B| of the sequential
 * result).  DOUBLE and FLOAT products are not affected. */
AMGT_API int amgt_spgemm_set_engine(int engine);

/* ------------------------------------------------ AMG setup + solve */
/* Galerkin hierarchy on mBSR and a PCG solve preconditioned by one V(1,1)
 * cycle with l1-Jacobi smoothing: the setup + solve that the two hooks
 * drive inside BoomerAMG-PCG (hypre_ParCSRMatrixRAPKT for the products,
 * hypre_BoomerAMGCycle with relax 18, krylov/pcg.c).  Coarsening and
 * interpolation are the caller's (they are BoomerAMG's, outside the AmgT
 * path): P[l] maps level l+1 to level l.  Level precisions follow
 * amgt_precision_for_level; the finest residual, the Krylov vectors and
 * dots, and the coarsest (dense, inverted) solve are always fp64. */
typedef struct {
    int max_levels;        /* cap on levels (default 25)                    */
    int max_coarse_rows;   /* largest coarsest level (dense inverse), 4096;
                              a larger coarsest level: AMGT_ERR_TOO_LARGE   */
    double tol;            /* ||b - A x|| / ||b|| target (default 1e-8)     */
    int max_iter;          /* default 200, at least 1                       */
    double relax_weight;   /* l1-Jacobi weight (default 1)                  */
    int flexible;          /* flexible CG (Polak-Ribiere beta), default 0   */
    int use_graph;         /* one CUDA graph per iteration (default 1)      */
    int galerkin_by_level; /* Galerkin products at each level's precision,
                              as AmgT's hypreDevice_CSRSpGemm does (0: fp64) */
    int smooth_prec0;      /* precision of the finest-level smoother SpMV   */
    int packed;            /* cycle / Krylov SpMVs on bitmap-packed values
                              (amgt_pbsr), default 0                        */
    int exact_storage;     /* fp64 operators whose values fp16 / fp32 hold
                              exactly are read from that shadow
                              (amgt_bsr_make_exact; same results), default 1 */
    int solver;            /* AMGT_SOLVER_PCG (default) or AMGT_SOLVER_FGMRES_IR */
    int restart;           /* FGMRES basis size m (default 30, 1 .. 32)      */
    double inner_tol;      /* an inner FGMRES solve stops when its residual
                              estimate is <= inner_tol times the outer
                              residual it started from (default 1e-4)      */
    int inner_prec0;       /* level-0 precision inside the inner solve: its
                              matvec and the cycle's level-0 residual
                              (default AMGT_FLOAT)                          */
    int max_outer;         /* refinement steps at most (default 20)        */
} amgt_amg_params;

/* FGMRES with iterative refinement (the reference's R/krylov/flexgmres.c
 * as the outer solver, refined in fp64): each refinement step computes the
 * fp64 residual r = b - A x (level 0 in fp64), solves A d = r with FGMRES(m)
 * preconditioned by the V-cycle, the inner matvec and the cycle's level-0
 * residual at inner_prec0 and the Krylov basis stored in fp32 (inner
 * products and the update of x in fp64), and adds d to x.  The inner loop is
 * one CUDA graph launch per refinement step. */
#define AMGT_SOLVER_PCG 0
#define AMGT_SOLVER_FGMRES_IR 1

typedef struct amgt_amg amgt_amg;

AMGT_API void amgt_amg_default_params(amgt_amg_params *p);
/* Host-blocking (sizes of every level).  The coarsest operator is inverted
 * on the GPU (Gauss-Jordan, partial pivoting); a singular one returns
 * AMGT_ERR_INVALID.  Rejected with AMGT_ERR_INVALID: max_iter outside
 * 1 .. 1000000, tol negative or NaN, max_coarse_rows outside 1 .. 16384. */
AMGT_API int amgt_amg_setup(const amgt_csr *A, int num_interp, const amgt_csr *P,
                            const amgt_amg_params *params, amgt_amg **out,
                            amgt_stream_t stream);
/* Level-by-level setup with the coarsening decided by the caller, once
 * each level's operator exists (the place of BoomerAMG's coarsening and
 * interpolation, R/parcsr_ls/par_amg_setup.c, which HYPRE runs per level on
 * A_l).  fn(level, A_l, P, prec, ctx) is called on the setup's host thread
 * for level = 0, 1, ...: it sets *prec to level l's precision (its
 * smoother and cycle SpMVs; the transfers of level l - 1 use it too) and
 * either returns 0 with *P the interpolation from level l + 1 to level l
 * (device CSR, A_l->row rows; the caller keeps its arrays alive until the
 * setup returns), or returns 1 to make A_l the coarsest level; a negative
 * return aborts the setup (AMGT_ERR_INVALID).  A_l is a borrowed view,
 * valid during the call; fn may run library calls on the same stream.
 * When params->max_levels ends the hierarchy, fn is called once more for
 * the coarsest level's precision.  The rest is amgt_amg_setup's. */
typedef int (*amgt_coarsen_fn)(int level, const amgt_bsr *A, amgt_csr *P, int *prec, void *ctx);
AMGT_API int amgt_amg_setup_adaptive(const amgt_csr *A, amgt_coarsen_fn fn, void *ctx, const amgt_amg_params *params,
                                     amgt_amg **out, amgt_stream_t stream);
/* x: initial guess in, solution out (device).  PCG: the iteration loop is
 * one CUDA graph launch and one read-back (one launch and an 8-byte read
 * per iteration where the runtime lacks conditional graph nodes).
 * FGMRES-IR: one read-back per refinement step; *iterations counts inner
 * FGMRES iterations, *rel_res is the last fp64 residual ||b - A x|| / ||b||. */
AMGT_API int amgt_amg_solve(amgt_amg *amg, const double *b, double *x,
                            int *iterations, double *rel_res, amgt_stream_t stream);
/* Many right-hand sides at once on the same hierarchy (the batching form):
 * B and X row-major n x nrhs (x_i of right-hand side v at X[i*nrhs + v]),
 * 1 <= nrhs <= 32; X holds the initial guesses and receives the solutions.
 * Refinement in fp64 (R = B - A X with fp64 values; X += D) around a
 * correction A D = R solved by PCG in lockstep over the columns, each with
 * its own scalars and its own stop (inner_tol * ||R_v||), preconditioned by
 * one V(1,1) cycle whose every operator is one amgt_spmm_rm over all
 * columns at its level's precision (reduced-precision levels on the tensor
 * cores; level 0 inside the correction at inner_prec0).  Each correction is
 * one CUDA graph launch.  Stops when every column reaches tol, or after
 * max_iter correction iterations in total, or max_outer refinements.
 * iterations[v]: correction iterations column v took; rel_res[v]: its
 * final ||B_v - A X_v|| / ||B_v|| in fp64 (both arrays may be NULL). */
AMGT_API int amgt_amg_solve_multi(amgt_amg *amg, int nrhs, const double *B, double *X, int *iterations,
                                  double *rel_res, amgt_stream_t stream);
/* A batch of independent systems of uneven size solved at once (the
 * batching form; no reference counterpart: HYPRE solves one system per
 * call).  A[s] (square, device CSR) and its interpolations P[s][0 ..
 * nlev[s] - 1], given flattened system after system in P, are concatenated
 * block-diagonally level by level (a system with fewer levels continues
 * with identity blocks, which leave its coarse operator unchanged), and
 * one hierarchy is set up for the concatenation (as amgt_amg_setup, with
 * its params).  Systems are rows offsets[s] .. offsets[s + 1] - 1 of the
 * concatenated vectors (amgt_batch_offsets). */
AMGT_API int amgt_batch_setup(int nsys, const amgt_csr *A, const int *nlev, const amgt_csr *P,
                              const amgt_amg_params *params, amgt_amg **out, amgt_stream_t stream);
/* One PCG per system in lockstep (each its own scalars; a system stops at
 * ||b_s - A_s x_s|| / ||b_s|| <= tol), preconditioned by one V(1,1) cycle
 * of the block-diagonal hierarchy, the whole iteration loop one CUDA graph
 * launch.  b, x: concatenated device vectors (x: initial guess in, solution
 * out).  iterations[s], rel_res[s] (fp64 residual of the returned x_s):
 * arrays of nsys, or NULL; *batch_iterations: the loop's iterations. */
AMGT_API int amgt_amg_solve_batch(amgt_amg *amg, const double *b, double *x, int *iterations, double *rel_res,
                                  int *batch_iterations, amgt_stream_t stream);
/* offsets[0 .. nsys] (cap entries at most); returns nsys, or -1 when amg
 * was not built by amgt_batch_setup. */
AMGT_API int amgt_batch_offsets(const amgt_amg *amg, int *offsets, int cap);
AMGT_API int amgt_amg_num_levels(const amgt_amg *amg);
/* Borrowed view of level `level`'s operator and its cycle precision. */
AMGT_API int amgt_amg_level(const amgt_amg *amg, int level, amgt_bsr *A_view, int *prec);
/* ms[0..3], stream time between phase ends: conversion of A, waits for the
 * interpolation operators (converted and transposed on a second stream,
 * overlapping the other phases), Galerkin SpGEMMs, smoother data + exact
 * and reduced-precision shadows + coarse inverse + vectors. */
AMGT_API int amgt_amg_setup_times(const amgt_amg *amg, double *ms);
/* Relative residual per iteration (entry 0 = initial); returns the count.
 * FGMRES-IR: the inner solves' residual estimates relative to ||b||, and at
 * each refinement step the fp64 residual. */
AMGT_API int amgt_amg_residual_history(const amgt_amg *amg, double *hist, int cap);
AMGT_API int amgt_amg_destroy(amgt_amg *amg, amgt_stream_t stream);

/* --------------------------------------- BoomerAMG coarsening (host) */
/* One level of BoomerAMG's coarsening and interpolation with the settings
 * the headline configurations name: HMIS (Ruge-Stueben first pass, then
 * PMIS; hypre_BoomerAMGCoarsenHMIS, R/parcsr_ls/par_coarsen.c:2845),
 * classical strength with threshold theta and max_row_sum
 * (hypre_BoomerAMGCreateS, par_strength.c), extended+i interpolation
 * (hypre_BoomerAMGBuildExtPIInterp, par_lr_interp.c:1025) truncated to p_max
 * entries per row with rescaling (hypre_ParCSRMatrixTruncate), one process.
 * Host code, as HYPRE 2.31's HMIS is.  No reference counterpart inside the
 * AmgT path: this is the caller's side of the SpGEMM hook (what produces
 * the P of the Galerkin products). */
typedef struct {
    double theta;        /* strength threshold (default 0.25)               */
    double max_row_sum;  /* rows with |sum| > max_row_sum |a_ii|: all weak;
                            1.0 turns the test off (default 1.0, the ij
                            driver's value, R/test/ij.c:290)               */
    int p_max;           /* interpolation entries per row (default 4, the ij
                            driver's, R/test/ij.c:244; 0: all)             */
    int coarsen_type;    /* 10: HMIS (default, the ij driver's,
                            R/test/ij.c:247); 8: PMIS (BoomerAMG's GPU
                            default, R/parcsr_ls/par_amg.c:304-316)        */
} amgt_boomer_params;
AMGT_API void amgt_boomer_default_params(amgt_boomer_params *p);
/* Host CSR in (rows with the diagonal first, as HYPRE stores them); P out in
 * HOST memory from malloc (free with amgt_boomer_free_host); cf_marker (host,
 * n, may be NULL): 1 for C points, -1 for F points. */
AMGT_API int amgt_boomer_coarsen_host(int n, const int *ia, const int *ja, const double *a,
                                      const amgt_boomer_params *prm, int *cf_marker, amgt_csr *P);
AMGT_API int amgt_boomer_free_host(amgt_csr *P);
/* The same for a device mBSR operator (copied to the host with its rows
 * reordered diagonal first); P in DEVICE memory from the allocator (free
 * with amgt_csr_free).  Blocks the host.  Usable as the coarsening of
 * amgt_amg_setup_adaptive. */
AMGT_API int amgt_boomer_interp(const amgt_bsr *A, const amgt_boomer_params *prm, amgt_csr *P, int *cf_marker,
                                amgt_stream_t stream);
/* The whole hierarchy on the host as HYPRE's CPU BoomerAMG builds it on one
 * process (hypre_BoomerAMGSetup, R/parcsr_ls/par_amg_setup.c): each level
 * as amgt_boomer_coarsen_host, then A_{l+1} = P^T (A_l P) in the order and
 * arithmetic of hypre_ParCSRMatrixRAPKTHost (R/parcsr_mv/
 * par_csr_triplemat.c:877-880; hypre_CSRMatrixMultiplyHost, R/seq_mv/
 * csr_matop.c:665), so the next level sees HYPRE's column order and its
 * truncation breaks ties as HYPRE's does.  A (host, n rows, each row's
 * diagonal first: HYPRE's storage).  Stops at a level of at most max_coarse
 * rows (HYPRE's default 9), at max_levels levels (default 25), or when a
 * level does not coarsen.  AMGT_ERR_UNSUPPORTED where HYPRE would switch to
 * CLJP coarsening (a coarse level of at least 3/4 of its fine level,
 * par_amg_setup.c:3166). */
typedef struct amgt_boomer_hier amgt_boomer_hier;
AMGT_API int amgt_boomer_hierarchy_host(int n, const int *ia, const int *ja, const double *a,
                                        const amgt_boomer_params *prm, int max_levels, int max_coarse,
                                        amgt_boomer_hier **out);
AMGT_API int amgt_boomer_hierarchy_levels(const amgt_boomer_hier *h);
/* Host views owned by h of level l's operator A_l (l < levels) and
 * interpolation P_l (l < levels - 1; zeroed on the coarsest level); either
 * output may be NULL. */
AMGT_API int amgt_boomer_hierarchy_level(const amgt_boomer_hier *h, int l, amgt_csr *A, amgt_csr *P);
AMGT_API void amgt_boomer_hierarchy_free(amgt_boomer_hier *h);

/* --------------------------------- learned precision / theta policy */
/* No reference counterpart: AmgT's precision per level is a fixed table
 * (get_calculationPrecison, R/seq_mv/csr_spgemm_device.c:1847-1862) and
 * BoomerAMG's strength threshold a fixed parameter
 * (HYPRE_BoomerAMGSetStrongThreshold).  These are the pieces of a policy
 * that picks both per level from cheap features of the level's operator. */
#define AMGT_MLP_IN 16
#define AMGT_MLP_HIDDEN 64
#define AMGT_MLP_OUT 4
#define AMGT_MLP_NPARAM 5508 /* W1 64x16, b1 64, W2 64x64, b2 64, W3 4x64, b3 4 */

/* 16 features of level `level`'s operator A (fp64 values), on an nx x ny x
 * nz grid dims[0..2] (the grid decodes a column offset into grid axes):
 * log10 rows, CSR nonzeros per row / 10, block fill, mean and minimum
 * diagonal dominance |a_ii| / sum_j!=i |a_ij| (capped at 10), mean and
 * spread of row sum / |a_ii|, share of positive off-diagonals, the shares
 * of coupling |a_ij| / |a_ii| along x, y, z and across axes, mean largest
 * off-diagonal / |a_ii|, level / 10, 3D flag, 1.  out: 16 host floats.
 * One host read-back. */
AMGT_API int amgt_level_features(const amgt_bsr *A, int level, const int *dims, float *out, amgt_stream_t stream);

/* Linear interpolation between vertex-centred structured grids along the
 * axes with coarsen[d] != 0 (coarse point j on fine point 2j), identity
 * along the others: P (device CSR from the allocator, free with
 * amgt_csr_free), cdims = the coarse grid.  One host read-back. */
AMGT_API int amgt_structured_interp(const int *dims, const int *coarsen, amgt_csr *P, int *cdims,
                                    amgt_stream_t stream);

/* Test and training problem (the learned policy's matrices): rotated
 * anisotropic diffusion -div(K grad u) on dims[0] x dims[1] x dims[2],
 * K = R(angle) diag(1, eps) R^T in the x-y plane and 1 along z, Dirichlet
 * boundary, unit spacing; 9-point x-y stencil (the mixed derivative by
 * central differences) plus the z neighbours.  Rows: diagonal first, then
 * ascending columns, as HYPRE's generators store them.  A: device CSR from
 * the allocator (free with amgt_csr_free).  One host read-back. */
AMGT_API int amgt_aniso_problem(const int *dims, double eps, double angle, amgt_csr *A, amgt_stream_t stream);

/* The 16 -> 64 -> 64 -> 4 MLP (fp32, ReLU; params: AMGT_MLP_NPARAM device
 * floats).  Output 0: logit of theta; 1 .. 3: logits of the level's
 * precision (fp64, fp32, fp16).  X: n x 16, out: n x 4 (device).
 * amgt_mlp_grad: the mean over the n samples of the gradient of
 * (sigmoid(o0) - T[2i])^2 + cross-entropy(softmax(o1..o3), class T[2i+1])
 * into grad (AMGT_MLP_NPARAM device floats) and the mean loss into *loss
 * (device, may be NULL).  amgt_mlp_train: Adam (beta 0.9, 0.999) over
 * `epochs` passes of seeded shuffles in minibatches of `batch`, params
 * updated in place; loss_hist (host, may be NULL): mean loss of each
 * epoch's last minibatch. */
AMGT_API int amgt_mlp_forward(const float *params, int n, const float *X, float *out, amgt_stream_t stream);
AMGT_API int amgt_mlp_grad(const float *params, int n, const float *X, const float *T, float *grad, float *loss,
                           amgt_stream_t stream);
AMGT_API int amgt_mlp_train(float *params, int n, const float *X, const float *T, int epochs, int batch, float lr,
                            unsigned seed, float *loss_hist, amgt_stream_t stream);

/* ------------------------------------------ HYPRE-facing mirror layer */
/* The fields of hypre_CSRMatrix that the AmgT path reads and writes
 * (R/seq_mv/seq_mv.h:154-199): the CSR arrays, the AmgT level tag and the
 * lazily built mBSR cache.  bsr_mat_T caches A^T for trans = 1 (the
 * reference ignores trans). */
typedef struct {
    int coasen_level;            /* hypre_Level(A)            */
    char bsr_spmv_balanced_tag;  /* hypre_BSRBALANCEDTAG(A)   */
    char bsr_tag;                /* hypre_BSRTAG(A)           */
    char mixed_precision_flag;   /* hypre_MixedPrecisionTag(A)*/
    char owns_data;              /* CSR arrays freed by Destroy */
    amgt_bsr *bsr_mat;           /* hypre_BSR(A)              */
    amgt_bsr *bsr_mat_T;         /* cached transpose (trans = 1) */
    amgt_csr csr;                /* i / j / data / sizes      */
} amgt_CSRMatrix;

/* Wraps caller-owned device CSR arrays (owns_data = 0). */
AMGT_API amgt_CSRMatrix *amgt_CSRMatrixCreate(int num_rows, int num_cols,
                                     int num_nonzeros, int *i, int *j,
                                     double *data, int level);
/* Frees the mBSR caches, and the CSR arrays when owns_data is set. */
AMGT_API int amgt_CSRMatrixDestroy(amgt_CSRMatrix *A);

/* Stream used by the mirror layer (HYPRE's hypre_HandleComputeStream). */
AMGT_API int amgt_set_stream(amgt_stream_t stream);

/* hypreDevice_CSRSpGemm (R/seq_mv/csr_spgemm_device.c:2579-2608): converts
 * A and B to mBSR on first use (cached), picks the precision from
 * hypre_Level(A) through amgt_precision_for_level, multiplies, and returns a
 * new matrix that owns its CSR arrays (from the allocator), carries C's mBSR
 * with bsr_tag = 1, and has C's level = A's level. */
AMGT_API int amgt_CSRSpGemm(amgt_CSRMatrix *A, amgt_CSRMatrix *B, amgt_CSRMatrix **C_ptr);

/* hypre_CSRMatrixMatvecCusparseNewAPI
 * (R/seq_mv/csr_matvec_device.c:2397-2437): y[offset:] = alpha * op(A) * x
 * + beta * y[offset:], op(A) = A^T when trans != 0 (built once and cached).
 * offset must be 0 (asserted by the caller in HYPRE, :142).  Multivectors
 * (num_vectors > 1) go through amgt_spmm.  Precision from hypre_Level(A). */
AMGT_API int amgt_CSRMatrixMatvec(int trans, double alpha, amgt_CSRMatrix *A,
                         const amgt_vector *x, double beta, amgt_vector *y,
                         int offset);

#ifdef __cplusplus
}
#endif

#endif /* AMGT_B200_H */
