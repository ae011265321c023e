// Multi-right-hand-side mBSR SpMM with row-major multivectors:
//   Y (m x nvec) <- alpha * A * X (n x nvec) + beta * Y,  nvec <= 32,
// X[i * nvec + v], Y[i * nvec + v], fp64 in memory.  The batching form's
// operator: one pass over A's values for all right-hand sides (the
// reference's hook ignores num_vectors, AmgT_HYPRE/src/seq_mv/
// csr_matvec_device.c:2409-2437; its tensor-core SpMV is bsr_spmv_tc_fp64,
// :452-507).
//
// Tensor-core form (values in fp32 / fp16 / bf16): one warp takes two block
// rows b1, b2 at a time and walks their blocks in step (block t of each
// row); per step one mma.m16n8k8 (tf32 in, fp32 accumulate) per 16
// right-hand sides computes
//   D (16 rhs x 8 outputs) += Xg (16 rhs x 8) * Bop (8 x 8)
// with K = [the 4 columns of b1's block t | the 4 columns of b2's block t]
// and N = [b1's 4 rows | b2's 4 rows]: Bop = [A1^T 0; 0 A2^T] (block
// diagonal), Xg the gathered rows of X.  Half of Bop is zero, and in
// exchange every lane loads exactly one value per step (lane l < 16: entry
// l of b1's block, l >= 16: entry l - 16 of b2's block, which is the
// mma's B fragment element for that lane) and no shuffle is needed.  fp32
// accuracy on the tf32 units: values and x are split as v = hi + lo
// (hi = tf32(v), lo = tf32(v - hi)) and D accumulates hi*hi + lo*hi + hi*lo
// (fp16 / bf16 values are exact in tf32: two products).  The op stays
// bandwidth-bound, so the extra mma work is free.
//
// CUDA-core forms (any precision, fp64 for fp64 values): one warp per block
// row, lane = right-hand side; block values are read once per warp and
// broadcast by shuffles; x rows are coalesced across lanes.
//
// Deterministic: every output sums its blocks in stored order.
#include "spmv_common.cuh"

namespace amgt {

__device__ __forceinline__ uint32_t to_tf32(float f)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(f));
    return r;
}

__device__ __forceinline__ void mma_tf32(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int PREC>
__device__ __forceinline__ float load_val1(const void *__restrict__ val, long long i)
{
    if constexpr (PREC == AMGT_FLOAT) return __ldcs(static_cast<const float *>(val) + i);
    else if constexpr (PREC == AMGT_HALF)
        return __half2float(__ushort_as_half(__ldcs(static_cast<const unsigned short *>(val) + i)));
    else return __bfloat162float(__ushort_as_bfloat16(__ldcs(static_cast<const unsigned short *>(val) + i)));
}

// NH halves of 16 right-hand sides (nvec <= 16 * NH); WPC warps per CTA.
template <int PREC, int NH, int WPC>
__global__ void __launch_bounds__(WPC * 32)
spmm_tc_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
               const void *__restrict__ val, double alpha, const double *__restrict__ X, int nvec, double beta,
               double *__restrict__ Y)
{
    grid_dependency_wait();
    constexpr bool kSplitA = PREC == AMGT_FLOAT;  // fp16 / bf16 values are exact in tf32
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int npairs = (brow + 1) >> 1;
    const bool upper = lane >= 16;  // this lane's block value comes from b2
    for (int p = warp; p < npairs; p += nwarps) {
        const int b1 = 2 * p, b2 = 2 * p + 1;
        const int s1 = ptr[b1], e1 = ptr[b1 + 1];
        const int s2 = b2 < brow ? ptr[b2] : 0, e2 = b2 < brow ? ptr[b2 + 1] : 0;
        const int len = max(e1 - s1, e2 - s2);
        const int ms = upper ? s2 : s1, me = upper ? e2 : e1;
        float acc[NH][4];
#pragma unroll
        for (int h = 0; h < NH; ++h)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[h][q] = 0.0f;
        for (int t = 0; t < len; ++t) {
            const int kb = ms + t;
            const bool mine = kb < me;
            const float a = mine ? load_val1<PREC>(val, 16LL * kb + (lane & 15)) : 0.0f;
            const int cm = mine ? __ldcs(idx + kb) : -1;
            const int c1 = __shfl_sync(FULL, cm, 0), c2 = __shfl_sync(FULL, cm, 16);
            const uint32_t ahi = to_tf32(a);
            const uint32_t b0h = upper ? 0u : ahi, b1h = upper ? ahi : 0u;
            uint32_t b0l = 0u, b1l = 0u;
            if constexpr (kSplitA) {
                const uint32_t alo = to_tf32(a - __uint_as_float(ahi));
                b0l = upper ? 0u : alo;
                b1l = upper ? alo : 0u;
            }
            const long long r1 = 4LL * c1 + tig, r2 = 4LL * c2 + tig;
            const bool ok1 = c1 >= 0 && r1 < n, ok2 = c2 >= 0 && r2 < n;
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int v0 = 16 * h + gid, v1 = v0 + 8;
                double xv[4];
                xv[0] = (ok1 && v0 < nvec) ? X[r1 * nvec + v0] : 0.0;
                xv[1] = (ok1 && v1 < nvec) ? X[r1 * nvec + v1] : 0.0;
                xv[2] = (ok2 && v0 < nvec) ? X[r2 * nvec + v0] : 0.0;
                xv[3] = (ok2 && v1 < nvec) ? X[r2 * nvec + v1] : 0.0;
                uint32_t xh[4], xl[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float f = (float)xv[q];
                    xh[q] = to_tf32(f);
                    xl[q] = to_tf32((float)(xv[q] - (double)__uint_as_float(xh[q])));
                }
                mma_tf32(acc[h], xh, b0h, b1h);
                mma_tf32(acc[h], xl, b0h, b1h);
                if constexpr (kSplitA) mma_tf32(acc[h], xh, b0l, b1l);
            }
        }
        // D fragment: (rhs gid, output 2 tig), (gid, 2 tig + 1), (gid + 8, 2 tig), (gid + 8, 2 tig + 1)
#pragma unroll
        for (int h = 0; h < NH; ++h)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int v = 16 * h + gid + ((q & 2) ? 8 : 0);
                const int o = 2 * tig + (q & 1);
                const int b = o < 4 ? b1 : b2;
                const int row = 4 * b + (o & 3);
                if (b < brow && row < m && v < nvec) {
                    double *yy = Y + (long long)row * nvec + v;
                    const double r = alpha * (double)acc[h][q];
                    *yy = (beta == 0.0) ? r : r + beta * *yy;
                }
            }
    }
}

// CUDA-core form: warp per block row, lane = right-hand side.
template <int PREC, int WPC>
__global__ void __launch_bounds__(WPC * 32)
spmm_cc_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
               const void *__restrict__ val, double alpha, const double *__restrict__ X, int nvec, double beta,
               double *__restrict__ Y)
{
    grid_dependency_wait();
    using acc_t = typename ValTraits<PREC>::acc_t;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool live = lane < nvec;
    for (int b = warp; b < brow; b += nwarps) {
        acc_t acc[4] = {0, 0, 0, 0};
        const int e = ptr[b + 1];
        for (int k = ptr[b]; k < e; ++k) {
            const int c = __ldcs(idx + k);
            acc_t vq;
            if constexpr (PREC == AMGT_DOUBLE) vq = __ldcs(static_cast<const double *>(val) + 16LL * k + (lane & 15));
            else vq = load_val1<PREC>(val, 16LL * k + (lane & 15));
            acc_t xk[4];
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const long long r = 4LL * c + cc;
                xk[cc] = (live && r < n) ? (acc_t)X[r * nvec + lane] : (acc_t)0;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) acc[r] = fma(__shfl_sync(FULL, vq, 4 * r + cc), xk[cc], acc[r]);
        }
        if (live)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = 4 * b + r;
                if (row < m) {
                    double *yy = Y + (long long)row * nvec + lane;
                    const double t = alpha * (double)acc[r];
                    *yy = (beta == 0.0) ? t : t + beta * *yy;
                }
            }
    }
}

// ---------------------------------------------------------------- launch
// kind: 0 CUDA cores, 1 tensor cores; wpc: warps per CTA (4 or 8).
template <int PREC, int WPC>
static int launch_rm(int kind, const amgt_bsr *A, const void *val, double alpha, const double *X, int nvec,
                     double beta, double *Y, cudaStream_t s, int sm_count)
{
    const int brow = A->blc_row;
    if (kind == 1) {
        if constexpr (PREC == AMGT_DOUBLE) {
            return AMGT_ERR_UNSUPPORTED;
        } else {
            const int grid = grid_for(WPC, (brow + 1) / 2, sm_count, 16);
            if (nvec <= 16)
                AMGT_LAUNCH_PDL((spmm_tc_kernel<PREC, 1, WPC>), grid, WPC * 32, 0, s, A->row, A->col, brow, A->blcPtr,
                                A->blcIdx, val, alpha, X, nvec, beta, Y);
            else
                AMGT_LAUNCH_PDL((spmm_tc_kernel<PREC, 2, WPC>), grid, WPC * 32, 0, s, A->row, A->col, brow, A->blcPtr,
                                A->blcIdx, val, alpha, X, nvec, beta, Y);
            return AMGT_OK;
        }
    }
    const int grid = grid_for(WPC, brow, sm_count, 16);
    AMGT_LAUNCH_PDL((spmm_cc_kernel<PREC, WPC>), grid, WPC * 32, 0, s, A->row, A->col, brow, A->blcPtr, A->blcIdx,
                    val, alpha, X, nvec, beta, Y);
    return AMGT_OK;
}

template <int PREC>
static int launch_rm_prec(int kind, int wpc, const amgt_bsr *A, const void *val, double alpha, const double *X,
                          int nvec, double beta, double *Y, cudaStream_t s, int sm_count)
{
    return wpc == 8 ? launch_rm<PREC, 8>(kind, A, val, alpha, X, nvec, beta, Y, s, sm_count)
                    : launch_rm<PREC, 4>(kind, A, val, alpha, X, nvec, beta, Y, s, sm_count);
}

static const void *rm_values(const amgt_bsr *A, int prec)
{
    switch (prec) {
    case AMGT_DOUBLE: return A->blcVal;
    case AMGT_FLOAT: return A->blcVal_fp32;
    case AMGT_HALF: return A->blcVal_fp16;
    case AMGT_BF16: return A->blcVal_bf16;
    default: return nullptr;
    }
}

// The storage read for `prec`: fp32 requests read an exact fp16 shadow
// (same inputs, half the bytes); fp64 keeps 8-byte values here.
static int rm_storage(const amgt_bsr *A, int prec)
{
    if (prec == AMGT_FLOAT && A->exact_prec == AMGT_HALF && A->blcVal_fp16) return AMGT_HALF;
    return prec;
}

int spmm_rowmajor(int prec, int kind, int wpc, const amgt_bsr *A, double alpha, const double *X, int nvec,
                  double beta, double *Y, cudaStream_t s, int sm_count)
{
    const int mode = rm_storage(A, prec);
    const void *val = rm_values(A, mode);
    if (!val) return AMGT_ERR_INVALID;
    if (mode == AMGT_DOUBLE && kind == 1) kind = 0;  // fp64 values: CUDA cores
    switch (mode) {
    case AMGT_DOUBLE: return launch_rm_prec<AMGT_DOUBLE>(kind, wpc, A, val, alpha, X, nvec, beta, Y, s, sm_count);
    case AMGT_FLOAT: return launch_rm_prec<AMGT_FLOAT>(kind, wpc, A, val, alpha, X, nvec, beta, Y, s, sm_count);
    case AMGT_HALF: return launch_rm_prec<AMGT_HALF>(kind, wpc, A, val, alpha, X, nvec, beta, Y, s, sm_count);
    default: return launch_rm_prec<AMGT_BF16>(kind, wpc, A, val, alpha, X, nvec, beta, Y, s, sm_count);
    }
}

}  // namespace amgt
