// mBSR SpMV / SpMM: y <- alpha * A * x + beta * y.
//
// Replaces spmv_amgT_fp64 / _fp32 / _fp16 and the bsr_spmv_* kernels
// (AmgT_HYPRE/src/seq_mv/csr_matvec_device.c:319-613, 1302-1542,
// 1654-2309).  The reference puts two 4x4 blocks in one m8n8k4 fp64 MMA and
// keeps the diagonal of the 8x8 result (1/8 of the MMA work is useful);
// SpMV is bound by HBM bytes, so here the tensor cores are not used at all
// and the kernel is shaped for bandwidth instead:
//   - 4 lanes per block, lane q owns block row q: its 4 values are 32
//     contiguous bytes (two 16-byte loads for fp64, one for fp32, one
//     8-byte load for fp16/bf16), so a warp streams whole 128-byte blocks;
//   - LPR lanes per block row (4, 8, 16 or 32) so that short rows do not
//     leave lanes idle; the LPR/4 groups of a row take every (LPR/4)-th
//     block and are combined with shuffles (fixed order: deterministic);
//   - values and block columns are read with evict-first hints so that x
//     stays in L2;
//   - beta * y is fused (no separate beta pass), beta == 0 does not read y;
//   - reduced precisions read the value shadow, convert x in registers and
//     accumulate in fp32; the result is combined with beta * y in fp64.
// Very long rows (longest row > 256 blocks and a segment table present) are
// cut into <= 64-block segments; partial sums go to scratch and a second
// kernel adds them in segment order (the reference uses fp64 atomicAdd,
// :593, which is not deterministic).
#include <cstdlib>

#include "spmv_common.cuh"

namespace amgt {

template <int PREC, bool SAFE>
__device__ __forceinline__ typename ValTraits<PREC>::acc_t block_row_dot(const void *__restrict__ val,
                                                                         const double *__restrict__ x, int n,
                                                                         long long k, int q, int col,
                                                                         typename ValTraits<PREC>::acc_t acc)
{
    using acc_t = typename ValTraits<PREC>::acc_t;
    acc_t v[4];
    double xv[4];
    load_block_row<PREC>(val, k, q, v);
    load_x4<SAFE>(x, col, n, xv);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc = fma(v[c], (acc_t)xv[c], acc);
    return acc;
}

// A lane group's blocks k, k + G, k + 2G, ... of one block row, two per
// step so that both loads are in flight before the FMAs; products are
// added in block order.  (Four per step measured slower here: the 128^3
// SpMV 77.7 -> 85.7 us, the interpolation 47.6 -> 77.7 us.)
template <int PREC, int G, bool SAFE>
__device__ __forceinline__ typename ValTraits<PREC>::acc_t row_dot(const void *__restrict__ val,
                                                                   const int *__restrict__ idx,
                                                                   const double *__restrict__ x, int n, int k,
                                                                   int end, int q, typename ValTraits<PREC>::acc_t acc)
{
    for (; k + G < end; k += 2 * G) {
        const int c0 = __ldcs(idx + k), c1 = __ldcs(idx + k + G);
        acc = block_row_dot<PREC, SAFE>(val, x, n, k, q, c0, acc);
        acc = block_row_dot<PREC, SAFE>(val, x, n, k + G, q, c1, acc);
    }
    if (k < end) acc = block_row_dot<PREC, SAFE>(val, x, n, k, q, __ldcs(idx + k), acc);
    return acc;
}

// The same walk with the blocks dealt alternately to two sums (a lane group
// standing for two of the row's segments: blocks k, k + 2G, ... and
// k + G, k + 3G, ...), with the loads and the order of each sum unchanged;
// four blocks per step (the level-0 passes over the exact fp16 shadow,
// 44 -> 40.5 us at 128^3).
template <int PREC, int G, bool SAFE>
__device__ __forceinline__ void row_dot2(const void *__restrict__ val, const int *__restrict__ idx,
                                         const double *__restrict__ x, int n, int k, int end, int q,
                                         typename ValTraits<PREC>::acc_t &a0, typename ValTraits<PREC>::acc_t &a1)
{
    for (; k + 3 * G < end; k += 4 * G) {
        const int c0 = __ldcs(idx + k), c1 = __ldcs(idx + k + G), c2 = __ldcs(idx + k + 2 * G),
                  c3 = __ldcs(idx + k + 3 * G);
        a0 = block_row_dot<PREC, SAFE>(val, x, n, k, q, c0, a0);
        a1 = block_row_dot<PREC, SAFE>(val, x, n, k + G, q, c1, a1);
        a0 = block_row_dot<PREC, SAFE>(val, x, n, k + 2 * G, q, c2, a0);
        a1 = block_row_dot<PREC, SAFE>(val, x, n, k + 3 * G, q, c3, a1);
    }
    for (; k + G < end; k += 2 * G) {
        const int c0 = __ldcs(idx + k), c1 = __ldcs(idx + k + G);
        a0 = block_row_dot<PREC, SAFE>(val, x, n, k, q, c0, a0);
        a1 = block_row_dot<PREC, SAFE>(val, x, n, k + G, q, c1, a1);
    }
    if (k < end) a0 = block_row_dot<PREC, SAFE>(val, x, n, k, q, __ldcs(idx + k), a0);
}

// Row sum of a block row: V == 1, LPR lanes per row as the row's segments;
// V == 2, LPR lanes stand for the 2 LPR-lane layout (each lane group holds
// segments g and g + LPR/4 of it): the segment sums are combined in that
// layout's order (first across groups, then the two halves), so both give
// the same bits.  Lanes with g == 0 hold the result.
template <int PREC, int LPR, bool SAFE, int V>
__device__ __forceinline__ typename ValTraits<PREC>::acc_t row_sum(const void *__restrict__ val,
                                                                   const int *__restrict__ idx,
                                                                   const double *__restrict__ x, int n, bool live,
                                                                   int k, int end, int q)
{
    using acc_t = typename ValTraits<PREC>::acc_t;
    constexpr int G = LPR / 4;
    if constexpr (V == 1) {
        acc_t acc = 0;
        if (live) acc = row_dot<PREC, G, SAFE>(val, idx, x, n, k, end, q, acc);
#pragma unroll
        for (int o = 4; o < LPR; o <<= 1) acc += __shfl_xor_sync(FULL, acc, o);
        return acc;
    } else {
        acc_t a0 = 0, a1 = 0;
        if (live) row_dot2<PREC, G, SAFE>(val, idx, x, n, k, end, q, a0, a1);
#pragma unroll
        for (int o = 4; o < LPR; o <<= 1) {
            a0 += __shfl_xor_sync(FULL, a0, o);
            a1 += __shfl_xor_sync(FULL, a1, o);
        }
        return a0 + a1;
    }
}

template <int PREC, int LPR, bool SAFE, int V = 1>
__global__ void __launch_bounds__(256)
spmv_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
            const void *__restrict__ val, double alpha, const double *__restrict__ x, double beta,
            double *__restrict__ y)
{
    grid_dependency_wait();
    using acc_t = typename ValTraits<PREC>::acc_t;
    constexpr int RPW = 32 / LPR;  // block rows per warp
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPR, l = lane % LPR, g = l >> 2, q = l & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int b0 = warp * RPW; b0 < brow; b0 += nwarps * RPW) {
        const int b = b0 + sub;
        const bool live = b < brow;
        const acc_t acc = row_sum<PREC, LPR, SAFE, V>(val, idx, x, n, live, live ? ptr[b] + g : 0,
                                                      live ? ptr[b + 1] : 0, q);
        if (live && g == 0) {
            const int row = 4 * b + q;
            if (row < m) {
                const double t = alpha * (double)acc;
                y[row] = (beta == 0.0) ? t : t + beta * y[row];
            }
        }
    }
}

// Long rows: one warp per <= 64-block segment, partial row sums to scratch.
template <int PREC, bool SAFE>
__global__ void __launch_bounds__(256)
spmv_segment_kernel(int n, int nseg, const int *__restrict__ segrow, const int *__restrict__ segptr,
                    const int *__restrict__ ptr, const int *__restrict__ idx, const void *__restrict__ val,
                    const double *__restrict__ x, double *__restrict__ part)
{
    using acc_t = typename ValTraits<PREC>::acc_t;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int sgi = warp; sgi < nseg; sgi += nwarps) {
        const int b = segrow[sgi];
        const int j = sgi - segptr[b];
        const int start = ptr[b] + 64 * j, end = min(ptr[b + 1], start + 64);
        acc_t acc = 0;
        for (int k = start + g; k < end; k += 8) acc = block_row_dot<PREC, SAFE>(val, x, n, k, q, __ldcs(idx + k), acc);
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) acc += __shfl_xor_sync(FULL, acc, o);
        if (g == 0) part[4LL * sgi + q] = (double)acc;
    }
}

__global__ void spmv_segment_combine(int m, int brow, const int *__restrict__ segptr,
                                     const double *__restrict__ part, double alpha, double beta,
                                     double *__restrict__ y, int lowp)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        const int b = row >> 2, q = row & 3;
        double t = 0.0;
        float tf = 0.0f;
        for (int sgi = segptr[b]; sgi < segptr[b + 1]; ++sgi) {
            if (lowp) tf += (float)part[4LL * sgi + q];
            else t += part[4LL * sgi + q];
        }
        if (lowp) t = (double)tf;
        const double r = alpha * t;
        y[row] = (beta == 0.0) ? r : r + beta * y[row];
    }
}

// SpMM: NV vectors per pass, the block row values loaded once for all.
template <int PREC, int LPR, int NV>
__global__ void __launch_bounds__(256)
spmm_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
            const void *__restrict__ val, double alpha, const double *__restrict__ x, int ldx, double beta,
            double *__restrict__ y, int ldy)
{
    using acc_t = typename ValTraits<PREC>::acc_t;
    constexpr int RPW = 32 / LPR;
    constexpr int G = LPR / 4;
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPR, l = lane % LPR, g = l >> 2, q = l & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int b0 = warp * RPW; b0 < brow; b0 += nwarps * RPW) {
        const int b = b0 + sub;
        acc_t acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = 0;
        if (b < brow) {
            for (int k = ptr[b] + g; k < ptr[b + 1]; k += G) {
                const int col = __ldcs(idx + k);
                acc_t a[4];
                load_block_row<PREC>(val, k, q, a);
#pragma unroll
                for (int v = 0; v < NV; ++v)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const long long j = 4LL * col + c;
                        const double xv = (j < n) ? __ldg(x + (long long)v * ldx + j) : 0.0;
                        acc[v] = fma(a[c], (acc_t)xv, acc[v]);
                    }
            }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int o = 4; o < LPR; o <<= 1) acc[v] += __shfl_xor_sync(FULL, acc[v], o);
        if (b < brow && g == 0) {
            const int row = 4 * b + q;
            if (row < m) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    double *yy = y + (long long)v * ldy + row;
                    const double t = alpha * (double)acc[v];
                    *yy = (beta == 0.0) ? t : t + beta * *yy;
                }
            }
        }
    }
}

// SpMV with a fused row epilogue (the smoother / residual / Krylov forms).
//   EPI_RESID : out = f - A u                          (residual, par_cycle.c:678)
//   EPI_JACOBI: out = u + w (f - A u) / l1             (Relax 18, par_relax.c:1178-1260)
//   EPI_DOT   : out = A u, and dot partials of u . out (PCG's p.q), one per CTA
//   EPI_RESTRICT_JACOBI0: out = A u (a restriction) and out2 = w out ./ l1
//               (the coarser level's l1-Jacobi sweep from a zero guess)
// x is u.  Same load pattern and per-row summation order as spmv_kernel.
enum { EPI_RESID = 0, EPI_JACOBI = 1, EPI_DOT = 2, EPI_RESTRICT_JACOBI0 = 3 };

struct EpiArgs {
    const double *f;       // RESID, JACOBI
    const double *inv_l1;  // JACOBI, RESTRICT_JACOBI0
    double w;              // JACOBI, RESTRICT_JACOBI0
    double *out;
    double *partial;       // DOT: [gridDim.x]
    double *out2;          // RESTRICT_JACOBI0
};

template <int PREC, int LPR, bool SAFE, int EPI, int V = 1>
__global__ void __launch_bounds__(256)
spmv_epi_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
                const void *__restrict__ val, const double *__restrict__ x, EpiArgs e)
{
    static_assert(V == 1 || EPI != EPI_DOT, "dot partials follow the one-segment-per-group layout");
    grid_dependency_wait();
    using acc_t = typename ValTraits<PREC>::acc_t;
    constexpr int RPW = 32 / LPR;
    __shared__ double sred[8];
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPR, l = lane % LPR, g = l >> 2, q = l & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double dot = 0.0;
    for (int b0 = warp * RPW; b0 < brow; b0 += nwarps * RPW) {
        const int b = b0 + sub;
        const bool live = b < brow;
        const acc_t acc = row_sum<PREC, LPR, SAFE, V>(val, idx, x, n, live, live ? ptr[b] + g : 0,
                                                      live ? ptr[b + 1] : 0, q);
        if (live && g == 0) {
            const int row = 4 * b + q;
            if (row < m) {
                const double ax = (double)acc;
                if constexpr (EPI == EPI_RESID) {
                    e.out[row] = e.f[row] - ax;
                } else if constexpr (EPI == EPI_JACOBI) {
                    e.out[row] = x[row] + e.w * (e.f[row] - ax) * e.inv_l1[row];
                } else if constexpr (EPI == EPI_RESTRICT_JACOBI0) {
                    e.out[row] = ax;
                    e.out2[row] = e.w * ax * e.inv_l1[row];
                } else {
                    e.out[row] = ax;
                    dot += x[row] * ax;
                }
            }
        }
    }
    if constexpr (EPI == EPI_DOT) {
        // fixed-order reduction: lanes, then warps (deterministic for a fixed grid)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(FULL, dot, o);
        if (lane == 0) sred[threadIdx.x >> 5] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sred[i];
            e.partial[blockIdx.x] = s;
        }
    }
}

// l1 row norms sum_j |a_ij| (hypre_ParCSRComputeL1Norms option 1,
// AmgT_HYPRE/src/parcsr_ls/ams.c:627-636), one thread per scalar row.
// PREC: the 8-byte values or an exact narrow shadow (same values, widened
// exactly: the same sums with fewer bytes read).
template <int PREC>
__global__ void l1_norm_kernel(int m, const int *__restrict__ ptr, const void *__restrict__ val,
                               double *__restrict__ l1, int invert)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        const int b = row >> 2, q = row & 3;
        double s = 0.0;
        for (int k = ptr[b]; k < ptr[b + 1]; ++k) {
            double v[4];
            load_block_row<PREC>(val, k, q, v);
            s += fabs(v[0]) + fabs(v[1]) + fabs(v[2]) + fabs(v[3]);
        }
        l1[row] = invert ? (s != 0.0 ? 1.0 / s : 0.0) : s;
    }
}

__global__ void scale_kernel(long long n, double beta, double *__restrict__ y)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (beta == 0.0) ? 0.0 : beta * y[i];
}

static const void *value_array(const amgt_bsr *A, int prec)
{
    switch (prec) {
    case AMGT_DOUBLE: return A->blcVal;
    case AMGT_FLOAT: return A->blcVal_fp32;
    case AMGT_HALF: return A->blcVal_fp16;
    case AMGT_BF16: return A->blcVal_bf16;
    case kExact32: return A->blcVal_fp32;
    case kExact16: return A->blcVal_fp16;
    default: return nullptr;
    }
}

// Storage a product reads: for fp64, the shadow that holds every value
// exactly when amgt_bsr_make_exact found one (same results, fewer bytes);
// for fp32, the fp16 shadow when it holds every value exactly (the same
// fp32 inputs and the same fp32 sums at half the bytes), so that a reduced
// precision never reads more value bytes than the fp64 form of the same
// operator.  bf16 keeps its own rounding.
static int storage_mode(const amgt_bsr *A, int prec)
{
    if (prec == AMGT_FLOAT && A->exact_prec == AMGT_HALF && A->blcVal_fp16) return AMGT_HALF;
    if (prec != AMGT_DOUBLE) return prec;
    if (A->exact_prec == AMGT_HALF && A->blcVal_fp16) return kExact16;
    if (A->exact_prec == AMGT_FLOAT && A->blcVal_fp32) return kExact32;
    return AMGT_DOUBLE;
}


// Lanes per block row: amgt_autotune's choice for this matrix when it has
// one, else from the mean block-row length (AMGT_SPMV_LPR overrides both).
static int pick_lpr(const amgt_bsr *A, int mode)
{
    // the choice depends on the structure only: with the same segment length
    // the exact narrow storage sums a row in the fp64 order, bit for bit
    (void)mode;
    static int env = -1;
    if (env < 0) {
        const char *e = getenv("AMGT_SPMV_LPR");
        env = e ? atoi(e) : 0;
    }
    if (env == 4 || env == 8 || env == 16 || env == 32) return env;
    const int tuned = tuned_lpr(A);  // amgt_autotune's measured choice for this matrix
    if (tuned) return tuned;
    const double avg = A->blc_row ? (double)A->blc_num / A->blc_row : 0.0;
    if (avg <= 4.0) return 4;    // interpolation 128^3 (3.3): 4 beat 8 for 8- and 2-byte values
    if (avg <= 10.0) return 8;   // 7-point 128^3 (6.9): 8 beat 4 and 16 for 8-byte values
    if (avg <= 20.0) return 16;
    return 32;
}

// Lanes a row is given when it runs: 2-byte values move few bytes per
// lane, so with the 8-lane segment layout half the lanes (each group
// holding two of its segments, same sums) keep more rows in flight
// (7-point 128^3, fp16 exact: 43.7 -> 37.0 us; at 32 lanes the same split
// measured 22.4 -> 23.5 us and is not used).  The fused dot form keeps the
// segment layout (its partials follow it).
static int run_lpr(int lpr, int mode)
{
    const bool narrow = mode == AMGT_HALF || mode == AMGT_BF16 || mode == kExact16;
    return (narrow && lpr == 8) ? 4 : lpr;
}

template <int PREC>
static int launch_spmv(const amgt_bsr *A, const void *val, double alpha, const double *x, double beta, double *y,
                       cudaStream_t s, int sm_count)
{
    const int brow = A->blc_row;
    const bool safe = (A->col % 4 != 0) || ((uintptr_t)x % 16 != 0);
    const int lpr = pick_lpr(A, PREC), run = run_lpr(lpr, PREC);
    const int rows_per_cta = 8 * (32 / run);
    const int grid = grid_for(rows_per_cta, brow, sm_count, 8);
#define AMGT_SPMV_CASE(L, V)                                                                                \
    if (run == L && lpr == L * V) {                                                                         \
        if (safe)                                                                                           \
            AMGT_LAUNCH_PDL((spmv_kernel<PREC, L, true, V>), grid, 256, 0, s, A->row, A->col, brow,          \
                            A->blcPtr, A->blcIdx, val, alpha, x, beta, y);                                  \
        else                                                                                                \
            AMGT_LAUNCH_PDL((spmv_kernel<PREC, L, false, V>), grid, 256, 0, s, A->row, A->col, brow,         \
                            A->blcPtr, A->blcIdx, val, alpha, x, beta, y);                                  \
        return AMGT_OK;                                                                                     \
    }
    AMGT_SPMV_CASE(4, 1)
    AMGT_SPMV_CASE(8, 1)
    AMGT_SPMV_CASE(16, 1)
    AMGT_SPMV_CASE(32, 1)
    if constexpr (PREC == AMGT_HALF || PREC == AMGT_BF16 || PREC == kExact16) {
        AMGT_SPMV_CASE(4, 2)
    }
#undef AMGT_SPMV_CASE
    return AMGT_ERR_INVALID;
}

template <int PREC>
static int launch_spmv_segmented(const amgt_bsr *A, const void *val, double alpha, const double *x, double beta,
                                 double *y, cudaStream_t s, int sm_count)
{
    const bool safe = (A->col % 4 != 0) || ((uintptr_t)x % 16 != 0);
    double *part = nullptr;
    AMGT_TRY(alloc_n(&part, 4LL * A->warpnum, s));
    const int grid = grid_for(8, A->warpnum, sm_count, 8);
    if (safe)
        AMGT_LAUNCH((spmv_segment_kernel<PREC, true>), grid, 256, 0, s, A->col, A->warpnum, A->rowIdxbyWarp,
                    A->rowPtrbyWarp, A->blcPtr, A->blcIdx, val, x, part);
    else
        AMGT_LAUNCH((spmv_segment_kernel<PREC, false>), grid, 256, 0, s, A->col, A->warpnum, A->rowIdxbyWarp,
                    A->rowPtrbyWarp, A->blcPtr, A->blcIdx, val, x, part);
    AMGT_LAUNCH(spmv_segment_combine, grid_for(256, A->row, sm_count, 8), 256, 0, s, A->row, A->blc_row,
                A->rowPtrbyWarp, part, alpha, beta, y, PREC != AMGT_DOUBLE);
    free_ptr(part, s);
    return AMGT_OK;
}

template <int PREC, int LPR>
static int launch_spmm_lpr(const amgt_bsr *A, const void *val, double alpha, int nvec, const double *x, int ldx,
                           double beta, double *y, int ldy, cudaStream_t s, int grid)
{
    int v0 = 0;
    while (v0 < nvec) {
        const int left = nvec - v0;
        const double *xx = x + (long long)v0 * ldx;
        double *yy = y + (long long)v0 * ldy;
        if (left >= 8) {
            AMGT_LAUNCH((spmm_kernel<PREC, LPR, 8>), grid, 256, 0, s, A->row, A->col, A->blc_row, A->blcPtr,
                        A->blcIdx, val, alpha, xx, ldx, beta, yy, ldy);
            v0 += 8;
        } else if (left >= 4) {
            AMGT_LAUNCH((spmm_kernel<PREC, LPR, 4>), grid, 256, 0, s, A->row, A->col, A->blc_row, A->blcPtr,
                        A->blcIdx, val, alpha, xx, ldx, beta, yy, ldy);
            v0 += 4;
        } else if (left >= 2) {
            AMGT_LAUNCH((spmm_kernel<PREC, LPR, 2>), grid, 256, 0, s, A->row, A->col, A->blc_row, A->blcPtr,
                        A->blcIdx, val, alpha, xx, ldx, beta, yy, ldy);
            v0 += 2;
        } else {
            AMGT_LAUNCH((spmm_kernel<PREC, LPR, 1>), grid, 256, 0, s, A->row, A->col, A->blc_row, A->blcPtr,
                        A->blcIdx, val, alpha, xx, ldx, beta, yy, ldy);
            v0 += 1;
        }
    }
    return AMGT_OK;
}

template <int PREC>
static int launch_spmm(const amgt_bsr *A, const void *val, double alpha, int nvec, const double *x, int ldx,
                       double beta, double *y, int ldy, cudaStream_t s, int sm_count)
{
    const int lpr = pick_lpr(A, AMGT_DOUBLE);
    const int grid = grid_for(8 * (32 / lpr), A->blc_row, sm_count, 8);
    switch (lpr) {
    case 4: return launch_spmm_lpr<PREC, 4>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, grid);
    case 8: return launch_spmm_lpr<PREC, 8>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, grid);
    case 16: return launch_spmm_lpr<PREC, 16>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, grid);
    default: return launch_spmm_lpr<PREC, 32>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, grid);
    }
}

template <int PREC>
static int launch_segmented_scratch(const amgt_bsr *A, const void *val, double alpha, const double *x,
                                    double beta, double *y, double *part, int sm_count, cudaStream_t s)
{
    const bool safe = (A->col % 4 != 0) || ((uintptr_t)x % 16 != 0);
    const int grid = grid_for(8, A->warpnum, sm_count, 8);
    if (safe)
        AMGT_LAUNCH((spmv_segment_kernel<PREC, true>), grid, 256, 0, s, A->col, A->warpnum, A->rowIdxbyWarp,
                    A->rowPtrbyWarp, A->blcPtr, A->blcIdx, val, x, part);
    else
        AMGT_LAUNCH((spmv_segment_kernel<PREC, false>), grid, 256, 0, s, A->col, A->warpnum, A->rowIdxbyWarp,
                    A->rowPtrbyWarp, A->blcPtr, A->blcIdx, val, x, part);
    AMGT_LAUNCH(spmv_segment_combine, grid_for(256, A->row, sm_count, 8), 256, 0, s, A->row, A->blc_row,
                A->rowPtrbyWarp, part, alpha, beta, y, PREC != AMGT_DOUBLE);
    return AMGT_OK;
}

// The segmented SpMV (same two kernels and summation order as the
// allocating path) writing its partial sums into caller-provided scratch of
// 4 * A->warpnum doubles.  Performs no allocation and no device query.
int spmv_segmented_with_scratch(int prec, double alpha, const amgt_bsr *A, const double *x, double beta, double *y,
                                double *part, int sm_count, cudaStream_t s)
{
    const void *val = value_array(A, prec);
    if (!val) return AMGT_ERR_INVALID;
    switch (prec) {
    case AMGT_DOUBLE: return launch_segmented_scratch<AMGT_DOUBLE>(A, val, alpha, x, beta, y, part, sm_count, s);
    case AMGT_FLOAT: return launch_segmented_scratch<AMGT_FLOAT>(A, val, alpha, x, beta, y, part, sm_count, s);
    case AMGT_HALF: return launch_segmented_scratch<AMGT_HALF>(A, val, alpha, x, beta, y, part, sm_count, s);
    case AMGT_BF16: return launch_segmented_scratch<AMGT_BF16>(A, val, alpha, x, beta, y, part, sm_count, s);
    default: return AMGT_ERR_INVALID;
    }
}

template <int PREC, int EPI>
static int launch_epi(const amgt_bsr *A, const void *val, const double *x, const EpiArgs &e, int grid,
                      cudaStream_t s, int sm_count)
{
    const bool safe = (A->col % 4 != 0) || ((uintptr_t)x % 16 != 0);
    const int lpr = pick_lpr(A, PREC);
    const int run = EPI == EPI_DOT ? lpr : run_lpr(lpr, PREC);
    if (run != lpr) grid = grid_for(8 * (32 / run), A->blc_row, sm_count, 8);  // no partials: any grid
#define AMGT_EPI_CASE(L, V)                                                                                  \
    if (run == L && lpr == L * V) {                                                                          \
        if (safe)                                                                                            \
            AMGT_LAUNCH_PDL((spmv_epi_kernel<PREC, L, true, EPI, V>), grid, 256, 0, s, A->row, A->col,        \
                            A->blc_row, A->blcPtr, A->blcIdx, val, x, e);                                    \
        else                                                                                                 \
            AMGT_LAUNCH_PDL((spmv_epi_kernel<PREC, L, false, EPI, V>), grid, 256, 0, s, A->row, A->col,       \
                            A->blc_row, A->blcPtr, A->blcIdx, val, x, e);                                    \
        return AMGT_OK;                                                                                      \
    }
    AMGT_EPI_CASE(4, 1)
    AMGT_EPI_CASE(8, 1)
    AMGT_EPI_CASE(16, 1)
    AMGT_EPI_CASE(32, 1)
    if constexpr (EPI != EPI_DOT && (PREC == AMGT_HALF || PREC == AMGT_BF16 || PREC == kExact16)) {
        AMGT_EPI_CASE(4, 2)
    }
#undef AMGT_EPI_CASE
    return AMGT_ERR_INVALID;
}

template <int EPI>
static int launch_epi_prec(int prec, const amgt_bsr *A, const double *x, const EpiArgs &e, int grid,
                           cudaStream_t s, int sm_count)
{
    const int mode = storage_mode(A, prec);
    const void *val = value_array(A, mode);
    if (!val) return AMGT_ERR_INVALID;
    switch (mode) {
    case AMGT_DOUBLE: return launch_epi<AMGT_DOUBLE, EPI>(A, val, x, e, grid, s, sm_count);
    case AMGT_FLOAT: return launch_epi<AMGT_FLOAT, EPI>(A, val, x, e, grid, s, sm_count);
    case AMGT_HALF: return launch_epi<AMGT_HALF, EPI>(A, val, x, e, grid, s, sm_count);
    case AMGT_BF16: return launch_epi<AMGT_BF16, EPI>(A, val, x, e, grid, s, sm_count);
    case kExact32: return launch_epi<kExact32, EPI>(A, val, x, e, grid, s, sm_count);
    case kExact16: return launch_epi<kExact16, EPI>(A, val, x, e, grid, s, sm_count);
    default: return AMGT_ERR_INVALID;
    }
}

int epi_grid(const amgt_bsr *A, int sm_count)
{
    const int lpr = pick_lpr(A, storage_mode(A, AMGT_DOUBLE));
    return grid_for(8 * (32 / lpr), A->blc_row, sm_count, 8);
}

int spmv_residual(int prec, const amgt_bsr *A, const double *f, const double *u, double *r, cudaStream_t s,
                  int sm_count)
{
    EpiArgs e{f, nullptr, 0.0, r, nullptr};
    return launch_epi_prec<EPI_RESID>(prec, A, u, e, epi_grid(A, sm_count), s, sm_count);
}

int spmv_jacobi(int prec, const amgt_bsr *A, const double *inv_l1, double w, const double *f, const double *u,
                double *u_out, cudaStream_t s, int sm_count)
{
    EpiArgs e{f, inv_l1, w, u_out, nullptr};
    return launch_epi_prec<EPI_JACOBI>(prec, A, u, e, epi_grid(A, sm_count), s, sm_count);
}

bool restrict_fusable(const amgt_bsr *R)
{
    const bool seg = R->rowPtrbyWarp && R->rowIdxbyWarp && R->warpnum > 0 && R->max_blc_per_row > 256;
    return R->row > 0 && R->blc_num > 0 && R->col > 0 && !seg;
}

int spmv_restrict_jacobi0(int prec, const amgt_bsr *R, const double *t, double *f, const double *inv_l1, double w,
                          double *u, cudaStream_t s, int sm_count)
{
    if (!restrict_fusable(R)) return AMGT_ERR_INVALID;
    EpiArgs e{nullptr, inv_l1, w, f, nullptr, u};
    return launch_epi_prec<EPI_RESTRICT_JACOBI0>(prec, R, t, e, epi_grid(R, sm_count), s, sm_count);
}

int spmv_dot(int prec, const amgt_bsr *A, const double *u, double *out, double *partial, int grid, cudaStream_t s)
{
    EpiArgs e{nullptr, nullptr, 0.0, out, partial};
    return launch_epi_prec<EPI_DOT>(prec, A, u, e, grid, s, 0);  // the segment layout: grid as given
}

int scale_vector(long long n, double beta, double *y, int sm_count, cudaStream_t s)
{
    AMGT_LAUNCH(scale_kernel, grid_for(256, n, sm_count, 8), 256, 0, s, n, beta, y);
    return AMGT_OK;
}

int bsr_l1_norms(const amgt_bsr *A, double *l1, int invert, cudaStream_t s, int sm_count)
{
    const int mode = storage_mode(A, AMGT_DOUBLE);
    const void *val = value_array(A, mode);
    const int grid = grid_for(256, A->row, sm_count, 8);
    if (mode == kExact16)
        AMGT_LAUNCH(l1_norm_kernel<kExact16>, grid, 256, 0, s, A->row, A->blcPtr, val, l1, invert);
    else if (mode == kExact32)
        AMGT_LAUNCH(l1_norm_kernel<kExact32>, grid, 256, 0, s, A->row, A->blcPtr, val, l1, invert);
    else
        AMGT_LAUNCH(l1_norm_kernel<AMGT_DOUBLE>, grid, 256, 0, s, A->row, A->blcPtr, A->blcVal, l1, invert);
    return AMGT_OK;
}

}  // namespace amgt

using namespace amgt;

extern "C" {

int amgt_spmv(int prec, double alpha, const amgt_bsr *A, const double *x, double beta, double *y,
              amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16) return AMGT_ERR_INVALID;
    if (A->row > 0 && !y) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    if (A->blc_num == 0 || A->col == 0) {
        AMGT_LAUNCH(scale_kernel, grid_for(256, A->row, st->sm_count, 8), 256, 0, s, (long long)A->row, beta, y);
        return AMGT_OK;
    }
    const bool seg = A->rowPtrbyWarp && A->rowIdxbyWarp && A->warpnum > 0 && A->max_blc_per_row > 256;
    const int mode = seg ? prec : storage_mode(A, prec);
    const void *val = value_array(A, mode);
    if (!val || !x || !A->blcPtr || !A->blcIdx) return AMGT_ERR_INVALID;
    switch (mode) {
    case kExact32: return launch_spmv<kExact32>(A, val, alpha, x, beta, y, s, st->sm_count);
    case kExact16: return launch_spmv<kExact16>(A, val, alpha, x, beta, y, s, st->sm_count);
    case AMGT_DOUBLE:
        return seg ? launch_spmv_segmented<AMGT_DOUBLE>(A, val, alpha, x, beta, y, s, st->sm_count)
                   : launch_spmv<AMGT_DOUBLE>(A, val, alpha, x, beta, y, s, st->sm_count);
    case AMGT_FLOAT:
        return seg ? launch_spmv_segmented<AMGT_FLOAT>(A, val, alpha, x, beta, y, s, st->sm_count)
                   : launch_spmv<AMGT_FLOAT>(A, val, alpha, x, beta, y, s, st->sm_count);
    case AMGT_HALF:
        return seg ? launch_spmv_segmented<AMGT_HALF>(A, val, alpha, x, beta, y, s, st->sm_count)
                   : launch_spmv<AMGT_HALF>(A, val, alpha, x, beta, y, s, st->sm_count);
    default:
        return seg ? launch_spmv_segmented<AMGT_BF16>(A, val, alpha, x, beta, y, s, st->sm_count)
                   : launch_spmv<AMGT_BF16>(A, val, alpha, x, beta, y, s, st->sm_count);
    }
}

int amgt_spmm(int prec, double alpha, const amgt_bsr *A, int nvec, const double *x, int ldx, double beta, double *y,
              int ldy, amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16 || nvec < 0) return AMGT_ERR_INVALID;
    if (nvec == 0 || A->row == 0) return AMGT_OK;
    if (!y || ldy < A->row || (A->col > 0 && ldx < A->col)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    if (A->blc_num == 0 || A->col == 0) {
        for (int v = 0; v < nvec; ++v)
            AMGT_LAUNCH(scale_kernel, grid_for(256, A->row, st->sm_count, 8), 256, 0, s, (long long)A->row, beta,
                        y + (long long)v * ldy);
        return AMGT_OK;
    }
    const void *val = value_array(A, prec);
    if (!val || !x) return AMGT_ERR_INVALID;
    switch (prec) {
    case AMGT_DOUBLE: return launch_spmm<AMGT_DOUBLE>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, st->sm_count);
    case AMGT_FLOAT: return launch_spmm<AMGT_FLOAT>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, st->sm_count);
    case AMGT_HALF: return launch_spmm<AMGT_HALF>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, st->sm_count);
    default: return launch_spmm<AMGT_BF16>(A, val, alpha, nvec, x, ldx, beta, y, ldy, s, st->sm_count);
    }
}

}  // extern "C"

extern "C" {

int amgt_bsr_l1_norms(const amgt_bsr *A, double *l1, amgt_stream_t stream)
{
    if (!A || (A->row > 0 && (!l1 || !A->blcPtr))) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return bsr_l1_norms(A, l1, 0, (cudaStream_t)stream, st->sm_count);
}

int amgt_bsr_residual(int prec, const amgt_bsr *A, const double *f, const double *u, double *r,
                      amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (!f || !u || !r || !A->blcPtr || !value_array(A, storage_mode(A, prec))) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return spmv_residual(prec, A, f, u, r, (cudaStream_t)stream, st->sm_count);
}

int amgt_bsr_jacobi(int prec, const amgt_bsr *A, const double *inv_l1, double weight, const double *f,
                    const double *u, double *u_out, amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16 || A->row != A->col) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (!inv_l1 || !f || !u || !u_out || u == u_out || !A->blcPtr || !value_array(A, storage_mode(A, prec)))
        return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return spmv_jacobi(prec, A, inv_l1, weight, f, u, u_out, (cudaStream_t)stream, st->sm_count);
}

}  // extern "C"
