// Galerkin AMG hierarchy on mBSR and a PCG solve preconditioned by one
// V(1,1) cycle with l1-Jacobi smoothing, for the setup + solve measurement.
//
// The coarsening and interpolation stay the caller's (in HYPRE they are
// BoomerAMG's, outside the AmgT path): the caller passes P_0 .. P_{L-2}.
// Everything else runs here, on the GPU, through the mBSR kernels:
//   setup  A_0 = CSR->mBSR; per level P_l -> mBSR, R_l = P_l^T (block
//          transpose), A_{l+1} = R_l (A_l P_l) (two SpGEMMs, the
//          Galerkin product of hypre_ParCSRMatrixRAPKT,
//          par_csr_triplemat_device.c:630-905), inverse l1 row norms
//          (relax 18, ams.c:627-636), value shadows, and the dense inverse
//          of the coarsest operator (HYPRE's coarse GE, relax 9);
//   cycle  pre-smooth from zero u = w f ./ l1; r = f - A u (fused);
//          f_c = R r; recurse; u += P e; post-smooth u + w (f - A u) ./ l1
//          (fused), as hypre_BoomerAMGCycle does with relax 18
//          (par_cycle.c:678-751, par_relax.c:1178-1260);
//   solve  PCG (krylov/pcg.c:405-580), optionally flexible (Polak-Ribiere
//          beta), with the scalars kept on the device; the whole iteration
//          loop is one CUDA graph launch (a conditional while node whose
//          body ends with the convergence test) and one read-back of the
//          iteration count and the ||r||^2 history (if the runtime does
//          not take the loop graph: one graph launch and one 8-byte read
//          per iteration).
// Dots are deterministic: fixed grids, per-CTA partials reduced in a fixed
// order by one CTA.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "amg_handle.cuh"

namespace amgt {

enum { S_BB = 0, S_RR = 1, S_RZ = 2, S_PQ = 3, S_ALPHA = 4, S_BETA = 5, S_ZRPREV = 6, S_NSCAL = 8 };
enum { OP_STORE = 0, OP_ALPHA = 1, OP_BETA = 2, OP_BETA_FLEX = 3 };

__global__ void __launch_bounds__(kDotThreads) dot_kernel(long long n, const double *__restrict__ a,
                                                         const double *__restrict__ b, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kDotThreads / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += a[i] * b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDotThreads / 32; ++w) t += sred[w];
        part[blockIdx.x] = t;
    }
}

// Sums np partials in a fixed order into scal[slot] and applies op.
__global__ void __launch_bounds__(kDotThreads) reduce_kernel(const double *__restrict__ part, int np,
                                                            double *__restrict__ scal, int slot, int op)
{
    grid_dependency_wait();
    __shared__ double sred[kDotThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDotThreads / 32; ++w) t += sred[w];
        if (op == OP_ALPHA) {
            scal[S_PQ] = t;
            scal[S_ALPHA] = (t != 0.0) ? scal[S_RZ] / t : 0.0;
        } else if (op == OP_BETA || op == OP_BETA_FLEX) {
            const double rz_old = scal[S_RZ];
            const double num = (op == OP_BETA_FLEX) ? t - scal[S_ZRPREV] : t;
            scal[S_BETA] = (rz_old != 0.0) ? num / rz_old : 0.0;
            scal[S_RZ] = t;
        } else {
            scal[slot] = t;
        }
    }
}

// x += alpha p; r -= alpha q; partials of r . r
__global__ void __launch_bounds__(kDotThreads) axpy2_dot_kernel(long long n, const double *__restrict__ scal,
                                                               const double *__restrict__ p,
                                                               const double *__restrict__ q, double *__restrict__ x,
                                                               double *__restrict__ r, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kDotThreads / 32];
    const double alpha = scal[S_ALPHA];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        s += ri * ri;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDotThreads / 32; ++w) t += sred[w];
        part[blockIdx.x] = t;
    }
}

// p = z + beta p
__global__ void xpby_kernel(long long n, const double *__restrict__ z, const double *__restrict__ scal,
                            double *__restrict__ p)
{
    grid_dependency_wait();
    const double beta = scal[S_BETA];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// u = w f ./ l1 (l1-Jacobi sweep from a zero guess)
__global__ void jacobi_zero_kernel(long long n, const double *__restrict__ f, const double *__restrict__ inv_l1,
                                   double w, double *__restrict__ u)
{
    grid_dependency_wait();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        u[i] = w * f[i] * inv_l1[i];
}

// u = M f with M the coarsest inverse: dense diagonal blocks, block b
// rows cb_off[b] .. cb_off[b+1]-1, row-major at M + cb_doff[b] (one block
// for a single system); one warp per row
__global__ void dense_mv_kernel(int nc, const int *__restrict__ row_blk, const int *__restrict__ cb_off,
                                const long long *__restrict__ cb_doff, const double *__restrict__ M,
                                const double *__restrict__ f, double *__restrict__ u)
{
    grid_dependency_wait();
    const int lane = threadIdx.x & 31;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nc; row += (gridDim.x * blockDim.x) >> 5) {
        const int b = row_blk[row], o = cb_off[b], nb = cb_off[b + 1] - o;
        const double *Mr = M + cb_doff[b] + (long long)(row - o) * nb;
        double s = 0.0;
        for (int j = lane; j < nb; j += 32) s += Mr[j] * f[o + j];
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(FULL, s, o2);
        if (lane == 0) u[row] = s;
    }
}

// mBSR -> dense diagonal blocks (row-major per block, as dense_mv_kernel
// reads them); entries outside a row's block are not stored (the
// operator is block-diagonal when there are several blocks)
__global__ void bsr_to_dense_kernel(int m, int n, const int *__restrict__ ptr, const int *__restrict__ idx,
                                    const double *__restrict__ val, const int *__restrict__ row_blk,
                                    const int *__restrict__ cb_off, const long long *__restrict__ cb_doff,
                                    double *__restrict__ D)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        const int b = row >> 2, q = row & 3;
        const int rb = row_blk[row], o = cb_off[rb], nb = cb_off[rb + 1] - o;
        double *Dr = D + cb_doff[rb] + (long long)(row - o) * nb;
        for (int k = ptr[b]; k < ptr[b + 1]; ++k)
            for (int c = 0; c < 4; ++c) {
                const int col = 4 * idx[k] + c;
                if (col < n && col >= o && col < o + nb) Dr[col - o] = val[16LL * k + 4 * q + c];
            }
    }
}

// Dense inverse of the coarsest operator on the GPU: Gauss-Jordan in
// exchange form with partial pivoting.  The table T starts as D (y = D x);
// a pivot (p, c), p the largest |T[r][c]| among rows not yet pivoted,
// exchanges unknown x_c with equation y_p:
//   T'[p][c] = 1/a, T'[p][k] = -T[p][k]/a, T'[r][c] = T[r][c]/a,
//   T'[r][k] = T[r][k] - T[r][c] T[p][k]/a          (a = T[p][c]).
// After every column has been pivoted, row p_c expresses x_c in the
// equations y_{p_k}: D^-1[c][p_k] = T[p_c][k] (gj_gather_kernel).  Each
// update needs only the element itself, the pivot row and the pivot column,
// which the pivot phase stages first, so the update runs in place.  A zero
// (or non-finite) pivot marks D singular in *bad and continues with a = 1.
// Candidate (v2, i2) beats (v1, i1): a row beats none, a number beats NaN,
// then the larger |value|, then the lower row.
__device__ __forceinline__ bool gj_better(double v2, int i2, double v1, int i1, int none)
{
    if (i2 == none) return false;
    if (i1 == none) return true;
    if (isnan(v1) != isnan(v2)) return isnan(v1);
    return v2 > v1 || (v2 == v1 && i2 < i1);
}

__device__ void gj_pivot_phase(int nc, int c, const double *__restrict__ T, int *__restrict__ used,
                               int *__restrict__ piv, double *__restrict__ rowp, double *__restrict__ colc,
                               int *__restrict__ bad, double *sval, int *sidx)
{
    const int t = threadIdx.x, nt = blockDim.x;  // nt: a power of two
    double best = 0.0;
    int bi = nc;
    for (int r = t; r < nc; r += nt) {
        if (used[r]) continue;
        const double v = fabs(T[(long long)r * nc + c]);
        if (gj_better(v, r, best, bi, nc)) { best = v; bi = r; }
    }
    sval[t] = best;
    sidx[t] = bi;
    __syncthreads();
    for (int o = nt / 2; o > 0; o >>= 1) {
        if (t < o && gj_better(sval[t + o], sidx[t + o], sval[t], sidx[t], nc)) {
            sval[t] = sval[t + o];
            sidx[t] = sidx[t + o];
        }
        __syncthreads();
    }
    // c < nc columns done so far leave at least one unpivoted row, so p < nc
    const int p = min(sidx[0], nc - 1);
    __syncthreads();
    for (int k = t; k < nc; k += nt) {
        rowp[k] = T[(long long)p * nc + k];
        colc[k] = T[(long long)k * nc + c];
    }
    if (t == 0) {
        used[p] = 1;
        piv[c] = p;
        const double a = T[(long long)p * nc + c];
        if (!(a != 0.0) || !isfinite(a)) *bad = 1;
    }
}

__device__ __forceinline__ double gj_update(double v, int r, int k, int p, int c, double a, const double *rowp,
                                            const double *colc)
{
    if (r == p) return (k == c) ? 1.0 / a : -rowp[k] / a;
    if (k == c) return colc[r] / a;
    return v - colc[r] * rowp[k] / a;
}

__device__ __forceinline__ double gj_pivot_value(int c, const double *rowp)
{
    const double a = rowp[c];
    return (a != 0.0 && isfinite(a)) ? a : 1.0;
}

// Whole inverse in one CTA (small coarsest levels): pivot phase, barrier,
// in-place update, barrier, per column.
__global__ void __launch_bounds__(1024) gj_small_kernel(int nc, double *__restrict__ T, int *__restrict__ used,
                                                       int *__restrict__ piv, double *__restrict__ rowp,
                                                       double *__restrict__ colc, int *__restrict__ bad)
{
    __shared__ double sval[1024];
    __shared__ int sidx[1024];
    for (int r = threadIdx.x; r < nc; r += blockDim.x) used[r] = 0;
    __syncthreads();
    for (int c = 0; c < nc; ++c) {
        gj_pivot_phase(nc, c, T, used, piv, rowp, colc, bad, sval, sidx);
        __syncthreads();
        const int p = piv[c];
        const double a = gj_pivot_value(c, rowp);
        for (long long e = threadIdx.x; e < (long long)nc * nc; e += blockDim.x) {
            const int r = (int)(e / nc), k = (int)(e % nc);
            T[e] = gj_update(T[e], r, k, p, c, a, rowp, colc);
        }
        __syncthreads();
    }
}

// Larger coarsest levels: one CTA finds and stages the pivot of column c ...
__global__ void __launch_bounds__(1024) gj_pivot_kernel(int nc, int c, const double *__restrict__ T,
                                                       int *__restrict__ used, int *__restrict__ piv,
                                                       double *__restrict__ rowp, double *__restrict__ colc,
                                                       int *__restrict__ bad)
{
    __shared__ double sval[1024];
    __shared__ int sidx[1024];
    gj_pivot_phase(nc, c, T, used, piv, rowp, colc, bad, sval, sidx);
}

// ... and the whole grid updates the table in place.
__global__ void gj_update_kernel(int nc, int c, double *__restrict__ T, const int *__restrict__ piv,
                                 const double *__restrict__ rowp, const double *__restrict__ colc)
{
    const int p = piv[c];
    const double a = gj_pivot_value(c, rowp);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)nc * nc;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / nc), k = (int)(e % nc);
        T[e] = gj_update(T[e], r, k, p, c, a, rowp, colc);
    }
}

__global__ void clear_int_kernel(int n, int *__restrict__ a)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0;
}

// D^-1[c][p_k] = T[p_c][k]
__global__ void gj_gather_kernel(int nc, const double *__restrict__ T, const int *__restrict__ piv,
                                 double *__restrict__ inv)
{
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)nc * nc;
         e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e / nc), k = (int)(e % nc);
        inv[(long long)c * nc + piv[k]] = T[(long long)piv[c] * nc + k];
    }
}

// Several diagonal blocks (a batch of systems): one CTA inverts each block
// in place with the same steps as gj_small_kernel, then gathers it.
__global__ void __launch_bounds__(1024) gj_blocks_kernel(const int *__restrict__ cb_off,
                                                        const long long *__restrict__ cb_doff, double *__restrict__ T,
                                                        double *__restrict__ inv, int *__restrict__ used,
                                                        int *__restrict__ piv, double *__restrict__ rowp,
                                                        double *__restrict__ colc, int *__restrict__ bad)
{
    __shared__ double sval[1024];
    __shared__ int sidx[1024];
    const int o = cb_off[blockIdx.x], nb = cb_off[blockIdx.x + 1] - o;
    double *Tb = T + cb_doff[blockIdx.x], *Ib = inv + cb_doff[blockIdx.x];
    int *ub = used + o, *pb = piv + o;
    double *rb = rowp + o, *cb = colc + o;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) ub[r] = 0;
    __syncthreads();
    for (int c = 0; c < nb; ++c) {
        gj_pivot_phase(nb, c, Tb, ub, pb, rb, cb, bad, sval, sidx);
        __syncthreads();
        const int p = pb[c];
        const double a = gj_pivot_value(c, rb);
        for (long long e = threadIdx.x; e < (long long)nb * nb; e += blockDim.x) {
            const int r = (int)(e / nb), k = (int)(e % nb);
            Tb[e] = gj_update(Tb[e], r, k, p, c, a, rb, cb);
        }
        __syncthreads();
    }
    for (long long e = threadIdx.x; e < (long long)nb * nb; e += blockDim.x) {
        const int c = (int)(e / nb), k = (int)(e % nb);
        Ib[(long long)c * nb + pb[k]] = Tb[(long long)pb[c] * nb + k];
    }
}

constexpr int kGjSmall = 256;  // one CTA up to this order, a launch pair per column above

// inv = D^-1 for the dense nc x nc matrix T (overwritten); *bad (device,
// zeroed by the caller) is raised when D is singular.
int dense_invert(int nc, double *T, double *inv, int *bad, int sm_count, cudaStream_t s)
{
    int *used = nullptr, *piv = nullptr;
    double *rowp = nullptr, *colc = nullptr;
    int rc = AMGT_OK;
    if ((rc = alloc_n(&used, nc, s)) || (rc = alloc_n(&piv, nc, s)) || (rc = alloc_n(&rowp, nc, s)) ||
        (rc = alloc_n(&colc, nc, s)))
        goto done;
    if (nc <= kGjSmall) {
        count_launch();
        gj_small_kernel<<<1, 1024, 0, s>>>(nc, T, used, piv, rowp, colc, bad);
    } else {
        count_launch();
        clear_int_kernel<<<grid_for(256, nc, sm_count, 4), 256, 0, s>>>(nc, used);
        const int grid = grid_for(256, (long long)nc * nc, sm_count, 8);
        for (int c = 0; c < nc; ++c) {
            count_launch();
            gj_pivot_kernel<<<1, 1024, 0, s>>>(nc, c, T, used, piv, rowp, colc, bad);
            count_launch();
            gj_update_kernel<<<grid, 256, 0, s>>>(nc, c, T, piv, rowp, colc);
        }
    }
    count_launch();
    gj_gather_kernel<<<grid_for(256, (long long)nc * nc, sm_count, 8), 256, 0, s>>>(nc, T, piv, inv);
    if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
done:
    free_ptr(used, s);
    free_ptr(piv, s);
    free_ptr(rowp, s);
    free_ptr(colc, s);
    return rc;
}

// ------------------------------------------------ FGMRES with refinement
// The inner solve of FGMRES-IR: flexible GMRES(m) (R/krylov/flexgmres.c)
// with the Krylov basis V (m + 1 vectors) and the preconditioned vectors Z
// (m vectors) stored in fp32, inner products and the Hessenberg
// least-squares problem in fp64.  The iteration index j lives on the device
// so that one captured iteration serves every j (the body of a while node):
//   vin (fixed, fp64) = V_j      written by the previous iteration's scale
//   zout = M vin                 V-cycle
//   Z_j = zout                   (fp32)
//   w = A zout                   level-0 matvec at the inner precision
//   H[i][j] = V_i . w, i <= j    classical Gram-Schmidt, one pass
//   w -= sum H[i][j] V_i; ||w||
//   Givens rotations on column j, residual estimate |g[j+1]|, j += 1
//   V_j = vin = w / ||w||
// Scalars (gm): H column-major (m + 1) x m, then cs[m], sn[m], g[m + 1],
// y[m], and the slots below.
constexpr int kGmMaxRestart = 32;
enum { GM_BETA0 = 0, GM_INVH = 1, GM_RES = 2, GM_NSLOT = 4 };

struct GmLayout {
    int m;
    __host__ __device__ int H(int i, int j) const { return i + j * (m + 1); }
    __host__ __device__ int cs() const { return (m + 1) * m; }
    __host__ __device__ int sn() const { return cs() + m; }
    __host__ __device__ int g() const { return sn() + m; }
    __host__ __device__ int y() const { return g() + m + 1; }
    __host__ __device__ int slot() const { return y() + m; }
    __host__ __device__ int size() const { return slot() + GM_NSLOT; }
};

// partials of V_i . w for i = 0 .. j, one row of partials per i; the basis
// is taken 8 vectors per sweep (w re-read from L2 between sweeps)
__global__ void __launch_bounds__(kDotThreads) gm_mdot_kernel(long long n, const float *__restrict__ V,
                                                             const int *__restrict__ jdev,
                                                             const double *__restrict__ w, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kDotThreads / 32][8];
    const int j = *jdev;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i0 = 0; i0 <= j; i0 += 8) {
        double acc[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) acc[t] = 0.0;
        for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
             e += (long long)gridDim.x * blockDim.x) {
            const double we = w[e];
#pragma unroll
            for (int t = 0; t < 8; ++t)
                if (i0 + t <= j) acc[t] += (double)V[(long long)(i0 + t) * n + e] * we;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            double v = acc[t];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
            if (lane == 0) sred[warp][t] = v;
        }
        __syncthreads();
        if (threadIdx.x < 8 && i0 + (int)threadIdx.x <= j) {
            double t = 0.0;
            for (int w8 = 0; w8 < kDotThreads / 32; ++w8) t += sred[w8][threadIdx.x];
            part[(long long)(i0 + threadIdx.x) * gridDim.x + blockIdx.x] = t;
        }
        __syncthreads();
    }
}

// H[i][j] = sum of the partials of vector i (warp i, fixed order)
__global__ void __launch_bounds__(1024) gm_mdot_reduce_kernel(const double *__restrict__ part, int np,
                                                             const int *__restrict__ jdev, int m,
                                                             double *__restrict__ gm)
{
    grid_dependency_wait();
    const int j = *jdev, lane = threadIdx.x & 31;
    const GmLayout L{m};
    for (int i = threadIdx.x >> 5; i <= j; i += blockDim.x >> 5) {
        double t = 0.0;
        for (int k = lane; k < np; k += 32) t += part[(long long)i * np + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
        if (lane == 0) gm[L.H(i, j)] = t;
    }
}

// w -= sum_{i <= j} H[i][j] V_i; partials of ||w||^2
__global__ void __launch_bounds__(kDotThreads) gm_orth_kernel(long long n, const float *__restrict__ V,
                                                             const int *__restrict__ jdev, int m,
                                                             const double *__restrict__ gm, double *__restrict__ w,
                                                             double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double hc[kGmMaxRestart + 1];
    __shared__ double sred[kDotThreads / 32];
    const int j = *jdev;
    const GmLayout L{m};
    for (int i = threadIdx.x; i <= j; i += blockDim.x) hc[i] = gm[L.H(i, j)];
    __syncthreads();
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double we = w[e];
        for (int i = 0; i <= j; ++i) we -= hc[i] * (double)V[(long long)i * n + e];
        w[e] = we;
        s += we * we;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kDotThreads / 32; ++k) t += sred[k];
        part[blockIdx.x] = t;
    }
}

// ||w|| from its partials, Givens rotations on column j, the residual
// estimate; j += 1; the while condition (inner tolerance, basis size,
// breakdown, total iteration cap).
__global__ void __launch_bounds__(kDotThreads) gm_givens_kernel(cudaGraphConditionalHandle cond, int use_cond,
                                                               const double *__restrict__ part, int np,
                                                               int *__restrict__ jdev, int m, double *__restrict__ gm,
                                                               double inner_tol, int *__restrict__ it_total,
                                                               int max_iter, double *__restrict__ hist)
{
    grid_dependency_wait();
    __shared__ double sred[kDotThreads / 32];
    double s = 0.0;
    for (int k = threadIdx.x; k < np; k += blockDim.x) s += part[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double wsq = 0.0;
    for (int k = 0; k < kDotThreads / 32; ++k) wsq += sred[k];
    const int j = *jdev;
    const GmLayout L{m};
    double *cs = gm + L.cs(), *sn = gm + L.sn(), *g = gm + L.g(), *sl = gm + L.slot();
    const double hn = sqrt(fmax(wsq, 0.0));
    for (int i = 0; i < j; ++i) {
        const double a = gm[L.H(i, j)], b = gm[L.H(i + 1, j)];
        gm[L.H(i, j)] = cs[i] * a + sn[i] * b;
        gm[L.H(i + 1, j)] = -sn[i] * a + cs[i] * b;
    }
    const double a = gm[L.H(j, j)];
    const double r = hypot(a, hn);
    const double c = r > 0.0 ? a / r : 1.0, sg = r > 0.0 ? hn / r : 0.0;
    cs[j] = c;
    sn[j] = sg;
    gm[L.H(j, j)] = r;
    gm[L.H(j + 1, j)] = 0.0;
    g[j + 1] = -sg * g[j];
    g[j] = c * g[j];
    const double res = fabs(g[j + 1]);
    sl[GM_RES] = res;
    sl[GM_INVH] = hn > 0.0 ? 1.0 / hn : 0.0;
    const int k = ++*it_total;
    hist[k] = res;
    *jdev = j + 1;
    const bool more = (j + 1 < m) && res > inner_tol * sl[GM_BETA0] && hn > 0.0 && k < max_iter;
    if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// V_j = vin = w / ||w|| (j already advanced)
__global__ void gm_scale_kernel(long long n, const double *__restrict__ w, const int *__restrict__ jdev, int m,
                                const double *__restrict__ gm, float *__restrict__ V, double *__restrict__ vin)
{
    grid_dependency_wait();
    const int j = *jdev;
    const double inv = gm[GmLayout{m}.slot() + GM_INVH];
    float *vj = V + (long long)j * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double v = w[e] * inv;
        const float f = (float)v;
        vj[e] = f;
        vin[e] = (double)f;  // the cycle sees the stored basis vector
    }
}

// Z_j = zout (fp32)
__global__ void gm_store_z_kernel(long long n, const double *__restrict__ zout, const int *__restrict__ jdev,
                                  float *__restrict__ Z)
{
    grid_dependency_wait();
    float *zj = Z + (long long)(*jdev) * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        zj[e] = (float)zout[e];
}

// start of an inner solve: r (fp64) in vin and V_0 = r / ||r||; g = (beta0, 0, ...)
__global__ void gm_start_kernel(int m, const double *__restrict__ scal, int slot_rr, double *__restrict__ gm,
                                int *__restrict__ jdev)
{
    const GmLayout L{m};
    const double beta0 = sqrt(fmax(scal[slot_rr], 0.0));
    double *g = gm + L.g();
    for (int i = 0; i <= m; ++i) g[i] = 0.0;
    g[0] = beta0;
    gm[L.slot() + GM_BETA0] = beta0;
    gm[L.slot() + GM_INVH] = beta0 > 0.0 ? 1.0 / beta0 : 0.0;
    *jdev = 0;
}

__global__ void gm_scale_first_kernel(long long n, const double *__restrict__ r, int m, const double *__restrict__ gm,
                                      float *__restrict__ V, double *__restrict__ vin)
{
    const double inv = gm[GmLayout{m}.slot() + GM_INVH];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float f = (float)(r[e] * inv);
        V[e] = f;
        vin[e] = (double)f;
    }
}

// y = R^-1 g over the k = j columns done (R: the rotated Hessenberg)
__global__ void gm_backsolve_kernel(int m, const int *__restrict__ jdev, double *__restrict__ gm)
{
    const GmLayout L{m};
    const int k = *jdev;
    const double *g = gm + L.g();
    double *y = gm + L.y();
    for (int i = k - 1; i >= 0; --i) {
        double t = g[i];
        for (int l = i + 1; l < k; ++l) t -= gm[L.H(i, l)] * y[l];
        const double d = gm[L.H(i, i)];
        y[i] = d != 0.0 ? t / d : 0.0;
    }
}

// x += sum_{i < k} y_i Z_i  (fp64 update of x)
__global__ void gm_update_kernel(long long n, const float *__restrict__ Z, const int *__restrict__ jdev, int m,
                                 const double *__restrict__ gm, double *__restrict__ x)
{
    __shared__ double ys[kGmMaxRestart];
    const int k = *jdev;
    const double *y = gm + GmLayout{m}.y();
    for (int i = threadIdx.x; i < k; i += blockDim.x) ys[i] = y[i];
    __syncthreads();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int i = 0; i < k; ++i) t += ys[i] * (double)Z[(long long)i * n + e];
        x[e] += t;
    }
}

}  // namespace amgt

using namespace amgt;

namespace {

void free_level(Level &v, cudaStream_t s)
{
    amgt_bsr_free(&v.A, (amgt_stream_t)s);
    amgt_bsr_free(&v.P, (amgt_stream_t)s);
    amgt_bsr_free(&v.R, (amgt_stream_t)s);
    amgt_pbsr_free(&v.pA, (amgt_stream_t)s);
    amgt_pbsr_free(&v.pAs, (amgt_stream_t)s);
    amgt_pbsr_free(&v.pP, (amgt_stream_t)s);
    amgt_pbsr_free(&v.pR, (amgt_stream_t)s);
    free_ptr(v.inv_l1, s);
    free_ptr(v.f, s);
    free_ptr(v.u, s);
    free_ptr(v.t, s);
    free_ptr(v.s, s);
}

void destroy_handle(amgt_amg *h, cudaStream_t s)
{
    if (!h) return;
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->loop) cudaGraphExecDestroy(h->loop);
    if (h->gm_loop) cudaGraphExecDestroy(h->gm_loop);
    free_ptr(h->gmV, s);
    free_ptr(h->gmZ, s);
    free_ptr(h->gm, s);
    free_ptr(h->gm_vin, s);
    free_ptr(h->gm_zout, s);
    free_ptr(h->gm_w, s);
    free_ptr(h->gm_part, s);
    free_ptr(h->gm_j, s);
    if (h->mr) free_multi_rhs(h->mr, s);
    if (h->batch) free_batch(h->batch, s);
    if (h->graph_stream) cudaStreamDestroy(h->graph_stream);
    free_ptr(h->loop_it, s);
    free_ptr(h->loop_rr, s);
    // loop_pinned and mr_pinned live inside the one pinned block h->pinned
    for (auto &v : h->lv) free_level(v, s);
    free_ptr(h->coarse_inv, s);
    free_ptr(h->cb_off, s);
    free_ptr(h->cb_doff, s);
    free_ptr(h->row_blk, s);
    free_ptr(h->r, s);
    free_ptr(h->z, s);
    free_ptr(h->p, s);
    free_ptr(h->q, s);
    free_ptr(h->scal, s);
    free_ptr(h->part, s);
    pinned_put(h->pinned);
    delete h;
}

// Interpolations are converted and transposed on a second stream while the
// first stream converts A and runs the products.  The work is issued from
// inside amgt_csr_to_bsr / amgt_spgemm (after their first kernels are
// queued and before they wait for a size), so that the host
// synchronisations of the second stream's own calls delay no work on the
// first: the pending transpose first (R_l, for level l's R (A P)), then the
// pending conversion (P_{l+1}), whose transpose waits for the next call.
// Events by level parity, so that level l + 1's records do not move the
// ones level l still waits on: p_ready[l % 2] after P_l, r_ready[l % 2]
// after R_l.
// With exact storage, a conversion whose every block row takes the sorted
// fill path also writes P_l's fp16 shadow and exactness bits (flag slot
// 3 l + 1 of xflags; fused16 records it), and the transpose then carries
// the shadow to R_l, whose values are P_l's: R_l's bits are P_l's.
struct NextInterp {
    cudaStream_t s2 = nullptr;
    cudaEvent_t p_ready[2] = {nullptr, nullptr}, r_ready[2] = {nullptr, nullptr};
    const amgt_csr *P = nullptr;  // pending conversion into Pb (R later into PRb)
    amgt_bsr *Pb = nullptr, *PRb = nullptr;
    int pslot = 0;
    int plevel = 0;  // level of the pending conversion
    bool exact = false;
    int64_t *xflags = nullptr;
    std::vector<char> *fused16 = nullptr;
    amgt_bsr *Tb = nullptr, *TRb = nullptr;  // pending transpose Tb -> TRb
    int rslot = 0;
    int tlevel = 0;  // level of the pending transpose
};

int transpose_pending(NextInterp *nx)
{
    if (!nx->Tb) return AMGT_OK;
    const bool with16 = (*nx->fused16)[3 * nx->tlevel + 1] != 0;
    // R = P^T carries P's fp16 candidate and, for a transfer used in fp32,
    // P's fp32 shadow written by the conversion
    AMGT_TRY(bsr_transpose_impl(nx->Tb, nx->TRb, (amgt_stream_t)nx->s2, with16, with16));
    if (with16) (*nx->fused16)[3 * nx->tlevel + 2] = 1;
    AMGT_CUDA_TRY(cudaEventRecord(nx->r_ready[nx->rslot], nx->s2));
    nx->Tb = nullptr;
    return AMGT_OK;
}

int prepare_interp(void *ctx)
{
    NextInterp *nx = static_cast<NextInterp *>(ctx);
    AMGT_TRY(transpose_pending(nx));
    if (!nx->P) return AMGT_OK;
    CvtFuse f;
    // transfers used in fp64 or fp32 are checked for exact fp16 storage by
    // the conversion's fill pass (the transpose then carries the result)
    const int tp = amgt_precision_for_level(nx->plevel + 1);
    f.want16 = nx->exact && (tp == AMGT_DOUBLE || tp == AMGT_FLOAT);
    f.want32 = f.want16 && tp == AMGT_FLOAT;
    f.flags = nx->xflags + 3 * nx->plevel + 1;
    AMGT_TRY(csr_to_bsr_impl(nx->P, nx->Pb, (amgt_stream_t)nx->s2, nullptr, nullptr, f.want16 ? &f : nullptr));
    if (f.want16 && f.fused) (*nx->fused16)[3 * nx->plevel + 1] = 1;
    AMGT_CUDA_TRY(cudaEventRecord(nx->p_ready[nx->pslot], nx->s2));
    nx->Tb = nx->Pb;
    nx->TRb = nx->PRb;
    nx->rslot = nx->pslot;
    nx->tlevel = nx->plevel;
    nx->P = nullptr;
    return AMGT_OK;
}

// Setup phase times from events recorded in stream order (no host
// synchronisation between phases): mark(p) closes an interval of phase p.
struct PhaseMarks {
    std::vector<cudaEvent_t> ev;
    std::vector<int> phase;
    void mark(int p, cudaStream_t s)
    {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess || cudaEventRecord(e, s) != cudaSuccess) {
            cudaGetLastError();
            if (e) cudaEventDestroy(e);
            return;
        }
        ev.push_back(e);
        phase.push_back(p);
    }
    void accumulate(double *ms)
    {
        if (!ev.empty() && cudaEventSynchronize(ev.back()) == cudaSuccess)
            for (size_t i = 1; i < ev.size(); ++i) {
                float t = 0.f;
                if (phase[i] >= 0 && cudaEventElapsedTime(&t, ev[i - 1], ev[i]) == cudaSuccess) ms[phase[i]] += t;
            }
        cudaGetLastError();
    }
    ~PhaseMarks()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};


int grid_n(amgt_amg *h, long long n) { return grid_for(256, n, h->sm_count, 8); }

// The value shadow a level's products at `prec` read; none for fp32 when
// the exact fp16 shadow serves them (the SpMV reads it instead).
int level_shadow(amgt_bsr *A, int prec, amgt_stream_t stream)
{
    if (prec == AMGT_FLOAT && A->exact_prec == AMGT_HALF && A->blcVal_fp16) return AMGT_OK;
    return amgt_bsr_make_shadow(A, prec, stream);
}

// z = M f: one V(1,1) cycle
int cycle(amgt_amg *h, const double *rhs0, double *out0, cudaStream_t s)
{
    auto &lv = h->lv;
    const int L = (int)lv.size();
    const double w = h->prm.relax_weight;
    const bool pk = h->prm.packed != 0;
    bool have_u = false;  // level l's sweep from a zero guess came with the restriction into it
    for (int l = 0; l < L - 1; ++l) {
        Level &v = lv[l];
        const double *f = (l == 0) ? rhs0 : v.f;
        if (!have_u)
            AMGT_LAUNCH_PDL(jacobi_zero_kernel, grid_n(h, v.n), 256, 0, s, (long long)v.n, f, v.inv_l1, w, v.u);
        have_u = false;
        if (pk) {
            AMGT_TRY(pbsr_residual(&v.pA, f, v.u, v.t, s, h->sm_count));
            AMGT_TRY(pbsr_spmv(&v.pR, 1.0, v.t, 0.0, lv[l + 1].f, s, h->sm_count));
        } else {
            AMGT_TRY(spmv_residual(l == 0 ? h->resid_prec0 : v.prec, &v.A, f, v.u, v.t, s, h->sm_count));
            Level &nx = lv[l + 1];
            if (l + 1 < L - 1 && restrict_fusable(&v.R)) {  // the next level smooths: fuse its first sweep
                AMGT_TRY(spmv_restrict_jacobi0(v.prec_transfer, &v.R, v.t, nx.f, nx.inv_l1, w, nx.u, s,
                                               h->sm_count));
                have_u = true;
            } else {
                AMGT_TRY(amgt_spmv(v.prec_transfer, 1.0, &v.R, v.t, 0.0, nx.f, (amgt_stream_t)s));
            }
        }
    }
    Level &c = lv[L - 1];
    const double *fc = (L == 1) ? rhs0 : c.f;
    double *uc = (L == 1) ? out0 : c.s;
    AMGT_LAUNCH_PDL(dense_mv_kernel, grid_for(8, c.n, h->sm_count, 8), 256, 0, s, c.n, (const int *)h->row_blk,
                    (const int *)h->cb_off, (const long long *)h->cb_doff, (const double *)h->coarse_inv, fc, uc);
    for (int l = L - 2; l >= 0; --l) {
        Level &v = lv[l];
        const double *f = (l == 0) ? rhs0 : v.f;
        double *out = (l == 0) ? out0 : v.s;
        if (pk) {
            AMGT_TRY(pbsr_spmv(&v.pP, 1.0, lv[l + 1].s, 1.0, v.u, s, h->sm_count));
            AMGT_TRY(pbsr_jacobi(l == 0 ? &v.pAs : &v.pA, v.inv_l1, w, f, v.u, out, s, h->sm_count));
        } else {
            AMGT_TRY(amgt_spmv(v.prec_transfer, 1.0, &v.P, lv[l + 1].s, 1.0, v.u, (amgt_stream_t)s));
            AMGT_TRY(spmv_jacobi(l == 0 ? h->prm.smooth_prec0 : v.prec, &v.A, v.inv_l1, w, f, v.u, out, s,
                                 h->sm_count));
        }
    }
    return AMGT_OK;
}

int dot(amgt_amg *h, const double *a, const double *b, int slot, int op, cudaStream_t s)
{
    AMGT_LAUNCH_PDL(dot_kernel, kDotGrid, kDotThreads, 0, s, h->n0, a, b, h->part);
    AMGT_LAUNCH_PDL(reduce_kernel, 1, kDotThreads, 0, s, h->part, kDotGrid, h->scal, slot, op);
    return AMGT_OK;
}

// One PCG iteration after the first (q = A p ... p = z + beta p).
int pcg_iteration(amgt_amg *h, double *x, cudaStream_t s)
{
    Level &v0 = h->lv[0];
    if (h->prm.packed) AMGT_TRY(pbsr_dot(&v0.pA, h->p, h->q, h->part, h->grid0, s));
    else AMGT_TRY(spmv_dot(AMGT_DOUBLE, &v0.A, h->p, h->q, h->part, h->grid0, s));
    AMGT_LAUNCH_PDL(reduce_kernel, 1, kDotThreads, 0, s, h->part, h->grid0, h->scal, (int)S_PQ, (int)OP_ALPHA);
    AMGT_LAUNCH_PDL(axpy2_dot_kernel, kDotGrid, kDotThreads, 0, s, h->n0, h->scal, h->p, h->q, x, h->r, h->part);
    AMGT_LAUNCH_PDL(reduce_kernel, 1, kDotThreads, 0, s, h->part, kDotGrid, h->scal, (int)S_RR, (int)OP_STORE);
    AMGT_CUDA_TRY(cudaMemcpyAsync(h->pinned, h->scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->prm.flexible) AMGT_TRY(dot(h, h->z, h->r, S_ZRPREV, OP_STORE, s));
    AMGT_TRY(cycle(h, h->r, h->z, s));
    AMGT_TRY(dot(h, h->r, h->z, S_RZ, h->prm.flexible ? OP_BETA_FLEX : OP_BETA, s));
    AMGT_LAUNCH_PDL(xpby_kernel, grid_n(h, h->n0), 256, 0, s, h->n0, h->z, h->scal, h->p);
    return AMGT_OK;
}

// End of a loop iteration inside the loop graph: counts it, keeps ||r||^2
// and sets the while condition with the host loop's test (relative
// residual above tol and fewer than max_iter iterations).
__global__ void pcg_continue_kernel(cudaGraphConditionalHandle cond, const double *__restrict__ scal, double tol,
                                    int max_iter, int *__restrict__ it, double *__restrict__ rr_hist)
{
    const int k = ++*it;
    const double rr = scal[S_RR];
    rr_hist[k] = rr;
    const double rel = sqrt(fmax(0.0, rr) / scal[S_BB]);
    cudaGraphSetConditional(cond, (k < max_iter && !(rel <= tol)) ? 1u : 0u);
}

// Builds h->loop: a while node whose body is one PCG iteration plus
// pcg_continue_kernel.  Returns an error (and the caller keeps the
// one-graph-per-iteration loop) if the runtime does not take it.
int build_loop_graph(amgt_amg *h, double *x)
{
    if (h->loop && h->loop_xout == x) return AMGT_OK;
    if (h->loop) {
        cudaGraphExecDestroy(h->loop);
        h->loop = nullptr;
    }
    if (!h->graph_stream) AMGT_CUDA_TRY(cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking));
    if (!h->loop_it || !h->loop_rr) return AMGT_ERR_INVALID;  // allocated by the setup
    if (!h->loop_pinned) return AMGT_ERR_INVALID;  // allocated by the setup
    cudaGraph_t g = nullptr;
    AMGT_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    cudaGraph_t body = nullptr;
    int rc = AMGT_OK;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    }
    if (e == cudaSuccess) {
        body = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(h->graph_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    }
    if (e == cudaSuccess) {
        const uint64_t c0 = amgt_kernel_launch_count();
        rc = pcg_iteration(h, x, h->graph_stream);
        if (rc == AMGT_OK) {
            count_launch();
            h->loop_launches = amgt_kernel_launch_count() - c0;
            pcg_continue_kernel<<<1, 1, 0, h->graph_stream>>>(cond, h->scal, h->prm.tol, h->prm.max_iter, h->loop_it,
                                                              h->loop_rr);
            e = cudaGetLastError();
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(h->graph_stream, &captured);
        if (e == cudaSuccess) e = ee;
    }
    if (e == cudaSuccess && rc == AMGT_OK) e = cudaGraphInstantiate(&h->loop, g, 0);
    cudaGraphDestroy(g);
    if (rc != AMGT_OK) return rc;
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->loop = nullptr;
        set_last_cuda_error(e, "loop graph", __FILE__, __LINE__);
        return AMGT_ERR_CUDA;
    }
    h->loop_xout = x;
    return AMGT_OK;
}

int build_graph(amgt_amg *h, double *x)
{
    if (h->graph && h->graph_xout == x) return AMGT_OK;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    if (!h->graph_stream) AMGT_CUDA_TRY(cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    AMGT_CUDA_TRY(cudaStreamBeginCapture(h->graph_stream, cudaStreamCaptureModeThreadLocal));
    const uint64_t c0 = amgt_kernel_launch_count();
    const int rc = pcg_iteration(h, x, h->graph_stream);
    h->graph_launches = amgt_kernel_launch_count() - c0;
    const cudaError_t e = cudaStreamEndCapture(h->graph_stream, &g);
    if (rc != AMGT_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    AMGT_CUDA_TRY(e);
    const cudaError_t ei = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    AMGT_CUDA_TRY(ei);
    h->graph_xout = x;
    return AMGT_OK;
}

// One inner FGMRES iteration (the body of the inner loop graph); see the
// kernel comments above.  use_cond: the Givens kernel sets the while node's
// condition.
int gm_iteration(amgt_amg *h, cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond)
{
    const int m = h->prm.restart;
    const long long n = h->n0;
    AMGT_TRY(cycle(h, h->gm_vin, h->gm_zout, s));
    AMGT_LAUNCH_PDL(gm_store_z_kernel, grid_n(h, n), 256, 0, s, n, (const double *)h->gm_zout, (const int *)h->gm_j,
                    h->gmZ);
    AMGT_TRY(amgt_spmv(h->prm.inner_prec0, 1.0, &h->lv[0].A, h->gm_zout, 0.0, h->gm_w, (amgt_stream_t)s));
    AMGT_LAUNCH_PDL(gm_mdot_kernel, kDotGrid, kDotThreads, 0, s, n, (const float *)h->gmV, (const int *)h->gm_j,
                    (const double *)h->gm_w, h->gm_part);
    AMGT_LAUNCH_PDL(gm_mdot_reduce_kernel, 1, 1024, 0, s, (const double *)h->gm_part, kDotGrid, (const int *)h->gm_j,
                    m, h->gm);
    AMGT_LAUNCH_PDL(gm_orth_kernel, kDotGrid, kDotThreads, 0, s, n, (const float *)h->gmV, (const int *)h->gm_j, m,
                    (const double *)h->gm, h->gm_w, h->gm_part);
    AMGT_LAUNCH_PDL(gm_givens_kernel, 1, kDotThreads, 0, s, cond, use_cond, (const double *)h->gm_part, kDotGrid,
                    h->gm_j, m, h->gm, h->prm.inner_tol, h->loop_it, h->prm.max_iter, h->loop_rr);
    AMGT_LAUNCH_PDL(gm_scale_kernel, grid_n(h, n), 256, 0, s, n, (const double *)h->gm_w, (const int *)h->gm_j, m,
                    (const double *)h->gm, h->gmV, h->gm_vin);
    return AMGT_OK;
}

// The inner loop as one graph: a while node whose body is gm_iteration.
int build_gm_loop(amgt_amg *h)
{
    if (h->gm_loop) return AMGT_OK;
    if (!h->graph_stream) AMGT_CUDA_TRY(cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    AMGT_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    int rc = AMGT_OK;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    }
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(h->graph_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const uint64_t c0 = amgt_kernel_launch_count();
        rc = gm_iteration(h, h->graph_stream, 1, cond);
        h->gm_loop_launches = amgt_kernel_launch_count() - c0;
        cudaGraph_t captured = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(h->graph_stream, &captured);
        if (e == cudaSuccess) e = ee;
    }
    if (e == cudaSuccess && rc == AMGT_OK) e = cudaGraphInstantiate(&h->gm_loop, g, 0);
    cudaGraphDestroy(g);
    if (rc != AMGT_OK) return rc;
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->gm_loop = nullptr;
        set_last_cuda_error(e, "FGMRES loop graph", __FILE__, __LINE__);
        return AMGT_ERR_CUDA;
    }
    return AMGT_OK;
}

// FGMRES(m) with iterative refinement: see amgt_amg_params.solver.
int fgmres_ir_solve(amgt_amg *h, const double *b, double *x, int *iterations, double *rel_res, cudaStream_t s)
{
    Level &v0 = h->lv[0];
    const int m = h->prm.restart;
    const long long n = h->n0;
    const int max_iter = h->prm.max_iter;
    if (!h->loop_pinned) return AMGT_ERR_INVALID;  // allocated by the setup
    h->hist.clear();
    AMGT_CUDA_TRY(cudaMemsetAsync(h->loop_it, 0, sizeof(int), s));
    AMGT_TRY(dot(h, b, b, S_BB, OP_STORE, s));
    double bb = 0.0, rel = 0.0;
    int total = 0, seen = 0;
    bool graph_ran = false;
    for (int outer = 0; outer < h->prm.max_outer + 1; ++outer) {
        // fp64 residual of the current x (the refinement's residual)
        AMGT_TRY(spmv_residual(AMGT_DOUBLE, &v0.A, b, x, h->r, s, h->sm_count));
        AMGT_TRY(dot(h, h->r, h->r, S_RR, OP_STORE, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(h->pinned, h->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(h->loop_pinned, h->loop_it, sizeof(int), cudaMemcpyDeviceToHost, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(h->loop_pinned + 1, h->loop_rr + 1, sizeof(double) * max_iter,
                                      cudaMemcpyDeviceToHost, s));
        AMGT_CUDA_TRY(cudaStreamSynchronize(s));
        bb = h->pinned[S_BB];
        const double sb = bb > 0.0 ? std::sqrt(bb) : 1.0;
        total = *reinterpret_cast<const int *>(h->loop_pinned);
        for (int k = seen + 1; k <= total; ++k) h->hist.push_back(h->loop_pinned[k] / sb);  // inner estimates
        if (graph_ran)  // the kernels the graph launched, per inner iteration
            for (long long k = 0; k < (long long)(total - seen) * (long long)h->gm_loop_launches; ++k) count_launch();
        graph_ran = false;
        seen = total;
        rel = bb > 0.0 ? std::sqrt(std::max(0.0, h->pinned[S_RR]) / bb) : 0.0;
        h->hist.push_back(rel);
        if (rel <= h->prm.tol || total >= max_iter || outer == h->prm.max_outer) break;
        // inner solve of A d = r; x += d
        AMGT_LAUNCH(gm_start_kernel, 1, 1, 0, s, m, (const double *)h->scal, (int)S_RR, h->gm, h->gm_j);
        AMGT_LAUNCH(gm_scale_first_kernel, grid_n(h, n), 256, 0, s, n, (const double *)h->r, m,
                    (const double *)h->gm, h->gmV, h->gm_vin);
        bool done = false;
        if (h->prm.use_graph && !h->gm_loop_failed) {
            const int lrc = build_gm_loop(h);
            if (lrc == AMGT_OK) {
                AMGT_CUDA_TRY(cudaGraphLaunch(h->gm_loop, s));
                done = graph_ran = true;
            } else if (lrc != AMGT_ERR_CUDA) {
                return lrc;
            } else {
                h->gm_loop_failed = true;
            }
        }
        if (!done) {
            // direct launches, the while test on the host
            for (int j = 0; j < m; ++j) {
                AMGT_TRY(gm_iteration(h, s, 0, 0));
                AMGT_CUDA_TRY(cudaMemcpyAsync(h->pinned + 2, h->gm + GmLayout{m}.slot(), 3 * sizeof(double),
                                              cudaMemcpyDeviceToHost, s));
                AMGT_CUDA_TRY(cudaMemcpyAsync(h->loop_pinned, h->loop_it, sizeof(int), cudaMemcpyDeviceToHost, s));
                AMGT_CUDA_TRY(cudaStreamSynchronize(s));
                const double beta0 = h->pinned[2 + GM_BETA0], invh = h->pinned[2 + GM_INVH],
                             res = h->pinned[2 + GM_RES];
                const int k = *reinterpret_cast<const int *>(h->loop_pinned);
                if (!(j + 1 < m && res > h->prm.inner_tol * beta0 && invh > 0.0 && k < max_iter)) break;
            }
        }
        AMGT_LAUNCH(gm_backsolve_kernel, 1, 1, 0, s, m, (const int *)h->gm_j, h->gm);
        AMGT_LAUNCH(gm_update_kernel, grid_n(h, n), 256, 0, s, n, (const float *)h->gmZ, (const int *)h->gm_j, m,
                    (const double *)h->gm, x);
    }
    if (iterations) *iterations = total;
    if (rel_res) *rel_res = rel;
    return AMGT_OK;
}

}  // namespace

int amgt::amg_cycle(amgt_amg *h, const double *rhs0, double *out0, cudaStream_t s) { return cycle(h, rhs0, out0, s); }

extern "C" {

void amgt_amg_default_params(amgt_amg_params *p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->max_levels = 25;
    p->max_coarse_rows = 4096;
    p->tol = 1e-8;
    p->max_iter = 200;
    p->relax_weight = 1.0;
    p->flexible = 0;
    p->use_graph = 1;
    p->galerkin_by_level = 0;
    p->smooth_prec0 = AMGT_DOUBLE;
    p->packed = 0;
    p->exact_storage = 1;
    p->solver = AMGT_SOLVER_PCG;
    p->restart = 30;
    p->inner_tol = 1e-4;
    p->inner_prec0 = AMGT_FLOAT;
    p->max_outer = 20;
}

int amgt_amg_setup(const amgt_csr *A, int num_interp, const amgt_csr *P, const amgt_amg_params *params,
                   amgt_amg **out, amgt_stream_t stream)
{
    return amgt::amg_setup_blocks(A, num_interp, P, params, out, stream, nullptr, nullptr, nullptr);
}

int amgt_amg_setup_adaptive(const amgt_csr *A, amgt_coarsen_fn fn, void *ctx, const amgt_amg_params *params,
                            amgt_amg **out, amgt_stream_t stream)
{
    if (!fn) return AMGT_ERR_INVALID;
    return amgt::amg_setup_blocks(A, 0, nullptr, params, out, stream, nullptr, fn, ctx);
}

}  // extern "C"

int amgt::amg_setup_blocks(const amgt_csr *A, int num_interp, const amgt_csr *P, const amgt_amg_params *params,
                           amgt_amg **out, amgt_stream_t stream, const std::vector<std::vector<int>> *sys_rows,
                           amgt_coarsen_fn cb, void *cb_ctx)
{
    // with a coarsening callback, P_l and level l's precision come from it,
    // level by level, once A_l exists (num_interp: the most it may give)
    std::vector<amgt_csr> Pcb;
    if (cb) {
        num_interp = (params ? params->max_levels : 25) - 1;
        if (num_interp < 0) num_interp = 0;
        Pcb.resize(num_interp + 1);
        P = Pcb.data();
    }
    if (!A || !out || num_interp < 0 || (num_interp > 0 && !P) || A->num_rows != A->num_cols || A->num_rows <= 0)
        return AMGT_ERR_INVALID;
    *out = nullptr;
    // the loop graph's body runs at least once and keeps max_iter + 1
    // residual norms: max_iter must be >= 1 (and bounded, so that its
    // buffers stay small)
    if (params && (params->max_iter < 1 || params->max_iter > 1000000 || !(params->tol >= 0.0) ||
                   params->max_coarse_rows < 1 || params->max_coarse_rows > 16384 ||
                   (params->solver != AMGT_SOLVER_PCG && params->solver != AMGT_SOLVER_FGMRES_IR)))
        return AMGT_ERR_INVALID;
    if (params && params->solver == AMGT_SOLVER_FGMRES_IR &&
        (params->restart < 1 || params->restart > kGmMaxRestart || params->inner_prec0 < AMGT_DOUBLE ||
         params->inner_prec0 > AMGT_BF16 || !(params->inner_tol >= 0.0) || params->max_outer < 1))
        return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    amgt_amg *h = new amgt_amg();
    if (params) h->prm = *params;
    else amgt_amg_default_params(&h->prm);
    if (h->prm.smooth_prec0 < AMGT_DOUBLE || h->prm.smooth_prec0 > AMGT_BF16) h->prm.smooth_prec0 = AMGT_DOUBLE;
    const bool fgm = h->prm.solver == AMGT_SOLVER_FGMRES_IR;
    h->resid_prec0 = fgm ? h->prm.inner_prec0 : AMGT_DOUBLE;
    h->sm_count = st->sm_count;
    int L = num_interp + 1;
    if (h->prm.max_levels > 0 && L > h->prm.max_levels) L = h->prm.max_levels;
    int rc = AMGT_OK;
    PhaseMarks pm;
    NextInterp nx;
    double *dense = nullptr;  // the coarsest operator, dense (inverted into h->coarse_inv)
    // exactness bits per operator (flag slots 3 l, 3 l + 1, 3 l + 2: A_l,
    // P_l, R_l), some written by the conversions' fill passes (fused16)
    int64_t *xflags = nullptr;
    std::vector<char> fused16(3 * (size_t)(num_interp + 1), 0);
    bool l1_fused0 = false;  // level 0's l1 norms written by A's conversion
    pm.mark(-1, s);
    if ((rc = alloc_n(&xflags, fused16.size(), s))) goto fail;
    if (cudaMemsetAsync(xflags, 0, sizeof(int64_t) * fused16.size(), s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    // the second stream starts after everything the caller queued on `s`
    // before this call (the inputs may still be arriving there)
    if (L > 1 && (cudaStreamCreateWithFlags(&nx.s2, cudaStreamNonBlocking) != cudaSuccess ||
                  cudaEventCreateWithFlags(&nx.p_ready[0], cudaEventDisableTiming) != cudaSuccess ||
                  cudaEventCreateWithFlags(&nx.p_ready[1], cudaEventDisableTiming) != cudaSuccess ||
                  cudaEventCreateWithFlags(&nx.r_ready[0], cudaEventDisableTiming) != cudaSuccess ||
                  cudaEventCreateWithFlags(&nx.r_ready[1], cudaEventDisableTiming) != cudaSuccess ||
                  cudaEventRecord(nx.p_ready[0], s) != cudaSuccess ||
                  cudaStreamWaitEvent(nx.s2, nx.p_ready[0], 0) != cudaSuccess)) {
        cudaGetLastError();
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    h->lv.resize(L);
    nx.exact = h->prm.exact_storage != 0 && !cb;  // fused checks follow the policy table
    nx.xflags = xflags;
    nx.fused16 = &fused16;
    // hierarchy: P_0 converted while A's conversion runs, R_l transposed
    // and P_{l+1} converted while level l's A P runs (with a callback, P_l
    // exists only once A_l does: each is converted when it arrives)
    if (L > 1 && !cb) {
        nx.P = &P[0];
        nx.Pb = &h->lv[0].P;
        nx.PRb = &h->lv[0].R;
        nx.pslot = 0;
        nx.plevel = 0;
    }
    if ((rc = alloc_n(&h->lv[0].inv_l1, A->num_rows, s))) goto fail;
    {
        // A's fill pass also writes level 0's inverse l1 norms and, with
        // exact storage, A's fp16 shadow and exactness bits
        CvtFuse f0;
        f0.want16 = h->prm.exact_storage != 0;
        f0.flags = xflags;
        f0.l1 = h->lv[0].inv_l1;
        f0.invert = 1;
        if ((rc = csr_to_bsr_impl(A, &h->lv[0].A, stream, prepare_interp, &nx, &f0))) goto fail;
        l1_fused0 = f0.fused;
        fused16[0] = f0.fused && f0.want16;
    }
    h->lv[0].n = A->num_rows;
    pm.mark(0, s);
    for (int l = 0; l < L - 1; ++l) {
        Level &v = h->lv[l];
        if (cb) {
            int prec_l = AMGT_DOUBLE;
            amgt_csr Pl{};
            const int r = cb(l, &v.A, &Pl, &prec_l, cb_ctx);
            if (r < 0 || prec_l < AMGT_DOUBLE || prec_l > AMGT_BF16) {
                rc = AMGT_ERR_INVALID;
                goto fail;
            }
            v.prec = prec_l;
            if (r == 1) {  // A_l is the coarsest level
                L = l + 1;
                h->lv.resize(L);
                break;
            }
            Pcb[l] = Pl;
            // P_l's arrays may still be arriving on the caller's stream:
            // the second stream converts it after them
            if (cudaEventRecord(nx.p_ready[l % 2], s) != cudaSuccess ||
                cudaStreamWaitEvent(nx.s2, nx.p_ready[l % 2], 0) != cudaSuccess) {
                rc = AMGT_ERR_CUDA;
                goto fail;
            }
            nx.P = &Pcb[l];
            nx.Pb = &v.P;
            nx.PRb = &v.R;
            nx.pslot = l % 2;
            nx.plevel = l;
        }
        if (P[l].num_rows != v.n || P[l].num_cols <= 0) { rc = AMGT_ERR_INVALID; goto fail; }
        if (!cb) {
            v.prec = amgt_precision_for_level(l);
            v.prec_transfer = amgt_precision_for_level(l + 1);
        }
        // A P waits for P_l only (converted now if no call issued it),
        // R (A P) for R_l (transposed now if A P's call did not)
        if (nx.P && (rc = prepare_interp(&nx))) goto fail;
        if (cudaStreamWaitEvent(s, nx.p_ready[l % 2], 0) != cudaSuccess) {
            rc = AMGT_ERR_CUDA;
            goto fail;
        }
        pm.mark(1, s);
        const int gp = h->prm.galerkin_by_level ? v.prec : AMGT_DOUBLE;
        amgt_bsr AP{};
        if (l + 1 < L - 1 && !cb) {
            nx.P = &P[l + 1];
            nx.Pb = &h->lv[l + 1].P;
            nx.PRb = &h->lv[l + 1].R;
            nx.pslot = (l + 1) % 2;
            nx.plevel = l + 1;
        }
        if ((rc = spgemm_impl(gp, &v.A, &v.P, &AP, nullptr, stream, prepare_interp, &nx))) goto fail;
        if (nx.Tb == &v.P && (rc = transpose_pending(&nx))) {
            amgt_bsr_free(&AP, stream);
            goto fail;
        }
        if (cudaStreamWaitEvent(s, nx.r_ready[l % 2], 0) != cudaSuccess) {
            amgt_bsr_free(&AP, stream);
            rc = AMGT_ERR_CUDA;
            goto fail;
        }
        {
            // A_{l+1} used in fp64 or fp32 is checked for exact fp16 storage
            // by the numeric pass, which also writes the fp32 shadow of an
            // fp64 product for a level used in fp32
            CvtFuse fz;
            const int np = amgt_precision_for_level(l + 1);
            fz.want16 = h->prm.exact_storage && !cb &&
                        ((gp == AMGT_DOUBLE && (np == AMGT_DOUBLE || np == AMGT_FLOAT)) ||
                         (gp == AMGT_FLOAT && np == AMGT_FLOAT));
            fz.want32 = fz.want16 && gp == AMGT_DOUBLE && np == AMGT_FLOAT;
            fz.flags = xflags + 3 * (l + 1);
            rc = spgemm_impl(gp, &v.R, &AP, &h->lv[l + 1].A, nullptr, stream, nullptr, nullptr,
                             fz.want16 ? &fz : nullptr);
            if (!rc && fz.fused) fused16[3 * (l + 1)] = 1;
        }
        amgt_bsr_free(&AP, stream);
        if (rc) goto fail;
        h->lv[l + 1].n = h->lv[l + 1].A.row;
        pm.mark(2, s);
    }
    if (cb) {
        // the coarsest level's precision when the level cap ended the loop,
        // and each transfer at its coarse level's precision
        if (L == num_interp + 1 || (h->prm.max_levels > 0 && L == h->prm.max_levels)) {
            int prec_l = AMGT_DOUBLE;
            amgt_csr unused{};
            if (cb(L - 1, &h->lv[L - 1].A, &unused, &prec_l, cb_ctx) < 0 || prec_l < AMGT_DOUBLE ||
                prec_l > AMGT_BF16) {
                rc = AMGT_ERR_INVALID;
                goto fail;
            }
            h->lv[L - 1].prec = prec_l;
        }
        for (int l = 0; l + 1 < L; ++l) h->lv[l].prec_transfer = h->lv[l + 1].prec;
    } else {
        h->lv[L - 1].prec = amgt_precision_for_level(L - 1);
    }
    // coarsest: dense diagonal blocks (one, or one per system of a batch)
    // and their inverses, on the GPU (Gauss-Jordan); the singularity flag is
    // read back with the exactness bits below
    h->nc = h->lv[L - 1].n;
    if (h->nc > h->prm.max_coarse_rows) {
        rc = AMGT_ERR_TOO_LARGE;
        goto fail;
    }
    {
        std::vector<int> boff{0};
        if (sys_rows)
            for (const auto &r : *sys_rows) boff.push_back(boff.back() + r[L - 1]);
        else
            boff.push_back(h->nc);
        if (boff.back() != h->nc) {
            rc = AMGT_ERR_INVALID;
            goto fail;
        }
        const int nb = (int)boff.size() - 1;
        std::vector<long long> doff{0};
        std::vector<int> rblk(h->nc);
        for (int b = 0; b < nb; ++b) {
            const long long w = boff[b + 1] - boff[b];
            doff.push_back(doff.back() + w * w);
            for (int r = boff[b]; r < boff[b + 1]; ++r) rblk[r] = b;
        }
        const size_t nn = (size_t)doff.back();
        int *bad = reinterpret_cast<int *>(xflags + 3 * num_interp + 2);
        h->ncb = nb;
        if ((rc = alloc_n(&dense, nn, s)) || (rc = alloc_n(&h->coarse_inv, nn, s)) ||
            (rc = alloc_n(&h->cb_off, (size_t)nb + 1, s)) || (rc = alloc_n(&h->cb_doff, (size_t)nb + 1, s)) ||
            (rc = alloc_n(&h->row_blk, (size_t)h->nc, s)))
            goto fail;
        if (cudaMemcpyAsync(h->cb_off, boff.data(), sizeof(int) * boff.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(h->cb_doff, doff.data(), sizeof(long long) * doff.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(h->row_blk, rblk.data(), sizeof(int) * rblk.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemsetAsync(dense, 0, sizeof(double) * nn, s) != cudaSuccess ||
            cudaMemsetAsync(xflags + 3 * num_interp + 2, 0, sizeof(int64_t), s) != cudaSuccess) {
            rc = AMGT_ERR_CUDA;
            goto fail;
        }
        AMGT_LAUNCH(bsr_to_dense_kernel, grid_for(256, h->nc, h->sm_count, 8), 256, 0, s, h->nc, h->nc,
                    h->lv[L - 1].A.blcPtr, h->lv[L - 1].A.blcIdx, h->lv[L - 1].A.blcVal, (const int *)h->row_blk,
                    (const int *)h->cb_off, (const long long *)h->cb_doff, dense);
        // the flag slot after the last operator's (never a P or R slot: the
        // coarsest level has none) holds the singular mark
        if (nb == 1) {
            if ((rc = dense_invert(h->nc, dense, h->coarse_inv, bad, h->sm_count, s))) goto fail;
        } else {
            int *used = nullptr, *piv = nullptr;
            double *rowp = nullptr, *colc = nullptr;
            if (!(rc = alloc_n(&used, h->nc, s)) && !(rc = alloc_n(&piv, h->nc, s)) &&
                !(rc = alloc_n(&rowp, h->nc, s)) && !(rc = alloc_n(&colc, h->nc, s))) {
                count_launch();
                gj_blocks_kernel<<<nb, 1024, 0, s>>>(h->cb_off, h->cb_doff, dense, h->coarse_inv, used, piv, rowp,
                                                     colc, bad);
                if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
            }
            free_ptr(used, s);
            free_ptr(piv, s);
            free_ptr(rowp, s);
            free_ptr(colc, s);
            if (rc) goto fail;
        }
        free_ptr(dense, s);
    }
    // exact narrow storage of the operators used in fp64 (level 0, fp64
    // levels and transfers): one value check each, one read-back per 15
    if (h->prm.exact_storage) {
        std::vector<std::pair<amgt_bsr *, int>> mats;  // operator, flag slot
        // fp32 operators too: one whose values fp16 holds is read from the
        // fp16 shadow (the same fp32 sums at half the bytes)
        for (int l = 0; l < L; ++l) {
            if (l == 0 || h->lv[l].prec == AMGT_DOUBLE || h->lv[l].prec == AMGT_FLOAT)
                mats.push_back({&h->lv[l].A, 3 * l});
            if (l < L - 1 && (h->lv[l].prec_transfer == AMGT_DOUBLE || h->lv[l].prec_transfer == AMGT_FLOAT)) {
                mats.push_back({&h->lv[l].P, 3 * l + 1});
                mats.push_back({&h->lv[l].R, 3 * l + 2});
            }
        }
        std::vector<char> own16(fused16.size(), 0);
        for (size_t i = 0; i < mats.size() && !rc; ++i) {
            const int slot = mats[i].second;
            if (fused16[slot]) {
                own16[slot] = 1;  // checked by its conversion, which allocated the shadow
                continue;
            }
            bool o = false;
            rc = bsr_exact_check(mats[i].first, xflags + slot, &o, s, h->sm_count);
            own16[slot] = o;
        }
        std::vector<int64_t> f(fused16.size(), 0);
        for (size_t i0 = 0; i0 < f.size() && !rc; i0 += 63) {
            const int k = (int)std::min<size_t>(63, f.size() - i0);
            const int64_t *hf = nullptr;
            if ((rc = read_back(xflags + i0, k, s, &hf))) break;
            for (int i = 0; i < k; ++i) f[i0 + i] = hf[i];  // the pinned slots are reused by later calls
        }
        for (size_t i = 0; i < mats.size() && !rc; ++i) {
            const int slot = mats[i].second;
            const int fs = (slot % 3 == 2 && fused16[slot]) ? slot - 1 : slot;  // R_l carried P_l's shadow
            rc = bsr_exact_apply(mats[i].first, f[fs], own16[slot] != 0, s);
        }
        if (rc) goto fail;
    }
    // smoother data, shadows, work vectors
    for (int l = 0; l < L; ++l) {
        Level &v = h->lv[l];
        if (!(l == 0 && l1_fused0)) {
            if (!v.inv_l1 && (rc = alloc_n(&v.inv_l1, v.n, s))) goto fail;
            if ((rc = bsr_l1_norms(&v.A, v.inv_l1, 1, s, h->sm_count))) goto fail;
        }
        if ((rc = level_shadow(&v.A, v.prec, stream))) goto fail;
        if (l == 0 && (rc = level_shadow(&v.A, h->prm.smooth_prec0, stream))) goto fail;
        if (l == 0 && fgm && (rc = level_shadow(&v.A, h->prm.inner_prec0, stream))) goto fail;
        if (l < L - 1) {
            if ((rc = level_shadow(&v.P, v.prec_transfer, stream))) goto fail;
            if ((rc = level_shadow(&v.R, v.prec_transfer, stream))) goto fail;
        }
        if (h->prm.packed) {
            // level 0: fp64 for the residual and the Krylov product, the
            // smoother at smooth_prec0; coarser levels at their precision
            if ((rc = amgt_bsr_pack(&v.A, l == 0 ? AMGT_DOUBLE : v.prec, &v.pA, stream))) goto fail;
            if (l == 0 && (rc = amgt_bsr_pack(&v.A, h->prm.smooth_prec0, &v.pAs, stream))) goto fail;
            if (l < L - 1 && ((rc = amgt_bsr_pack(&v.P, v.prec_transfer, &v.pP, stream)) ||
                              (rc = amgt_bsr_pack(&v.R, v.prec_transfer, &v.pR, stream))))
                goto fail;
        }
        if ((rc = alloc_n(&v.u, v.n, s)) || (rc = alloc_n(&v.t, v.n, s))) goto fail;
        if (l > 0 && ((rc = alloc_n(&v.f, v.n, s)) || (rc = alloc_n(&v.s, v.n, s)))) goto fail;
    }
    // coarsest: the inverse's singularity mark (one read-back)
    {
        const int64_t *hf = nullptr;
        if ((rc = read_back(xflags + 3 * num_interp + 2, 1, s, &hf))) goto fail;
        if (hf[0] != 0) {
            rc = AMGT_ERR_INVALID;  // singular coarsest operator
            goto fail;
        }
        if (L == 1) h->lv[L - 1].s = nullptr;
    }
    // Krylov vectors and scalars
    h->n0 = h->lv[0].n;
    h->grid0 = h->prm.packed ? pbsr_grid(&h->lv[0].pA, h->sm_count) : epi_grid(&h->lv[0].A, h->sm_count);
    if ((rc = alloc_n(&h->r, h->n0, s)) || (rc = alloc_n(&h->z, h->n0, s)) || (rc = alloc_n(&h->p, h->n0, s)) ||
        (rc = alloc_n(&h->q, h->n0, s)) || (rc = alloc_n(&h->scal, S_NSCAL, s)) ||
        (rc = alloc_n(&h->part, std::max(h->grid0, kDotGrid), s)) || (rc = alloc_n(&h->loop_it, 1, s)) ||
        (rc = alloc_n(&h->loop_rr, (size_t)h->prm.max_iter + 1, s)))
        goto fail;
    if (fgm) {
        const int m = h->prm.restart;
        if ((rc = alloc_n(&h->gmV, (size_t)(m + 1) * h->n0, s)) || (rc = alloc_n(&h->gmZ, (size_t)m * h->n0, s)) ||
            (rc = alloc_n(&h->gm, (size_t)GmLayout{m}.size(), s)) || (rc = alloc_n(&h->gm_vin, h->n0, s)) ||
            (rc = alloc_n(&h->gm_zout, h->n0, s)) || (rc = alloc_n(&h->gm_w, h->n0, s)) ||
            (rc = alloc_n(&h->gm_part, (size_t)(m + 1) * kDotGrid, s)) || (rc = alloc_n(&h->gm_j, 1, s)))
            goto fail;
        if (cudaMemsetAsync(h->gm, 0, sizeof(double) * GmLayout{m}.size(), s) != cudaSuccess) {
            rc = AMGT_ERR_CUDA;
            goto fail;
        }
    }
    AMGT_CUDA_TRY(cudaMemsetAsync(h->scal, 0, sizeof(double) * S_NSCAL, s));
    // every host read-back slot of the solvers in one pinned block, so that
    // no solve allocates: 8 scalars, the multi-right-hand-side solve's 160,
    // and the loop's iteration count and max_iter + 1 residual norms
    {
        void *pb = nullptr;
        if ((rc = pinned_get(sizeof(double) * (8 + 160 + (size_t)h->prm.max_iter + 2), &pb))) goto fail;
        h->pinned = static_cast<double *>(pb);
    }
    h->mr_pinned = h->pinned + 8;
    h->loop_pinned = h->pinned + 168;
    free_ptr(xflags, s);
    pm.mark(3, s);
    pm.accumulate(h->setup_ms);  // waits for the setup's last work
    if (nx.s2) cudaStreamDestroy(nx.s2);
    for (int i = 0; i < 2; ++i) {
        if (nx.p_ready[i]) cudaEventDestroy(nx.p_ready[i]);
        if (nx.r_ready[i]) cudaEventDestroy(nx.r_ready[i]);
    }
    *out = h;
    return AMGT_OK;
fail:
    if (nx.s2) {  // its conversions may still use arrays the handle frees
        cudaStreamSynchronize(nx.s2);
        cudaStreamDestroy(nx.s2);
    }
    cudaStreamSynchronize(s);  // no kernel of this setup in flight
    if (xflags) free_ptr(xflags, s);
    if (dense) free_ptr(dense, s);
    for (int i = 0; i < 2; ++i) {
        if (nx.p_ready[i]) cudaEventDestroy(nx.p_ready[i]);
        if (nx.r_ready[i]) cudaEventDestroy(nx.r_ready[i]);
    }
    cudaGetLastError();
    destroy_handle(h, s);
    return rc;
}

extern "C" {

int amgt_amg_solve(amgt_amg *h, const double *b, double *x, int *iterations, double *rel_res, amgt_stream_t stream)
{
    if (!h || !b || !x) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (h->prm.solver == AMGT_SOLVER_FGMRES_IR) return fgmres_ir_solve(h, b, x, iterations, rel_res, s);
    Level &v0 = h->lv[0];
    h->hist.clear();
    // r = b - A x, ||b||^2, ||r||^2
    AMGT_TRY(spmv_residual(AMGT_DOUBLE, &v0.A, b, x, h->r, s, h->sm_count));
    AMGT_TRY(dot(h, b, b, S_BB, OP_STORE, s));
    AMGT_TRY(dot(h, h->r, h->r, S_RR, OP_STORE, s));
    AMGT_CUDA_TRY(cudaMemcpyAsync(h->pinned, h->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaStreamSynchronize(s));
    const double bb = h->pinned[S_BB];
    double rel = bb > 0 ? std::sqrt(h->pinned[S_RR] / bb) : 0.0;
    h->hist.push_back(rel);
    int it = 0;
    if (rel > h->prm.tol) {
        AMGT_TRY(cycle(h, h->r, h->z, s));
        AMGT_TRY(dot(h, h->r, h->z, S_RZ, OP_STORE, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(h->p, h->z, sizeof(double) * h->n0, cudaMemcpyDeviceToDevice, s));
        uint64_t per_iter = 0;
        if (h->prm.use_graph && !h->loop_failed) {
            // one launch for the whole loop; one read-back at its end
            const int lrc = build_loop_graph(h, x);
            per_iter = h->loop_launches;
            if (lrc == AMGT_OK) {
                AMGT_CUDA_TRY(cudaMemsetAsync(h->loop_it, 0, sizeof(int), s));
                AMGT_CUDA_TRY(cudaGraphLaunch(h->loop, s));
                AMGT_CUDA_TRY(cudaMemcpyAsync(h->loop_pinned, h->loop_it, sizeof(int), cudaMemcpyDeviceToHost, s));
                AMGT_CUDA_TRY(cudaMemcpyAsync(h->loop_pinned + 1, h->loop_rr + 1, sizeof(double) * h->prm.max_iter,
                                              cudaMemcpyDeviceToHost, s));
                AMGT_CUDA_TRY(cudaStreamSynchronize(s));
                it = *reinterpret_cast<const int *>(h->loop_pinned);
                for (int k = 1; k <= it; ++k) {
                    rel = std::sqrt(std::max(0.0, h->loop_pinned[k]) / bb);
                    h->hist.push_back(rel);
                }
                for (int k = 0; k < it; ++k)
                    for (uint64_t j = 0; j < per_iter; ++j) count_launch();
                if (iterations) *iterations = it;
                if (rel_res) *rel_res = rel;
                return AMGT_OK;
            }
            if (lrc != AMGT_ERR_CUDA) return lrc;
            h->loop_failed = true;  // the runtime did not take the loop graph: one graph per iteration
        }
        if (h->prm.use_graph) {
            AMGT_TRY(build_graph(h, x));
            per_iter = h->graph_launches;
        }
        for (it = 1; it <= h->prm.max_iter; ++it) {
            if (h->prm.use_graph) {
                AMGT_CUDA_TRY(cudaGraphLaunch(h->graph, s));
                for (uint64_t k = 0; k < per_iter; ++k) count_launch();
            } else {
                AMGT_TRY(pcg_iteration(h, x, s));
            }
            AMGT_CUDA_TRY(cudaStreamSynchronize(s));
            rel = std::sqrt(std::max(0.0, h->pinned[0]) / bb);
            h->hist.push_back(rel);
            if (rel <= h->prm.tol) break;
        }
        if (it > h->prm.max_iter) it = h->prm.max_iter;
    }
    if (iterations) *iterations = it;
    if (rel_res) *rel_res = rel;
    return AMGT_OK;
}

int amgt_amg_num_levels(const amgt_amg *h) { return h ? (int)h->lv.size() : 0; }

int amgt_amg_level(const amgt_amg *h, int level, amgt_bsr *A_view, int *prec)
{
    if (!h || level < 0 || level >= (int)h->lv.size()) return AMGT_ERR_INVALID;
    if (A_view) *A_view = h->lv[level].A;
    if (prec) *prec = h->lv[level].prec;
    return AMGT_OK;
}

int amgt_amg_setup_times(const amgt_amg *h, double *ms)
{
    if (!h || !ms) return AMGT_ERR_INVALID;
    for (int i = 0; i < 4; ++i) ms[i] = h->setup_ms[i];
    return AMGT_OK;
}

int amgt_amg_residual_history(const amgt_amg *h, double *hist, int cap)
{
    if (!h) return -1;
    const int n = (int)h->hist.size();
    for (int i = 0; i < n && i < cap && hist; ++i) hist[i] = h->hist[i];
    return n;
}

int amgt_amg_destroy(amgt_amg *h, amgt_stream_t stream)
{
    destroy_handle(h, (cudaStream_t)stream);
    return AMGT_OK;
}

}  // extern "C"
