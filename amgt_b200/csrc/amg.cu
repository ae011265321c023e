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

#include "amgt_internal.cuh"

namespace amgt {

constexpr int kDotGrid = 1184;  // 8 x 148 SMs
constexpr int kDotThreads = 256;

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

// u = M f with M dense (row-major, nc x nc), one warp per row
__global__ void dense_mv_kernel(int nc, const double *__restrict__ M, const double *__restrict__ f,
                                double *__restrict__ u)
{
    grid_dependency_wait();
    const int lane = threadIdx.x & 31;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nc; row += (gridDim.x * blockDim.x) >> 5) {
        double s = 0.0;
        for (int j = lane; j < nc; j += 32) s += M[(long long)row * nc + j] * f[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) u[row] = s;
    }
}

// mBSR -> dense (row-major), for the coarsest operator
__global__ void bsr_to_dense_kernel(int m, int n, const int *__restrict__ ptr, const int *__restrict__ idx,
                                    const double *__restrict__ val, double *__restrict__ D)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        const int b = row >> 2, q = row & 3;
        for (int k = ptr[b]; k < ptr[b + 1]; ++k)
            for (int c = 0; c < 4; ++c) {
                const int col = 4 * idx[k] + c;
                if (col < n) D[(long long)row * n + col] = val[16LL * k + 4 * q + c];
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

struct Level {
    amgt_bsr A{}, P{}, R{};
    amgt_pbsr pA{}, pAs{}, pP{}, pR{};  // packed: cycle operator, level-0 smoother, transfers
    double *inv_l1 = nullptr;
    double *f = nullptr, *u = nullptr, *t = nullptr, *s = nullptr;
    int n = 0;
    int prec = AMGT_DOUBLE;           // smoother SpMVs on A_l
    int prec_transfer = AMGT_DOUBLE;  // R_l / P_l SpMVs
};

}  // namespace amgt

// Opaque handle of the C ABI.
struct amgt_amg {
    std::vector<amgt::Level> lv;
    amgt_amg_params prm;
    double *coarse_inv = nullptr;
    int nc = 0;
    long long n0 = 0;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    double *scal = nullptr, *part = nullptr;
    double *pinned = nullptr;  // host: ||r||^2 read-back
    int sm_count = 0, grid0 = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    const double *graph_b = nullptr;
    double *graph_xout = nullptr;
    // the whole iteration loop as one graph (a conditional while node); the
    // loop's iteration count and ||r||^2 per iteration stay on the device
    cudaGraphExec_t loop = nullptr;
    double *loop_xout = nullptr;
    bool loop_failed = false;
    int *loop_it = nullptr;     // device: iterations done
    double *loop_rr = nullptr;  // device: ||r||^2 after iteration k, k = 1 .. max_iter
    double *loop_pinned = nullptr;
    uint64_t graph_launches = 0, loop_launches = 0;  // our kernels per iteration in each graph
    double setup_ms[5] = {0, 0, 0, 0, 0};
    std::vector<double> hist;
};

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
    if (h->graph_stream) cudaStreamDestroy(h->graph_stream);
    free_ptr(h->loop_it, s);
    free_ptr(h->loop_rr, s);
    if (h->loop_pinned) cudaFreeHost(h->loop_pinned);
    for (auto &v : h->lv) free_level(v, s);
    free_ptr(h->coarse_inv, s);
    free_ptr(h->r, s);
    free_ptr(h->z, s);
    free_ptr(h->p, s);
    free_ptr(h->q, s);
    free_ptr(h->scal, s);
    free_ptr(h->part, s);
    if (h->pinned) cudaFreeHost(h->pinned);
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
    AMGT_TRY(bsr_transpose_impl(nx->Tb, nx->TRb, (amgt_stream_t)nx->s2, with16));
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
    f.want16 = nx->exact && amgt_precision_for_level(nx->plevel + 1) == AMGT_DOUBLE;
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

// z = M f: one V(1,1) cycle
int cycle(amgt_amg *h, const double *rhs0, double *out0, cudaStream_t s)
{
    auto &lv = h->lv;
    const int L = (int)lv.size();
    const double w = h->prm.relax_weight;
    const bool pk = h->prm.packed != 0;
    for (int l = 0; l < L - 1; ++l) {
        Level &v = lv[l];
        const double *f = (l == 0) ? rhs0 : v.f;
        AMGT_LAUNCH_PDL(jacobi_zero_kernel, grid_n(h, v.n), 256, 0, s, (long long)v.n, f, v.inv_l1, w, v.u);
        if (pk) {
            AMGT_TRY(pbsr_residual(&v.pA, f, v.u, v.t, s, h->sm_count));
            AMGT_TRY(pbsr_spmv(&v.pR, 1.0, v.t, 0.0, lv[l + 1].f, s, h->sm_count));
        } else {
            AMGT_TRY(spmv_residual(l == 0 ? AMGT_DOUBLE : v.prec, &v.A, f, v.u, v.t, s, h->sm_count));
            AMGT_TRY(amgt_spmv(v.prec_transfer, 1.0, &v.R, v.t, 0.0, lv[l + 1].f, (amgt_stream_t)s));
        }
    }
    Level &c = lv[L - 1];
    const double *fc = (L == 1) ? rhs0 : c.f;
    double *uc = (L == 1) ? out0 : c.s;
    AMGT_LAUNCH_PDL(dense_mv_kernel, grid_for(8, c.n, h->sm_count, 8), 256, 0, s, c.n, h->coarse_inv, fc, uc);
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
    if (!h->loop_pinned) AMGT_CUDA_TRY(cudaMallocHost(&h->loop_pinned, sizeof(double) * (h->prm.max_iter + 2)));
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

}  // namespace

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
}

int amgt_amg_setup(const amgt_csr *A, int num_interp, const amgt_csr *P, const amgt_amg_params *params,
                   amgt_amg **out, amgt_stream_t stream)
{
    if (!A || !out || num_interp < 0 || (num_interp > 0 && !P) || A->num_rows != A->num_cols || A->num_rows <= 0)
        return AMGT_ERR_INVALID;
    *out = nullptr;
    // the loop graph's body runs at least once and keeps max_iter + 1
    // residual norms: max_iter must be >= 1 (and bounded, so that its
    // buffers stay small)
    if (params && (params->max_iter < 1 || params->max_iter > 1000000 || !(params->tol >= 0.0) ||
                   params->max_coarse_rows < 1 || params->max_coarse_rows > 16384))
        return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    amgt_amg *h = new amgt_amg();
    if (params) h->prm = *params;
    else amgt_amg_default_params(&h->prm);
    if (h->prm.smooth_prec0 < AMGT_DOUBLE || h->prm.smooth_prec0 > AMGT_BF16) h->prm.smooth_prec0 = AMGT_DOUBLE;
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
    nx.exact = h->prm.exact_storage != 0;
    nx.xflags = xflags;
    nx.fused16 = &fused16;
    // hierarchy: P_0 converted while A's conversion runs, R_l transposed
    // and P_{l+1} converted while level l's A P runs
    if (L > 1) {
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
        if (P[l].num_rows != v.n || P[l].num_cols <= 0) { rc = AMGT_ERR_INVALID; goto fail; }
        v.prec = amgt_precision_for_level(l);
        v.prec_transfer = amgt_precision_for_level(l + 1);
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
        if (l + 1 < L - 1) {
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
            // A_{l+1} in fp64 is checked for exact storage by the numeric pass
            CvtFuse fz;
            fz.want16 = h->prm.exact_storage && gp == AMGT_DOUBLE &&
                        amgt_precision_for_level(l + 1) == AMGT_DOUBLE;
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
    h->lv[L - 1].prec = amgt_precision_for_level(L - 1);
    // coarsest: dense form and its inverse, on the GPU (Gauss-Jordan); the
    // singularity flag is read back with the exactness bits below
    h->nc = h->lv[L - 1].n;
    if (h->nc > h->prm.max_coarse_rows) {
        rc = AMGT_ERR_TOO_LARGE;
        goto fail;
    }
    {
        const size_t nn = (size_t)h->nc * h->nc;
        if ((rc = alloc_n(&dense, nn, s)) || (rc = alloc_n(&h->coarse_inv, nn, s))) goto fail;
        if (cudaMemsetAsync(dense, 0, sizeof(double) * nn, s) != cudaSuccess ||
            cudaMemsetAsync(xflags + 3 * num_interp + 2, 0, sizeof(int64_t), s) != cudaSuccess) {
            rc = AMGT_ERR_CUDA;
            goto fail;
        }
        AMGT_LAUNCH(bsr_to_dense_kernel, grid_for(256, h->nc, h->sm_count, 8), 256, 0, s, h->nc, h->nc,
                    h->lv[L - 1].A.blcPtr, h->lv[L - 1].A.blcIdx, h->lv[L - 1].A.blcVal, dense);
        // the flag slot after the last operator's (never a P or R slot: the
        // coarsest level has none) holds the singular mark
        if ((rc = dense_invert(h->nc, dense, h->coarse_inv, reinterpret_cast<int *>(xflags + 3 * num_interp + 2),
                               h->sm_count, s)))
            goto fail;
        free_ptr(dense, s);
    }
    // exact narrow storage of the operators used in fp64 (level 0, fp64
    // levels and transfers): one value check each, one read-back per 15
    if (h->prm.exact_storage) {
        std::vector<std::pair<amgt_bsr *, int>> mats;  // operator, flag slot
        for (int l = 0; l < L; ++l) {
            if (l == 0 || h->lv[l].prec == AMGT_DOUBLE) mats.push_back({&h->lv[l].A, 3 * l});
            if (l < L - 1 && h->lv[l].prec_transfer == AMGT_DOUBLE) {
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
        if ((rc = amgt_bsr_make_shadow(&v.A, v.prec, stream))) goto fail;
        if (l == 0 && (rc = amgt_bsr_make_shadow(&v.A, h->prm.smooth_prec0, stream))) goto fail;
        if (l < L - 1) {
            if ((rc = amgt_bsr_make_shadow(&v.P, v.prec_transfer, stream))) goto fail;
            if ((rc = amgt_bsr_make_shadow(&v.R, v.prec_transfer, stream))) goto fail;
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
    AMGT_CUDA_TRY(cudaMemsetAsync(h->scal, 0, sizeof(double) * S_NSCAL, s));
    AMGT_CUDA_TRY(cudaMallocHost(&h->pinned, sizeof(double) * 4));
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

int amgt_amg_solve(amgt_amg *h, const double *b, double *x, int *iterations, double *rel_res, amgt_stream_t stream)
{
    if (!h || !b || !x) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
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
