// amgt_amg_solve_multi: many right-hand sides on one hierarchy at once.
//
// X and B are row-major n x nv (nv <= 32): x_i of right-hand side v at
// X[i * nv + v], the layout of amgt_spmm_rm, so that every operator of the
// cycle is one SpMM over all right-hand sides (one pass over the operator's
// values instead of nv passes).  Solve:
//   refinement (fp64)   R = B - A X with fp64 values on the CUDA cores;
//                       per column ||R_v|| / ||B_v||; stop when every
//                       column is at tol;
//   correction          A D = R by PCG in lockstep over the columns (each
//                       column its own alpha, beta, and its own stop at
//                       inner_tol * ||R_v||), preconditioned by one V(1,1)
//                       cycle; every operator through amgt_spmm_rm at its
//                       level's precision (fp32 / fp16 / bf16 levels on the
//                       tensor cores; level 0 at inner_prec0); X += D.
// The correction's iteration loop is one CUDA graph launch (a conditional
// while node whose body ends with the per-column convergence test).
// Kernels use a lane per right-hand side and warps striding over rows, so
// the vector passes are coalesced (nv = 32: 256 bytes per warp per row).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "amg_handle.cuh"

namespace amgt {

int spmm_rowmajor(int prec, int kind, int wpc, const amgt_bsr *A, double alpha, const double *X, int nvec,
                  double beta, double *Y, cudaStream_t s, int sm_count);

// per-column scalars: scal[slot * 32 + v]
enum { MS_BB = 0, MS_RR = 1, MS_RZ = 2, MS_PQ = 3, MS_ALPHA = 4, MS_BETA = 5, MS_RR0 = 6, MS_ACTIVE = 7,
       MS_NSLOT = 8 };
enum { MOP_STORE = 0, MOP_ALPHA = 1, MOP_BETA = 2, MOP_RR_TEST = 3, MOP_START = 4 };

struct MultiRhsLevel {
    double *f = nullptr, *u = nullptr, *t = nullptr, *s = nullptr;  // n_l x nv
};

struct MultiRhs {
    int nv = 0;
    std::vector<MultiRhsLevel> lv;
    double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *d = nullptr, *res = nullptr;
    double *scal = nullptr, *part = nullptr;
    int *cnt = nullptr;   // device: [32] iterations per column, [32] total inner iterations
    double *pinned = nullptr;  // host, the handle's: 2 * 32 norms, counts, the loop flag
    cudaGraphExec_t loop = nullptr;
    bool loop_failed = false;
    uint64_t loop_launches = 0;
};

void free_multi_rhs(MultiRhs *mr, cudaStream_t s)
{
    if (!mr) return;
    if (mr->loop) cudaGraphExecDestroy(mr->loop);
    for (auto &l : mr->lv) {
        free_ptr(l.f, s);
        free_ptr(l.u, s);
        free_ptr(l.t, s);
        free_ptr(l.s, s);
    }
    free_ptr(mr->r, s);
    free_ptr(mr->z, s);
    free_ptr(mr->p, s);
    free_ptr(mr->q, s);
    free_ptr(mr->d, s);
    free_ptr(mr->res, s);
    free_ptr(mr->scal, s);
    free_ptr(mr->part, s);
    free_ptr(mr->cnt, s);
    delete mr;
}

constexpr int kMvThreads = 256;
constexpr int kMvGrid = 592;  // 4 x 148 SMs

#define MV_LOOP(rowvar, nrows)                                                                     \
    const int lane = threadIdx.x & 31;                                                             \
    const bool live = lane < nv;                                                                   \
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;                  \
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;                                 \
    for (long long rowvar = gw; rowvar < (nrows); rowvar += nw)

// partials of a_v . b_v per CTA: part[cta * 32 + v]
__global__ void __launch_bounds__(kMvThreads) mv_dot_kernel(long long n, int nv, const double *__restrict__ a,
                                                           const double *__restrict__ b, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kMvThreads / 32][32];
    double s = 0.0;
    MV_LOOP(r, n)
    {
        if (live) s += a[r * nv + lane] * b[r * nv + lane];
    }
    sred[threadIdx.x >> 5][lane] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = 0.0;
        for (int w = 0; w < kMvThreads / 32; ++w) t += sred[w][threadIdx.x];
        part[blockIdx.x * 32 + threadIdx.x] = t;
    }
}

// sums the partials per column (warp v, fixed order) and applies op
__global__ void __launch_bounds__(1024) mv_reduce_kernel(const double *__restrict__ part, int np, int nv,
                                                        double *__restrict__ scal, int slot, int op,
                                                        double inner_tol)
{
    grid_dependency_wait();
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (v >= nv) return;
    double t = 0.0;
    for (int k = lane; k < np; k += 32) t += part[k * 32 + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
    if (lane != 0) return;
    double *sc = scal;
    if (op == MOP_STORE) {
        sc[slot * 32 + v] = t;
    } else if (op == MOP_ALPHA) {
        sc[MS_PQ * 32 + v] = t;
        sc[MS_ALPHA * 32 + v] = (sc[MS_ACTIVE * 32 + v] != 0.0 && t != 0.0) ? sc[MS_RZ * 32 + v] / t : 0.0;
    } else if (op == MOP_BETA) {
        const double rz_old = sc[MS_RZ * 32 + v];
        sc[MS_BETA * 32 + v] = rz_old != 0.0 ? t / rz_old : 0.0;
        sc[MS_RZ * 32 + v] = t;
    } else if (op == MOP_RR_TEST) {
        sc[MS_RR * 32 + v] = t;
        if (!(sqrt(fmax(t, 0.0)) > inner_tol * sqrt(sc[MS_RR0 * 32 + v]))) sc[MS_ACTIVE * 32 + v] = 0.0;
    } else {  // MOP_START: rr0 = ||r||^2, a column with r = 0 starts inactive
        sc[MS_RR0 * 32 + v] = t;
        sc[MS_RR * 32 + v] = t;
        sc[MS_ACTIVE * 32 + v] = (t > 0.0 && sc[MS_ACTIVE * 32 + v] != 0.0) ? 1.0 : 0.0;
    }
}

// d += alpha_v p; r -= alpha_v q; partials of r_v . r_v
__global__ void __launch_bounds__(kMvThreads) mv_axpy2_dot_kernel(long long n, int nv,
                                                                 const double *__restrict__ scal,
                                                                 const double *__restrict__ p,
                                                                 const double *__restrict__ q, double *__restrict__ d,
                                                                 double *__restrict__ r, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kMvThreads / 32][32];
    const double alpha = (threadIdx.x & 31) < nv ? scal[MS_ALPHA * 32 + (threadIdx.x & 31)] : 0.0;
    double s = 0.0;
    MV_LOOP(i, n)
    {
        if (!live) continue;
        const long long e = i * nv + lane;
        d[e] += alpha * p[e];
        const double ri = r[e] - alpha * q[e];
        r[e] = ri;
        s += ri * ri;
    }
    sred[threadIdx.x >> 5][lane] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = 0.0;
        for (int w = 0; w < kMvThreads / 32; ++w) t += sred[w][threadIdx.x];
        part[blockIdx.x * 32 + threadIdx.x] = t;
    }
}

// p = z + beta_v p
__global__ void mv_xpby_kernel(long long n, int nv, const double *__restrict__ z, const double *__restrict__ scal,
                               double *__restrict__ p)
{
    grid_dependency_wait();
    const double beta = (threadIdx.x & 31) < nv ? scal[MS_BETA * 32 + (threadIdx.x & 31)] : 0.0;
    MV_LOOP(i, n)
    {
        if (live) p[i * nv + lane] = z[i * nv + lane] + beta * p[i * nv + lane];
    }
}

// u = w f .* inv_l1 (smoothing from zero)
__global__ void mv_jacobi_zero_kernel(long long n, int nv, const double *__restrict__ f,
                                      const double *__restrict__ inv_l1, double w, double *__restrict__ u)
{
    grid_dependency_wait();
    MV_LOOP(i, n)
    {
        if (live) u[i * nv + lane] = w * f[i * nv + lane] * inv_l1[i];
    }
}

// out = u + w t .* inv_l1 (t = f - A u)
__global__ void mv_jacobi_update_kernel(long long n, int nv, const double *__restrict__ u,
                                        const double *__restrict__ t, const double *__restrict__ inv_l1, double w,
                                        double *__restrict__ out)
{
    grid_dependency_wait();
    MV_LOOP(i, n)
    {
        if (live) out[i * nv + lane] = u[i * nv + lane] + w * t[i * nv + lane] * inv_l1[i];
    }
}

__global__ void mv_copy_kernel(long long count, const double *__restrict__ a, double *__restrict__ b)
{
    grid_dependency_wait();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        b[e] = a[e];
}

__global__ void mv_add_kernel(long long count, const double *__restrict__ a, double *__restrict__ b)
{
    grid_dependency_wait();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        b[e] += a[e];
}

// U = M F for the coarsest inverse M (dense diagonal blocks, as
// dense_mv_kernel reads them): warp per row, lane per column
__global__ void mv_dense_kernel(int nc, int nv, const int *__restrict__ row_blk, const int *__restrict__ cb_off,
                                const long long *__restrict__ cb_doff, const double *__restrict__ M,
                                const double *__restrict__ f, double *__restrict__ u)
{
    grid_dependency_wait();
    MV_LOOP(row, nc)
    {
        const int b = row_blk[row], o = cb_off[b], nb = cb_off[b + 1] - o;
        const double *Mr = M + cb_doff[b] + (row - o) * nb;
        double s = 0.0;
        if (live)
            for (int j = 0; j < nb; ++j) s += Mr[j] * f[(long long)(o + j) * nv + lane];
        if (live) u[row * nv + lane] = s;
    }
}

// end of a correction iteration: per-column iteration counts, the while
// condition (a column still active and the iteration cap not reached)
__global__ void mv_continue_kernel(cudaGraphConditionalHandle cond, int use_cond, int nv,
                                   const double *__restrict__ scal, int *__restrict__ cnt, int max_iter,
                                   int *__restrict__ more_out)
{
    int any = 0;
    for (int v = 0; v < nv; ++v) {
        if (scal[MS_ALPHA * 32 + v] != 0.0) ++cnt[v];  // the column took this iteration's step
        any |= scal[MS_ACTIVE * 32 + v] != 0.0;        // and still needs one
    }
    const int k = ++cnt[32];
    const int more = (any && k < max_iter) ? 1 : 0;
    *more_out = more;
    if (use_cond) cudaGraphSetConditional(cond, (unsigned)more);
}

}  // namespace amgt

using namespace amgt;

namespace {

int mv_grid(long long n, int sm_count) { return grid_for(kMvThreads / 32, n, sm_count, 4); }

// operator application through the SpMM (auto engine: autotuned or tensor cores)
int apply(const amgt_amg *, int prec, const amgt_bsr *A, double alpha, const double *X, int nv, double beta,
          double *Y, cudaStream_t s)
{
    return amgt_spmm_rm(prec, AMGT_ENGINE_AUTO, alpha, A, nv, X, beta, Y, (amgt_stream_t)s);
}

// Z = M R: one V(1,1) cycle on nv columns (the single-vector cycle of
// amg.cu with every operator as an SpMM)
int mv_cycle(amgt_amg *h, MultiRhs *mr, const double *rhs0, double *out0, cudaStream_t s)
{
    auto &lv = h->lv;
    const int L = (int)lv.size(), nv = mr->nv;
    const double w = h->prm.relax_weight;
    const int p0 = h->prm.inner_prec0;
    for (int l = 0; l < L - 1; ++l) {
        Level &v = lv[l];
        MultiRhsLevel &m = mr->lv[l];
        const double *f = (l == 0) ? rhs0 : m.f;
        const int pl = l == 0 ? p0 : v.prec;
        AMGT_LAUNCH_PDL(mv_jacobi_zero_kernel, mv_grid(v.n, h->sm_count), kMvThreads, 0, s, (long long)v.n, nv, f,
                        (const double *)v.inv_l1, w, m.u);
        AMGT_LAUNCH_PDL(mv_copy_kernel, grid_for(256, (long long)v.n * nv, h->sm_count, 8), 256, 0, s,
                        (long long)v.n * nv, f, m.t);
        AMGT_TRY(apply(h, pl, &v.A, -1.0, m.u, nv, 1.0, m.t, s));
        AMGT_TRY(apply(h, v.prec_transfer, &v.R, 1.0, m.t, nv, 0.0, mr->lv[l + 1].f, s));
    }
    Level &c = lv[L - 1];
    MultiRhsLevel &cm = mr->lv[L - 1];
    const double *fc = (L == 1) ? rhs0 : cm.f;
    double *uc = (L == 1) ? out0 : cm.s;
    AMGT_LAUNCH_PDL(mv_dense_kernel, mv_grid(c.n, h->sm_count), kMvThreads, 0, s, c.n, nv,
                    (const int *)h->row_blk, (const int *)h->cb_off, (const long long *)h->cb_doff,
                    (const double *)h->coarse_inv, fc, uc);
    for (int l = L - 2; l >= 0; --l) {
        Level &v = lv[l];
        MultiRhsLevel &m = mr->lv[l];
        const double *f = (l == 0) ? rhs0 : m.f;
        double *out = (l == 0) ? out0 : m.s;
        const int pl = l == 0 ? p0 : v.prec;
        AMGT_TRY(apply(h, v.prec_transfer, &v.P, 1.0, mr->lv[l + 1].s, nv, 1.0, m.u, s));
        AMGT_LAUNCH_PDL(mv_copy_kernel, grid_for(256, (long long)v.n * nv, h->sm_count, 8), 256, 0, s,
                        (long long)v.n * nv, f, m.t);
        AMGT_TRY(apply(h, pl, &v.A, -1.0, m.u, nv, 1.0, m.t, s));
        AMGT_LAUNCH_PDL(mv_jacobi_update_kernel, mv_grid(v.n, h->sm_count), kMvThreads, 0, s, (long long)v.n, nv,
                        (const double *)m.u, (const double *)m.t, (const double *)v.inv_l1, w, out);
    }
    return AMGT_OK;
}

int mv_dot(amgt_amg *h, MultiRhs *mr, const double *a, const double *b, int slot, int op, cudaStream_t s)
{
    AMGT_LAUNCH_PDL(mv_dot_kernel, kMvGrid, kMvThreads, 0, s, h->n0, mr->nv, a, b, mr->part);
    AMGT_LAUNCH_PDL(mv_reduce_kernel, 1, 1024, 0, s, (const double *)mr->part, kMvGrid, mr->nv, mr->scal, slot, op,
                    h->prm.inner_tol);
    return AMGT_OK;
}

// one lockstep PCG iteration of the correction (body of the loop graph)
int mv_iteration(amgt_amg *h, MultiRhs *mr, cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond)
{
    const int nv = mr->nv;
    const long long n = h->n0;
    AMGT_TRY(apply(h, h->prm.inner_prec0, &h->lv[0].A, 1.0, mr->p, nv, 0.0, mr->q, s));
    AMGT_TRY(mv_dot(h, mr, mr->p, mr->q, MS_PQ, MOP_ALPHA, s));
    AMGT_LAUNCH_PDL(mv_axpy2_dot_kernel, kMvGrid, kMvThreads, 0, s, n, nv, (const double *)mr->scal,
                    (const double *)mr->p, (const double *)mr->q, mr->d, mr->r, mr->part);
    AMGT_LAUNCH_PDL(mv_reduce_kernel, 1, 1024, 0, s, (const double *)mr->part, kMvGrid, nv, mr->scal, (int)MS_RR,
                    (int)MOP_RR_TEST, h->prm.inner_tol);
    AMGT_TRY(mv_cycle(h, mr, mr->r, mr->z, s));
    AMGT_TRY(mv_dot(h, mr, mr->r, mr->z, MS_RZ, MOP_BETA, s));
    AMGT_LAUNCH_PDL(mv_xpby_kernel, mv_grid(n, h->sm_count), kMvThreads, 0, s, n, nv, (const double *)mr->z,
                    (const double *)mr->scal, mr->p);
    count_launch();
    mv_continue_kernel<<<1, 1, 0, s>>>(cond, use_cond, nv, mr->scal, mr->cnt, h->prm.max_iter, mr->cnt + 33);
    AMGT_CUDA_TRY(cudaGetLastError());
    return AMGT_OK;
}

int build_mv_loop(amgt_amg *h, MultiRhs *mr)
{
    if (mr->loop) return AMGT_OK;
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
        rc = mv_iteration(h, mr, h->graph_stream, 1, cond);
        mr->loop_launches = amgt_kernel_launch_count() - c0;
        cudaGraph_t captured = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(h->graph_stream, &captured);
        if (e == cudaSuccess) e = ee;
    }
    if (e == cudaSuccess && rc == AMGT_OK) e = cudaGraphInstantiate(&mr->loop, g, 0);
    cudaGraphDestroy(g);
    if (rc != AMGT_OK) return rc;
    if (e != cudaSuccess) {
        cudaGetLastError();
        mr->loop = nullptr;
        set_last_cuda_error(e, "multi-RHS loop graph", __FILE__, __LINE__);
        return AMGT_ERR_CUDA;
    }
    return AMGT_OK;
}

int make_multi_rhs(amgt_amg *h, int nv, cudaStream_t s, MultiRhs **out)
{
    if (h->mr && h->mr->nv == nv) {
        *out = h->mr;
        return AMGT_OK;
    }
    if (h->mr) {
        free_multi_rhs(h->mr, s);
        h->mr = nullptr;
    }
    MultiRhs *mr = new MultiRhs();
    mr->nv = nv;
    mr->lv.resize(h->lv.size());
    const size_t n0 = (size_t)h->n0 * nv;
    int rc = AMGT_OK;
    for (size_t l = 0; l < h->lv.size() && !rc; ++l) {
        const size_t nl = (size_t)h->lv[l].n * nv;
        MultiRhsLevel &m = mr->lv[l];
        if ((rc = alloc_n(&m.u, nl, s)) || (rc = alloc_n(&m.t, nl, s)) || (rc = alloc_n(&m.f, nl, s)) ||
            (rc = alloc_n(&m.s, nl, s)))
            break;
    }
    if (!rc && ((rc = alloc_n(&mr->r, n0, s)) || (rc = alloc_n(&mr->z, n0, s)) || (rc = alloc_n(&mr->p, n0, s)) ||
                (rc = alloc_n(&mr->q, n0, s)) || (rc = alloc_n(&mr->d, n0, s)) || (rc = alloc_n(&mr->res, n0, s)) ||
                (rc = alloc_n(&mr->scal, (size_t)MS_NSLOT * 32, s)) ||
                (rc = alloc_n(&mr->part, (size_t)kMvGrid * 32, s)) || (rc = alloc_n(&mr->cnt, 40, s))))
        rc = rc ? rc : AMGT_ERR_ALLOC;
    mr->pinned = h->mr_pinned;  // the handle's pinned block (no allocation here)
    if (!rc && cudaMemsetAsync(mr->scal, 0, sizeof(double) * MS_NSLOT * 32, s) != cudaSuccess) rc = AMGT_ERR_CUDA;
    if (rc) {
        cudaGetLastError();
        free_multi_rhs(mr, s);
        return rc;
    }
    h->mr = mr;
    *out = mr;
    return AMGT_OK;
}

__global__ void mv_set_active_kernel(int nv, const double *__restrict__ rel, double tol, double *__restrict__ scal)
{
    for (int v = threadIdx.x; v < nv; v += blockDim.x) scal[MS_ACTIVE * 32 + v] = rel[v] > tol ? 1.0 : 0.0;
}

}  // namespace

extern "C" int amgt_amg_solve_multi(amgt_amg *h, int nrhs, const double *B, double *X, int *iterations,
                                    double *rel_res, amgt_stream_t stream)
{
    if (!h || nrhs < 1 || nrhs > 32 || !B || !X) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    MultiRhs *mr = nullptr;
    AMGT_TRY(make_multi_rhs(h, nrhs, s, &mr));
    Level &v0 = h->lv[0];
    // level 0 inside the correction reads inner_prec0's values
    if (!(h->prm.inner_prec0 == AMGT_FLOAT && v0.A.exact_prec == AMGT_HALF && v0.A.blcVal_fp16))
        AMGT_TRY(amgt_bsr_make_shadow(&v0.A, h->prm.inner_prec0, stream));
    const long long n = h->n0, cnt_all = n * nrhs;
    const int nv = nrhs;
    AMGT_CUDA_TRY(cudaMemsetAsync(mr->cnt, 0, sizeof(int) * 40, s));
    AMGT_TRY(mv_dot(h, mr, B, B, MS_BB, MOP_STORE, s));
    std::vector<double> rel(nv, 0.0);
    double *rel_dev = mr->q;  // scratch for the per-column relative residuals (nv doubles)
    bool graph_ran = false;
    int seen = 0;
    for (int outer = 0; outer <= h->prm.max_outer; ++outer) {
        // fp64 residual R = B - A X (8-byte values, CUDA cores)
        AMGT_LAUNCH_PDL(mv_copy_kernel, grid_for(256, cnt_all, h->sm_count, 8), 256, 0, s, cnt_all, B, mr->res);
        AMGT_TRY(spmm_rowmajor(AMGT_DOUBLE, 0, 8, &v0.A, -1.0, X, nv, 1.0, mr->res, s, h->sm_count));
        AMGT_TRY(mv_dot(h, mr, mr->res, mr->res, MS_RR, MOP_STORE, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(mr->pinned, mr->scal, sizeof(double) * 64, cudaMemcpyDeviceToHost, s));
        AMGT_CUDA_TRY(cudaMemcpyAsync(mr->pinned + 64, mr->cnt, sizeof(int) * 34, cudaMemcpyDeviceToHost, s));
        AMGT_CUDA_TRY(cudaStreamSynchronize(s));
        const int *cnt_h = reinterpret_cast<const int *>(mr->pinned + 64);
        const int total = cnt_h[32];
        if (graph_ran)
            for (long long k = 0; k < (long long)(total - seen) * (long long)mr->loop_launches; ++k) count_launch();
        graph_ran = false;
        seen = total;
        bool all = true;
        for (int v = 0; v < nv; ++v) {
            const double bb = mr->pinned[MS_BB * 32 + v], rr = mr->pinned[MS_RR * 32 + v];
            rel[v] = bb > 0.0 ? std::sqrt(std::max(rr, 0.0) / bb) : std::sqrt(std::max(rr, 0.0));
            all = all && rel[v] <= h->prm.tol;
        }
        if (all || total >= h->prm.max_iter || outer == h->prm.max_outer) {
            for (int v = 0; v < nv; ++v) {
                if (iterations) iterations[v] = cnt_h[v];
                if (rel_res) rel_res[v] = rel[v];
            }
            return AMGT_OK;
        }
        // correction: A D = R, lockstep PCG; columns already at tol stay idle
        AMGT_CUDA_TRY(cudaMemcpyAsync(rel_dev, rel.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, s));
        AMGT_LAUNCH(mv_set_active_kernel, 1, 32, 0, s, nv, (const double *)rel_dev, h->prm.tol, mr->scal);
        AMGT_CUDA_TRY(cudaMemsetAsync(mr->d, 0, sizeof(double) * cnt_all, s));
        AMGT_LAUNCH_PDL(mv_copy_kernel, grid_for(256, cnt_all, h->sm_count, 8), 256, 0, s, cnt_all,
                        (const double *)mr->res, mr->r);
        AMGT_TRY(mv_dot(h, mr, mr->r, mr->r, MS_RR0, MOP_START, s));
        AMGT_TRY(mv_cycle(h, mr, mr->r, mr->z, s));
        AMGT_TRY(mv_dot(h, mr, mr->r, mr->z, MS_RZ, MOP_STORE, s));
        AMGT_LAUNCH_PDL(mv_copy_kernel, grid_for(256, cnt_all, h->sm_count, 8), 256, 0, s, cnt_all,
                        (const double *)mr->z, mr->p);
        bool done = false;
        if (h->prm.use_graph && !mr->loop_failed) {
            const int lrc = build_mv_loop(h, mr);
            if (lrc == AMGT_OK) {
                AMGT_CUDA_TRY(cudaGraphLaunch(mr->loop, s));
                done = graph_ran = true;
            } else if (lrc != AMGT_ERR_CUDA) {
                return lrc;
            } else {
                mr->loop_failed = true;
            }
        }
        if (!done) {
            for (;;) {
                AMGT_TRY(mv_iteration(h, mr, s, 0, 0));
                AMGT_CUDA_TRY(cudaMemcpyAsync(mr->pinned + 100, mr->cnt + 33, sizeof(int), cudaMemcpyDeviceToHost, s));
                AMGT_CUDA_TRY(cudaStreamSynchronize(s));
                if (*reinterpret_cast<const int *>(mr->pinned + 100) == 0) break;
            }
        }
        AMGT_LAUNCH_PDL(mv_add_kernel, grid_for(256, cnt_all, h->sm_count, 8), 256, 0, s, cnt_all,
                        (const double *)mr->d, X);
    }
    return AMGT_OK;
}
