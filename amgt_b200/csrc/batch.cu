// Many independent systems of uneven size in one solve (the batching form):
// amgt_batch_setup concatenates the systems block-diagonally, level by
// level, and builds one hierarchy; amgt_amg_solve_batch runs one PCG per
// system in lockstep, each with its own scalars and its own stop, the
// whole iteration loop as one CUDA graph launch.
//
// Block-diagonal concatenation: A = diag(A_0, ..., A_{S-1}), and per level
// P_l = diag(P_l^s), where a system whose own hierarchy has fewer levels
// contributes an identity block at its coarsest size.  Every operator of
// the hierarchy is then block-diagonal, so no system ever sees another's
// values; a system carried down by identity blocks reaches the coarsest
// level unchanged (R A P = A), where the dense inverse of the block-
// diagonal operator is the block-diagonal of the inverses, so its coarse
// correction is still its own exact coarse solve.  One SpMV, one cycle,
// one launch of each kernel serves all systems.
//
// Per-system scalars: level-0 rows are cut into tiles of at most
// kTileRows rows that never cross a system boundary; dots reduce per tile
// (fixed order) and then per system over its tiles (fixed order), and the
// vector updates read their system's scalar through the tile.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "amg_handle.cuh"

namespace amgt {

constexpr int kTileRows = 4096;
constexpr int kBThreads = 256;

enum { BS_BB = 0, BS_RR = 1, BS_RZ = 2, BS_PQ = 3, BS_ALPHA = 4, BS_BETA = 5, BS_ACTIVE = 6, BS_NSLOT = 7 };
enum { BOP_STORE = 0, BOP_ALPHA = 1, BOP_BETA = 2, BOP_RR_TEST = 3 };

struct Batch {
    int nsys = 0, ntiles = 0;
    int *tile_sys = nullptr;      // device [ntiles]: system of the tile
    int *tile_beg = nullptr;      // device [ntiles + 1]: first row (tiles ascend)
    int *sys_tile = nullptr;      // device [nsys + 1]: first tile of each system
    double *scal = nullptr;       // device [BS_NSLOT * nsys]
    double *part = nullptr;       // device [ntiles]
    int *cnt = nullptr;           // device [nsys + 2]: iterations per system, total, more
    double *pinned = nullptr;     // host [2 * nsys + nsys + 2]
    std::vector<int> rows;        // rows per system (level 0)
    cudaGraphExec_t loop = nullptr;
    double *loop_x = nullptr;  // the x the loop graph updates
    bool loop_failed = false;
    uint64_t loop_launches = 0;
};

struct CatDesc {
    const int *ia, *ja;
    const double *a;
    int rows, nnz, row_off, col_off, nnz_off, identity;
};

// one system per blockIdx.y: rows, columns and values with offsets
__global__ void cat_kernel(const CatDesc *__restrict__ d, int *__restrict__ ia, int *__restrict__ ja,
                           double *__restrict__ a)
{
    const CatDesc c = d[blockIdx.y];
    const int top = max(c.rows, c.nnz);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < top; i += gridDim.x * blockDim.x) {
        if (i < c.rows) ia[c.row_off + i] = (c.identity ? i : c.ia[i]) + c.nnz_off;
        if (i < c.nnz) {
            ja[c.nnz_off + i] = (c.identity ? i : c.ja[i]) + c.col_off;
            a[c.nnz_off + i] = c.identity ? 1.0 : c.a[i];
        }
    }
}

__global__ void set_int_kernel(int *__restrict__ p, int v) { *p = v; }

// partial dot per tile
__global__ void __launch_bounds__(kBThreads) b_dot_kernel(int ntiles, const int *__restrict__ tile_beg,
                                                         const double *__restrict__ a, const double *__restrict__ b,
                                                         double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kBThreads / 32];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        double s = 0.0;
        for (int i = tile_beg[t] + threadIdx.x; i < tile_beg[t + 1]; i += blockDim.x) s += a[i] * b[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double u = 0.0;
            for (int w = 0; w < kBThreads / 32; ++w) u += sred[w];
            part[t] = u;
        }
        __syncthreads();
    }
}

// per system: sum of its tiles in order (a warp per system), then op
__global__ void b_reduce_kernel(int nsys, const int *__restrict__ sys_tile, const double *__restrict__ part,
                                double *__restrict__ scal, int slot, int op, double tol)
{
    grid_dependency_wait();
    const int lane = threadIdx.x & 31;
    for (int sy = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sy < nsys; sy += (gridDim.x * blockDim.x) >> 5) {
        double t = 0.0;
        for (int k = sys_tile[sy] + lane; k < sys_tile[sy + 1]; k += 32) t += part[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
        if (lane != 0) continue;
        double *sc = scal;
        if (op == BOP_STORE) {
            sc[slot * nsys + sy] = t;
        } else if (op == BOP_ALPHA) {
            sc[BS_PQ * nsys + sy] = t;
            sc[BS_ALPHA * nsys + sy] = (sc[BS_ACTIVE * nsys + sy] != 0.0 && t != 0.0) ? sc[BS_RZ * nsys + sy] / t : 0.0;
        } else if (op == BOP_BETA) {
            const double rz_old = sc[BS_RZ * nsys + sy];
            sc[BS_BETA * nsys + sy] = rz_old != 0.0 ? t / rz_old : 0.0;
            sc[BS_RZ * nsys + sy] = t;
        } else {  // BOP_RR_TEST: ||r|| / ||b|| <= tol stops the system
            sc[BS_RR * nsys + sy] = t;
            const double bb = sc[BS_BB * nsys + sy];
            const double rel = bb > 0.0 ? sqrt(fmax(t, 0.0) / bb) : sqrt(fmax(t, 0.0));
            sc[BS_ACTIVE * nsys + sy] = (rel > tol) ? 1.0 : 0.0;
        }
    }
}

// x += alpha_s p; r -= alpha_s q; partial r . r per tile
__global__ void __launch_bounds__(kBThreads) b_axpy2_dot_kernel(int ntiles, int nsys, const int *__restrict__ tile_beg,
                                                               const int *__restrict__ tile_sys,
                                                               const double *__restrict__ scal,
                                                               const double *__restrict__ p,
                                                               const double *__restrict__ q, double *__restrict__ x,
                                                               double *__restrict__ r, double *__restrict__ part)
{
    grid_dependency_wait();
    __shared__ double sred[kBThreads / 32];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const double alpha = scal[BS_ALPHA * nsys + tile_sys[t]];
        double s = 0.0;
        for (int i = tile_beg[t] + threadIdx.x; i < tile_beg[t + 1]; i += blockDim.x) {
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
            double u = 0.0;
            for (int w = 0; w < kBThreads / 32; ++w) u += sred[w];
            part[t] = u;
        }
        __syncthreads();
    }
}

// p = z + beta_s p
__global__ void b_xpby_kernel(int ntiles, int nsys, const int *__restrict__ tile_beg, const int *__restrict__ tile_sys,
                              const double *__restrict__ scal, const double *__restrict__ z, double *__restrict__ p)
{
    grid_dependency_wait();
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const double beta = scal[BS_BETA * nsys + tile_sys[t]];
        for (int i = tile_beg[t] + threadIdx.x; i < tile_beg[t + 1]; i += blockDim.x) p[i] = z[i] + beta * p[i];
    }
}

// end of an iteration: iterations per system, the while condition
__global__ void b_continue_kernel(cudaGraphConditionalHandle cond, int use_cond, int nsys,
                                  const double *__restrict__ scal, int *__restrict__ cnt, int max_iter)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int sy = threadIdx.x; sy < nsys; sy += blockDim.x) {
        if (scal[BS_ALPHA * nsys + sy] != 0.0) ++cnt[sy];  // took this iteration's step
        if (scal[BS_ACTIVE * nsys + sy] != 0.0) any = 1;  // benign race: every writer stores 1
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int k = ++cnt[nsys];
        const int more = (any && k < max_iter) ? 1 : 0;
        cnt[nsys + 1] = more;
        if (use_cond) cudaGraphSetConditional(cond, (unsigned)more);
    }
}

void free_batch(Batch *b, cudaStream_t s)
{
    if (!b) return;
    if (b->loop) cudaGraphExecDestroy(b->loop);
    free_ptr(b->tile_sys, s);
    free_ptr(b->tile_beg, s);
    free_ptr(b->sys_tile, s);
    free_ptr(b->scal, s);
    free_ptr(b->part, s);
    free_ptr(b->cnt, s);
    pinned_put(b->pinned);
    delete b;
}

}  // namespace amgt

using namespace amgt;

namespace {

int dot_b(amgt_amg *h, Batch *b, const double *x, const double *y, int slot, int op, cudaStream_t s)
{
    const int grid = std::min(b->ntiles, 8 * h->sm_count);
    AMGT_LAUNCH_PDL(b_dot_kernel, grid, kBThreads, 0, s, b->ntiles, (const int *)b->tile_beg, x, y, b->part);
    AMGT_LAUNCH_PDL(b_reduce_kernel, grid_for(8, b->nsys, h->sm_count, 4), 256, 0, s, b->nsys,
                    (const int *)b->sys_tile, (const double *)b->part, b->scal, slot, op, h->prm.tol);
    return AMGT_OK;
}

int b_iteration(amgt_amg *h, Batch *b, double *x, cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond)
{
    Level &v0 = h->lv[0];
    const int grid = std::min(b->ntiles, 8 * h->sm_count);
    AMGT_TRY(amgt_spmv(AMGT_DOUBLE, 1.0, &v0.A, h->p, 0.0, h->q, (amgt_stream_t)s));
    AMGT_TRY(dot_b(h, b, h->p, h->q, BS_PQ, BOP_ALPHA, s));
    AMGT_LAUNCH_PDL(b_axpy2_dot_kernel, grid, kBThreads, 0, s, b->ntiles, b->nsys, (const int *)b->tile_beg,
                    (const int *)b->tile_sys, (const double *)b->scal, (const double *)h->p, (const double *)h->q, x,
                    h->r, b->part);
    AMGT_LAUNCH_PDL(b_reduce_kernel, grid_for(8, b->nsys, h->sm_count, 4), 256, 0, s, b->nsys,
                    (const int *)b->sys_tile, (const double *)b->part, b->scal, (int)BS_RR, (int)BOP_RR_TEST,
                    h->prm.tol);
    AMGT_TRY(amg_cycle(h, h->r, h->z, s));
    AMGT_TRY(dot_b(h, b, h->r, h->z, BS_RZ, BOP_BETA, s));
    AMGT_LAUNCH_PDL(b_xpby_kernel, grid, kBThreads, 0, s, b->ntiles, b->nsys, (const int *)b->tile_beg,
                    (const int *)b->tile_sys, (const double *)b->scal, (const double *)h->z, h->p);
    count_launch();
    b_continue_kernel<<<1, 256, 0, s>>>(cond, use_cond, b->nsys, b->scal, b->cnt, h->prm.max_iter);
    AMGT_CUDA_TRY(cudaGetLastError());
    return AMGT_OK;
}

int build_b_loop(amgt_amg *h, Batch *b, double *x)
{
    if (b->loop) return AMGT_OK;
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
        rc = b_iteration(h, b, x, h->graph_stream, 1, cond);
        b->loop_launches = amgt_kernel_launch_count() - c0;
        cudaGraph_t captured = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(h->graph_stream, &captured);
        if (e == cudaSuccess) e = ee;
    }
    if (e == cudaSuccess && rc == AMGT_OK) e = cudaGraphInstantiate(&b->loop, g, 0);
    cudaGraphDestroy(g);
    if (rc != AMGT_OK) return rc;
    if (e != cudaSuccess) {
        cudaGetLastError();
        b->loop = nullptr;
        set_last_cuda_error(e, "batch loop graph", __FILE__, __LINE__);
        return AMGT_ERR_CUDA;
    }
    b->loop_x = x;
    return AMGT_OK;
}

}  // namespace

extern "C" {

int amgt_batch_setup(int nsys, const amgt_csr *A, const int *nlev, const amgt_csr *P, const amgt_amg_params *params,
                     amgt_amg **out, amgt_stream_t stream)
{
    if (!A || !nlev || !out || nsys < 1 || nsys > 65535) return AMGT_ERR_INVALID;
    *out = nullptr;
    // per system: level sizes; identity blocks below a system's own coarsest level
    int Lmax = 0;
    long long np_total = 0;
    for (int s = 0; s < nsys; ++s) {
        if (A[s].num_rows <= 0 || A[s].num_rows != A[s].num_cols || A[s].num_nonzeros < 0 || nlev[s] < 0)
            return AMGT_ERR_INVALID;
        Lmax = std::max(Lmax, nlev[s]);
        np_total += nlev[s];
    }
    if (np_total > 0 && !P) return AMGT_ERR_INVALID;
    std::vector<long long> poff(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) poff[s + 1] = poff[s] + nlev[s];
    std::vector<std::vector<int>> rows(nsys);
    for (int s = 0; s < nsys; ++s) {
        rows[s].push_back(A[s].num_rows);
        for (int l = 0; l < nlev[s]; ++l) {
            const amgt_csr &p = P[poff[s] + l];
            if (p.num_rows != rows[s].back() || p.num_cols <= 0 || p.num_nonzeros < 0) return AMGT_ERR_INVALID;
            rows[s].push_back(p.num_cols);
        }
        while ((int)rows[s].size() < Lmax + 1) rows[s].push_back(rows[s].back());
    }
    long long tot_rows0 = 0;
    for (int s = 0; s < nsys; ++s) tot_rows0 += rows[s][0];
    if (tot_rows0 > 0x7fffffffLL) return AMGT_ERR_TOO_LARGE;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    // concatenations: index 0 = A, 1 + l = P_l
    std::vector<amgt_csr> cat(Lmax + 1);
    CatDesc *ddesc = nullptr;
    int rc = AMGT_OK;
    amgt_amg *h = nullptr;
    if ((rc = alloc_n(&ddesc, (size_t)nsys, s))) return rc;
    for (int k = 0; k <= Lmax && !rc; ++k) {
        std::vector<CatDesc> d(nsys);
        long long ro = 0, co = 0, no = 0;
        for (int sy = 0; sy < nsys; ++sy) {
            CatDesc &c = d[sy];
            if (k == 0) {
                c = CatDesc{A[sy].i, A[sy].j, A[sy].data, A[sy].num_rows, A[sy].num_nonzeros, (int)ro, (int)co,
                            (int)no, 0};
                co += A[sy].num_rows;
            } else if (k - 1 < nlev[sy]) {
                const amgt_csr &p = P[poff[sy] + k - 1];
                c = CatDesc{p.i, p.j, p.data, p.num_rows, p.num_nonzeros, (int)ro, (int)co, (int)no, 0};
                co += p.num_cols;
            } else {
                const int n = rows[sy][k - 1];
                c = CatDesc{nullptr, nullptr, nullptr, n, n, (int)ro, (int)co, (int)no, 1};
                co += n;
            }
            ro += c.rows;
            no += c.nnz;
            if (no > 0x7fffffffLL || ro > 0x7fffffffLL || co > 0x7fffffffLL) rc = AMGT_ERR_TOO_LARGE;
        }
        if (rc) break;
        amgt_csr &C = cat[k];
        C.num_rows = (int)ro;
        C.num_cols = (int)co;
        C.num_nonzeros = (int)no;
        if ((rc = alloc_n(&C.i, (size_t)ro + 1, s)) || (rc = alloc_n(&C.j, (size_t)no, s)) ||
            (rc = alloc_n(&C.data, (size_t)no, s)))
            break;
        // pageable source: the copy is complete when cudaMemcpyAsync returns
        if (cudaMemcpyAsync(ddesc, d.data(), sizeof(CatDesc) * nsys, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            rc = AMGT_ERR_CUDA;
            break;
        }
        count_launch();
        cat_kernel<<<dim3(std::max(1, std::min(64, (int)((std::max(ro, no) / nsys + 255) / 256))), nsys), 256, 0, s>>>(
            ddesc, C.i, C.j, C.data);
        count_launch();
        set_int_kernel<<<1, 1, 0, s>>>(C.i + ro, (int)no);
        if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
        if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = AMGT_ERR_CUDA;  // ddesc is reused next level
    }
    if (!rc) rc = amg_setup_blocks(&cat[0], Lmax, Lmax > 0 ? &cat[1] : nullptr, params, &h, stream, &rows, nullptr,
                                  nullptr);
    for (auto &C : cat) {
        free_ptr(C.i, s);
        free_ptr(C.j, s);
        free_ptr(C.data, s);
    }
    free_ptr(ddesc, s);
    if (rc) return rc;
    // tiles of <= kTileRows level-0 rows, never across systems
    Batch *b = new Batch();
    b->nsys = nsys;
    std::vector<int> tsys, tbeg, stile;
    int r0 = 0;
    for (int sy = 0; sy < nsys; ++sy) {
        stile.push_back((int)tsys.size());
        b->rows.push_back(rows[sy][0]);
        for (int i = 0; i < rows[sy][0]; i += kTileRows) {
            tsys.push_back(sy);
            tbeg.push_back(r0 + i);
        }
        r0 += rows[sy][0];
    }
    stile.push_back((int)tsys.size());
    tbeg.push_back(r0);
    b->ntiles = (int)tsys.size();
    if ((rc = alloc_n(&b->tile_sys, tsys.size(), s)) || (rc = alloc_n(&b->tile_beg, tbeg.size(), s)) ||
        (rc = alloc_n(&b->sys_tile, stile.size(), s)) || (rc = alloc_n(&b->scal, (size_t)BS_NSLOT * nsys, s)) ||
        (rc = alloc_n(&b->part, (size_t)b->ntiles, s)) || (rc = alloc_n(&b->cnt, (size_t)nsys + 2, s))) {
        free_batch(b, s);
        amgt_amg_destroy(h, stream);
        return rc;
    }
    if (cudaMemcpyAsync(b->tile_sys, tsys.data(), sizeof(int) * tsys.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->tile_beg, tbeg.data(), sizeof(int) * tbeg.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->sys_tile, stile.data(), sizeof(int) * stile.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(b->scal, 0, sizeof(double) * BS_NSLOT * nsys, s) != cudaSuccess ||
        pinned_get(sizeof(double) * (3 * (size_t)nsys + 4), reinterpret_cast<void **>(&b->pinned)) != AMGT_OK) {
        cudaGetLastError();
        free_batch(b, s);
        amgt_amg_destroy(h, stream);
        return AMGT_ERR_CUDA;
    }
    h->batch = b;
    *out = h;
    return AMGT_OK;
}

int amgt_amg_solve_batch(amgt_amg *h, const double *bvec, double *x, int *iterations, double *rel_res,
                         int *batch_iterations, amgt_stream_t stream)
{
    if (!h || !h->batch || !bvec || !x) return AMGT_ERR_INVALID;
    Batch *b = h->batch;
    cudaStream_t s = (cudaStream_t)stream;
    Level &v0 = h->lv[0];
    const int ns = b->nsys;
    AMGT_CUDA_TRY(cudaMemsetAsync(b->cnt, 0, sizeof(int) * (ns + 2), s));
    AMGT_CUDA_TRY(cudaMemsetAsync(b->scal, 0, sizeof(double) * BS_NSLOT * ns, s));
    AMGT_TRY(spmv_residual(AMGT_DOUBLE, &v0.A, bvec, x, h->r, s, h->sm_count));
    AMGT_TRY(dot_b(h, b, bvec, bvec, BS_BB, BOP_STORE, s));
    AMGT_TRY(dot_b(h, b, h->r, h->r, BS_RR, BOP_RR_TEST, s));
    AMGT_TRY(amg_cycle(h, h->r, h->z, s));
    AMGT_TRY(dot_b(h, b, h->r, h->z, BS_RZ, BOP_STORE, s));
    AMGT_CUDA_TRY(cudaMemcpyAsync(h->p, h->z, sizeof(double) * h->n0, cudaMemcpyDeviceToDevice, s));
    bool graph = false;
    if (h->prm.use_graph && !b->loop_failed) {
        if (b->loop && b->loop_x != x) {
            cudaGraphExecDestroy(b->loop);
            b->loop = nullptr;
        }
        const int lrc = build_b_loop(h, b, x);
        if (lrc == AMGT_OK) {
            AMGT_CUDA_TRY(cudaGraphLaunch(b->loop, s));
            graph = true;
        } else if (lrc != AMGT_ERR_CUDA) {
            return lrc;
        } else {
            b->loop_failed = true;
        }
    }
    if (!graph) {
        for (;;) {
            AMGT_TRY(b_iteration(h, b, x, s, 0, 0));
            int *pin = reinterpret_cast<int *>(b->pinned);
            AMGT_CUDA_TRY(cudaMemcpyAsync(pin, b->cnt + ns + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            AMGT_CUDA_TRY(cudaStreamSynchronize(s));
            if (*pin == 0) break;
        }
    }
    // true residuals of the returned x, per system
    AMGT_TRY(spmv_residual(AMGT_DOUBLE, &v0.A, bvec, x, h->r, s, h->sm_count));
    AMGT_TRY(dot_b(h, b, h->r, h->r, BS_RR, BOP_STORE, s));
    AMGT_CUDA_TRY(cudaMemcpyAsync(b->pinned, b->scal, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaMemcpyAsync(b->pinned + 2 * ns, b->cnt, sizeof(int) * (ns + 2), cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaStreamSynchronize(s));
    const int *cnt = reinterpret_cast<const int *>(b->pinned + 2 * ns);
    if (graph)
        for (long long k = 0; k < (long long)cnt[ns] * (long long)b->loop_launches; ++k) count_launch();
    for (int sy = 0; sy < ns; ++sy) {
        const double bb = b->pinned[BS_BB * ns + sy], rr = b->pinned[BS_RR * ns + sy];
        if (iterations) iterations[sy] = cnt[sy];
        if (rel_res) rel_res[sy] = bb > 0.0 ? std::sqrt(std::max(rr, 0.0) / bb) : std::sqrt(std::max(rr, 0.0));
    }
    if (batch_iterations) *batch_iterations = cnt[ns];
    return AMGT_OK;
}

int amgt_batch_offsets(const amgt_amg *h, int *offsets, int cap)
{
    if (!h || !h->batch) return -1;
    const Batch *b = h->batch;
    int o = 0;
    for (int sy = 0; sy <= b->nsys && sy < cap && offsets; ++sy) {
        offsets[sy] = o;
        if (sy < b->nsys) o += b->rows[sy];
    }
    return b->nsys;
}

}  // extern "C"
