// Internal: the AMG handle (amgt_amg) and its levels, shared by the
// single-vector solvers (amg.cu) and the multi-right-hand-side solve
// (multirhs.cu).  Not part of the C ABI.
#pragma once

#include <vector>

#include "amgt_internal.cuh"

namespace amgt {

constexpr int kDotGrid = 1184;  // 8 x 148 SMs
constexpr int kDotThreads = 256;

struct MultiRhs;  // multi-right-hand-side work vectors (multirhs.cu)
void free_multi_rhs(MultiRhs *mr, cudaStream_t s);
struct Batch;     // per-system data of a batch of systems (batch.cu)
void free_batch(Batch *b, cudaStream_t s);

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
    double *coarse_inv = nullptr;  // inverse of the coarsest operator: dense diagonal blocks
    int nc = 0, ncb = 0;           // its rows; its blocks (1, or one per system of a batch)
    int *cb_off = nullptr;         // device [ncb + 1]: first row of each block
    long long *cb_doff = nullptr;  // device [ncb + 1]: offset of each block's dense values
    int *row_blk = nullptr;        // device [nc]: block of each row
    long long n0 = 0;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    double *scal = nullptr, *part = nullptr;
    double *pinned = nullptr;  // host: one pinned block of every read-back slot (setup allocates it)
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
    double *loop_pinned = nullptr;  // host, inside the pinned block (below)
    double *mr_pinned = nullptr;    // host, 160 slots of the multi-right-hand-side solve
    uint64_t graph_launches = 0, loop_launches = 0;  // our kernels per iteration in each graph
    double setup_ms[5] = {0, 0, 0, 0, 0};
    std::vector<double> hist;
    // FGMRES with iterative refinement (solver = AMGT_SOLVER_FGMRES_IR)
    int resid_prec0 = AMGT_DOUBLE;  // the cycle's level-0 residual precision
    float *gmV = nullptr, *gmZ = nullptr;  // basis (m + 1 vectors), preconditioned vectors (m)
    double *gm = nullptr;                  // Hessenberg, rotations, g, y, slots (GmLayout)
    double *gm_vin = nullptr, *gm_zout = nullptr, *gm_w = nullptr, *gm_part = nullptr;
    int *gm_j = nullptr;                   // device: inner iteration index
    cudaGraphExec_t gm_loop = nullptr;
    bool gm_loop_failed = false;
    uint64_t gm_loop_launches = 0;
    amgt::MultiRhs *mr = nullptr;  // amgt_amg_solve_multi's vectors, built on first use
    amgt::Batch *batch = nullptr;  // systems of amgt_batch_setup
};

namespace amgt {
// z = M r: one V(1,1) cycle of h's hierarchy (amg.cu)
int amg_cycle(amgt_amg *h, const double *rhs0, double *out0, cudaStream_t s);
// amgt_amg_setup with the coarsest operator inverted per diagonal block:
// block s has sys_rows[s][L - 1] rows, L the levels set up (nullptr: one
// block).
// With cb: P_l and level l's precision from the callback, once A_l exists
// (amgt_amg_setup_adaptive).
int amg_setup_blocks(const amgt_csr *A, int num_interp, const amgt_csr *P, const amgt_amg_params *params,
                     amgt_amg **out, amgt_stream_t stream, const std::vector<std::vector<int>> *sys_rows,
                     amgt_coarsen_fn cb, void *cb_ctx);
}  // namespace amgt


