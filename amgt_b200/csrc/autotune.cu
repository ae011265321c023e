// Autotuner of the SpMV / SpMM launch shapes, and the row-major SpMM entry
// point that uses its choice.
//
// The tunables are the ones that decide how a block row meets the warps:
//   SpMV (one vector):   lanes per block row, LPR in {4, 8, 16, 32} (a
//                        warp takes 32 / LPR block rows; the row's LPR / 4
//                        lane groups each take every (LPR/4)-th block);
//   SpMM (nvec vectors): engine (CUDA cores: a warp per block row, a lane
//                        per right-hand side; tensor cores: a warp per two
//                        block rows, mma.m16n8k8 tf32) and warps per CTA
//                        (4 or 8; the CTA tile of block rows).
// amgt_autotune times every candidate on the matrix itself (CUDA events,
// 3 warm-up and 10 timed launches each, on the caller's stream) and keeps
// the fastest in a table keyed by the matrix (its block-row pointer array,
// block rows, blocks) and the precision / vector count; amgt_spmv and
// amgt_spmm_rm (engine AUTO) then use it.  The choice changes the order in
// which a row's blocks are summed for the SpMV (as any LPR does), never the
// set of terms.  The reference has a fixed shape (WARP_NUM_SPMV = 4 warps,
// one warp per block row, AmgT_HYPRE/src/seq_mv/seq_mv.h:84-99) and a fixed
// adaptive switch (stand >= 12, csr_matvec_device.c:1302-1411).
#include <map>
#include <mutex>
#include <tuple>

#include "amgt_internal.cuh"

namespace amgt {

int spmm_rowmajor(int prec, int kind, int wpc, const amgt_bsr *A, double alpha, const double *X, int nvec,
                  double beta, double *Y, cudaStream_t s, int sm_count);

namespace {

using Key = std::tuple<const void *, int, int, int, int>;  // blcPtr, blc_row, blc_num, prec, nvec
struct Choice {
    int a, b;  // SpMV: lpr, 0; SpMM: engine, warps per CTA
};
std::mutex g_mu;
std::map<Key, Choice> g_table;

Key key_of(const amgt_bsr *A, int prec, int nvec) { return Key(A->blcPtr, A->blc_row, A->blc_num, prec, nvec); }

bool lookup(const amgt_bsr *A, int prec, int nvec, Choice *c)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find(key_of(A, prec, nvec));
    if (it == g_table.end()) return false;
    *c = it->second;
    return true;
}

thread_local int t_force_lpr = 0;  // set while the tuner times an SpMV candidate

}  // namespace

int tuned_lpr(const amgt_bsr *A)
{
    if (t_force_lpr) return t_force_lpr;
    if (!A->blcPtr) return 0;
    Choice c;
    // the SpMV's shape depends on the structure only (the same for every
    // value array, so exact narrow storage keeps the fp64 sums)
    return lookup(A, -1, 1, &c) ? c.a : 0;
}

void tune_forget(const amgt_bsr *A)
{
    if (!A->blcPtr) return;
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_table.begin(); it != g_table.end();) {
        if (std::get<0>(it->first) == A->blcPtr) it = g_table.erase(it);
        else ++it;
    }
}

}  // namespace amgt

using namespace amgt;

namespace {

// mean of `reps` launches of fn after 3 warm-ups, in ms
template <typename F>
int time_it(F fn, cudaStream_t s, float *ms)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = AMGT_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
    } else {
        for (int i = 0; i < 3 && !rc; ++i) rc = fn();
        if (!rc && cudaEventRecord(e0, s) != cudaSuccess) rc = AMGT_ERR_CUDA;
        for (int i = 0; i < 10 && !rc; ++i) rc = fn();
        if (!rc && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(ms, e0, e1) != cudaSuccess))
            rc = AMGT_ERR_CUDA;
        if (!rc) *ms /= 10.0f;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGetLastError();
    return rc;
}

}  // namespace

extern "C" {

int amgt_spmm_rm(int prec, int engine, double alpha, const amgt_bsr *A, int nvec, const double *X, double beta,
                 double *Y, amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16 || nvec < 1 || nvec > 32 || engine < AMGT_ENGINE_AUTO ||
        engine > AMGT_ENGINE_TENSOR_CORE)
        return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (!Y) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    if (A->blc_num == 0 || A->col == 0) return scale_vector((long long)A->row * nvec, beta, Y, st->sm_count, s);
    if (!X || !A->blcPtr || !A->blcIdx) return AMGT_ERR_INVALID;
    int kind = 1, wpc = 8;
    if (engine == AMGT_ENGINE_CUDA_CORE) kind = 0;
    if (engine == AMGT_ENGINE_AUTO) {
        Choice c;
        if (lookup(A, prec, nvec, &c)) {
            kind = c.a;
            wpc = c.b;
        }
    }
    return spmm_rowmajor(prec, kind, wpc, A, alpha, X, nvec, beta, Y, s, st->sm_count);
}

int amgt_autotune(const amgt_bsr *A, int prec, int nvec, amgt_tune_result *out, amgt_stream_t stream)
{
    if (!A || !out || prec < AMGT_DOUBLE || prec > AMGT_BF16 || nvec < 1 || nvec > 32) return AMGT_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    if (A->row == 0 || A->blc_num == 0) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    double *x = nullptr, *y = nullptr;
    int rc = AMGT_OK;
    if ((rc = alloc_n(&x, (size_t)A->col * nvec, s)) || (rc = alloc_n(&y, (size_t)A->row * nvec, s))) goto done;
    if (cudaMemsetAsync(x, 0, sizeof(double) * (size_t)A->col * nvec, s) != cudaSuccess ||
        cudaMemsetAsync(y, 0, sizeof(double) * (size_t)A->row * nvec, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto done;
    }
    if (nvec == 1) {
        static const int lprs[4] = {4, 8, 16, 32};
        float best = 0.0f;
        for (int i = 0; i < 4 && !rc; ++i) {
            float ms = 0.0f;
            t_force_lpr = lprs[i];
            rc = time_it([&] { return amgt_spmv(prec, 1.0, A, x, 0.0, y, stream); }, s, &ms);
            t_force_lpr = 0;
            out->candidate[i] = lprs[i];
            out->ms[i] = ms;
            if (!rc && (i == 0 || ms < best)) {
                best = ms;
                out->choice = lprs[i];
            }
        }
        out->count = 4;
        if (!rc) {
            std::lock_guard<std::mutex> lk(g_mu);
            g_table[key_of(A, -1, 1)] = Choice{out->choice, 0};
        }
    } else {
        // candidate code: 10 * engine + warps per CTA
        static const int cands[4][2] = {{0, 4}, {0, 8}, {1, 4}, {1, 8}};
        float best = 0.0f;
        int n = 0;
        for (int i = 0; i < 4 && !rc; ++i) {
            if (cands[i][0] == 1 && prec == AMGT_DOUBLE) continue;  // fp64 values: CUDA cores only
            float ms = 0.0f;
            rc = time_it([&] { return spmm_rowmajor(prec, cands[i][0], cands[i][1], A, 1.0, x, nvec, 0.0, y, s,
                                                    st->sm_count); }, s, &ms);
            out->candidate[n] = 10 * cands[i][0] + cands[i][1];
            out->ms[n] = ms;
            if (!rc && (n == 0 || ms < best)) {
                best = ms;
                out->choice = out->candidate[n];
            }
            ++n;
        }
        out->count = n;
        if (!rc) {
            std::lock_guard<std::mutex> lk(g_mu);
            g_table[key_of(A, prec, nvec)] = Choice{out->choice / 10, out->choice % 10};
        }
    }
done:
    free_ptr(x, s);
    free_ptr(y, s);
    return rc;
}

int amgt_autotune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
    return AMGT_OK;
}

}  // extern "C"
