// amgt_spmv_segmented_noalloc: the long-row (segmented) SpMV with its
// partial-sum scratch in a fixed device array instead of the allocator.
//
// Some callers cannot allocate device memory at the moment they run a
// matvec: a solver whose device memory was handed, whole, to a pool sized at
// set-up time and that must not grow afterwards; a caller whose allocator
// hook may not be invoked from the thread issuing the solve; a caller that
// cannot afford cudaMalloc / cudaFree, which can synchronise the device and
// so stall every other stream.  For them the segmented SpMV, the one SpMV
// path that needs scratch (4 doubles per segment of <= 64 blocks), takes it
// from the array below.
//
// The array is g_noalloc_part: AMGT_NOALLOC_MAX_SEGMENTS * 4 doubles (8 MiB)
// of file-scope __device__ memory, which every GPU that loads the library
// holds until the process exits.  Host code cannot use the array's name as a
// device address (on the host it names a host-side stand-in), so the first
// call on each device, with that device current, looks the address up with
// cudaGetSymbolAddress and keeps it; that first call should therefore come
// before any stream capture.  Nothing in the array has to start at zero: the
// first kernel writes every partial sum the second kernel reads.  All calls
// share the array, so calls whose kernels overlap on the GPU (two streams,
// or two host threads) race on it and must be ordered by the caller.
#include <mutex>

#include "amgt_internal.cuh"

namespace {

__device__ __align__(256) double g_noalloc_part[4 * AMGT_NOALLOC_MAX_SEGMENTS];

constexpr int kMaxDev = 64;
double *g_part_addr[kMaxDev];
int g_sm_count[kMaxDev];
bool g_ready[kMaxDev];
std::mutex g_mu;

// Per-device set-up: device address of the array and the SM count.  Uses
// no allocating call.
int noalloc_setup(double **part, int *sm_count)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        amgt::set_last_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
        return AMGT_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDev) return AMGT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ready[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_part);
        if (e != cudaSuccess) {
            amgt::set_last_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_part)", __FILE__, __LINE__);
            return AMGT_ERR_CUDA;
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            amgt::set_last_cuda_error(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
            return AMGT_ERR_CUDA;
        }
        g_part_addr[dev] = static_cast<double *>(p);
        g_sm_count[dev] = sms;
        g_ready[dev] = true;
    }
    *part = g_part_addr[dev];
    *sm_count = g_sm_count[dev];
    return AMGT_OK;
}

}  // namespace

extern "C" int amgt_spmv_segmented_noalloc(int prec, double alpha, const amgt_bsr *A, const double *x, double beta,
                                           double *y, amgt_stream_t stream)
{
    if (!A || prec < AMGT_DOUBLE || prec > AMGT_BF16) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (!y) return AMGT_ERR_INVALID;
    double *part = nullptr;
    int sm_count = 0;
    if (A->blc_num == 0 || A->col == 0) {
        // no stored block: y = beta * y, as amgt_spmv does (no scratch needed)
        const int rc = noalloc_setup(&part, &sm_count);
        if (rc != AMGT_OK) return rc;
        return amgt::scale_vector(A->row, beta, y, sm_count, (cudaStream_t)stream);
    }
    if (!x || !A->blcPtr || !A->blcIdx || !A->rowPtrbyWarp || !A->rowIdxbyWarp || A->warpnum <= 0)
        return AMGT_ERR_INVALID;  // needs the segment table of amgt_bsr_balance
    if (A->warpnum > AMGT_NOALLOC_MAX_SEGMENTS) return AMGT_ERR_TOO_LARGE;
    const int rc = noalloc_setup(&part, &sm_count);
    if (rc != AMGT_OK) return rc;
    return amgt::spmv_segmented_with_scratch(prec, alpha, A, x, beta, y, part, sm_count, (cudaStream_t)stream);
}
