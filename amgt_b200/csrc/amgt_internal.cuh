// Internal helpers shared by the mBSR kernels (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/amgt_b200.h"

namespace amgt {

// ------------------------------------------------------------------ status
#define AMGT_CUDA_TRY(expr)                                                   \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) {                                              \
            amgt::set_last_cuda_error(_e, #expr, __FILE__, __LINE__);         \
            return AMGT_ERR_CUDA;                                             \
        }                                                                     \
    } while (0)

#define AMGT_TRY(expr)                                                        \
    do {                                                                      \
        int _s = (expr);                                                      \
        if (_s != AMGT_OK) return _s;                                         \
    } while (0)

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);

// Every kernel launch of the library goes through this so that the launch
// counter (amgt_kernel_launch_count) is exact.
void count_launch();
#define AMGT_LAUNCH(kernel, grid, block, smem, stream, ...)                   \
    do {                                                                      \
        amgt::count_launch();                                                 \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);           \
        AMGT_CUDA_TRY(cudaGetLastError());                                    \
    } while (0)

// Launch with programmatic dependent launch (solve-path kernels): the grid
// may be scheduled while the previous kernel on the stream is finishing,
// which hides most of the launch gap between dependent kernels (also inside
// CUDA graphs, where capture turns it into a programmatic edge).  Every
// kernel launched this way calls grid_dependency_wait() before it touches
// memory; without a programmatic dependency the wait returns at once.
#define AMGT_LAUNCH_PDL(kernel, grid, block, smem, strm, ...)                 \
    do {                                                                      \
        amgt::count_launch();                                                 \
        cudaLaunchConfig_t _cfg = {};                                         \
        _cfg.gridDim = dim3(grid);                                            \
        _cfg.blockDim = dim3(block);                                          \
        _cfg.dynamicSmemBytes = (smem);                                       \
        _cfg.stream = (strm);                                                 \
        cudaLaunchAttribute _at[1];                                           \
        _at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;       \
        _at[0].val.programmaticStreamSerializationAllowed = 1;                \
        _cfg.attrs = _at;                                                     \
        _cfg.numAttrs = 1;                                                    \
        AMGT_CUDA_TRY(cudaLaunchKernelEx(&_cfg, kernel, __VA_ARGS__));        \
    } while (0)

__device__ __forceinline__ void grid_dependency_wait()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

// ------------------------------------------------------------- allocation
void *dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);

template <typename T>
int alloc_n(T **out, size_t n, cudaStream_t s)
{
    *out = nullptr;
    if (n == 0) n = 1;  // keep a valid pointer for empty arrays
    *out = static_cast<T *>(dev_alloc(n * sizeof(T), s));
    return *out ? AMGT_OK : AMGT_ERR_ALLOC;
}

template <typename T>
void free_ptr(T *&p, cudaStream_t s)
{
    if (p) dev_free((void *)p, s);
    p = nullptr;
}

// Per-device state: a device error word that kernels raise instead of
// trapping, and the SM count.
struct DeviceState {
    int *err;            // device: 0 = ok, else first error code raised
    int sm_count;
};
int device_state(DeviceState **st);

// Reports the device error word as the calling thread's last read_back on
// this device copied it (no further synchronisation) and clears a raised
// word.  Call right after a read_back.
int check_device_error(cudaStream_t s);

// Error codes a kernel may raise into DeviceState::err
enum : int {
    DEV_ERR_PROBE = 1,   // bounded probe / loop limit exceeded
    DEV_ERR_INDEX = 2,   // index out of range in the input
    DEV_ERR_CAPACITY = 3 // a per-row work buffer was too small
};

__device__ __forceinline__ void raise_error(int *err, int code)
{
    atomicCAS(err, 0, code);
}

// Longest block row and spread of block-row lengths (max_blc_per_row,
// stand) of an mBSR matrix; one host read-back.
int block_row_stats(amgt_bsr *A, cudaStream_t s);

// Segmented SpMV (long-row path) with caller-provided partial-sum scratch
// of 4 * A->warpnum doubles; allocates nothing (spmv.cu).
int spmv_segmented_with_scratch(int prec, double alpha, const amgt_bsr *A, const double *x, double beta, double *y,
                                double *part, int sm_count, cudaStream_t s);

// Autotuner table (autotune.cu): the SpMV lanes per block row chosen for
// A (0: none), and dropping A's entries when it is freed.
int tuned_lpr(const amgt_bsr *A);
void tune_forget(const amgt_bsr *A);

// y = beta * y (y = 0 when beta == 0) over n entries (spmv.cu).
int scale_vector(long long n, double beta, double *y, int sm_count, cudaStream_t s);

// Fused SpMV forms (spmv.cu): r = f - A u; u_out = u + w (f - A u) .* inv_l1;
// out = A u with per-CTA partials of u . out (grid CTAs, from epi_grid);
// l1 row norms (or their inverses).
int epi_grid(const amgt_bsr *A, int sm_count);
int spmv_residual(int prec, const amgt_bsr *A, const double *f, const double *u, double *r, cudaStream_t s,
                  int sm_count);
int spmv_jacobi(int prec, const amgt_bsr *A, const double *inv_l1, double w, const double *f, const double *u,
                double *u_out, cudaStream_t s, int sm_count);
int spmv_dot(int prec, const amgt_bsr *A, const double *u, double *out, double *partial, int grid, cudaStream_t s);
// f = R t with amgt_spmv's arithmetic (alpha 1, beta 0) and, in the same
// pass, u = w f ./ l1 (jacobi_zero_kernel's arithmetic): a restriction and
// the coarser level's first l1-Jacobi sweep from a zero guess.  R must be
// restrict_fusable (non-empty, not on the segmented path).
bool restrict_fusable(const amgt_bsr *R);
int spmv_restrict_jacobi0(int prec, const amgt_bsr *R, const double *t, double *f, const double *inv_l1, double w,
                          double *u, cudaStream_t s, int sm_count);
int bsr_l1_norms(const amgt_bsr *A, double *l1, int invert, cudaStream_t s, int sm_count);

// Packed-value forms (packed.cu), same contracts as the dense ones.
int pbsr_grid(const amgt_pbsr *A, int sm_count);
int pbsr_spmv(const amgt_pbsr *A, double alpha, const double *x, double beta, double *y, cudaStream_t s,
              int sm_count);
int pbsr_residual(const amgt_pbsr *A, const double *f, const double *u, double *r, cudaStream_t s, int sm_count);
int pbsr_jacobi(const amgt_pbsr *A, const double *inv_l1, double w, const double *f, const double *u, double *u_out,
                cudaStream_t s, int sm_count);
int pbsr_dot(const amgt_pbsr *A, const double *u, double *out, double *partial, int grid, cudaStream_t s);

// Exact narrow storage (convert.cu): launch the value check of A into
// *flag (bit 0: not all fp32 values, bit 1: not all fp16 values; *flag
// zeroed by the caller), then, with the flag read back, build the exact
// shadow and set A->exact_prec.
// bsr_exact_check also writes the fp16 shadow (allocating it when absent:
// *own16 set), so that fp16-exact matrices need no second pass.
int bsr_exact_check(amgt_bsr *A, int64_t *flag, bool *own16, cudaStream_t s, int sm_count);
int bsr_exact_apply(amgt_bsr *A, int64_t flag, bool own16, cudaStream_t s);

// Work the conversion's fill pass can do on the values it writes, when
// every block row takes the sorted path (else `fused` stays false and the
// caller runs the separate passes): with want16, the exactness check of
// bsr_exact_check (the fp16 shadow, allocated here, and the flag bits in
// *flags), and with want32 the fp32 shadow as well; with l1, the row norms
// of bsr_l1_norms (1 / norm when invert), the same bits.  spgemm_impl takes
// the same request for its product: fp64 products write the fp16 shadow and
// the bits (and with want32 the fp32 shadow), fp32 products the fp16
// candidate beside their fp32 values and its bit.
struct CvtFuse {
    bool want16 = false;
    bool want32 = false;  // with want16: write the fp32 shadow as well (an operator used in fp32)
    int64_t *flags = nullptr;
    double *l1 = nullptr;
    int invert = 0;
    bool fused = false;  // out
};

// amgt_csr_to_bsr with a host callback run between the queued count pass
// and the wait for the block count, and the optional fused work above
// (convert.cu).
int csr_to_bsr_impl(const amgt_csr *A, amgt_bsr *out, amgt_stream_t stream, int (*between)(void *), void *ctx,
                    CvtFuse *fuse = nullptr);

// amgt_spgemm with a host callback run between the queued symbolic pass
// and the wait for C's size (spgemm.cu); at fp64 with fuse->want16 the
// numeric pass also writes C's fp16 shadow and exactness bits (fuse->l1
// unused).
int spgemm_impl(int prec, const amgt_bsr *A, const amgt_bsr *B, amgt_bsr *C, amgt_csr *Ccsr, amgt_stream_t stream,
                int (*between)(void *), void *ctx, CvtFuse *fuse = nullptr);

// amgt_bsr_transpose; with16: A's fp16 shadow, when present, is
// transposed with the values (convert.cu).
int bsr_transpose_impl(const amgt_bsr *A, amgt_bsr *out, amgt_stream_t stream, bool with16, bool with32 = false);

// Exclusive scan of n ints (in may equal out), CUB with allocator scratch.
int exclusive_scan_int(const int *in, int *out, int n, cudaStream_t s);
// Exclusive scan of n 64-bit ints.
int exclusive_scan_i64(const int64_t *in, int64_t *out, int n, cudaStream_t s);

// Device-to-host read of `count` (<= 63) int64 slots into the calling
// thread's pinned staging for this device, and a stream synchronize;
// returns a pointer to the pinned slots (valid until the thread's next
// read_back on the device).
int read_back(const int64_t *dev, int count, cudaStream_t s, const int64_t **host);
// Pinned host blocks for the handles' read-back slots, from a library cache
// reused across handles (cudaMallocHost only on a miss); pinned_put returns
// a block to the cache, amgt_trim_pool frees the cached ones.
int pinned_get(size_t bytes, void **out);
void pinned_put(void *p);

// ----------------------------------------------------------------- bitmaps
// Boolean 4x4 product of two block bitmaps (bit r*4+c = entry (r, c)): OR
// over k of column k of a (bits r*4+k) times row k of b (bits 4k..4k+3).
__host__ __device__ __forceinline__ uint32_t bitmap_mul(uint32_t a, uint32_t b)
{
    uint32_t res = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t colk = (a >> k) & 0x1111u;
        uint32_t rowk = (b >> (4 * k)) & 0xFu;
        res |= (colk * 0xFu) & (rowk * 0x1111u);
    }
    return res & 0xFFFFu;
}

// Transpose of a 4x4 block bitmap.
__host__ __device__ __forceinline__ uint32_t bitmap_transpose(uint32_t m)
{
    uint32_t t = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (m & (1u << (4 * r + c))) t |= 1u << (4 * c + r);
    return t;
}

constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int *total)
{
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    *total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// Sum over the full warp (one redux.sync; two's complement wraps alike).
__device__ __forceinline__ int warp_sum(int v) { return (int)__reduce_add_sync(FULL, (unsigned)v); }

// Grid sizes: a multiple of the SM count, capped by the work.
inline int grid_for(int units_per_cta, long long units, int sm_count, int ctas_per_sm = 8)
{
    long long need = (units + units_per_cta - 1) / units_per_cta;
    long long cap = (long long)sm_count * ctas_per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

}  // namespace amgt
