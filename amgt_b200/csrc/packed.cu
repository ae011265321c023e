// Bitmap-packed mBSR values and the SpMV / smoother kernels on them.
//
// mBSR stores 16 values per 4x4 block; AMG operators fill about 4 of them
// (7-point Poisson at 128^3: 14.6M nonzeros in 3.6M blocks), so a
// bandwidth-bound SpMV reads ~3x more value bytes than it needs.  The
// packed form keeps the block structure (block-row pointers, block columns
// and bitmaps, borrowed from the mBSR matrix) and stores only the values of
// set bits, block after block, in bitmap order (row-major inside the
// block), plus each block's and each block row's offset into that array.
// Bytes per block: 4 (column) + 2 (bitmap) + 4 (offset) + s * set bits.
#include <cstdlib>

#include "spmv_common.cuh"

namespace amgt {

enum { PEPI_AXPBY = 0, PEPI_RESID = 1, PEPI_JACOBI = 2, PEPI_DOT = 3 };

struct PEpiArgs {
    double alpha, beta;    // AXPBY
    const double *f;       // RESID, JACOBI
    const double *inv_l1;  // JACOBI
    double w;              // JACOBI
    double *out;           // y (AXPBY reads it when beta != 0)
    double *partial;       // DOT: [gridDim.x]
};

template <int PREC>
struct PackedT {
    using val_t = double;
};
template <>
struct PackedT<AMGT_FLOAT> {
    using val_t = float;
};
template <>
struct PackedT<AMGT_HALF> {
    using val_t = unsigned short;
};
template <>
struct PackedT<AMGT_BF16> {
    using val_t = unsigned short;
};

template <int PREC>
__device__ __forceinline__ typename ValTraits<PREC>::acc_t widen(typename PackedT<PREC>::val_t v)
{
    if constexpr (PREC == AMGT_HALF) return __half2float(__ushort_as_half(v));
    else if constexpr (PREC == AMGT_BF16) return __bfloat162float(__ushort_as_bfloat16(v));
    else return v;
}

// SpMV on the packed values, each block's first value given (blcVoff):
// laid out like the 16-value kernel — LPR lanes per block row, 4 lanes per block,
// lane q taking block row q, the row's blocks dealt to the LPR/4 lane
// groups two per step — with lane q reading only its row's stored values
// (popc of its bitmap nibble, from voff[k] + the set bits before it) and an
// FMA for every column, zero where the bit is clear: the sums of the
// 16-value kernel at the same lanes per row, bit for bit, from a third of
// the bytes at AMG fills.  A block's column, bitmap and value offset load
// together, its values and x one trip later.
template <int PREC, bool SAFE>
__device__ __forceinline__ typename ValTraits<PREC>::acc_t pblock_dot(const typename PackedT<PREC>::val_t *__restrict__ val,
                                                                      const double *__restrict__ x, int n, int vo,
                                                                      uint32_t mp, int q, int col,
                                                                      typename ValTraits<PREC>::acc_t acc)
{
    using acc_t = typename ValTraits<PREC>::acc_t;
    const uint32_t nib = (mp >> (4 * q)) & 0xFu;
    int o = vo + __popc(mp & ((1u << (4 * q)) - 1u));
    double xv[4];
    load_x4<SAFE>(x, col, n, xv);
    acc_t w[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        w[c] = (acc_t)0;
        if ((nib >> c) & 1u) w[c] = widen<PREC>(__ldcs(val + o++));
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) acc = fma(w[c], (acc_t)xv[c], acc);
    return acc;
}

template <int PREC, int LPR, bool SAFE, int EPI>
__global__ void __launch_bounds__(256)
pspmv_off_kernel(int m, int n, int brow, const int *__restrict__ ptr, const int *__restrict__ idx,
                 const uint16_t *__restrict__ map, const int *__restrict__ voff, const void *__restrict__ valv,
                 const double *__restrict__ x, PEpiArgs e)
{
    grid_dependency_wait();  // launched with programmatic dependent launch
    using acc_t = typename ValTraits<PREC>::acc_t;
    using val_t = typename PackedT<PREC>::val_t;
    constexpr int RPW = 32 / LPR;
    constexpr int G = LPR / 4;
    __shared__ double sred[8];
    const val_t *__restrict__ val = static_cast<const val_t *>(valv);
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPR, l = lane % LPR, g = l >> 2, q = l & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double dot = 0.0;
    for (int b0 = warp * RPW; b0 < brow; b0 += nwarps * RPW) {
        const int b = b0 + sub;
        const bool live = b < brow;
        acc_t acc = 0;
        if (live) {
            int k = ptr[b] + g;
            const int end = ptr[b + 1];
            for (; k + G < end; k += 2 * G) {
                const int c0 = __ldcs(idx + k), c1 = __ldcs(idx + k + G);
                const uint32_t m0 = __ldcs(map + k), m1 = __ldcs(map + k + G);
                const int o0 = __ldcs(voff + k), o1 = __ldcs(voff + k + G);
                acc = pblock_dot<PREC, SAFE>(val, x, n, o0, m0, q, c0, acc);
                acc = pblock_dot<PREC, SAFE>(val, x, n, o1, m1, q, c1, acc);
            }
            if (k < end) acc = pblock_dot<PREC, SAFE>(val, x, n, __ldcs(voff + k), __ldcs(map + k), q, __ldcs(idx + k), acc);
        }
#pragma unroll
        for (int o = 4; o < LPR; o <<= 1) acc += __shfl_xor_sync(FULL, acc, o);
        if (live && g == 0) {
            const int row = 4 * b + q;
            if (row < m) {
                const double ax = (double)acc;
                if constexpr (EPI == PEPI_AXPBY) {
                    const double t = e.alpha * ax;
                    e.out[row] = (e.beta == 0.0) ? t : t + e.beta * e.out[row];
                } else if constexpr (EPI == PEPI_RESID) {
                    e.out[row] = e.f[row] - ax;
                } else if constexpr (EPI == PEPI_JACOBI) {
                    e.out[row] = x[row] + e.w * (e.f[row] - ax) * e.inv_l1[row];
                } else {
                    e.out[row] = ax;
                    dot += x[row] * ax;
                }
            }
        }
    }
    if constexpr (EPI == PEPI_DOT) {
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

// ------------------------------------------------------------- packing
__global__ void popc_kernel(int nblk, const uint16_t *__restrict__ map, int *__restrict__ cnt)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nblk; k += gridDim.x * blockDim.x)
        cnt[k] = __popc((uint32_t)map[k]);
}

// row offset = value offset of the row's first block
__global__ void row_offset_kernel(int brow, const int *__restrict__ ptr, const int *__restrict__ voff,
                                  int *__restrict__ rvoff)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= brow; b += gridDim.x * blockDim.x)
        rvoff[b] = voff[ptr[b]];
}

template <int PREC>
__global__ void pack_kernel(long long nblk, const uint16_t *__restrict__ map, const int *__restrict__ voff,
                            const double *__restrict__ val, void *__restrict__ out)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < 16 * nblk;
         t += (long long)gridDim.x * blockDim.x) {
        const long long k = t >> 4;
        const int e = (int)(t & 15);
        const uint32_t mp = map[k];
        if (!((mp >> e) & 1u)) continue;
        const long long dst = voff[k] + __popc(mp & ((1u << e) - 1u));
        const double v = val[t];
        if (PREC == AMGT_DOUBLE) static_cast<double *>(out)[dst] = v;
        else if (PREC == AMGT_FLOAT) static_cast<float *>(out)[dst] = __double2float_rn(v);
        else if (PREC == AMGT_HALF) static_cast<__half *>(out)[dst] = __double2half(v);
        else static_cast<__nv_bfloat16 *>(out)[dst] = __double2bfloat16(v);
    }
}

static int packed_lpr(const amgt_pbsr *A)
{
    static int env = -1;
    if (env < 0) {
        const char *ev = getenv("AMGT_PSPMV_LPR");
        env = ev ? atoi(ev) : 0;
    }
    if (env == 4 || env == 8 || env == 16 || env == 32) return env;
    // the 16-value kernel's choice from the mean block-row length, so that
    // the offset kernel's sums are that kernel's
    const double avg = A->blc_row ? (double)A->blc_num / A->blc_row : 0.0;
    if (avg <= 4.0) return 4;
    if (avg <= 10.0) return 8;
    if (avg <= 20.0) return 16;
    return 32;
}

int pbsr_grid(const amgt_pbsr *A, int sm_count)
{
    return grid_for(8 * (32 / packed_lpr(A)), A->blc_row, sm_count, 8);
}

template <int PREC, int EPI>
static int launch_packed(const amgt_pbsr *A, const double *x, const PEpiArgs &e, int grid, cudaStream_t s)
{
    const bool safe = (A->col % 4 != 0) || ((uintptr_t)x % 16 != 0);
    const int lpr = packed_lpr(A);
#define AMGT_P_CASE(L)                                                                                       \
    if (lpr == L) {                                                                                          \
        if (safe)                                                                                            \
            AMGT_LAUNCH_PDL((pspmv_off_kernel<PREC, L, true, EPI>), grid, 256, 0, s, A->row, A->col,          \
                            A->blc_row, A->blcPtr, A->blcIdx, A->blcMap, A->blcVoff, A->val, x, e);          \
        else                                                                                                 \
            AMGT_LAUNCH_PDL((pspmv_off_kernel<PREC, L, false, EPI>), grid, 256, 0, s, A->row, A->col,         \
                            A->blc_row, A->blcPtr, A->blcIdx, A->blcMap, A->blcVoff, A->val, x, e);          \
        return AMGT_OK;                                                                                      \
    }
    AMGT_P_CASE(4)
    AMGT_P_CASE(8)
    AMGT_P_CASE(16)
    AMGT_P_CASE(32)
#undef AMGT_P_CASE
    return AMGT_ERR_INVALID;
}

template <int EPI>
static int launch_packed_prec(const amgt_pbsr *A, const double *x, const PEpiArgs &e, int grid, cudaStream_t s)
{
    switch (A->prec) {
    case AMGT_DOUBLE: return launch_packed<AMGT_DOUBLE, EPI>(A, x, e, grid, s);
    case AMGT_FLOAT: return launch_packed<AMGT_FLOAT, EPI>(A, x, e, grid, s);
    case AMGT_HALF: return launch_packed<AMGT_HALF, EPI>(A, x, e, grid, s);
    case AMGT_BF16: return launch_packed<AMGT_BF16, EPI>(A, x, e, grid, s);
    default: return AMGT_ERR_INVALID;
    }
}

int pbsr_spmv(const amgt_pbsr *A, double alpha, const double *x, double beta, double *y, cudaStream_t s,
              int sm_count)
{
    PEpiArgs e{alpha, beta, nullptr, nullptr, 0.0, y, nullptr};
    return launch_packed_prec<PEPI_AXPBY>(A, x, e, pbsr_grid(A, sm_count), s);
}

int pbsr_residual(const amgt_pbsr *A, const double *f, const double *u, double *r, cudaStream_t s, int sm_count)
{
    PEpiArgs e{0.0, 0.0, f, nullptr, 0.0, r, nullptr};
    return launch_packed_prec<PEPI_RESID>(A, u, e, pbsr_grid(A, sm_count), s);
}

int pbsr_jacobi(const amgt_pbsr *A, const double *inv_l1, double w, const double *f, const double *u, double *u_out,
                cudaStream_t s, int sm_count)
{
    PEpiArgs e{0.0, 0.0, f, inv_l1, w, u_out, nullptr};
    return launch_packed_prec<PEPI_JACOBI>(A, u, e, pbsr_grid(A, sm_count), s);
}

int pbsr_dot(const amgt_pbsr *A, const double *u, double *out, double *partial, int grid, cudaStream_t s)
{
    PEpiArgs e{0.0, 0.0, nullptr, nullptr, 0.0, out, partial};
    return launch_packed_prec<PEPI_DOT>(A, u, e, grid, s);
}

}  // namespace amgt

using namespace amgt;

extern "C" {

int amgt_pbsr_free(amgt_pbsr *A, amgt_stream_t stream)
{
    if (!A) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    free_ptr(A->rowVoff, s);
    free_ptr(A->blcVoff, s);
    free_ptr(A->val, s);
    memset(A, 0, sizeof(*A));
    return AMGT_OK;
}

int amgt_bsr_pack(const amgt_bsr *A, int prec, amgt_pbsr *out, amgt_stream_t stream)
{
    if (!A || !out || prec < AMGT_DOUBLE || prec > AMGT_BF16) return AMGT_ERR_INVALID;
    if (A->blc_num > 0 && (!A->blcVal || !A->blcMap)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    memset(out, 0, sizeof(*out));
    out->row = A->row;
    out->col = A->col;
    out->blc_row = A->blc_row;
    out->blc_col = A->blc_col;
    out->blc_num = A->blc_num;
    out->prec = prec;
    out->blcPtr = A->blcPtr;
    out->blcIdx = A->blcIdx;
    out->blcMap = A->blcMap;
    out->max_blc_per_row = A->max_blc_per_row;
    const int nb = A->blc_num;
    int *cnt = nullptr, *voff = nullptr;
    int64_t *tot = nullptr;
    const int64_t *h = nullptr;
    int rc = AMGT_OK;
    const size_t vs = prec == AMGT_DOUBLE ? 8 : (prec == AMGT_FLOAT ? 4 : 2);
    if ((rc = alloc_n(&voff, (size_t)nb + 1, s)) || (rc = alloc_n(&out->rowVoff, (size_t)A->blc_row + 1, s)) ||
        (rc = alloc_n(&cnt, (size_t)nb + 1, s)) || (rc = alloc_n(&tot, 1, s)))
        goto fail;
    AMGT_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nb + 1), s));
    AMGT_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(int64_t), s));
    if (nb > 0) AMGT_LAUNCH(popc_kernel, grid_for(256, nb, st->sm_count, 8), 256, 0, s, nb, A->blcMap, cnt);
    if ((rc = exclusive_scan_int(cnt, voff, nb + 1, s))) goto fail;
    AMGT_LAUNCH(row_offset_kernel, grid_for(256, A->blc_row + 1LL, st->sm_count, 8), 256, 0, s, A->blc_row,
                A->blcPtr, voff, out->rowVoff);
    if (A->csr_nnz > 0 || nb == 0) {
        out->nnz = A->csr_nnz;  // number of set bits, known: no read-back
    } else {
        AMGT_CUDA_TRY(cudaMemcpyAsync(tot, voff + nb, sizeof(int), cudaMemcpyDeviceToDevice, s));
        if ((rc = read_back(tot, 1, s, &h))) goto fail;
        out->nnz = (int)h[0];
    }
    // 4 values of padding: the kernels read a row's 4 candidates unconditionally
    out->val = dev_alloc(((size_t)out->nnz + 4) * vs, s);
    if (!out->val) { rc = AMGT_ERR_ALLOC; goto fail; }
    AMGT_CUDA_TRY(cudaMemsetAsync((char *)out->val + (size_t)out->nnz * vs, 0, 4 * vs, s));
    if (nb > 0) {
        const int grid = grid_for(256, 16LL * nb, st->sm_count, 8);
        switch (prec) {
        case AMGT_DOUBLE: AMGT_LAUNCH(pack_kernel<AMGT_DOUBLE>, grid, 256, 0, s, (long long)nb, A->blcMap, voff, A->blcVal, out->val); break;
        case AMGT_FLOAT: AMGT_LAUNCH(pack_kernel<AMGT_FLOAT>, grid, 256, 0, s, (long long)nb, A->blcMap, voff, A->blcVal, out->val); break;
        case AMGT_HALF: AMGT_LAUNCH(pack_kernel<AMGT_HALF>, grid, 256, 0, s, (long long)nb, A->blcMap, voff, A->blcVal, out->val); break;
        default: AMGT_LAUNCH(pack_kernel<AMGT_BF16>, grid, 256, 0, s, (long long)nb, A->blcMap, voff, A->blcVal, out->val); break;
        }
    }
    free_ptr(cnt, s);
    free_ptr(tot, s);
    out->blcVoff = voff;  // each block's first value (the offset kernel's index)
    return AMGT_OK;
fail:
    free_ptr(cnt, s);
    free_ptr(tot, s);
    free_ptr(voff, s);
    amgt_pbsr_free(out, stream);
    return rc;
}

int amgt_pbsr_spmv(double alpha, const amgt_pbsr *A, const double *x, double beta, double *y, amgt_stream_t stream)
{
    if (!A || (A->row > 0 && !y)) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (A->blc_num > 0 && (!x || !A->val || !A->rowVoff)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return pbsr_spmv(A, alpha, x, beta, y, (cudaStream_t)stream, st->sm_count);
}

int amgt_pbsr_residual(const amgt_pbsr *A, const double *f, const double *u, double *r, amgt_stream_t stream)
{
    if (!A || (A->row > 0 && (!f || !u || !r))) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return pbsr_residual(A, f, u, r, (cudaStream_t)stream, st->sm_count);
}

int amgt_pbsr_jacobi(const amgt_pbsr *A, const double *inv_l1, double weight, const double *f, const double *u,
                     double *u_out, amgt_stream_t stream)
{
    if (!A || A->row != A->col) return AMGT_ERR_INVALID;
    if (A->row == 0) return AMGT_OK;
    if (!inv_l1 || !f || !u || !u_out || u == u_out) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    return pbsr_jacobi(A, inv_l1, weight, f, u, u_out, (cudaStream_t)stream, st->sm_count);
}

}  // extern "C"
