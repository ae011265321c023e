// Value loaders shared by the dense and the packed mBSR SpMV kernels.
#pragma once

#include "amgt_internal.cuh"

namespace amgt {

template <int PREC>
struct ValTraits;
template <>
struct ValTraits<AMGT_DOUBLE> {
    using acc_t = double;
};
template <>
struct ValTraits<AMGT_FLOAT> {
    using acc_t = float;
};
template <>
struct ValTraits<AMGT_HALF> {
    using acc_t = float;
};
template <>
struct ValTraits<AMGT_BF16> {
    using acc_t = float;
};
// Internal storage modes for fp64 arithmetic on values that the fp32 or
// fp16 shadow holds exactly (amgt_bsr.exact_prec): the shadow is read and
// widened exactly, the sums are the fp64 kernel's, bit for bit.
constexpr int kExact32 = 4;
constexpr int kExact16 = 5;
template <>
struct ValTraits<kExact32> {
    using acc_t = double;
};
template <>
struct ValTraits<kExact16> {
    using acc_t = double;
};

// Row q of block k as 4 values in the accumulation type.
template <int PREC>
__device__ __forceinline__ void load_block_row(const void *__restrict__ val, long long k, int q,
                                               typename ValTraits<PREC>::acc_t v[4])
{
    if constexpr (PREC == AMGT_DOUBLE) {
        const double2 *p = reinterpret_cast<const double2 *>(val) + (k * 8 + q * 2);
        const double2 a = __ldcs(p), b = __ldcs(p + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else if constexpr (PREC == AMGT_FLOAT || PREC == kExact32) {
        const float4 a = __ldcs(reinterpret_cast<const float4 *>(val) + (k * 4 + q));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
        const uint2 a = __ldcs(reinterpret_cast<const uint2 *>(val) + (k * 4 + q));
        if constexpr (PREC == AMGT_HALF || PREC == kExact16) {
            const float2 f0 = __half22float2(*reinterpret_cast<const __half2 *>(&a.x));
            const float2 f1 = __half22float2(*reinterpret_cast<const __half2 *>(&a.y));
            v[0] = f0.x; v[1] = f0.y; v[2] = f1.x; v[3] = f1.y;
        } else {
            const float2 f0 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&a.x));
            const float2 f1 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&a.y));
            v[0] = f0.x; v[1] = f0.y; v[2] = f1.x; v[3] = f1.y;
        }
    }
}

// x[4*col .. 4*col+3]; SAFE: scalar loads with the n bound (last block
// column when n % 4 != 0, or x not 16-byte aligned).
template <bool SAFE>
__device__ __forceinline__ void load_x4(const double *__restrict__ x, int col, int n, double xv[4])
{
    if constexpr (!SAFE) {
        const double2 *p = reinterpret_cast<const double2 *>(x + 4LL * col);
        const double2 a = __ldg(p), b = __ldg(p + 1);
        xv[0] = a.x; xv[1] = a.y; xv[2] = b.x; xv[3] = b.y;
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long long j = 4LL * col + c;
            xv[c] = (j < n) ? __ldg(x + j) : 0.0;
        }
    }
}

}  // namespace amgt
