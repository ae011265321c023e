// Sorted union of (key, bitmap) pairs for one block row, done by one warp.
//
// Both the CSR -> mBSR conversion (keys = block columns of the 4 CSR rows'
// entries) and the SpGEMM symbolic phase (keys = block columns of B blocks
// whose bitmap product with the A block is non-zero) reduce a block row's
// list of pairs to its sorted distinct keys with the OR of their bitmaps.
// Pairs are packed into 64 bits as key << 32 | tag << 16 | bitmap, so one
// ascending sort orders by key and then by the producer's tag (entry index),
// which keeps every output independent of thread timing.
#pragma once

#include "amgt_internal.cuh"

namespace amgt {

constexpr unsigned long long kSentinel = ~0ull;  // sorts last

__device__ __forceinline__ unsigned long long pack_pair(int key, int tag, uint32_t map)
{
    return ((unsigned long long)(unsigned)key << 32) | ((unsigned long long)(tag & 0xFFFF) << 16) |
           (unsigned long long)(map & 0xFFFFu);
}
__device__ __forceinline__ int pair_key(unsigned long long p) { return (int)(p >> 32); }
__device__ __forceinline__ int pair_tag(unsigned long long p) { return (int)((p >> 16) & 0xFFFF); }
__device__ __forceinline__ uint32_t pair_map(unsigned long long p) { return (uint32_t)(p & 0xFFFFu); }

// Bitonic sort of 32 values held one per lane, ascending by lane.
__device__ __forceinline__ unsigned long long warp_sort32(unsigned long long v, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            unsigned long long o = __shfl_xor_sync(FULL, v, j);
            bool up = (lane & k) == 0;
            bool lower = (lane & j) == 0;
            unsigned long long lo = v < o ? v : o, hi = v < o ? o : v;
            v = (lower == up) ? lo : hi;
        }
    }
    return v;
}

// Bitonic sort of n (power of two, >= 64) values in shared memory by one warp.
__device__ __forceinline__ void warp_sort_smem(unsigned long long *s, int n, int lane)
{
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < n; i += 32) {
                int ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long a = s[i], b = s[ixj];
                    bool asc = (i & k) == 0;
                    if ((a > b) == asc) {
                        s[i] = b;
                        s[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Lanes hold sorted pairs (one per lane, sentinels last).  Returns, per
// lane, whether it heads a run of equal keys, and in *orv the OR of the
// bitmaps of the run that starts at this lane (valid on heads).
__device__ __forceinline__ bool warp_runs32(unsigned long long v, int lane, uint32_t *orv)
{
    const int key = pair_key(v);
    const bool valid = v != kSentinel;
    const int prev = __shfl_up_sync(FULL, key, 1);
    const bool head = valid && (lane == 0 || prev != key);
    uint32_t m = pair_map(v);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t om = __shfl_down_sync(FULL, m, o);
        int ok = __shfl_down_sync(FULL, key, o);
        bool ov = __shfl_down_sync(FULL, valid ? 1 : 0, o);
        if (lane + o < 32 && ov && ok == key) m |= om;
    }
    *orv = m;
    return head;
}

__device__ __forceinline__ int next_pow2_min64(int n)
{
    int p = 64;
    while (p < n) p <<= 1;
    return p;
}

}  // namespace amgt
