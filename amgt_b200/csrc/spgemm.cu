// mBSR SpGEMM: C = A * B.
//
// Replaces spgemm_amgT_fp64 / _fp32 / _fp16 and the kernels compute_Cub_bin,
// set_bin, symbolic_spgemm_step1/2 (+_large, _gl), numeric_spgemm_hybrid
// (+_tf32, _f16) and bsr2csr_* (AmgT_HYPRE/src/seq_mv/csr_spgemm_device.c:
// 82-1440, 1527-2578).
//
// Symbolic.  One warp owns one block row of A.  For each A block (row
// order) the lanes walk the B row it selects; every B block whose bitmap
// product with the A block is non-zero (bitMatrixMul, :189-205) becomes a
// (B block column, product bitmap) pair, appended to the warp's shared
// memory list.  Equal columns are merged with an OR of their bitmaps and
// the distinct columns sorted (rows of <= 32 pairs in registers, <= 256
// through a shared hash table and a sort of the distinct columns, <= 1024
// pairs inserted straight into the hash table as they are formed): that is
// C's block pattern and C's bitmap, bit for bit.  Rows with more than 1024
// pairs go to a CTA that sweeps the column range in windows of 8192 with a
// shared-memory bitmap table.  One pass: each
// row's sorted pattern goes to its slice of a scratch array (offsets from a
// scan of the per-row pair bounds) with its block and CSR counts; one host
// read-back then sizes C, and the numeric kernel moves the pattern into C.
//
// Numeric.  One warp per A block row; the row's (A block, B block) pairs
// are flattened and taken 8 at a time, 4 lanes per pair (lane r: row r of
// the 4x4 product), B blocks staged through shared memory, so that every
// load of a step is in flight at once.  In fp64, entry (r, c) of a product
// is the fused multiply-add chain t = fma(a[r][k], b[k][c], t) over k
// ascending from zero, and products are added to their C block in A block
// order: the arithmetic of the reference's fp64 kernel, whose scalar
// branch's `temp += a * b` (:1317) nvcc contracts into that chain and
// whose m8n8k4 branch (:1173-1262) takes every k term; so the fp64 result
// equals the oracle's restatement of that arithmetic bit for bit (for
// finite values: unstored entries are zero, and a zero term leaves an FMA
// chain unchanged).  The fp32 / fp16 / bf16 forms use separate fp32
// multiply and add.  C rows of up to 16, 24, 32 or 64 blocks (by the
// product's row lengths) accumulate in shared memory, longer rows in place.  FP64
// arithmetic on the CUDA cores: the 4x4 products are too small for tcgen05
// (M >= 64), and on B200 the fp64 MMA rate equals the fp64 FMA rate.  The
// CSR form of C is written by the same kernel (no separate BSR2CSR pass).
#include <atomic>

#include "rowunion.cuh"

namespace amgt {

constexpr int kSymWarps = 4;
constexpr int kSymCap = 1024;     // pairs a warp sorts in shared memory
constexpr int kSymWin = 8192;     // key window of the large-row path
constexpr int kSymLargeThreads = 256;
constexpr int kNumWarps = 4;
constexpr int kNumCap = 32;       // C blocks a warp accumulates in shared memory (products of short C rows)
constexpr int kNumCapWide = 64;   // the same for products whose C rows mostly exceed kNumCap blocks
constexpr int kNumCapNarrow = 16; // the same for products of at most 16 C blocks per row
constexpr int kNumCapMid = 24;    // ... and of at most 24
// CTAs per SM of the numeric kernel for an accumulator capacity: shared
// memory and registers (64 / 72 / 80 / 128 per thread) both allow that many
__host__ __device__ constexpr int num_ctas_per_sm(int cap)
{
    return cap <= 16 ? 8 : cap <= 24 ? 7 : cap <= 32 ? 6 : 4;
}
constexpr int kNumWin = 128;      // pairs per window of the numeric's pair list
constexpr int kOrdCap = 512;      // C blocks of a row the order kernel counts in shared memory

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// A row of the symbolic pass: its block row, A block range and scratch
// slice (offset, capacity = the pair bound, saturated).
struct SymRow {
    int b, a0, a1, ub;
    long long base;
};

// The row of work item t (b = -1 past the end), read ahead of its use.
__device__ __forceinline__ SymRow sym_row(int t, int nr, const int *__restrict__ rows, const int *__restrict__ aptr,
                                          const int64_t *__restrict__ ub_off)
{
    SymRow h{-1, 0, 0, 0, 0};
    if (t < nr) {
        h.b = rows ? rows[t] : t;
        h.a0 = aptr[h.b];
        h.a1 = aptr[h.b + 1];
        h.base = ub_off[h.b];
        const long long u = ub_off[h.b + 1] - h.base;
        h.ub = u > 0x7FFFFFFF ? 0x7FFFFFFF : (int)u;
    }
    return h;
}

// This lane's A block of a row's first 32 (column k, bitmap) and the range
// of the B row it selects, read in two steps a row ahead of their use.
struct SymLane {
    int k, j0, len;
    uint32_t ma;
};
template <int CAP>
__device__ __forceinline__ void sym_lane_a(const SymRow &h, int lane, const int *__restrict__ aidx,
                                           const uint16_t *__restrict__ amap, SymLane &l)
{
    l.k = -1;
    l.ma = 0;
    if (h.b >= 0 && h.ub <= CAP && h.a0 + lane < h.a1) {
        l.k = aidx[h.a0 + lane];
        l.ma = amap[h.a0 + lane];
    }
}
__device__ __forceinline__ void sym_lane_b(SymLane &l, const int *__restrict__ bptr)
{
    l.j0 = 0;
    l.len = 0;
    if (l.k >= 0) {
        l.j0 = bptr[l.k];
        l.len = bptr[l.k + 1] - l.j0;
    }
}

// Appends the row's non-zero-product pairs to the warp's list s[]; returns
// the count (the caller bounds it via the upper bound).  Up to 32 A blocks
// at a time: lane i fetches A block i's B row range (for the first 32,
// `pre`, read ahead by the caller), a warp scan of the range lengths
// flattens the (A block, B block) pairs, and lane t takes pair t, finding
// its A block by a five-step shuffle search; so every load of a chunk is in
// flight at once.  Pairs come out in (A block, B block)
// order, tagged with their ordinal in the row (< 65536: rows here have at
// most kSymCap pairs); pslot[ordinal] = 0xFFFF marks the pairs whose
// bitmap product is zero (they add nothing to C).
__device__ __forceinline__ int sym_collect(int lane, int a0, int a1, const SymLane &pre,
                                           const int *__restrict__ aidx, const uint16_t *__restrict__ amap,
                                           const int *__restrict__ bptr, const int *__restrict__ bidx,
                                           const uint16_t *__restrict__ bmap, unsigned long long *s,
                                           uint16_t *__restrict__ pslot)
{
    int cnt = 0, qbase = 0;
    for (int ib = a0; ib < a1; ib += 32) {
        const int i = ib + lane;
        int j0 = 0, len = 0;
        uint32_t ma = 0;
        if (ib == a0) {
            j0 = pre.j0;
            len = pre.len;
            ma = pre.ma;
        } else if (i < a1) {
            const int k = aidx[i];
            ma = amap[i];
            j0 = bptr[k];
            len = bptr[k + 1] - j0;
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        const int excl = incl - len;
        for (int t0 = 0; t0 < total; t0 += 32) {
            const int t = t0 + lane;
            int src = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(FULL, incl, min(src + step - 1, 31));
                if (v <= t) src += step;
            }
            src = min(src, 31);
            const int sj0 = __shfl_sync(FULL, j0, src), sex = __shfl_sync(FULL, excl, src);
            const uint32_t sma = __shfl_sync(FULL, ma, src);
            uint32_t mc = 0;
            int key = 0;
            if (t < total) {
                const int j = sj0 + (t - sex);
                mc = bitmap_mul(sma, bmap[j]);
                key = bidx[j];
                if (!mc) pslot[qbase + t] = 0xFFFF;
            }
            const unsigned bal = __ballot_sync(FULL, mc != 0);
            if (mc) s[cnt + __popc(bal & lanemask_lt(lane))] = pack_pair(key, qbase + t, mc);
            cnt += __popc(bal);
        }
        qbase += total;
    }
    __syncwarp();
    return cnt;
}

// Upper bound of the row's pairs: sum of the selected B row lengths.
__device__ __forceinline__ long long sym_upper_bound(int lane, int a0, int a1, const int *__restrict__ aidx,
                                                     const int *__restrict__ bptr)
{
    long long ub = 0;
    for (int i = a0 + lane; i < a1; i += 32) {
        const int k = aidx[i];
        ub += bptr[k + 1] - bptr[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ub += __shfl_xor_sync(FULL, ub, o);
    return ub;
}

// Sorted distinct keys with OR-ed bitmaps of the warp's list s[0..cnt),
// cnt <= 32 (one pair per lane).  Lanes with equal keys match
// (__match_any_sync); the lowest lane of each group is its leader, and a
// key's rank among the distinct keys comes from comparing it with every
// leader's key, so no sort is needed.  The group's bitmaps are OR-ed in
// shared memory (s[] is reused for that once the pairs are in registers).
// Writes the distinct keys in ascending order to cidx/cmap, the index of
// each pair's C block to pslot (by the pair's tag, its ordinal in the row),
// and returns the distinct count and the per-scalar-row CSR counts
// (popcount of each bitmap nibble).
__device__ __forceinline__ int sym_reduce32(int lane, int cnt, unsigned long long *s, int *__restrict__ cidx,
                                            uint16_t *__restrict__ cmap, int csr[4], uint16_t *__restrict__ pslot)
{
    const bool valid = lane < cnt;
    const unsigned long long v = valid ? s[lane] : kSentinel;
    const int key = valid ? pair_key(v) : -1 - lane;
    const unsigned peers = __match_any_sync(FULL, key);
    const bool leader = valid && (__ffs(peers) - 1) == lane;
    unsigned lm = __ballot_sync(FULL, leader);
    const int u = __popc(lm);
    int rank = 0;
    while (lm) {  // warp-uniform: the distinct keys
        const int l = __ffs(lm) - 1;
        lm &= lm - 1;
        rank += __shfl_sync(FULL, key, l) < key;
    }
    unsigned *so = reinterpret_cast<unsigned *>(s);
    __syncwarp();
    so[lane] = 0;
    __syncwarp();
    if (valid) {
        atomicOr(&so[rank], pair_map(v));
        pslot[pair_tag(v)] = (uint16_t)rank;
    }
    __syncwarp();
    csr[0] = csr[1] = csr[2] = csr[3] = 0;
    if (leader) {
        const uint32_t orv = so[rank];
        cidx[rank] = key;
        cmap[rank] = (uint16_t)orv;
#pragma unroll
        for (int q = 0; q < 4; ++q) csr[q] = __popc((orv >> (4 * q)) & 0xFu);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) csr[q] = warp_sum(csr[q]);
    return u;
}

// The same for rows of more than 32 pairs (cnt <= H, H a power of two and
// a multiple of 32).  The pairs' columns are first made distinct through a
// shared hash table of H slots (atomicCAS on the column, atomicOr on the
// bitmap; linear probing, bounded by H), so only the distinct columns are
// sorted (C rows here hold a tenth of their pairs' count or fewer); each
// pair's C block is found through its table slot.  The result equals
// sorting all pairs: C's columns ascending with OR-ed bitmaps, and the rank
// of each pair's column.  pslot first receives the pairs' table slots and
// then, in a second pass over the row's npairs ordinals, their ranks.
template <int H>
__device__ int sym_reduce_hashed(int lane, int cnt, unsigned long long *s, int *tkey, unsigned *tval,
                                 int *__restrict__ cidx, uint16_t *__restrict__ cmap, int csr[4],
                                 uint16_t *__restrict__ pslot, int npairs, int *__restrict__ err)
{
    constexpr int LOG2H = __builtin_ctz(H);
    for (int i = lane; i < H; i += 32) {
        tkey[i] = -1;
        tval[i] = 0;
    }
    __syncwarp();
    for (int i = lane; i < cnt; i += 32) {
        const unsigned long long v = s[i];
        const int key = pair_key(v);
        unsigned h = ((unsigned)key * 0x9E3779B1u) >> (32 - LOG2H);
        int probe = 0;
        for (; probe < H; ++probe) {
            const int prev = atomicCAS(&tkey[h], -1, key);
            if (prev == -1 || prev == key) break;
            h = (h + 1) & (H - 1);
        }
        if (probe == H) {  // cannot happen (cnt <= H); kept as a bound
            raise_error(err, DEV_ERR_PROBE);
            continue;
        }
        atomicOr(&tval[h], pair_map(v));
        pslot[pair_tag(v)] = (uint16_t)h;
    }
    __syncwarp();
    // distinct columns -> s[0..u), tagged with their table slot
    int u = 0;
    for (int i0 = 0; i0 < H; i0 += 32) {
        const int i = i0 + lane;
        const int key = tkey[i];
        const unsigned bal = __ballot_sync(FULL, key >= 0);
        if (key >= 0) s[u + __popc(bal & lanemask_lt(lane))] = pack_pair(key, i, tval[i]);
        u += __popc(bal);
    }
    __syncwarp();
    csr[0] = csr[1] = csr[2] = csr[3] = 0;
    if (u <= 32) {  // distinct keys: rank each by comparing with all u
        const unsigned long long v = (lane < u) ? s[lane] : kSentinel;
        const int key = pair_key(v);
        int rank = 0;
        for (int l = 0; l < u; ++l) rank += __shfl_sync(FULL, key, l) < key;
        if (lane < u) {
            const uint32_t mp = pair_map(v);
            cidx[rank] = key;
            cmap[rank] = (uint16_t)mp;
            tval[pair_tag(v)] = (unsigned)rank;  // rank of the column
#pragma unroll
            for (int q = 0; q < 4; ++q) csr[q] = __popc((mp >> (4 * q)) & 0xFu);
        }
    } else {
        const int N = next_pow2_min64(u);
        for (int i = u + lane; i < N; i += 32) s[i] = kSentinel;
        __syncwarp();
        warp_sort_smem(s, N, lane);
        for (int i = lane; i < u; i += 32) {
            const unsigned long long v = s[i];
            const uint32_t mp = pair_map(v);
            cidx[i] = pair_key(v);
            cmap[i] = (uint16_t)mp;
            tval[pair_tag(v)] = (unsigned)i;
#pragma unroll
            for (int q = 0; q < 4; ++q) csr[q] += __popc((mp >> (4 * q)) & 0xFu);
        }
    }
    __syncwarp();
    for (int q = lane; q < npairs; q += 32) {
        const uint16_t h = pslot[q];
        if (h != 0xFFFF) pslot[q] = (uint16_t)tval[h];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) csr[q] = warp_sum(csr[q]);
    return u;
}

// Upper bound of pairs per A block row (sum of the selected B row
// lengths); ub[brA] = 0 so that an exclusive scan gives scratch offsets.
// Also clears the symbolic pass's counters: ccnt[0 .. brA], csrcnt[0 .. m],
// stats[0 .. 3] and *nmedium.
__global__ void spgemm_ub_kernel(int m, int brA, const int *__restrict__ aptr, const int *__restrict__ aidx,
                                 const int *__restrict__ bptr, int64_t *__restrict__ ub, int *__restrict__ ccnt,
                                 int *__restrict__ csrcnt, int64_t *__restrict__ stats, int *__restrict__ nmedium)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= brA; b += gridDim.x * blockDim.x) {
        long long t = 0;
        if (b < brA)
            for (int i = aptr[b]; i < aptr[b + 1]; ++i) {
                const int k = aidx[i];
                t += bptr[k + 1] - bptr[k];
            }
        ub[b] = t;
        ccnt[b] = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (4 * b + q <= m) csrcnt[4 * b + q] = 0;
        if (b == 0) {
            stats[0] = stats[1] = stats[2] = stats[3] = 0;
            *nmedium = 0;
        }
    }
}

// One pass: per A block row, the sorted C block columns and bitmaps go to
// the row's scratch slice (offset ub_off[b], capacity ub[b]); C blocks per
// row -> ccnt[b], CSR nonzeros per scalar row -> csrcnt[4b+q].  Launched
// with CAP = 256 over all rows (small shared buffer, high occupancy),
// passing rows with more pairs to spgemm_symbolic_hashed_kernel (up to
// 1024 pairs) through a list (rows[], count in *nrows), which passes rows
// beyond that to the window kernel's list.  (Given rows[], the kernel takes
// a list the same way.)
template <int CAP, int WARPS>
__global__ void __launch_bounds__(32 * WARPS)
spgemm_symbolic_kernel(int m, int brA, const int *__restrict__ aptr, const int *__restrict__ aidx,
                       const uint16_t *__restrict__ amap, const int *__restrict__ bptr,
                       const int *__restrict__ bidx, const uint16_t *__restrict__ bmap, int *__restrict__ ccnt,
                       int *__restrict__ csrcnt, int *__restrict__ large, int64_t *__restrict__ stats,
                       const int64_t *__restrict__ ub_off, int *__restrict__ skey, uint16_t *__restrict__ smap,
                       const int *__restrict__ rows, const int *__restrict__ nrows, int *__restrict__ over,
                       int *__restrict__ nover, uint16_t *__restrict__ pslot, int *__restrict__ err)
{
    __shared__ unsigned long long sbuf[WARPS][CAP];
    __shared__ int stkey[WARPS][CAP];       // hash table of the long rows
    __shared__ unsigned stval[WARPS][CAP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long *s = sbuf[warp];
    unsigned long long wmax = 0, wsq = 0;  // per-warp statistics, one atomic each at the end
    const int nr = rows ? *nrows : brA;
    // rows are read ahead so that a row's chain of dependent loads (row
    // pointers -> A blocks -> B row ranges) overlaps the previous rows'
    // work: the row pointers two rows ahead, the A blocks and B ranges one
    const int stride = gridDim.x * WARPS;
    int t = blockIdx.x * WARPS + warp;
    SymRow cur = sym_row(t, nr, rows, aptr, ub_off), nxt = sym_row(t + stride, nr, rows, aptr, ub_off);
    SymLane cl;
    sym_lane_a<CAP>(cur, lane, aidx, amap, cl);
    sym_lane_b(cl, bptr);
    for (; t < nr; t += stride) {
        SymLane nl;
        sym_lane_a<CAP>(nxt, lane, aidx, amap, nl);
        const SymRow nxt2 = sym_row(t + 2 * stride, nr, rows, aptr, ub_off);
        const int b = cur.b;
        if (cur.ub > CAP) {
            if (lane == 0) over[atomicAdd(nover, 1)] = b;
            sym_lane_b(nl, bptr);
        } else {
            const long long base = cur.base;
            const int cnt = sym_collect(lane, cur.a0, cur.a1, cl, aidx, amap, bptr, bidx, bmap, s, pslot + base);
            sym_lane_b(nl, bptr);
            int csr[4];
            const int u = cnt <= 32 ? sym_reduce32(lane, cnt, s, skey + base, smap + base, csr, pslot + base)
                                    : sym_reduce_hashed<CAP>(lane, cnt, s, stkey[warp], stval[warp], skey + base,
                                                             smap + base, csr, pslot + base, cur.ub, err);
            if (lane == 0) {
                ccnt[b] = u;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (4 * b + q < m) csrcnt[4 * b + q] = csr[q];
                wmax = wmax > (unsigned long long)u ? wmax : (unsigned long long)u;
                wsq += (unsigned long long)u * (unsigned long long)u;
            }
        }
        cur = nxt;
        nxt = nxt2;
        cl = nl;
    }
    if (lane == 0 && wsq) {
        atomicMax((unsigned long long *)&stats[0], wmax);
        atomicAdd((unsigned long long *)&stats[1], wsq);
    }
}

// Bitonic sort of n ints (a power of two) in shared memory by one warp.
__device__ __forceinline__ void warp_sort_smem_int(int *s, int n, int lane)
{
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < n; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = s[i], b = s[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        s[i] = b;
                        s[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Home slot of `key` in a shared hash table of H slots (linear probing
// from there).
template <int H>
__device__ __forceinline__ int hash_slot(int key)
{
    return (int)(((unsigned)key * 0x9E3779B1u) >> (32 - __builtin_ctz(H)));
}

// Rows of 257 .. H pairs (the 256-pair instance's list): every pair with a
// non-zero bitmap product goes straight into a shared hash table of the
// row's C blocks (atomicCAS on the column, atomicOr on the bitmap, the
// pair's table slot into pslot) as it is formed, with no list of the
// row's pairs; the distinct columns are then sorted (a bitonic sort of
// the keys, each key's slot found again by probing), and a second pass
// over the row's pairs turns slots into ranks.  Same output as the
// 256-pair instance (C's columns ascending with OR-ed bitmaps, each pair's
// C block), in 12 KB of shared memory per warp, so that 18 warps per SM
// hold rows.  Rows beyond H pairs go on to the window kernel's list.
template <int H, int WARPS>
__global__ void __launch_bounds__(32 * WARPS)
spgemm_symbolic_hashed_kernel(int m, const int *__restrict__ aptr, const int *__restrict__ aidx,
                              const uint16_t *__restrict__ amap, const int *__restrict__ bptr,
                              const int *__restrict__ bidx, const uint16_t *__restrict__ bmap,
                              int *__restrict__ ccnt, int *__restrict__ csrcnt, int64_t *__restrict__ stats,
                              const int64_t *__restrict__ ub_off, int *__restrict__ skey,
                              uint16_t *__restrict__ smap, const int *__restrict__ rows,
                              const int *__restrict__ nrows, int *__restrict__ over, int *__restrict__ nover,
                              uint16_t *__restrict__ pslot, int *__restrict__ err)
{
    __shared__ int tkey_s[WARPS][H];
    __shared__ unsigned tval_s[WARPS][H];
    __shared__ int kbuf_s[WARPS][H];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *tkey = tkey_s[warp], *kbuf = kbuf_s[warp];
    unsigned *tval = tval_s[warp];
    unsigned long long wmax = 0, wsq = 0;
    const int nr = *nrows;
    for (int t = blockIdx.x * WARPS + warp; t < nr; t += gridDim.x * WARPS) {
        const int b = rows[t];
        const int a0 = aptr[b], a1 = aptr[b + 1];
        const long long base = ub_off[b], ub = ub_off[b + 1] - base;
        if (ub > H) {
            if (lane == 0) over[atomicAdd(nover, 1)] = b;
            continue;
        }
        for (int i = lane; i < H; i += 32) {
            tkey[i] = -1;
            tval[i] = 0;
        }
        __syncwarp();
        // pairs, 32 at a time (flattened as in sym_collect), into the table
        int qbase = 0;
        for (int ib = a0; ib < a1; ib += 32) {
            const int i = ib + lane;
            int j0 = 0, len = 0;
            uint32_t ma = 0;
            if (i < a1) {
                const int k = aidx[i];
                ma = amap[i];
                j0 = bptr[k];
                len = bptr[k + 1] - j0;
            }
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(FULL, incl, 31);
            const int excl = incl - len;
            for (int t0 = 0; t0 < total; t0 += 32) {
                const int tq = t0 + lane;
                int src = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int v = __shfl_sync(FULL, incl, min(src + step - 1, 31));
                    if (v <= tq) src += step;
                }
                src = min(src, 31);
                const int sj0 = __shfl_sync(FULL, j0, src), sex = __shfl_sync(FULL, excl, src);
                const uint32_t sma = __shfl_sync(FULL, ma, src);
                if (tq < total) {
                    const int j = sj0 + (tq - sex);
                    const uint32_t mc = bitmap_mul(sma, bmap[j]);
                    uint16_t slot = 0xFFFF;
                    if (mc) {
                        const int key = bidx[j];
                        int h = hash_slot<H>(key), probe = 0;
                        for (; probe < H; ++probe) {
                            const int prev = atomicCAS(&tkey[h], -1, key);
                            if (prev == -1 || prev == key) break;
                            h = (h + 1) & (H - 1);
                        }
                        if (probe == H) {  // cannot happen (at most H pairs); kept as a bound
                            raise_error(err, DEV_ERR_PROBE);
                        } else {
                            atomicOr(&tval[h], mc);
                            slot = (uint16_t)h;
                        }
                    }
                    pslot[base + qbase + tq] = slot;
                }
            }
            qbase += total;
        }
        __syncwarp();
        // distinct columns -> kbuf[0 .. u), then ascending
        int u = 0;
        for (int i0 = 0; i0 < H; i0 += 32) {
            const int key = tkey[i0 + lane];
            const unsigned bal = __ballot_sync(FULL, key >= 0);
            if (key >= 0) kbuf[u + __popc(bal & lanemask_lt(lane))] = key;
            u += __popc(bal);
        }
        __syncwarp();
        if (u > 32) {
            int n = 64;
            while (n < u) n <<= 1;
            for (int i = u + lane; i < n; i += 32) kbuf[i] = 0x7FFFFFFF;
            __syncwarp();
            warp_sort_smem_int(kbuf, n, lane);
        } else {  // rank among at most 32 keys by comparing with all
            const int key = lane < u ? kbuf[lane] : 0x7FFFFFFF;
            int rank = 0;
            for (int l = 0; l < u; ++l) rank += __shfl_sync(FULL, key, l) < key;
            __syncwarp();
            if (lane < u) kbuf[rank] = key;
            __syncwarp();
        }
        // C block p: its column, OR-ed bitmap and CSR counts; its table slot
        // then holds its rank
        int c01 = 0, c23 = 0;  // CSR counts of scalar rows 0 / 1 and 2 / 3, 16 bits each
        for (int p = lane; p < u; p += 32) {
            const int key = kbuf[p];
            int h = hash_slot<H>(key);
            for (int probe = 0; probe < H && tkey[h] != key; ++probe) h = (h + 1) & (H - 1);
            const uint32_t mp = tval[h];
            skey[base + p] = key;
            smap[base + p] = (uint16_t)mp;
            c01 += __popc(mp & 0xFu) | (__popc((mp >> 4) & 0xFu) << 16);
            c23 += __popc((mp >> 8) & 0xFu) | (__popc((mp >> 12) & 0xFu) << 16);
            tval[h] = (unsigned)p;
        }
        __syncwarp();
        for (int q = lane; q < ub; q += 32) {
            const uint16_t h = pslot[base + q];
            if (h != 0xFFFF) pslot[base + q] = (uint16_t)tval[h];
        }
        c01 = warp_sum(c01);
        c23 = warp_sum(c23);
        if (lane == 0) {
            ccnt[b] = u;
            const int csr[4] = {c01 & 0xFFFF, c01 >> 16, c23 & 0xFFFF, c23 >> 16};
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (4 * b + q < m) csrcnt[4 * b + q] = csr[q];
            wmax = wmax > (unsigned long long)u ? wmax : (unsigned long long)u;
            wsq += (unsigned long long)u * (unsigned long long)u;
        }
        __syncwarp();
    }
    if (lane == 0 && wsq) {
        atomicMax((unsigned long long *)&stats[0], wmax);
        atomicAdd((unsigned long long *)&stats[1], wsq);
    }
}

// The row's (A block, B block) pairs with a non-zero bitmap product, given
// to f(column, product bitmap): warp `warp` of `nw` takes A blocks a0 +
// warp + nw * l, 32 of them at a time (lane l fetches A block l's B row
// range, a warp scan of the lengths flattens the pairs, lane t takes pair
// t, finding its A block by a five-step shuffle search), so that every load
// of a chunk is in flight at once.
template <typename F>
__device__ __forceinline__ void for_row_pairs(int a0, int a1, int warp, int nw, int lane,
                                              const int *__restrict__ aidx, const uint16_t *__restrict__ amap,
                                              const int *__restrict__ bptr, const int *__restrict__ bidx,
                                              const uint16_t *__restrict__ bmap, F f)
{
    for (int c0 = a0 + warp; c0 < a1; c0 += 32 * nw) {
        const int i = c0 + nw * lane;
        int j0 = 0, len = 0;
        uint32_t ma = 0;
        if (i < a1) {
            const int k = aidx[i];
            ma = amap[i];
            j0 = bptr[k];
            len = bptr[k + 1] - j0;
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        const int excl = incl - len;
        for (int t0 = 0; t0 < total; t0 += 32) {
            const int t = t0 + lane;
            int src = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(FULL, incl, min(src + step - 1, 31));
                if (v <= t) src += step;
            }
            src = min(src, 31);
            const int sj0 = __shfl_sync(FULL, j0, src), sex = __shfl_sync(FULL, excl, src);
            const uint32_t sma = __shfl_sync(FULL, ma, src);
            if (t < total) {
                const int j = sj0 + (t - sex);
                const uint32_t mc = bitmap_mul(sma, bmap[j]);
                if (mc) f(bidx[j], mc);
            }
        }
    }
}

// Rows with more than kSymCap pairs: window sweep over the reachable block
// columns, the row's pairs flattened over the CTA's warps (for_row_pairs).
__global__ void __launch_bounds__(kSymLargeThreads)
spgemm_symbolic_large_kernel(int m, const int *__restrict__ aptr, const int *__restrict__ aidx,
                             const uint16_t *__restrict__ amap, const int *__restrict__ bptr,
                             const int *__restrict__ bidx, const uint16_t *__restrict__ bmap,
                             const int *__restrict__ large, int64_t *__restrict__ stats, int *__restrict__ ccnt,
                             int *__restrict__ csrcnt, const int64_t *__restrict__ ub_off, int *__restrict__ skey,
                             uint16_t *__restrict__ smap)
{
    __shared__ uint32_t maps[kSymWin];
    __shared__ int sh[16];
    __shared__ int smin, smax, scsr[4];
    const int nlarge = (int)stats[3];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int t = blockIdx.x; t < nlarge; t += gridDim.x) {
        const int b = large[t];
        const int a0 = aptr[b], a1 = aptr[b + 1];
        if (tid == 0) {
            smin = 0x7FFFFFFF;
            smax = -1;
            scsr[0] = scsr[1] = scsr[2] = scsr[3] = 0;
        }
        __syncthreads();
        int lo = 0x7FFFFFFF, hi = -1;
        for_row_pairs(a0, a1, warp, nw, lane, aidx, amap, bptr, bidx, bmap, [&](int key, uint32_t) {
            lo = min(lo, key);
            hi = max(hi, key);
        });
        atomicMin(&smin, lo);
        atomicMax(&smax, hi);
        __syncthreads();
        const int kmin = smin, kmax = smax;
        const long long base = ub_off[b];
        int total = 0;
        int c4[4] = {0, 0, 0, 0};
        for (long long w0 = kmin; w0 <= kmax; w0 += kSymWin) {
            for (int i = tid; i < kSymWin; i += blockDim.x) maps[i] = 0;
            __syncthreads();
            for_row_pairs(a0, a1, warp, nw, lane, aidx, amap, bptr, bidx, bmap, [&](int col, uint32_t mc) {
                const long long key = col - w0;
                if (key >= 0 && key < kSymWin) atomicOr(&maps[key], mc);
            });
            __syncthreads();
            const int s0 = tid * (kSymWin / kSymLargeThreads);
            int c = 0;
            for (int i = 0; i < kSymWin / kSymLargeThreads; ++i) {
                const uint32_t mp = maps[s0 + i];
                if (mp) {
                    ++c;
#pragma unroll
                    for (int q = 0; q < 4; ++q) c4[q] += __popc((mp >> (4 * q)) & 0xFu);
                }
            }
            // block exclusive scan of c
            int wt;
            int off = warp_excl_scan(c, lane, &wt);
            if (lane == 0) sh[warp] = wt;
            __syncthreads();
            if (warp == 0) {
                int tv = (lane < 8) ? sh[lane] : 0, tt;
                int e = warp_excl_scan(tv, lane, &tt);
                if (lane < 8) sh[lane] = e;
                if (lane == 0) sh[8] = tt;
            }
            __syncthreads();
            off += sh[warp];
            const int wtotal = sh[8];
            {
                long long o = base + total + off;
                for (int i = 0; i < kSymWin / kSymLargeThreads; ++i) {
                    const uint32_t mp = maps[s0 + i];
                    if (mp) {
                        skey[o] = (int)(w0 + s0 + i);
                        smap[o] = (uint16_t)mp;
                        ++o;
                    }
                }
            }
            total += wtotal;
            __syncthreads();
        }
        {
#pragma unroll
            for (int q = 0; q < 4; ++q) atomicAdd(&scsr[q], c4[q]);
            __syncthreads();
            if (tid == 0) {
                ccnt[b] = total;
                for (int q = 0; q < 4; ++q)
                    if (4 * b + q < m) csrcnt[4 * b + q] = scsr[q];
                atomicMax((unsigned long long *)&stats[0], (unsigned long long)total);
                atomicAdd((unsigned long long *)&stats[1], (unsigned long long)total * (unsigned long long)total);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- numeric
template <int PREC>
struct NumT;
template <>
struct NumT<AMGT_DOUBLE> {
    using val_t = double;
    using acc_t = double;
    __device__ static double ld(const double *p, long long i) { return p[i]; }
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    // product entry step: the reference's contracted `temp += a * b`
    __device__ static double madd(double a, double b, double t, bool first)
    {
        return __fma_rn(a, b, first ? 0.0 : t);
    }
};
template <>
struct NumT<AMGT_FLOAT> {
    using val_t = float;
    using acc_t = float;
    __device__ static float ld(const float *p, long long i) { return p[i]; }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float madd(float a, float b, float t, bool first)
    {
        return first ? mul(a, b) : add(t, mul(a, b));
    }
};
template <>
struct NumT<AMGT_HALF> {
    using val_t = __half;
    using acc_t = float;
    __device__ static float ld(const __half *p, long long i) { return __half2float(p[i]); }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float madd(float a, float b, float t, bool first)
    {
        return first ? mul(a, b) : add(t, mul(a, b));
    }
};
template <>
struct NumT<AMGT_BF16> {
    using val_t = __nv_bfloat16;
    using acc_t = float;
    __device__ static float ld(const __nv_bfloat16 *p, long long i) { return __bfloat162float(p[i]); }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float madd(float a, float b, float t, bool first)
    {
        return first ? mul(a, b) : add(t, mul(a, b));
    }
};

template <int PREC>
__device__ __forceinline__ void store_shadow(void *sh, long long i, typename NumT<PREC>::acc_t v)
{
    if constexpr (PREC == AMGT_FLOAT) static_cast<float *>(sh)[i] = v;
    else if constexpr (PREC == AMGT_HALF) static_cast<__half *>(sh)[i] = __float2half_rn(v);
    else if constexpr (PREC == AMGT_BF16) static_cast<__nv_bfloat16 *>(sh)[i] = __float2bfloat16_rn(v);
}

__device__ __forceinline__ int search_sorted(const int *keys, int n, int key)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Accumulator stride (elements) per C block: 16 values plus a 16-byte pad,
// so that the 16-byte row accesses of the 8 pairs of one step fall in
// distinct banks.
template <typename acc_t>
struct NumStride {
    static constexpr int v = 16 + 16 / (int)sizeof(acc_t);
};

// Asynchronous global -> shared copies of 16 bytes (8 for half-precision
// A rows); completion is awaited per step with wait_group.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Four consecutive stored values (one block row) from shared memory,
// widened to the accumulator type.
template <int PREC>
__device__ __forceinline__ void row4_smem(const unsigned char *p, typename NumT<PREC>::acc_t out[4])
{
    if constexpr (PREC == AMGT_DOUBLE) {
        const double2 u = reinterpret_cast<const double2 *>(p)[0], w = reinterpret_cast<const double2 *>(p)[1];
        out[0] = u.x; out[1] = u.y; out[2] = w.x; out[3] = w.y;
    } else if constexpr (PREC == AMGT_FLOAT) {
        const float4 u = *reinterpret_cast<const float4 *>(p);
        out[0] = u.x; out[1] = u.y; out[2] = u.z; out[3] = u.w;
    } else {
        const typename NumT<PREC>::val_t *v = reinterpret_cast<const typename NumT<PREC>::val_t *>(p);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = NumT<PREC>::ld(v, q);
    }
}

// Four accumulators of one C block row (16-byte aligned: the stride of a
// block and the offset of a row are multiples of 16 bytes) as two double2
// or one float4 access.
template <typename acc_t>
__device__ __forceinline__ void acc4_load(const acc_t *p, acc_t v[4])
{
    if constexpr (sizeof(acc_t) == 8) {
        const double2 u = reinterpret_cast<const double2 *>(p)[0], w = reinterpret_cast<const double2 *>(p)[1];
        v[0] = u.x; v[1] = u.y; v[2] = w.x; v[3] = w.y;
    } else {
        const float4 u = *reinterpret_cast<const float4 *>(p);
        v[0] = u.x; v[1] = u.y; v[2] = u.z; v[3] = u.w;
    }
}
template <typename acc_t>
__device__ __forceinline__ void acc4_store(acc_t *p, const acc_t v[4])
{
    if constexpr (sizeof(acc_t) == 8) {
        reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
    } else {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// Shared memory of the numeric kernel per warp: C accumulators (CAP C
// blocks), two stages of 8 staged B blocks (16 values + 16-byte pad) and
// 8 x 4 A rows, and the window's list of pairs with a product.
template <int PREC, int CAP>
struct NumSmem {
    using V = typename NumT<PREC>::val_t;
    using acc_t = typename NumT<PREC>::acc_t;
    static constexpr int BB = 16 * (int)sizeof(V) + 16;  // staged B block bytes
    static constexpr int AR = 4 * (int)sizeof(V);        // staged A row bytes
    static constexpr int b_off = CAP * NumStride<acc_t>::v * (int)sizeof(acc_t);
    static constexpr int a_off = b_off + 2 * 8 * BB;
    static constexpr int p_off = a_off + 2 * 32 * AR;
    static constexpr int per_warp = (p_off + 2 * kNumWin + 15) / 16 * 16;
};

// Numeric phase.  One warp per A block row; the row's (A block, B block)
// pairs are flattened (up to 32 A blocks at a time: lane i holds A block
// i's B row range, a warp scan of the lengths numbers the pairs, and a
// shared list holds, for a window of 128 pairs, those whose bitmap product
// is non-zero, in order, with their A block) and taken 8 at a time, 4
// lanes per pair, lane r computing row r of the 4x4 product.  Steps are double-buffered: while step k is computed from
// shared memory, the asynchronous copies of step k+1's B blocks and A rows
// (each lane copies its own rows of its own pair) and its pairs' C slots
// are in flight.  A pair's C block comes from the symbolic pass (pslot, by
// pair ordinal; 0xFFFF = zero bitmap product) on rows of at most kSymCap
// pairs, else from a binary search of the row's sorted pattern.  Every term
// of the product is computed (unstored entries are zero): for finite values
// this gives the stored-term sums of the reference's scalar branch bit for
// bit, because adding a zero product leaves a non-zero partial sum
// unchanged and a partial sum started from +0 never becomes -0.  Products
// are added to their C block in pair order (= A block order): pairs of one
// step that hit the same C block row are applied in rounds, lowest lane
// first (match_any), so the accumulation order is the sequential one.  Rows
// of up to CAP C blocks (16, 24, 32 or 64 by C's row lengths, at 32, 28,
// 24 or 16 warps per SM) accumulate in shared memory, longer rows in place
// in C.  For fp64 with cshadow given, the final store also writes the fp16
// rounding of every C value and the exactness bits of exact_check_kernel
// into *cflags (bit 0: some value not an fp32 value, bit 1: not fp16).
template <int PREC, int CAP>
__global__ void __launch_bounds__(32 * kNumWarps, num_ctas_per_sm(CAP))
spgemm_numeric_kernel(int m, int brA, const int *__restrict__ aptr, const int *__restrict__ aidx,
                      const typename NumT<PREC>::val_t *__restrict__ aval, const int *__restrict__ bptr,
                      const int *__restrict__ bidx, const typename NumT<PREC>::val_t *__restrict__ bval,
                      const int *__restrict__ cptr, int *__restrict__ cidx, uint16_t *__restrict__ cmap,
                      double *__restrict__ cval, void *__restrict__ cshadow, const int *__restrict__ csr_i,
                      int *__restrict__ csr_j, double *__restrict__ csr_a, const int64_t *__restrict__ ub_off,
                      const int *__restrict__ skey, const uint16_t *__restrict__ smap,
                      const uint16_t *__restrict__ pslot, unsigned long long *__restrict__ cflags,
                      void *__restrict__ cextra)
{
    bool not32 = false, not16 = false;
    using T = NumT<PREC>;
    using V = typename T::val_t;
    using acc_t = typename T::acc_t;
    using SM = NumSmem<PREC, CAP>;
    constexpr int SS = NumStride<acc_t>::v;
    constexpr int CH = (int)sizeof(V);  // 16-byte chunks per block (16 values)
    constexpr int CPL = (CH + 3) / 4;   // B chunks copied per lane
    constexpr int BB = SM::BB, AR = SM::AR;
    extern __shared__ __align__(16) unsigned char num_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ps = lane >> 2, r = lane & 3;
    unsigned char *wbase = num_smem + warp * SM::per_warp;
    acc_t *sa = reinterpret_cast<acc_t *>(wbase);
    unsigned char *sB = wbase + SM::b_off, *sA = wbase + SM::a_off;
    uint16_t *sp = reinterpret_cast<uint16_t *>(wbase + SM::p_off);
    for (int b = blockIdx.x * kNumWarps + warp; b < brA; b += gridDim.x * kNumWarps) {
        const int c0 = cptr[b], cn = cptr[b + 1] - c0;
        // the row's pattern, sorted by the symbolic pass, moves from scratch to C
        const long long sbase = ub_off[b];
        const bool direct = ub_off[b + 1] - sbase <= kSymCap;
        // the first 32 pattern entries are read now and stored at the end,
        // so that no store waits on its load
        int pkey = 0;
        uint32_t pmap = 0;
        if (lane < cn) {
            pkey = skey[sbase + lane];
            pmap = smap[sbase + lane];
        }
        const bool small = cn <= CAP;
        double *ga = cval + 16LL * c0;
        // zeroed one block row (4 values) per lane and iteration
        if (small) {
            const acc_t z[4] = {(acc_t)0, (acc_t)0, (acc_t)0, (acc_t)0};
            for (int t = lane; t < 4 * cn; t += 32) acc4_store(sa + (t >> 2) * SS + 4 * (t & 3), z);
        } else {
            for (int t = lane; t < 4 * cn; t += 32) {
                double2 *d = reinterpret_cast<double2 *>(ga + 4LL * t);
                d[0] = make_double2(0.0, 0.0);
                d[1] = make_double2(0.0, 0.0);
            }
        }
        __syncwarp();
        const int a0 = aptr[b], a1 = aptr[b + 1];
        long long qbase = sbase;  // scratch index of the chunk's first pair
        for (int ib = a0; ib < a1; ib += 32) {
            int j0 = 0, len = 0;
            if (ib + lane < a1) {
                const int k = aidx[ib + lane];
                j0 = bptr[k];
                len = bptr[k + 1] - j0;
            }
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(FULL, incl, 31);
            const int excl = incl - len;
            const int jd = j0 - excl;  // B block of pair q of A block i: q + jd[i]
            for (int w0 = 0; w0 < total; w0 += kNumWin) {
                const int wlen = min(total - w0, kNumWin);
                for (int q = max(excl, w0); q < min(incl, w0 + wlen); ++q) sp[q - w0] = (uint16_t)lane;
                __syncwarp();
                // the window's pairs with a non-zero bitmap product, in pair
                // order, compacted in place: (ordinal in the window << 8) |
                // lane of the A block (rows beyond kSymCap pairs keep all)
                int nq = 0;
                for (int i0 = 0; i0 < wlen; i0 += 32) {
                    const int i = i0 + lane;
                    const bool in = i < wlen;
                    const int src = in ? sp[i] : 0;
                    const bool nz = in && (!direct || pslot[qbase + w0 + i] != 0xFFFF);
                    const unsigned bal = __ballot_sync(FULL, nz);
                    __syncwarp();  // every read of this chunk precedes the writes
                    if (nz) sp[nq + __popc(bal & lanemask_lt(lane))] = (uint16_t)((i << 8) | src);
                    nq += __popc(bal);
                }
                __syncwarp();
                if (nq == 0) continue;  // warp-uniform
                // issue of one step into stage `st`: copies of the lane's B
                // rows and A row, and the pair's C slot (-1: no product)
                auto issue = [&](int k0, int st) -> int {
                    const int k = k0 + ps;
                    const bool valid = k < nq;
                    const int e = valid ? sp[k] : 0;
                    const int src = e & 0xFF, q = w0 + (e >> 8);
                    const int j = q + __shfl_sync(FULL, jd, src);
                    int t = -1;
                    if (valid) {
                        const unsigned char *bsrc = reinterpret_cast<const unsigned char *>(bval + 16LL * j);
                        unsigned char *bdst = sB + (st * 8 + ps) * BB;
#pragma unroll
                        for (int h = 0; h < CPL; ++h) {
                            const int w = r * CPL + h;
                            if (w < CH) cp_async16(bdst + 16 * w, bsrc + 16 * w);
                        }
                        const unsigned char *asrc =
                            reinterpret_cast<const unsigned char *>(aval + 16LL * (ib + src) + 4 * r);
                        unsigned char *adst = sA + (st * 32 + lane) * AR;
                        if constexpr (AR == 32) {
                            cp_async16(adst, asrc);
                            cp_async16(adst + 16, asrc + 16);
                        } else if constexpr (AR == 16) {
                            cp_async16(adst, asrc);
                        } else {
                            cp_async8(adst, asrc);
                        }
                        if (direct) {
                            t = pslot[qbase + q];
                        } else {
                            const int key = bidx[j];
                            const int tt = cn > 0 ? search_sorted(skey + sbase, cn, key) : 0;
                            t = (tt < cn && skey[sbase + tt] == key) ? tt : -1;
                        }
                    }
                    cp_async_commit();
                    return t;
                };
                int tcur = issue(0, 0);
                int st = 0;
                for (int k0 = 0; k0 < nq; k0 += 8, st ^= 1) {
                    int tnext = -1;
                    if (k0 + 8 < nq) {
                        tnext = issue(k0 + 8, st ^ 1);
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                    __syncwarp();
                    const int t = tcur;
                    const bool found = (unsigned)t < (unsigned)cn;  // pslot 0xFFFF: no product
                    acc_t s[4];
                    if (found) {
                        acc_t ar[4];
                        row4_smem<PREC>(sA + (st * 32 + lane) * AR, ar);
                        const unsigned char *bp = sB + (st * 8 + ps) * BB;
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            acc_t bk[4];
                            row4_smem<PREC>(bp + kk * AR, bk);
#pragma unroll
                            for (int c = 0; c < 4; ++c)
                                s[c] = T::madd(ar[kk], bk[c], s[c], kk == 0);
                        }
                    }
                    // ordered accumulation: same C block row -> rounds in lane order
                    const int tag = found ? 4 * t + r : -1 - lane;
                    const unsigned peers = __match_any_sync(FULL, tag);
                    const int rank = __popc(peers & lanemask_lt(lane));
                    const int rounds = __reduce_max_sync(FULL, found ? rank : 0);
                    for (int rd = 0; rd <= rounds; ++rd) {
                        if (found && rank == rd) {
                            if (small) {
                                acc_t *d = sa + t * SS + 4 * r, v[4];
                                acc4_load(d, v);
#pragma unroll
                                for (int c = 0; c < 4; ++c) v[c] = T::add(v[c], s[c]);
                                acc4_store(d, v);
                            } else {
                                double *d = ga + 16LL * t + 4 * r;
#pragma unroll
                                for (int c = 0; c < 4; ++c) d[c] = (double)T::add((acc_t)d[c], s[c]);
                            }
                        }
                        __syncwarp();
                    }
                    tcur = tnext;
                }
            }
            qbase += total;
        }
        // pattern, C values (+ shadow)
        if (lane < cn) {
            cidx[c0 + lane] = pkey;
            cmap[c0 + lane] = (uint16_t)pmap;
        }
        for (int t = 32 + lane; t < cn; t += 32) {
            cidx[c0 + t] = skey[sbase + t];
            cmap[c0 + t] = smap[sbase + t];
        }
        // C values (+ shadow), one block row (4 values) per lane and iteration
        for (int t = lane; t < 4 * cn; t += 32) {
            acc_t v[4];
            if (small) {
                acc4_load(sa + (t >> 2) * SS + 4 * (t & 3), v);
            } else {
#pragma unroll
                for (int c = 0; c < 4; ++c) v[c] = (acc_t)ga[4LL * t + c];
            }
            double2 *g = reinterpret_cast<double2 *>(ga + 4LL * t);
            g[0] = make_double2((double)v[0], (double)v[1]);
            g[1] = make_double2((double)v[2], (double)v[3]);
            if constexpr (PREC == AMGT_DOUBLE) {
                if (cshadow) {
                    __half hv[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        hv[c] = __double2half(v[c]);
                        if ((double)__double2float_rn(v[c]) != v[c]) not32 = true;
                        if ((double)__half2float(hv[c]) != v[c]) not16 = true;
                    }
                    __half2 *hs = reinterpret_cast<__half2 *>(static_cast<__half *>(cshadow) + 16LL * c0 + 4LL * t);
                    hs[0] = __halves2half2(hv[0], hv[1]);
                    hs[1] = __halves2half2(hv[2], hv[3]);
                }
                if (cextra)  // the fp32 shadow of a level used in fp32
                    *reinterpret_cast<float4 *>(static_cast<float *>(cextra) + 16LL * c0 + 4LL * t) =
                        make_float4(__double2float_rn(v[0]), __double2float_rn(v[1]), __double2float_rn(v[2]),
                                    __double2float_rn(v[3]));
            } else if (cshadow) {
#pragma unroll
                for (int c = 0; c < 4; ++c) store_shadow<PREC>(cshadow, 16LL * c0 + 4LL * t + c, v[c]);
                if constexpr (PREC == AMGT_FLOAT) {
                    if (cextra) {  // fp16 candidate shadow and its exactness bit
                        __half hv[4];
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            hv[c] = __float2half_rn(v[c]);
                            if (__half2float(hv[c]) != v[c]) not16 = true;
                        }
                        __half2 *hs = reinterpret_cast<__half2 *>(static_cast<__half *>(cextra) + 16LL * c0 + 4LL * t);
                        hs[0] = __halves2half2(hv[0], hv[1]);
                        hs[1] = __halves2half2(hv[2], hv[3]);
                    }
                }
            }
        }
        __syncwarp();
        // CSR rows 4b..4b+3 (BSR2CSR fused)
        if (csr_i) {
            for (int qr = 0; qr < 4 && 4 * b + qr < m; ++qr) {
                int out = csr_i[4 * b + qr];
                for (int tt = 0; tt < cn; tt += 32) {
                    const int t = tt + lane;
                    uint32_t nib = 0;
                    int col0 = 0;
                    if (t < cn) {
                        nib = (cmap[c0 + t] >> (4 * qr)) & 0xFu;
                        col0 = 4 * cidx[c0 + t];
                    }
                    int tot;
                    const int off = warp_excl_scan(__popc(nib), lane, &tot);
                    if (nib) {
                        int o = out + off;
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc)
                            if (nib & (1u << cc)) {
                                csr_j[o] = col0 + cc;
                                csr_a[o] = ga[16 * t + 4 * qr + cc];
                                ++o;
                            }
                    }
                    out += tot;
                }
            }
        }
        __syncwarp();
    }
    // the row loop is warp-uniform: all lanes are here
    if ((PREC == AMGT_DOUBLE && cshadow) || (PREC == AMGT_FLOAT && cextra)) {
        const unsigned b32 = __ballot_sync(FULL, not32), b16 = __ballot_sync(FULL, not16);
        if (lane == 0 && (b32 | b16)) atomicOr(cflags, (b32 ? 1ull : 0ull) | (b16 ? 2ull : 0ull));
    }
}

// ------------------------------------------------------- gathered numeric
// The numeric phase by C block: every C block gathers its own ordered list
// of (A block, B block) pairs, so that the work spreads over all C blocks
// of the product whatever the row lengths (a few long rows of a coarse
// level no longer serialise on a few warps), and no two lanes ever add to
// the same C value (no ordering rounds).  Two kernels:
//   order   one warp per A block row moves the row's sorted pattern into C
//           and sorts the row's pairs by C block, stably (pair order = A
//           block order), into the row's scratch slice: glist[gbeg[c] ..
//           gbeg[c] + gnum[c]) lists C block c's pairs in the order the
//           sequential product adds them.  Rows of at most kOrdCap C
//           blocks: a flattened pass over 32 pairs at a time with
//           shared-memory counters, equal C blocks of a step ranked in lane
//           order; each pair's C block is the symbolic pass's pair slot
//           (rows of at most kSymCap pairs) or a search of the row's sorted
//           pattern copied to shared memory.  Rows of more C blocks go one A
//           block at a time (the B blocks of one A block hit distinct C
//           blocks), with the counters in gnum.
//   Used for products of fewer than 64 A block rows per SM (the coarse
//   levels, whose few long rows leave the staged kernel's warps idle) or
//   with more than an eighth of their rows beyond kSymCap pairs; the staged
//   kernel keeps the others.
//   gather  four lanes per C block (lane r: row r), the C block's pairs
//           streamed through a ring of kGatherSlots shared-memory slots per
//           C block (lane r copies row r of the pair's A block and of its B
//           block with cp.async, kGatherSlots - 1 pairs ahead, the list
//           entries four to eight ahead in registers, the next C block's
//           bounds and first entries during this one), so that several
//           pairs' loads of every C block are in flight; the product entry the
//           same fused chain as the staged kernel, the products added in
//           list order: C equals the staged kernel's result bit for bit.
// Writes C's values (+ shadow, + the fused exactness bits); the CSR form,
// when wanted, comes from spgemm_csr_kernel.
__global__ void __launch_bounds__(32 * kNumWarps)
spgemm_order_kernel(int brA, const int *__restrict__ aptr, const int *__restrict__ aidx,
                    const int *__restrict__ bptr, const int *__restrict__ bidx, const int *__restrict__ cptr,
                    int *__restrict__ cidx, uint16_t *__restrict__ cmap, const int64_t *__restrict__ ub_off,
                    const int *__restrict__ skey, const uint16_t *__restrict__ smap,
                    uint16_t *__restrict__ pslot, int2 *__restrict__ glist, long long *__restrict__ gbeg,
                    int *__restrict__ gnum)
{
    __shared__ int cnt_s[kNumWarps][kOrdCap];
    __shared__ int key_s[kNumWarps][kOrdCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *cnt = cnt_s[warp], *keys = key_s[warp];
    for (int b = blockIdx.x * kNumWarps + warp; b < brA; b += gridDim.x * kNumWarps) {
        const int c0 = cptr[b], cn = cptr[b + 1] - c0;
        const long long sbase = ub_off[b], npairs = ub_off[b + 1] - sbase;
        for (int t = lane; t < cn; t += 32) {
            cidx[c0 + t] = skey[sbase + t];
            cmap[c0 + t] = smap[sbase + t];
        }
        const int a0 = aptr[b], a1 = aptr[b + 1];
        const bool direct = npairs <= kSymCap;  // pair slots from the symbolic pass
        if (cn <= kOrdCap) {
            for (int t = lane; t < cn; t += 32) {
                cnt[t] = 0;
                if (!direct) keys[t] = skey[sbase + t];
            }
            __syncwarp();
            // pass 0 counts, pass 1 places; pairs enumerated in row order
            for (int pass = 0; pass < 2; ++pass) {
                long long qbase = sbase;
                for (int ib = a0; ib < a1; ib += 32) {
                    int j0 = 0, len = 0;
                    if (ib + lane < a1) {
                        const int k = aidx[ib + lane];
                        j0 = bptr[k];
                        len = bptr[k + 1] - j0;
                    }
                    int total;
                    const int excl = warp_excl_scan(len, lane, &total);
                    for (int q0 = 0; q0 < total; q0 += 32) {
                        const int q = q0 + lane;
                        // the A block of pair q: the last lane whose first pair is <= q
                        // (every lane searches, so that the shuffles are uniform)
                        int src = 0;
#pragma unroll
                        for (int st = 16; st > 0; st >>= 1) {
                            const int e = __shfl_sync(FULL, excl, src + st);
                            if (e <= q) src += st;
                        }
                        const int sj0 = __shfl_sync(FULL, j0, src), sex = __shfl_sync(FULL, excl, src);
                        int t = -1;
                        if (q < total) {
                            if (direct || pass == 1) {
                                const unsigned short ps = pslot[qbase + q];
                                t = ps < cn ? (int)ps : -1;
                            } else {  // the pair's C block from the row's sorted pattern, kept for pass 1
                                const int key = bidx[sj0 + (q - sex)];
                                int lo = 0, hi = cn - 1;
                                while (lo < hi) {
                                    const int mid = (lo + hi) >> 1;
                                    if (keys[mid] < key) lo = mid + 1;
                                    else hi = mid;
                                }
                                t = (cn > 0 && keys[lo] == key) ? lo : -1;
                                pslot[qbase + q] = t >= 0 ? (unsigned short)t : (unsigned short)0xFFFF;
                            }
                        }
                        if (pass == 0) {
                            if (t >= 0) atomicAdd(&cnt[t], 1);
                        } else {
                            const unsigned peers = __match_any_sync(FULL, t >= 0 ? t : -1 - lane);
                            if (t >= 0) {
                                const int rank = __popc(peers & lanemask_lt(lane));
                                glist[sbase + cnt[t] + rank] = make_int2(ib + src, sj0 + (q - sex));
                            }
                            __syncwarp();
                            if (t >= 0 && (peers & lanemask_lt(lane)) == 0) cnt[t] += __popc(peers);
                        }
                        __syncwarp();
                    }
                    qbase += total;
                }
                __syncwarp();
                if (pass == 0) {  // counts -> list starts (cnt then runs from the start)
                    int carry = 0;
                    for (int t0 = 0; t0 < cn; t0 += 32) {
                        const int t = t0 + lane;
                        const int c = t < cn ? cnt[t] : 0;
                        int tot;
                        const int off = warp_excl_scan(c, lane, &tot) + carry;
                        if (t < cn) {
                            gbeg[c0 + t] = sbase + off;
                            gnum[c0 + t] = c;
                            cnt[t] = off;
                        }
                        carry += tot;
                    }
                    __syncwarp();
                }
            }
        } else {
            // a row of more than kOrdCap C blocks: one A block at a time,
            // counters in gnum (cleared by the caller)
            for (int pass = 0; pass < 2; ++pass) {
                for (int i = a0; i < a1; ++i) {
                    const int k = aidx[i];
                    for (int j = bptr[k] + lane; j < bptr[k + 1]; j += 32) {
                        const int key = bidx[j];
                        const int tt = search_sorted(skey + sbase, cn, key);
                        if (tt < cn && skey[sbase + tt] == key) {
                            if (pass == 0) {
                                atomicAdd(&gnum[c0 + tt], 1);
                            } else {
                                glist[gbeg[c0 + tt] + gnum[c0 + tt]] = make_int2(i, j);
                                gnum[c0 + tt] += 1;  // the B blocks of one A block hit distinct C blocks
                            }
                        }
                    }
                    __syncwarp();
                }
                __syncwarp();
                if (pass == 0) {
                    long long carry = sbase;
                    for (int t0 = 0; t0 < cn; t0 += 32) {
                        const int t = t0 + lane;
                        const int c = t < cn ? gnum[c0 + t] : 0;
                        int tot;
                        const int off = warp_excl_scan(c, lane, &tot);
                        if (t < cn) {
                            gbeg[c0 + t] = carry + off;
                            gnum[c0 + t] = 0;
                        }
                        carry += tot;
                    }
                    __syncwarp();
                }
            }
        }
    }
}

constexpr int kGatherSlots = 4;     // ring slots per C block: pairs in flight = kGatherSlots - 1
constexpr int kGatherThreads = 128;  // 32 C blocks per CTA
template <int PREC>
struct GatherSmem {
    static constexpr int AR = 4 * (int)sizeof(typename NumT<PREC>::val_t);  // one block row
    static constexpr int slot = 8 * AR;                                     // A block, then B block
    // a C block's ring, padded by 16 bytes so that the eight C blocks of a
    // warp, reading the same row of their B blocks, hit distinct banks
    static constexpr int group = kGatherSlots * slot + 16;
    static constexpr int per_cta = (kGatherThreads / 4) * group;
};

template <int PREC>
__global__ void __launch_bounds__(kGatherThreads, 6)
spgemm_gather_kernel(int nbC, const typename NumT<PREC>::val_t *__restrict__ aval,
                     const typename NumT<PREC>::val_t *__restrict__ bval, const int2 *__restrict__ glist,
                     const long long *__restrict__ gbeg, const int *__restrict__ gnum, double *__restrict__ cval,
                     void *__restrict__ cshadow, unsigned long long *__restrict__ cflags, void *__restrict__ cextra)
{
    using T = NumT<PREC>;
    using acc_t = typename T::acc_t;
    using GS = GatherSmem<PREC>;
    constexpr int AR = GS::AR, SLOT = GS::slot, S = kGatherSlots;
    extern __shared__ __align__(16) unsigned char gather_smem[];
    const int r = threadIdx.x & 3;
    const unsigned gmask = 0xFu << (threadIdx.x & 28);  // this C block's four lanes
    unsigned char *ring = gather_smem + (threadIdx.x >> 2) * GS::group;
    bool not32 = false, not16 = false;
    const long long g0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 2;
    const long long gstride = ((long long)gridDim.x * blockDim.x) >> 2;
    // copies of row r of pair pr's A block and B block into slot `sl`
    auto issue = [&](int2 pr, int sl) {
        const unsigned char *asrc = reinterpret_cast<const unsigned char *>(aval + 16LL * pr.x + 4 * r);
        const unsigned char *bsrc = reinterpret_cast<const unsigned char *>(bval + 16LL * pr.y + 4 * r);
        unsigned char *adst = ring + sl * SLOT + r * AR, *bdst = adst + 4 * AR;
        if constexpr (AR == 32) {
            cp_async16(adst, asrc);
            cp_async16(adst + 16, asrc + 16);
            cp_async16(bdst, bsrc);
            cp_async16(bdst + 16, bsrc + 16);
        } else if constexpr (AR == 16) {
            cp_async16(adst, asrc);
            cp_async16(bdst, bsrc);
        } else {
            cp_async8(adst, asrc);
            cp_async8(bdst, bsrc);
        }
    };
    // list entries travel in batches of four, lane r holding entry 4m + r of
    // its C block's list and handing it to the group by a shuffle: the batch
    // after the one being issued is already in flight, and the next C
    // block's bounds and first batch are read while this one is computed
    const int gl = threadIdx.x & 28;  // the group's first lane in the warp
    auto entry = [&](long long beg, int n, int i) -> int2 {
        return i < n ? __ldg(glist + beg + i) : make_int2(0, 0);
    };
    long long beg = 0, begN = 0;
    int n = 0, nN = 0;
    int2 ent = make_int2(0, 0);
    if (g0 < nbC) {
        beg = gbeg[g0];
        n = gnum[g0];
        ent = entry(beg, n, r);
    }
    if (g0 + gstride < nbC) {
        begN = gbeg[g0 + gstride];
        nN = gnum[g0 + gstride];
    }
    for (long long g = g0; g < nbC; g += gstride) {
        // the C block after next: its bounds; the next one: its first batch
        long long begNN = 0;
        int nNN = 0;
        if (g + 2 * gstride < nbC) {
            begNN = gbeg[g + 2 * gstride];
            nNN = gnum[g + 2 * gstride];
        }
        const int2 entNext = entry(begN, nN, r);
        int2 entn = entry(beg, n, 4 + r);
        int kb = 0;  // first entry of the batch in `ent`
        auto take = [&](int i) -> int2 {  // entry i (kb <= i < kb + 4) from its lane
            const int src = gl | (i - kb);
            return make_int2(__shfl_sync(gmask, ent.x, src), __shfl_sync(gmask, ent.y, src));
        };
        // pairs 0 .. S-2 in flight
#pragma unroll
        for (int u = 0; u < S - 1; ++u) {
            const int2 pr = take(u);
            if (u < n) issue(pr, u);
            cp_async_commit();
        }
        acc_t acc[4] = {(acc_t)0, (acc_t)0, (acc_t)0, (acc_t)0};
        for (int k = 0; k < n; ++k) {
            const int ka = k + S - 1;  // the pair issued now
            if (ka == kb + 4) {        // next batch; the one after it goes in flight
                ent = entn;
                kb += 4;
                entn = entry(beg, n, kb + 4 + r);
            }
            const int2 pr = take(ka);
            if (ka < n) issue(pr, ka % S);
            cp_async_commit();
            cp_async_wait<S - 1>();  // pair k's copies are complete
            __syncwarp(gmask);
            const unsigned char *sl = ring + (k % S) * SLOT;
            acc_t ar[4], s[4];
            row4_smem<PREC>(sl + r * AR, ar);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                acc_t bk[4];
                row4_smem<PREC>(sl + 4 * AR + kk * AR, bk);
#pragma unroll
                for (int c = 0; c < 4; ++c) s[c] = T::madd(ar[kk], bk[c], s[c], kk == 0);
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[c] = T::add(acc[c], s[c]);
            __syncwarp(gmask);  // slot k % S is refilled by the next iteration's issue
        }
        cp_async_wait<0>();
        double *d = cval + 16 * g + 4 * r;
        reinterpret_cast<double2 *>(d)[0] = make_double2((double)acc[0], (double)acc[1]);
        reinterpret_cast<double2 *>(d)[1] = make_double2((double)acc[2], (double)acc[3]);
        if constexpr (PREC == AMGT_DOUBLE) {
            if (cshadow) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const __half hv = __double2half(acc[c]);
                    static_cast<__half *>(cshadow)[16 * g + 4 * r + c] = hv;
                    if ((double)__double2float_rn(acc[c]) != acc[c]) not32 = true;
                    if ((double)__half2float(hv) != acc[c]) not16 = true;
                }
            }
            if (cextra)  // the fp32 shadow of a level used in fp32
#pragma unroll
                for (int c = 0; c < 4; ++c) static_cast<float *>(cextra)[16 * g + 4 * r + c] = __double2float_rn(acc[c]);
        } else if (cshadow) {
#pragma unroll
            for (int c = 0; c < 4; ++c) store_shadow<PREC>(cshadow, 16 * g + 4 * r + c, acc[c]);
            if constexpr (PREC == AMGT_FLOAT) {
                if (cextra) {  // fp16 candidate shadow and its exactness bit
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const __half hv = __float2half_rn(acc[c]);
                        static_cast<__half *>(cextra)[16 * g + 4 * r + c] = hv;
                        if (__half2float(hv) != acc[c]) not16 = true;
                    }
                }
            }
        }
        beg = begN;
        n = nN;
        begN = begNN;
        nN = nNN;
        ent = entNext;
    }
    if ((PREC == AMGT_DOUBLE && cshadow) || (PREC == AMGT_FLOAT && cextra)) {
        const unsigned b32 = __ballot_sync(FULL, not32), b16 = __ballot_sync(FULL, not16);
        if ((threadIdx.x & 31) == 0 && (b32 | b16)) atomicOr(cflags, (b32 ? 1ull : 0ull) | (b16 ? 2ull : 0ull));
    }
}

// Tensor-core form of the gathered numeric for fp16 / bf16 values
// (amgt_spgemm_set_engine(AMGT_ENGINE_TENSOR_CORE)): one warp, four C
// blocks, one mma.m16n8k16 per step with fp32 accumulation.  The four 4x4
// products of a step (the k-th pair of each C block) sit block-diagonally
// in the MMA: C block i's A block in rows 4i..4i+3, columns 4i..4i+3 of
// the 16x16 A tile, its B block in rows 4i..4i+3, columns 0..3 of the 16x8
// B tile, so rows 4i..4i+3, columns 0..3 of the accumulator are C block i
// and the other products of the tile are zero terms (a quarter of the
// tile's rows and half its columns carry data).  A C block with fewer pairs
// takes zero blocks in the later steps.  Each entry is the tensor core's
// sum of its products and the running fp32 value, in the tensor core's
// order: not the sequential order of the CUDA-core form, so its parity is
// a tolerance, not bit-exactness.
template <int PREC>
__device__ __forceinline__ uint32_t pack_pair_bits(uint16_t lo, uint16_t hi)
{
    return (uint32_t)lo | ((uint32_t)hi << 16);
}

template <int PREC>
__device__ __forceinline__ void mma_16816(float d[4], const uint32_t a[4], const uint32_t b[2])
{
    if constexpr (PREC == AMGT_HALF) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    } else {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    }
}

template <int PREC>
__global__ void __launch_bounds__(128)
spgemm_gather_mma_kernel(int nbC, const uint16_t *__restrict__ aval, const uint16_t *__restrict__ bval,
                         const int2 *__restrict__ glist, const long long *__restrict__ gbeg,
                         const int *__restrict__ gnum, double *__restrict__ cval, void *__restrict__ cshadow)
{
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int ib = g >> 2, rr = g & 3, kk = (2 * t) & 3;
    const bool aload = (t >> 1) == ib;  // this lane's A elements lie in the diagonal blocks
    const int s0 = t >> 1, s1 = 2 + (t >> 1);
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; 4 * w < nbC; w += nwarps) {
        const long long c0 = 4 * w;
        // lane i < 4 holds C block c0 + i's list
        long long beg = 0;
        int n = 0;
        if (lane < 4 && c0 + lane < nbC) {
            beg = gbeg[c0 + lane];
            n = gnum[c0 + lane];
        }
        int nmax = n;
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) nmax = max(nmax, __shfl_xor_sync(FULL, nmax, o));
        nmax = __shfl_sync(FULL, nmax, 0);
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < nmax; ++k) {
            int2 p = make_int2(-1, -1);
            if (lane < 4 && k < n) p = __ldg(glist + beg + k);
            int px[4], py[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                px[i] = __shfl_sync(FULL, p.x, i);
                py[i] = __shfl_sync(FULL, p.y, i);
            }
            uint32_t a[4] = {0u, 0u, 0u, 0u}, b[2] = {0u, 0u};
            if (aload) {
                if (px[ib] >= 0) a[0] = __ldg(reinterpret_cast<const uint32_t *>(aval + 16LL * px[ib] + 4 * rr + kk));
                if (px[2 + ib] >= 0)
                    a[3] = __ldg(reinterpret_cast<const uint32_t *>(aval + 16LL * px[2 + ib] + 4 * rr + kk));
            }
            if (g < 4) {
                if (py[s0] >= 0) {
                    const uint16_t *q = bval + 16LL * py[s0] + 4 * kk + g;
                    b[0] = pack_pair_bits<PREC>(__ldg(q), __ldg(q + 4));
                }
                if (py[s1] >= 0) {
                    const uint16_t *q = bval + 16LL * py[s1] + 4 * kk + g;
                    b[1] = pack_pair_bits<PREC>(__ldg(q), __ldg(q + 4));
                }
            }
            mma_16816<PREC>(d, a, b);
        }
        // rows g (C block ib) and g + 8 (C block 2 + ib), columns 2t, 2t + 1
        if (t < 2) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long cb = c0 + (h ? 2 + ib : ib);
                if (cb < nbC) {
                    const long long o = 16 * cb + 4 * rr + 2 * t;
                    cval[o] = (double)d[2 * h];
                    cval[o + 1] = (double)d[2 * h + 1];
                    if (cshadow) {
                        store_shadow<PREC>(cshadow, o, d[2 * h]);
                        store_shadow<PREC>(cshadow, o + 1, d[2 * h + 1]);
                    }
                }
            }
        }
    }
}

// CSR form of C from its blocks: one warp per block row, scalar row by
// scalar row, entries in ascending column order.
__global__ void __launch_bounds__(32 * kNumWarps)
spgemm_csr_kernel(int m, int brA, const int *__restrict__ cptr, const int *__restrict__ cidx,
                  const uint16_t *__restrict__ cmap, const double *__restrict__ cval, const int *__restrict__ csr_i,
                  int *__restrict__ csr_j, double *__restrict__ csr_a)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = blockIdx.x * kNumWarps + warp; b < brA; b += gridDim.x * kNumWarps) {
        const int c0 = cptr[b], cn = cptr[b + 1] - c0;
        for (int qr = 0; qr < 4 && 4 * b + qr < m; ++qr) {
            int out = csr_i[4 * b + qr];
            for (int tt = 0; tt < cn; tt += 32) {
                const int t = tt + lane;
                uint32_t nib = 0;
                int col0 = 0;
                if (t < cn) {
                    nib = (cmap[c0 + t] >> (4 * qr)) & 0xFu;
                    col0 = 4 * cidx[c0 + t];
                }
                int tot;
                const int off = warp_excl_scan(__popc(nib), lane, &tot);
                if (nib) {
                    int o = out + off;
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc)
                        if (nib & (1u << cc)) {
                            csr_j[o] = col0 + cc;
                            csr_a[o] = cval[16LL * (c0 + t) + 4 * qr + cc];
                            ++o;
                        }
                }
                out += tot;
            }
        }
    }
}

template <int PREC, int CAP>
static int launch_numeric_cap(const amgt_bsr *A, const void *aval, const amgt_bsr *B, const void *bval, amgt_bsr *C,
                              void *cshadow, amgt_csr *Ccsr, const int64_t *ub_off, const int *skey,
                              const uint16_t *smap, const uint16_t *pslot, cudaStream_t s, int sm_count,
                              unsigned long long *cflags, void *cextra)
{
    using V = typename NumT<PREC>::val_t;
    constexpr int smem = kNumWarps * NumSmem<PREC, CAP>::per_warp;
    constexpr int per_sm = num_ctas_per_sm(CAP);
    AMGT_CUDA_TRY(cudaFuncSetAttribute(spgemm_numeric_kernel<PREC, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
    AMGT_LAUNCH((spgemm_numeric_kernel<PREC, CAP>), grid_for(kNumWarps, A->blc_row, sm_count, per_sm),
                32 * kNumWarps, smem, s, A->row, A->blc_row, A->blcPtr, A->blcIdx, (const V *)aval, B->blcPtr, B->blcIdx, (const V *)bval,
                C->blcPtr, C->blcIdx, C->blcMap, C->blcVal, cshadow, Ccsr ? Ccsr->i : nullptr,
                Ccsr ? Ccsr->j : nullptr, Ccsr ? Ccsr->data : nullptr, ub_off, skey, smap, pslot, cflags, cextra);
    return AMGT_OK;
}

// The staged numeric with the accumulator capacity for C's row lengths:
// 16 or 24 C blocks when no C row is longer (32 / 28 warps per SM), 64 when
// the average C row exceeds 24 blocks (most rows would otherwise accumulate
// in global memory; 16 warps per SM), else 32 (24 warps per SM).
template <int PREC>
static int launch_numeric(const amgt_bsr *A, const void *aval, const amgt_bsr *B, const void *bval, amgt_bsr *C,
                          void *cshadow, amgt_csr *Ccsr, const int64_t *ub_off, const int *skey,
                          const uint16_t *smap, const uint16_t *pslot, cudaStream_t s, int sm_count,
                          unsigned long long *cflags = nullptr, void *cextra = nullptr)
{
    if (A->blc_row == 0) return AMGT_OK;
    if (C->max_blc_per_row <= kNumCapNarrow)
        return launch_numeric_cap<PREC, kNumCapNarrow>(A, aval, B, bval, C, cshadow, Ccsr, ub_off, skey, smap, pslot,
                                                       s, sm_count, cflags, cextra);
    if (C->max_blc_per_row <= kNumCapMid)
        return launch_numeric_cap<PREC, kNumCapMid>(A, aval, B, bval, C, cshadow, Ccsr, ub_off, skey, smap, pslot, s,
                                                    sm_count, cflags, cextra);
    if (C->max_blc_per_row > kNumCap && 24LL * A->blc_row < (long long)C->blc_num)
        return launch_numeric_cap<PREC, kNumCapWide>(A, aval, B, bval, C, cshadow, Ccsr, ub_off, skey, smap, pslot, s,
                                                     sm_count, cflags, cextra);
    return launch_numeric_cap<PREC, kNumCap>(A, aval, B, bval, C, cshadow, Ccsr, ub_off, skey, smap, pslot, s,
                                             sm_count, cflags, cextra);
}

static void *shadow_of(const amgt_bsr *A, int prec)
{
    switch (prec) {
    case AMGT_FLOAT: return A->blcVal_fp32;
    case AMGT_HALF: return A->blcVal_fp16;
    case AMGT_BF16: return A->blcVal_bf16;
    default: return A->blcVal;
    }
}

}  // namespace amgt

using namespace amgt;

namespace amgt {

// Engine of the fp16 / bf16 block products (amgt_spgemm_set_engine).
static std::atomic<int> g_spgemm_engine{AMGT_ENGINE_AUTO};

// amgt_spgemm with an optional host callback `between`, run after the
// symbolic kernels are queued and before the host waits for C's size:
// host work that can overlap them (the AMG setup converts the next
// level's interpolation there, on its own stream).
int spgemm_impl(int prec, const amgt_bsr *A, const amgt_bsr *B, amgt_bsr *C, amgt_csr *Ccsr, amgt_stream_t stream,
                int (*between)(void *), void *ctx, CvtFuse *fuse)
{
    if (!A || !B || !C || prec < AMGT_DOUBLE || prec > AMGT_BF16) return AMGT_ERR_INVALID;
    if (A->col != B->row) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int m = A->row, brA = A->blc_row;
    memset(C, 0, sizeof(*C));
    if (Ccsr) memset(Ccsr, 0, sizeof(*Ccsr));
    C->row = m;
    C->col = B->col;
    C->blc_row = brA;
    C->blc_col = B->blc_col;

    // reduced precisions read A / B shadows; build temporaries when absent
    amgt_bsr Atmp = *A, Btmp = *B;
    bool ownA = false, ownB = false;
    int rc = AMGT_OK;
    unsigned char *arena = nullptr, *arena2 = nullptr;  // scratch (pieces below point into them)
    int *ccnt = nullptr, *csrcnt = nullptr, *large = nullptr, *csr_i = nullptr, *csr_tmp = nullptr;
    int64_t *stats = nullptr, *ub = nullptr, *ub_off = nullptr;
    int *skey = nullptr;
    uint16_t *smap = nullptr, *pslot = nullptr;  // scratch: pattern, per-pair C block
    const int64_t *h = nullptr;
    int nbC = 0, nnzC = 0;
    long long cap = 0;  // scratch capacity in pairs
    int nlarge = 0;     // rows of more than kSymCap pairs
    long long npairs = 0;  // (A block, B block) pairs of the product
    const bool tensor =  // fp16 / bf16 block products on the tensor cores
        g_spgemm_engine.load() == AMGT_ENGINE_TENSOR_CORE && (prec == AMGT_HALF || prec == AMGT_BF16);
    unsigned char *arena3 = nullptr;  // gathered numeric: pair lists and their starts / lengths
    void *cshadow = nullptr;
    void *cextra = nullptr;  // fp64 products: the fp32 shadow; fp32 products: the fp16 candidate (CvtFuse)
    if (prec != AMGT_DOUBLE) {
        if (!shadow_of(A, prec)) {
            Atmp.blcVal_fp32 = nullptr; Atmp.blcVal_fp16 = nullptr; Atmp.blcVal_bf16 = nullptr;
            if ((rc = amgt_bsr_make_shadow(&Atmp, prec, stream))) return rc;
            ownA = true;
        }
        if (!shadow_of(B, prec)) {
            Btmp.blcVal_fp32 = nullptr; Btmp.blcVal_fp16 = nullptr; Btmp.blcVal_bf16 = nullptr;
            if ((rc = amgt_bsr_make_shadow(&Btmp, prec, stream))) goto fail;
            ownB = true;
        }
    }
    {
        // the per-row scratch in one allocation (256-byte aligned pieces)
        const size_t o_stats = 0, o_ub = o_stats + 256, o_uboff = o_ub + align256(8 * ((size_t)brA + 1)),
                     o_ccnt = o_uboff + align256(8 * ((size_t)brA + 1)),
                     o_csr = o_ccnt + align256(4 * ((size_t)brA + 1)),
                     o_large = o_csr + align256(4 * ((size_t)m + 1)),
                     o_end = o_large + align256(4 * (2 * (size_t)brA + 1));
        if ((rc = alloc_n(&C->blcPtr, brA + 1, s)) || (rc = alloc_n(&arena, o_end, s))) goto fail;
        stats = reinterpret_cast<int64_t *>(arena + o_stats);
        ub = reinterpret_cast<int64_t *>(arena + o_ub);
        ub_off = reinterpret_cast<int64_t *>(arena + o_uboff);
        ccnt = reinterpret_cast<int *>(arena + o_ccnt);
        csrcnt = reinterpret_cast<int *>(arena + o_csr);
        large = reinterpret_cast<int *>(arena + o_large);
    }
    // per-row pair bounds -> scratch offsets for the rows' sorted patterns
    // (the kernel also clears the counters)
    AMGT_LAUNCH(spgemm_ub_kernel, grid_for(256, brA + 1LL, st->sm_count, 8), 256, 0, s, m, brA, A->blcPtr,
                A->blcIdx, B->blcPtr, ub, ccnt, csrcnt, stats, large + 2 * brA);
    if ((rc = exclusive_scan_i64(ub, ub_off, brA + 1, s))) goto fail;
    {
        // scratch size: the host-side bound nblk(A) * longest B row when it is
        // modest (<= 32 Mi pairs, 256 MB of scratch), else the exact total
        // (one read-back): a bound of gigabytes made the pool map and unmap
        // memory inside the product
        cap = (B->max_blc_per_row > 0 || B->blc_num == 0)
                            ? (long long)A->blc_num * (long long)B->max_blc_per_row
                            : -1;
        if (cap < 0 || cap > (32LL << 20)) {
            AMGT_CUDA_TRY(cudaMemcpyAsync(&stats[2], ub_off + brA, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
            if ((rc = read_back(stats, 4, s, &h))) goto fail;
            cap = h[2];
            AMGT_CUDA_TRY(cudaMemsetAsync(&stats[2], 0, sizeof(int64_t), s));
        }
        // pattern keys, bitmaps and pair slots in one allocation
        const size_t o_map = align256(4 * (size_t)cap), o_slot = o_map + align256(2 * (size_t)cap),
                     o_end = o_slot + align256(2 * (size_t)cap);
        if ((rc = alloc_n(&arena2, o_end, s))) goto fail;
        skey = reinterpret_cast<int *>(arena2);
        smap = reinterpret_cast<uint16_t *>(arena2 + o_map);
        pslot = reinterpret_cast<uint16_t *>(arena2 + o_slot);
    }
    if (brA > 0) {
        // medium-row list and count live behind the large list (2 * brA + 1 ints)
        int *medium = large + brA, *nmedium = large + 2 * brA;  // *nmedium cleared by spgemm_ub_kernel
        // as many CTAs as are resident at once: the rows are shared out
        // evenly, and no CTA waits for a slot to take its share
        static const int sym_resident = [] {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spgemm_symbolic_kernel<256, kSymWarps>,
                                                              32 * kSymWarps, 0) != cudaSuccess || n < 1) {
                (void)cudaGetLastError();  // clear the error of the query; a default grid follows
                n = 8;
            }
            return n;
        }();
        AMGT_LAUNCH((spgemm_symbolic_kernel<256, kSymWarps>), grid_for(kSymWarps, brA, st->sm_count, sym_resident),
                    32 * kSymWarps, 0, s, m, brA, A->blcPtr, A->blcIdx, A->blcMap, B->blcPtr, B->blcIdx, B->blcMap,
                    ccnt, csrcnt, large, stats, ub_off, skey, smap, nullptr, nullptr, medium, nmedium, pslot,
                    st->err);
        AMGT_LAUNCH((spgemm_symbolic_hashed_kernel<kSymCap, 2>), 9 * st->sm_count, 64, 0, s, m, A->blcPtr,
                    A->blcIdx, A->blcMap, B->blcPtr, B->blcIdx, B->blcMap, ccnt, csrcnt, stats, ub_off, skey, smap,
                    medium, nmedium, large, (int *)&stats[3], pslot, st->err);
        AMGT_LAUNCH(spgemm_symbolic_large_kernel, 6 * st->sm_count, kSymLargeThreads, 0, s, m, A->blcPtr, A->blcIdx,
                    A->blcMap, B->blcPtr, B->blcIdx, B->blcMap, large, stats, ccnt, csrcnt, ub_off, skey, smap);
    }
    if ((rc = exclusive_scan_int(ccnt, C->blcPtr, brA + 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemcpyAsync(&stats[2], C->blcPtr + brA, sizeof(int), cudaMemcpyDeviceToDevice, s));
    // CSR row pointer of C (into Ccsr->i, or a temporary when only the
    // nonzero count is wanted)
    if (Ccsr) {
        Ccsr->num_rows = m;
        Ccsr->num_cols = B->col;
        if ((rc = alloc_n(&Ccsr->i, m + 1, s))) goto fail;
        csr_i = Ccsr->i;
    } else if ((rc = alloc_n(&csr_tmp, m + 1, s))) {
        goto fail;
    } else {
        csr_i = csr_tmp;
    }
    if ((rc = exclusive_scan_int(csrcnt, csr_i, m + 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemcpyAsync((int *)&stats[2] + 1, csr_i + m, sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (between && (rc = between(ctx))) goto fail;
    // the exact pair count rides along (it sizes the gathered numeric's lists)
    AMGT_CUDA_TRY(cudaMemcpyAsync(&stats[4], ub_off + brA, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    if ((rc = read_back(stats, 5, s, &h))) goto fail;
    npairs = h[4];
    nbC = (int)(h[2] & 0xFFFFFFFF);
    nlarge = (int)(h[3] & 0xFFFFFFFF);
    nnzC = (int)(h[2] >> 32);
    C->max_blc_per_row = (int)h[0];
    {
        const double avg = brA ? (double)nbC / brA : 0.0;
        const double var = brA ? (double)h[1] / brA - avg * avg : 0.0;
        C->stand = var > 0 ? sqrt(var) : 0.0;
    }
    C->blc_num = nbC;
    C->nnz = (int)(16LL * nbC > 0x7FFFFFFF ? 0x7FFFFFFF : 16LL * nbC);  // saturates
    if ((rc = check_device_error(s))) goto fail;
    if ((rc = alloc_n(&C->blcIdx, nbC, s)) || (rc = alloc_n(&C->blcMap, nbC, s)) ||
        (rc = alloc_n(&C->blcVal, 16LL * nbC, s)))
        goto fail;
    if (prec == AMGT_FLOAT) {
        if ((rc = alloc_n(&C->blcVal_fp32, 16LL * nbC, s))) goto fail;
        cshadow = C->blcVal_fp32;
        if (fuse && fuse->want16 && nbC > 0) {  // fp16 exactness of the fp32 values fused too
            if ((rc = alloc_n(&C->blcVal_fp16, 16LL * nbC, s))) goto fail;
            cextra = C->blcVal_fp16;
            fuse->fused = true;
        }
    } else if (prec == AMGT_HALF) {
        if ((rc = alloc_n(&C->blcVal_fp16, 16LL * nbC, s))) goto fail;
        cshadow = C->blcVal_fp16;
    } else if (prec == AMGT_BF16) {
        if ((rc = alloc_n(&C->blcVal_bf16, 16LL * nbC, s))) goto fail;
        cshadow = C->blcVal_bf16;
    } else if (fuse && fuse->want16 && nbC > 0) {  // fp64: exactness check fused into the store
        if ((rc = alloc_n(&C->blcVal_fp16, 16LL * nbC, s))) goto fail;
        cshadow = C->blcVal_fp16;
        fuse->fused = true;
        if (fuse->want32) {  // and the fp32 shadow of a level used in fp32
            if ((rc = alloc_n(&C->blcVal_fp32, 16LL * nbC, s))) goto fail;
            cextra = C->blcVal_fp32;
        }
    }
    if (Ccsr) {
        Ccsr->num_nonzeros = nnzC;
        if ((rc = alloc_n(&Ccsr->j, nnzC, s)) || (rc = alloc_n(&Ccsr->data, nnzC, s))) goto fail;
    }
    // products of few A block rows (coarse levels) or with many rows beyond
    // kSymCap pairs: the gathered numeric; others:
    // the staged one, whose warp-per-row layout keeps every SM busy on short
    // rows and reads each A row once (both give the same C bit for bit).  fp16 / bf16 products on the tensor-core engine: always the
    // gathered form, its block products on the tensor cores.
    if (brA < 64 * st->sm_count || tensor || 8LL * nlarge > brA) {
        const size_t o_beg = align256(8 * (size_t)npairs), o_num = o_beg + align256(8 * (size_t)nbC + 8),
                     o_end = o_num + align256(4 * (size_t)nbC + 4);
        if ((rc = alloc_n(&arena3, o_end, s))) goto fail;
        int2 *glist = reinterpret_cast<int2 *>(arena3);
        long long *gbeg = reinterpret_cast<long long *>(arena3 + o_beg);
        int *gnum = reinterpret_cast<int *>(arena3 + o_num);
        if (brA > 0) {
            AMGT_CUDA_TRY(cudaMemsetAsync(gnum, 0, 4 * (size_t)nbC + 4, s));
            static const int ord_resident = [] {  // CTAs resident at once
                int n = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spgemm_order_kernel, 32 * kNumWarps, 0) !=
                        cudaSuccess ||
                    n < 1) {
                    (void)cudaGetLastError();  // clear the error of the query; a default grid follows
                    n = 8;
                }
                return n;
            }();
            AMGT_LAUNCH(spgemm_order_kernel, grid_for(kNumWarps, brA, st->sm_count, ord_resident), 32 * kNumWarps, 0,
                        s, brA,
                        A->blcPtr, A->blcIdx, B->blcPtr, B->blcIdx, C->blcPtr, C->blcIdx, C->blcMap, ub_off, skey,
                        smap, pslot, glist, gbeg, gnum);
        }
        if (nbC > 0 && tensor) {
            const long long want = (nbC + 15) / 16;  // 4 warps of 4 C blocks per CTA
            const int grid = (int)std::min<long long>(want, 16LL * st->sm_count);
            if (prec == AMGT_HALF)
                AMGT_LAUNCH(spgemm_gather_mma_kernel<AMGT_HALF>, grid, 128, 0, s, nbC, Atmp.blcVal_fp16,
                            Btmp.blcVal_fp16, glist, gbeg, gnum, C->blcVal, cshadow);
            else
                AMGT_LAUNCH(spgemm_gather_mma_kernel<AMGT_BF16>, grid, 128, 0, s, nbC, Atmp.blcVal_bf16,
                            Btmp.blcVal_bf16, glist, gbeg, gnum, C->blcVal, cshadow);
        } else if (nbC > 0) {
            // four lanes per C block; as many CTAs as are resident at once
            const long long want = (4LL * nbC + kGatherThreads - 1) / kGatherThreads;
            const int grid = (int)std::min<long long>(want, 6LL * st->sm_count);
            unsigned long long *flags = fuse ? reinterpret_cast<unsigned long long *>(fuse->flags) : nullptr;
            switch (prec) {
            case AMGT_DOUBLE:
                AMGT_LAUNCH(spgemm_gather_kernel<AMGT_DOUBLE>, grid, kGatherThreads, GatherSmem<AMGT_DOUBLE>::per_cta,
                            s, nbC, A->blcVal, B->blcVal, glist, gbeg, gnum, C->blcVal, cshadow, flags, cextra);
                break;
            case AMGT_FLOAT:
                AMGT_LAUNCH(spgemm_gather_kernel<AMGT_FLOAT>, grid, kGatherThreads, GatherSmem<AMGT_FLOAT>::per_cta, s,
                            nbC, Atmp.blcVal_fp32, Btmp.blcVal_fp32, glist, gbeg, gnum, C->blcVal, cshadow, flags,
                            cextra);
                break;
            case AMGT_HALF:
                AMGT_LAUNCH(spgemm_gather_kernel<AMGT_HALF>, grid, kGatherThreads, GatherSmem<AMGT_HALF>::per_cta, s,
                            nbC, (const __half *)Atmp.blcVal_fp16, (const __half *)Btmp.blcVal_fp16, glist, gbeg, gnum,
                            C->blcVal, cshadow, nullptr, nullptr);
                break;
            default:
                AMGT_LAUNCH(spgemm_gather_kernel<AMGT_BF16>, grid, kGatherThreads, GatherSmem<AMGT_BF16>::per_cta, s,
                            nbC, (const __nv_bfloat16 *)Atmp.blcVal_bf16, (const __nv_bfloat16 *)Btmp.blcVal_bf16,
                            glist, gbeg, gnum, C->blcVal, cshadow, nullptr, nullptr);
                break;
            }
        }
        if (Ccsr && brA > 0)
            AMGT_LAUNCH(spgemm_csr_kernel, grid_for(kNumWarps, brA, st->sm_count, 8), 32 * kNumWarps, 0, s, m, brA,
                        C->blcPtr, C->blcIdx, C->blcMap, C->blcVal, Ccsr->i, Ccsr->j, Ccsr->data);
    } else
    switch (prec) {
    case AMGT_DOUBLE:
        rc = launch_numeric<AMGT_DOUBLE>(A, A->blcVal, B, B->blcVal, C, cshadow, Ccsr, ub_off, skey, smap, pslot, s,
                                         st->sm_count, fuse ? reinterpret_cast<unsigned long long *>(fuse->flags)
                                                            : nullptr,
                                         cextra);
        break;
    case AMGT_FLOAT:
        rc = launch_numeric<AMGT_FLOAT>(A, Atmp.blcVal_fp32, B, Btmp.blcVal_fp32, C, cshadow, Ccsr, ub_off, skey,
                                        smap, pslot, s, st->sm_count,
                                        fuse ? reinterpret_cast<unsigned long long *>(fuse->flags) : nullptr, cextra);
        break;
    case AMGT_HALF:
        rc = launch_numeric<AMGT_HALF>(A, Atmp.blcVal_fp16, B, Btmp.blcVal_fp16, C, cshadow, Ccsr, ub_off, skey,
                                       smap, pslot, s, st->sm_count);
        break;
    default:
        rc = launch_numeric<AMGT_BF16>(A, Atmp.blcVal_bf16, B, Btmp.blcVal_bf16, C, cshadow, Ccsr, ub_off, skey,
                                       smap, pslot, s, st->sm_count);
        break;
    }
    if (rc) goto fail;
    C->csr_nnz = nnzC;
    C->avg_nnz = nbC ? (double)nnzC / nbC : 0.0;
    free_ptr(arena, s); free_ptr(arena2, s); free_ptr(arena3, s); free_ptr(csr_tmp, s);
    if (ownA) { free_ptr(Atmp.blcVal_fp32, s); free_ptr(Atmp.blcVal_fp16, s); free_ptr(Atmp.blcVal_bf16, s); }
    if (ownB) { free_ptr(Btmp.blcVal_fp32, s); free_ptr(Btmp.blcVal_fp16, s); free_ptr(Btmp.blcVal_bf16, s); }
    return AMGT_OK;
fail:
    free_ptr(arena, s); free_ptr(arena2, s); free_ptr(arena3, s); free_ptr(csr_tmp, s);
    if (ownA) { free_ptr(Atmp.blcVal_fp32, s); free_ptr(Atmp.blcVal_fp16, s); free_ptr(Atmp.blcVal_bf16, s); }
    if (ownB) { free_ptr(Btmp.blcVal_fp32, s); free_ptr(Btmp.blcVal_fp16, s); free_ptr(Btmp.blcVal_bf16, s); }
    amgt_bsr_free(C, stream);
    if (Ccsr) amgt_csr_free(Ccsr, stream);
    return rc;
}

}  // namespace amgt

extern "C" {

int amgt_spgemm(int prec, const amgt_bsr *A, const amgt_bsr *B, amgt_bsr *C, amgt_csr *Ccsr, amgt_stream_t stream)
{
    return amgt::spgemm_impl(prec, A, B, C, Ccsr, stream, nullptr, nullptr);
}

int amgt_spgemm_set_engine(int engine)
{
    if (engine < AMGT_ENGINE_AUTO || engine > AMGT_ENGINE_TENSOR_CORE) return AMGT_ERR_INVALID;
    amgt::g_spgemm_engine.store(engine);
    return AMGT_OK;
}

}  // extern "C"
