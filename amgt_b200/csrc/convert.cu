// CSR <-> mBSR conversions, block transpose, value shadows and the
// long-row segment table.
//
// CSR -> mBSR (replaces CSR2BSR_GPU and its csr2bsr_* kernels,
// AmgT_HYPRE/src/seq_mv/csr_matvec_device.c:683-1267).  One warp owns one
// block row (4 CSR rows).  Its entries become (block column, bit) pairs that
// are sorted in registers (<= 32 entries) or in the warp's shared-memory
// slice (<= 512 entries); block rows with more entries go to a CTA that
// sweeps the block-column range in windows of 8192 with a shared-memory
// bitmap table.  Two passes: count (sorts, keeps the sorted pairs in
// scratch, sizes the arrays with one host read-back), then fill (block
// columns, bitmaps, zero-padded values from the kept pairs).
#include <atomic>

#include <cub/device/device_radix_sort.cuh>

#include "rowunion.cuh"

namespace amgt {

constexpr int kWarpCap = 512;   // entries a warp sorts in shared memory
constexpr int kCvtWarps = 4;    // warps per CTA in the warp paths
constexpr int kWin = 8192;      // key window of the large-row path
constexpr int kLargeThreads = 256;

__device__ __forceinline__ unsigned lanemask_le(int lane) { return (lane == 31) ? FULL : ((2u << lane) - 1u); }

// Entry p of block row b -> packed (block column, local index, bit).
__device__ __forceinline__ unsigned long long csr_entry_pair(const int *ja, int p, int p0, int q_of_p, int n,
                                                             int *err)
{
    const int col = ja[p];
    if (col < 0 || col >= n) {
        raise_error(err, DEV_ERR_INDEX);
        return kSentinel;
    }
    return pack_pair(col >> 2, p - p0, 1u << (q_of_p * 4 + (col & 3)));
}

// Which of the block row's CSR rows holds entry p (rows r0..r0+3).
__device__ __forceinline__ int row_in_block(int p, int e1, int e2, int e3)
{
    return (p >= e1) + (p >= e2) + (p >= e3);
}

struct BlockRowRange {
    int p0, p1, e1, e2, e3;
};

__device__ __forceinline__ BlockRowRange block_row_range(const int *ia, int m, int b)
{
    const int r0 = 4 * b;
    BlockRowRange r;
    r.p0 = ia[r0];
    r.e1 = ia[min(r0 + 1, m)];
    r.e2 = ia[min(r0 + 2, m)];
    r.e3 = ia[min(r0 + 3, m)];
    r.p1 = ia[min(r0 + 4, m)];
    return r;
}

// ------------------------------------------------- sorted count pass
// One thread per block row.  When each of its 4 CSR rows lists block
// columns in non-decreasing order after its first entry (sorted CSR, or
// HYPRE's diagonal-first order), the block row's distinct block columns are
// an 8-way merge (each row's first entry, and the rest of the row): every
// entry gets its column's rank (slot) and a first-of-column flag in slotb,
// and the count goes to cnt[b], with no sorting and no warp-wide matching.  The
// entries of a warp's 32 block rows are first copied into shared memory
// with coalesced loads when they fit.  Block rows of more than kStRowMax
// entries or more than 32 block columns (a slot byte holds 5 bits), with
// unsorted columns or with an index out of range go to slow[] (and
// slowf[b] = 1) for the warp kernel below (which writes their slotb / cnt,
// or reports the bad index).  27-point operators (108 entries and about 27
// block columns per block row) stay on this path.
constexpr int kStWarps = 4;
constexpr int kStCap = 1024;    // entries of a warp's 32 block rows held in shared memory
constexpr int kStRowMax = 128;  // entries of a block row on this path

__global__ void __launch_bounds__(32 * kStWarps)
csr2bsr_count_sorted_kernel(int m, int n, const int *__restrict__ ia, const int *__restrict__ ja, int brow,
                            int *__restrict__ cnt, int *__restrict__ slow, int *__restrict__ nslow,
                            unsigned char *__restrict__ slowf, int64_t *__restrict__ stats,
                            unsigned char *__restrict__ slotb)
{
    __shared__ int scol[kStWarps][kStCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *sc = scol[warp];
    unsigned long long wmax = 0, wsq = 0;
    const int ngroups = (brow + 31) / 32;
    for (int gi = blockIdx.x * kStWarps + warp; gi < ngroups; gi += gridDim.x * kStWarps) {
        const int b = gi * 32 + lane;
        const bool live = b < brow;
        int r[5];
#pragma unroll
        for (int o = 0; o < 5; ++o) r[o] = live ? __ldg(ia + min(4 * b + o, m)) : 0;
        const int P0 = __shfl_sync(FULL, r[0], 0);
        const int P1 = __shfl_sync(FULL, r[4], min(31, brow - 1 - gi * 32));
        const bool staged = P1 - P0 <= kStCap;  // warp-uniform
        if (staged)
            for (int e = P0 + lane; e < P1; e += 32) sc[e - P0] = __ldg(ja + e);
        __syncwarp();
        auto col_at = [&](int p) { return staged ? sc[p - P0] : __ldg(ja + p); };
        bool ok = live && r[4] - r[0] <= kStRowMax;
        int u = 0;
        if (ok) {
            // lists in entry order: row q's first entry (list 2q) and the
            // rest of row q (list 2q + 1), so that the first entry popped
            // for a column is its lowest-numbered one
            int h[8], e[8], c[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                h[2 * q] = r[q];
                e[2 * q] = min(r[q] + 1, r[q + 1]);
                h[2 * q + 1] = r[q] + 1;
                e[2 * q + 1] = r[q + 1];
            }
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                c[l] = 0x7FFFFFFF;
                if (h[l] < e[l]) {
                    const int col = col_at(h[l]);
                    if (col < 0 || col >= n) ok = false;
                    c[l] = col >> 2;
                }
            }
            while (ok) {
                int mn = c[0];
#pragma unroll
                for (int l = 1; l < 8; ++l) mn = min(mn, c[l]);
                if (mn == 0x7FFFFFFF) break;
                if (u == 32) {  // a 33rd block column: slot bytes hold 0..31
                    ok = false;
                    break;
                }
                unsigned lead = 0x80;
#pragma unroll
                for (int l = 0; l < 8; ++l) {
                    while (c[l] == mn) {
                        slotb[h[l]] = (unsigned char)(u | lead);
                        lead = 0;
                        int next = 0x7FFFFFFF;
                        if (++h[l] < e[l]) {
                            const int col = col_at(h[l]);
                            if (col < 0 || col >= n || (col >> 2) < mn) ok = false;  // bad index / unsorted
                            next = (col >> 2) < mn ? 0x7FFFFFFF : col >> 2;
                        }
                        c[l] = next;
                    }
                }
                ++u;
            }
        }
        if (live) slowf[b] = ok ? 0 : 1;
        if (ok) {
            cnt[b] = u;
            wmax = wmax > (unsigned long long)u ? wmax : (unsigned long long)u;
            wsq += (unsigned long long)u * (unsigned long long)u;
        }
        const unsigned left = __ballot_sync(FULL, live && !ok);
        if (left) {
            int at = 0;
            if (lane == 0) at = atomicAdd(nslow, __popc(left));
            at = __shfl_sync(FULL, at, 0);
            if (live && !ok) slow[at + __popc(left & ((1u << lane) - 1))] = b;
        }
        __syncwarp();  // the shared entries are reused by the next group
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long om = __shfl_xor_sync(FULL, wmax, o);
        wmax = wmax > om ? wmax : om;
        wsq += __shfl_xor_sync(FULL, wsq, o);
    }
    if (lane == 0 && wsq) {
        atomicMax((unsigned long long *)&stats[0], wmax);
        atomicAdd((unsigned long long *)&stats[1], wsq);
    }
}

// ------------------------------------------------------------ count pass
// A warp takes kCvtGroup block rows at a time: their row pointers arrive
// in one load and their entries (rows of at most 32) in independent loads,
// so G block rows cost two memory round trips instead of 2 G.  Each block row is then sorted on its own
// (registers for <= 32 entries, the warp's shared-memory slice for <= 512);
// longer ones go to the large list.
constexpr int kCvtGroup = 4;

// rows == nullptr: every block row, in groups of kCvtGroup consecutive ones;
// else the *nrows block rows listed in rows[] (those the one-thread-per-row
// pass below left: unsorted columns, more than 32 entries, bad indices).
__global__ void __launch_bounds__(32 * kCvtWarps)
csr2bsr_count_kernel(int m, int n, const int *__restrict__ ia, const int *__restrict__ ja, int brow,
                     const int *__restrict__ rows, const int *__restrict__ nrows, int *__restrict__ cnt,
                     int *__restrict__ large, int64_t *__restrict__ stats, int *err,
                     unsigned long long *__restrict__ sorted, unsigned char *__restrict__ slotb)
{
    __shared__ unsigned long long sbuf[kCvtWarps][kWarpCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long *s = sbuf[warp];
    unsigned long long wmax = 0, wsq = 0;  // per-warp statistics, one atomic each at the end
    const int total = rows ? *nrows : brow;
    const int ngroups = (total + kCvtGroup - 1) / kCvtGroup;
    for (int g = blockIdx.x * kCvtWarps + warp; g < ngroups; g += gridDim.x * kCvtWarps) {
        const int nb = min(kCvtGroup, total - g * kCvtGroup);
        // lanes 5j .. 5j + 4 hold ia[min(4 b_j + o, m)], o = 0..4, for the
        // group's block rows b_j, j < nb (rows past m are empty)
        const int jl = lane / 5, ol = lane - 5 * jl;
        const int bl = (jl < nb) ? (rows ? rows[g * kCvtGroup + jl] : g * kCvtGroup + jl) : 0;
        const int iav = (jl < nb) ? ia[min(4 * bl + ol, m)] : 0;
        auto range = [&](int j) {  // block row b_j's entries and row ends
            BlockRowRange r;
            r.p0 = __shfl_sync(FULL, iav, 5 * j);
            r.e1 = __shfl_sync(FULL, iav, 5 * j + 1);
            r.e2 = __shfl_sync(FULL, iav, 5 * j + 2);
            r.e3 = __shfl_sync(FULL, iav, 5 * j + 3);
            r.p1 = __shfl_sync(FULL, iav, 5 * j + 4);
            return r;
        };
        unsigned long long v[kCvtGroup];
#pragma unroll
        for (int j = 0; j < kCvtGroup; ++j) {
            const BlockRowRange r = range(j);
            v[j] = kSentinel;
            const int L = r.p1 - r.p0;
            if (j < nb && L <= 32 && lane < L) {
                const int p = r.p0 + lane;
                v[j] = csr_entry_pair(ja, p, r.p0, row_in_block(p, r.e1, r.e2, r.e3), n, err);
            }
        }
#pragma unroll
        for (int j = 0; j < kCvtGroup; ++j) {
            const BlockRowRange Rj = range(j);
            const int b = __shfl_sync(FULL, bl, 5 * j);
            const int L = Rj.p1 - Rj.p0;
            if (j >= nb) {
                // past the last block row (warp-uniform)
            } else if (L > kWarpCap) {
                if (lane == 0) large[atomicAdd((int *)&stats[3], 1)] = b;
            } else {
            int u = 0;
            if (L <= 32) {
                // distinct block columns: lanes with equal columns match,
                // the lowest lane of each group counts it (no sort needed)
                const bool valid = v[j] != kSentinel;
                const int key = valid ? pair_key(v[j]) : -1 - lane;
                const unsigned peers = __match_any_sync(FULL, key);
                const bool leader = valid && (__ffs(peers) - 1) == lane;
                unsigned lm = __ballot_sync(FULL, leader);
                u = __popc(lm);
                int slot = 0;  // rank of the entry's column among the row's distinct columns
                while (lm) {   // warp-uniform
                    const int l = __ffs(lm) - 1;
                    lm &= lm - 1;
                    slot += __shfl_sync(FULL, key, l) < key;
                }
                if (valid) slotb[Rj.p0 + lane] = (unsigned char)(slot | (leader ? 0x80 : 0));
            } else {
                const int N = next_pow2_min64(L);
                for (int i = lane; i < N; i += 32) {
                    unsigned long long x = kSentinel;
                    if (i < L) {
                        const int p = Rj.p0 + i;
                        x = csr_entry_pair(ja, p, Rj.p0, row_in_block(p, Rj.e1, Rj.e2, Rj.e3), n, err);
                    }
                    s[i] = x;
                }
                __syncwarp();
                warp_sort_smem(s, N, lane);
                for (int i0 = 0; i0 < L; i0 += 32) {
                    const int i = i0 + lane;
                    bool head = false;
                    if (i < L) sorted[Rj.p0 + i] = s[i];  // reused by the fill pass
                    if (i < L && s[i] != kSentinel) head = (i == 0) || pair_key(s[i]) != pair_key(s[i - 1]);
                    u += __popc(__ballot_sync(FULL, head));
                }
                __syncwarp();
            }
            if (lane == 0) {
                cnt[b] = u;
                wmax = wmax > (unsigned long long)u ? wmax : (unsigned long long)u;
                wsq += (unsigned long long)u * (unsigned long long)u;
            }
            }
        }
    }
    if (lane == 0 && wsq) {
        atomicMax((unsigned long long *)&stats[0], wmax);
        atomicAdd((unsigned long long *)&stats[1], wsq);
    }
}

// Block-wide min / max of the block columns of a long block row.
__device__ void large_row_key_range(const int *ja, int p0, int p1, int n, int *smin, int *smax, int *kmin,
                                    int *kmax)
{
    if (threadIdx.x == 0) {
        *smin = 0x7FFFFFFF;
        *smax = -1;
    }
    __syncthreads();
    int lo = 0x7FFFFFFF, hi = -1;
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        int col = ja[p];
        if (col < 0 || col >= n) continue;
        lo = min(lo, col >> 2);
        hi = max(hi, col >> 2);
    }
    atomicMin(smin, lo);
    atomicMax(smax, hi);
    __syncthreads();
    *kmin = *smin;
    *kmax = *smax;
    __syncthreads();
}

// Block-wide exclusive scan of one int per thread (blockDim.x == 256).
__device__ int block_excl_scan256(int v, int *sh, int *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int wt;
    int x = warp_excl_scan(v, lane, &wt);
    if (lane == 0) sh[warp] = wt;
    __syncthreads();
    if (warp == 0) {
        int t = (lane < 8) ? sh[lane] : 0, tt;
        int e = warp_excl_scan(t, lane, &tt);
        if (lane < 8) sh[lane] = e;
        if (lane == 0) sh[8] = tt;
    }
    __syncthreads();
    x += sh[warp];
    *total = sh[8];
    __syncthreads();
    return x;
}

// Large block rows: window sweep with a shared-memory bitmap table.
// fill == false: count.  fill == true: write columns, bitmaps and values.
template <bool FILL>
__global__ void __launch_bounds__(kLargeThreads)
csr2bsr_large_kernel(int m, int n, const int *__restrict__ ia, const int *__restrict__ ja,
                     const double *__restrict__ a, const int *__restrict__ large, const int64_t *stats,
                     int *__restrict__ cnt, const int *__restrict__ bptr, int *__restrict__ bidx,
                     uint16_t *__restrict__ bmap, double *__restrict__ bval, int64_t *stats_out)
{
    extern __shared__ uint32_t smem[];
    uint32_t *maps = smem;                      // [kWin]
    int *pos = (int *)(smem + kWin);            // [kWin] (fill only)
    __shared__ int sh[16];
    __shared__ int smin, smax;
    const int nlarge = (int)stats[3];
    const int tid = threadIdx.x;
    for (int t = blockIdx.x; t < nlarge; t += gridDim.x) {
        const int b = large[t];
        const BlockRowRange R = block_row_range(ia, m, b);
        int kmin, kmax;
        large_row_key_range(ja, R.p0, R.p1, n, &smin, &smax, &kmin, &kmax);
        int total = 0;
        const int base = FILL ? bptr[b] : 0;
        for (long long w0 = kmin; w0 <= kmax; w0 += kWin) {
            for (int i = tid; i < kWin; i += blockDim.x) maps[i] = 0;
            __syncthreads();
            for (int p = R.p0 + tid; p < R.p1; p += blockDim.x) {
                const int col = ja[p];
                if (col < 0 || col >= n) continue;
                const long long k = (col >> 2) - w0;
                if (k < 0 || k >= kWin) continue;
                const int q = row_in_block(p, R.e1, R.e2, R.e3);
                atomicOr(&maps[k], 1u << (q * 4 + (col & 3)));
            }
            __syncthreads();
            // each thread owns 32 consecutive slots
            const int s0 = tid * (kWin / kLargeThreads);
            int c = 0;
            for (int i = 0; i < kWin / kLargeThreads; ++i) c += maps[s0 + i] != 0;
            int wtotal;
            int off = block_excl_scan256(c, sh, &wtotal);
            if (FILL) {
                int o = base + total + off;
                for (int i = 0; i < kWin / kLargeThreads; ++i) {
                    const uint32_t mp = maps[s0 + i];
                    if (mp) {
                        pos[s0 + i] = o;
                        bidx[o] = (int)(w0 + s0 + i);
                        bmap[o] = (uint16_t)mp;
                        ++o;
                    }
                }
                // zero this window's blocks, then scatter its entries
                double2 *z = reinterpret_cast<double2 *>(bval + (size_t)16 * (base + total));
                for (int i = tid; i < 8 * wtotal; i += blockDim.x) z[i] = make_double2(0.0, 0.0);
                __syncthreads();
                for (int p = R.p0 + tid; p < R.p1; p += blockDim.x) {
                    const int col = ja[p];
                    if (col < 0 || col >= n) continue;
                    const long long k = (col >> 2) - w0;
                    if (k < 0 || k >= kWin) continue;
                    const int q = row_in_block(p, R.e1, R.e2, R.e3);
                    bval[(size_t)16 * pos[k] + q * 4 + (col & 3)] = a[p];
                }
            }
            total += wtotal;
            __syncthreads();
        }
        if (!FILL && tid == 0) {
            cnt[b] = total;
            atomicMax((unsigned long long *)&stats_out[0], (unsigned long long)total);
            atomicAdd((unsigned long long *)&stats_out[1], (unsigned long long)total * (unsigned long long)total);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- fill pass
// Fill for the block rows of the sorted count pass (slowf[b] == 0): 4 lanes
// per block row, lane q walks CSR row q (its first entry, then the rest in
// column order, so in slot order) slot by slot and writes row q of every
// block once, zeros included; the 4 lanes together write whole 128-byte
// blocks.  A block's bitmap is the OR of the 4 lanes' nibbles (shuffles in
// the group), and the first entry of a column writes the block column.  A
// warp takes 8 block rows at a time and first copies their entries (column,
// value, slot byte) into shared memory with coalesced loads.
// With every block row on this path the pass can also write, from the
// values it holds: the fp16 rounding of each stored value and the
// exactness bits of exact_check_kernel (v16, flags), the fp32 rounding
// (v32, for an operator used in fp32), and each row's l1 norm
// summed as l1_norm_kernel sums it (blocks in order, |v0| + |v1| + |v2| +
// |v3| per block; 1 / norm with l1_invert).
constexpr int kFsWarps = 4;
constexpr int kFsCap = 256;  // entries of a warp's 8 block rows held in shared memory

struct FillExtras {
    __half *v16;                // nullable
    unsigned long long *flags;  // with v16
    float *v32;                 // nullable
    double *l1;                 // nullable
    int l1_invert;
};

__global__ void __launch_bounds__(32 * kFsWarps)
csr2bsr_fill_sorted_kernel(int m, const int *__restrict__ ia, const int *__restrict__ ja,
                           const double *__restrict__ a, int brow, const unsigned char *__restrict__ slowf,
                           const int *__restrict__ bptr, int *__restrict__ bidx, uint16_t *__restrict__ bmap,
                           double *__restrict__ bval, const unsigned char *__restrict__ slotb, FillExtras fx)
{
    bool not32 = false, not16 = false;
    __shared__ double sval[kFsWarps][kFsCap];
    __shared__ int scol[kFsWarps][kFsCap];
    __shared__ unsigned char sslot[kFsWarps][kFsCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = lane & 3;
    const unsigned gmask = 0xFu << (lane & ~3);
    const int nwg = (brow + 7) / 8;
    for (int wg = blockIdx.x * kFsWarps + warp; wg < nwg; wg += gridDim.x * kFsWarps) {
        const int b0 = 8 * wg;
        const int E0 = __ldg(ia + 4 * b0), E1 = __ldg(ia + min(4 * (b0 + 8), m));
        const bool staged = E1 - E0 <= kFsCap;  // warp-uniform
        if (staged)
            for (int e = E0 + lane; e < E1; e += 32) {
                scol[warp][e - E0] = __ldg(ja + e);
                sval[warp][e - E0] = __ldg(a + e);
                sslot[warp][e - E0] = __ldg(slotb + e);
            }
        __syncwarp();
        auto entry = [&](int p, int &sb, int &c, double &v) {
            if (staged) {
                sb = sslot[warp][p - E0];
                c = scol[warp][p - E0];
                v = sval[warp][p - E0];
            } else {
                sb = __ldg(slotb + p);
                c = __ldg(ja + p);
                v = __ldg(a + p);
            }
        };
        const int b = b0 + (lane >> 2);
        if (b < brow && !slowf[b]) {  // the same for the 4 lanes of a group
            const int base = bptr[b], u = bptr[b + 1] - base;
            const int r = 4 * b + q;
            int p = 0, pe = 0;
            if (r < m) {
                p = ia[r];
                pe = ia[r + 1];
            }
            int hs = -1, hc = 0, hsb = 0;
            double hv = 0.0;
            if (p < pe) {
                entry(p, hsb, hc, hv);
                hs = hsb & 0x1F;
                ++p;
            }
            int ts = -1, tc = 0, tsb = 0;
            double tv = 0.0;
            if (p < pe) {
                entry(p, tsb, tc, tv);
                ts = tsb & 0x1F;
            }
            double l1s = 0.0;
            for (int sl = 0; sl < u; ++sl) {
                double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
                unsigned bits = 0;
                if (hs == sl) {
                    const int c = hc & 3;
                    v0 = c == 0 ? hv : v0; v1 = c == 1 ? hv : v1; v2 = c == 2 ? hv : v2; v3 = c == 3 ? hv : v3;
                    bits |= 1u << c;
                    if (hsb & 0x80) bidx[base + sl] = hc >> 2;
                }
                while (ts == sl) {
                    const int c = tc & 3;
                    v0 = c == 0 ? tv : v0; v1 = c == 1 ? tv : v1; v2 = c == 2 ? tv : v2; v3 = c == 3 ? tv : v3;
                    bits |= 1u << c;
                    if (tsb & 0x80) bidx[base + sl] = tc >> 2;
                    ts = -1;
                    if (++p < pe) {
                        entry(p, tsb, tc, tv);
                        ts = tsb & 0x1F;
                    }
                }
                double2 *dst = reinterpret_cast<double2 *>(bval + 16LL * (base + sl) + 4 * q);
                dst[0] = make_double2(v0, v1);
                dst[1] = make_double2(v2, v3);
                if (fx.v16) {
                    const double vv[4] = {v0, v1, v2, v3};
                    __half hh[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        hh[c] = __double2half(vv[c]);
                        if ((double)__double2float_rn(vv[c]) != vv[c]) not32 = true;
                        if ((double)__half2float(hh[c]) != vv[c]) not16 = true;
                    }
                    __half2 *d16 = reinterpret_cast<__half2 *>(fx.v16 + 16LL * (base + sl) + 4 * q);
                    d16[0] = __halves2half2(hh[0], hh[1]);
                    d16[1] = __halves2half2(hh[2], hh[3]);
                }
                if (fx.v32)
                    *reinterpret_cast<float4 *>(fx.v32 + 16LL * (base + sl) + 4 * q) =
                        make_float4(__double2float_rn(v0), __double2float_rn(v1), __double2float_rn(v2),
                                    __double2float_rn(v3));
                l1s += fabs(v0) + fabs(v1) + fabs(v2) + fabs(v3);
                unsigned mp = bits << (4 * q);
                mp |= __shfl_xor_sync(gmask, mp, 1);
                mp |= __shfl_xor_sync(gmask, mp, 2);
                if (q == 0) bmap[base + sl] = (uint16_t)mp;
            }
            if (fx.l1 && r < m) fx.l1[r] = fx.l1_invert ? (l1s != 0.0 ? 1.0 / l1s : 0.0) : l1s;
        }
        __syncwarp();  // the shared entries are reused by the next group
    }
    if (fx.v16) {  // the warp's loop trip count is uniform: all lanes are here
        const unsigned b32 = __ballot_sync(FULL, not32), b16 = __ballot_sync(FULL, not16);
        if (lane == 0 && (b32 | b16)) atomicOr(fx.flags, (b32 ? 1ull : 0ull) | (b16 ? 2ull : 0ull));
    }
}

// Takes each block row's pairs as the count pass sorted them (scratch at the
// block row's CSR offset) and writes block columns, OR-ed bitmaps and the
// zero-padded values.
// rows == nullptr: every block row; else the *nrows listed ones (as in the
// count pass).
__global__ void __launch_bounds__(32 * kCvtWarps)
csr2bsr_fill_kernel(int m, int n, const int *__restrict__ ia, const int *__restrict__ ja,
                    const double *__restrict__ a, int brow, const int *__restrict__ rows,
                    const int *__restrict__ nrows, const int *__restrict__ bptr, int *__restrict__ bidx,
                    uint16_t *__restrict__ bmap, double *__restrict__ bval,
                    const unsigned long long *__restrict__ sorted, const unsigned char *__restrict__ slotb, int *err)
{
    __shared__ unsigned sorv[kCvtWarps][32];  // per-slot OR of the bitmaps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned *so = sorv[warp];
    const int total = rows ? *nrows : brow;
    const int ngroups = (total + kCvtGroup - 1) / kCvtGroup;
    for (int g = blockIdx.x * kCvtWarps + warp; g < ngroups; g += gridDim.x * kCvtWarps) {
        // kCvtGroup block rows at a time, as in the count pass: row pointers
        // (lanes 5j .. 5j + 4) and block offsets (lanes 2j, 2j + 1) in one
        // load each, sorted pairs and values of the short rows in
        // independent loads
        const int nb = min(kCvtGroup, total - g * kCvtGroup);
        const int jl = lane / 5, ol = lane - 5 * jl;
        const int bl = (jl < nb) ? (rows ? rows[g * kCvtGroup + jl] : g * kCvtGroup + jl) : 0;
        const int iav = (jl < nb) ? ia[min(4 * bl + ol, m)] : 0;
        const int jb = lane >> 1;
        const int bb = __shfl_sync(FULL, bl, 5 * min(jb, kCvtGroup - 1));  // every lane shuffles
        const int bpv = (jb < nb) ? bptr[bb + (lane & 1)] : 0;
        unsigned long long v[kCvtGroup];
        double av[kCvtGroup];
        int sl[kCvtGroup];  // slot | 0x80 on the first entry of its column (from the count pass)
#pragma unroll
        for (int j = 0; j < kCvtGroup; ++j) {
            const int p0 = __shfl_sync(FULL, iav, 5 * j), e1 = __shfl_sync(FULL, iav, 5 * j + 1),
                      e2 = __shfl_sync(FULL, iav, 5 * j + 2), e3 = __shfl_sync(FULL, iav, 5 * j + 3),
                      p1 = __shfl_sync(FULL, iav, 5 * j + 4);
            const int L = p1 - p0;
            v[j] = kSentinel;
            av[j] = 0.0;
            sl[j] = 0;
            if (j < nb && L <= 32 && lane < L) {  // short rows: entries straight from ja / a
                const int p = p0 + lane;
                v[j] = csr_entry_pair(ja, p, p0, row_in_block(p, e1, e2, e3), n, err);
                av[j] = a[p];
                sl[j] = slotb[p];
            }
        }
#pragma unroll
        for (int j = 0; j < kCvtGroup; ++j) {
            const int p0 = __shfl_sync(FULL, iav, 5 * j), p1 = __shfl_sync(FULL, iav, 5 * j + 4);
            const int L = p1 - p0;
            const int base = __shfl_sync(FULL, bpv, 2 * j), u = __shfl_sync(FULL, bpv, 2 * j + 1) - base;
            if (j < nb && L <= kWarpCap) {  // warp-uniform; longer rows: large-row kernel
                double2 *z = reinterpret_cast<double2 *>(bval + (size_t)16 * base);
                for (int i = lane; i < 8 * u; i += 32) z[i] = make_double2(0.0, 0.0);
                __syncwarp();
                if (L <= 32) {
                    // group the entries by block column (match), OR the
                    // group's bits, rank the column among the row's distinct
                    // columns by comparing with each group's leader
                    const bool valid = v[j] != kSentinel;
                    const int key = pair_key(v[j]);
                    const int slot = sl[j] & 0x1F;
                    const bool leader = valid && (sl[j] & 0x80);
                    so[lane] = 0;
                    __syncwarp();
                    if (valid) atomicOr(&so[slot], pair_map(v[j]));
                    __syncwarp();
                    if (valid) {
                        if (leader) {
                            bidx[base + slot] = key;
                            bmap[base + slot] = (uint16_t)so[slot];
                        }
                        const int bit = __ffs(pair_map(v[j])) - 1;
                        bval[(size_t)16 * (base + slot) + bit] = av[j];
                    }
                } else {
                    const unsigned long long *sp = sorted + p0;
                    int running = 0;
                    for (int i0 = 0; i0 < L; i0 += 32) {
                        const int i = i0 + lane;
                        const unsigned long long w = (i < L) ? sp[i] : kSentinel;
                        bool head = false;
                        if (w != kSentinel) head = (i == 0) || pair_key(w) != pair_key(sp[i - 1]);
                        const unsigned hb = __ballot_sync(FULL, head);
                        const int slot = running + __popc(hb & lanemask_le(lane)) - 1;
                        if (w != kSentinel) {
                            if (head) {
                                uint32_t orv = 0;
                                const int key = pair_key(w);
                                for (int jj = i; jj < L && sp[jj] != kSentinel && pair_key(sp[jj]) == key; ++jj)
                                    orv |= pair_map(sp[jj]);
                                bidx[base + slot] = key;
                                bmap[base + slot] = (uint16_t)orv;
                            }
                            const int bit = __ffs(pair_map(w)) - 1;
                            bval[(size_t)16 * (base + slot) + bit] = a[p0 + pair_tag(w)];
                        }
                        running += __popc(hb);
                    }
                }
            }
        }
    }
}

// --------------------------------------------------------- mBSR -> CSR
// Row counts: popcount of nibble q of every bitmap of block row b.
__global__ void bsr2csr_count_kernel(int m, int brow, const int *__restrict__ bptr,
                                     const uint16_t *__restrict__ bmap, int *__restrict__ rowcnt)
{
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;
    for (int b = blockIdx.x * wpc + (threadIdx.x >> 5); b < brow; b += gridDim.x * wpc) {
        int c0 = 0, c1 = 0, c2 = 0, c3 = 0;
        for (int k = bptr[b] + lane; k < bptr[b + 1]; k += 32) {
            const uint32_t mp = bmap[k];
            c0 += __popc(mp & 0xFu);
            c1 += __popc(mp & 0xF0u);
            c2 += __popc(mp & 0xF00u);
            c3 += __popc(mp & 0xF000u);
        }
        c0 = warp_sum(c0); c1 = warp_sum(c1); c2 = warp_sum(c2); c3 = warp_sum(c3);
        if (lane < 4) {
            const int r = 4 * b + lane;
            const int c = lane == 0 ? c0 : lane == 1 ? c1 : lane == 2 ? c2 : c3;
            if (r < m) rowcnt[r] = c;
        }
    }
}

// Emission: for each CSR row of the block row, walk the blocks 32 at a time,
// one block per lane, and place the nibble's set bits with a warp scan.
__global__ void bsr2csr_fill_kernel(int m, int brow, const int *__restrict__ bptr, const int *__restrict__ bidx,
                                    const uint16_t *__restrict__ bmap, const double *__restrict__ bval,
                                    const int *__restrict__ ia, int *__restrict__ ja, double *__restrict__ a)
{
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;
    for (int b = blockIdx.x * wpc + (threadIdx.x >> 5); b < brow; b += gridDim.x * wpc) {
        const int k0 = bptr[b], k1 = bptr[b + 1];
        for (int q = 0; q < 4 && 4 * b + q < m; ++q) {
            int out = ia[4 * b + q];
            for (int kk = k0; kk < k1; kk += 32) {
                const int k = kk + lane;
                uint32_t nib = 0;
                int col0 = 0;
                if (k < k1) {
                    nib = (bmap[k] >> (4 * q)) & 0xFu;
                    col0 = 4 * bidx[k];
                }
                int tot;
                int off = warp_excl_scan(__popc(nib), lane, &tot);
                if (nib) {
                    const double *v = bval + (size_t)16 * k + 4 * q;
                    int o = out + off;
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (nib & (1u << c)) {
                            ja[o] = col0 + c;
                            a[o] = v[c];
                            ++o;
                        }
                }
                out += tot;
            }
        }
    }
}

// ------------------------------------------------------ segment table
// Long block rows are cut into segments of at most 64 blocks
// (get_rowPtrbyWarp / get_rowIdxbyWarp, csr_matvec_device.c:615-637).
constexpr int kSegmentBlocks = 64;

__global__ void seg_count_kernel(int brow, const int *__restrict__ bptr, int *__restrict__ segcnt)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < brow; b += gridDim.x * blockDim.x) {
        const int len = bptr[b + 1] - bptr[b];
        segcnt[b] = (len + kSegmentBlocks - 1) / kSegmentBlocks;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) segcnt[brow] = 0;
}

__global__ void seg_fill_kernel(int brow, const int *__restrict__ segptr, int *__restrict__ segrow)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < brow; b += gridDim.x * blockDim.x)
        for (int s = segptr[b]; s < segptr[b + 1]; ++s) segrow[s] = b;
}

// ------------------------------------------------------------ shadows
template <int PREC>
__global__ void shadow_kernel(long long n, const double *__restrict__ v, void *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double d = v[i];
        if (PREC == AMGT_FLOAT) static_cast<float *>(out)[i] = __double2float_rn(d);
        else if (PREC == AMGT_HALF) static_cast<__half *>(out)[i] = __double2half(d);
        else static_cast<__nv_bfloat16 *>(out)[i] = __double2bfloat16(d);
    }
}

// Exactness of stored values, fused with the fp16 shadow: writes the
// fp16 rounding of every value and sets bit 0 of *flags when some value is
// not an fp32 value, bit 1 when some value is not an fp16 value (round trip
// through the format changes it; NaN counts as inexact).
__global__ void exact_check_kernel(long long n, const double *__restrict__ v, __half *__restrict__ v16,
                                   unsigned long long *flags)
{
    bool not32 = false, not16 = false;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double d = v[i];
        const __half h = __double2half(d);
        v16[i] = h;
        if ((double)__double2float_rn(d) != d) not32 = true;
        if ((double)__half2float(h) != d) not16 = true;
    }
    const unsigned b32 = __ballot_sync(FULL, not32), b16 = __ballot_sync(FULL, not16);
    if ((threadIdx.x & 31) == 0 && (b32 | b16))
        atomicOr(flags, (b32 ? 1ull : 0ull) | (b16 ? 2ull : 0ull));
}

int bsr_exact_check(amgt_bsr *A, int64_t *flag, bool *own16, cudaStream_t s, int sm_count)
{
    *own16 = false;
    if (A->blc_num == 0) return AMGT_OK;
    const long long n = 16LL * A->blc_num;
    if (!A->blcVal_fp16) {
        AMGT_TRY(alloc_n(&A->blcVal_fp16, (size_t)n, s));
        *own16 = true;
    }
    AMGT_LAUNCH(exact_check_kernel, grid_for(256 * 4, n, sm_count, 8), 256, 0, s, n, A->blcVal,
                reinterpret_cast<__half *>(A->blcVal_fp16), (unsigned long long *)flag);
    return AMGT_OK;
}

int bsr_exact_apply(amgt_bsr *A, int64_t flag, bool own16, cudaStream_t s)
{
    A->exact_prec = AMGT_DOUBLE;
    if (A->blc_num == 0) return AMGT_OK;
    if (!(flag & 2)) {
        A->exact_prec = AMGT_HALF;  // the fp16 shadow written by the check holds every value
        return AMGT_OK;
    }
    if (own16) free_ptr(A->blcVal_fp16, s);  // speculative shadow not needed
    if (flag & 1) return AMGT_OK;
    AMGT_TRY(amgt_bsr_make_shadow(A, AMGT_FLOAT, (amgt_stream_t)s));  // exact, so equal to any existing shadow
    A->exact_prec = AMGT_FLOAT;
    return AMGT_OK;
}

// ------------------------------------------------- block-row statistics
// out[0] = longest block row (max), out[1] = sum of squared lengths.
__global__ void row_stats_kernel(int brow, const int *__restrict__ bptr, int64_t *__restrict__ out)
{
    long long mx = 0, s2 = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < brow; b += gridDim.x * blockDim.x) {
        const long long len = bptr[b + 1] - bptr[b];
        mx = len > mx ? len : mx;
        s2 += len * len;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        long long om = __shfl_xor_sync(FULL, mx, o);
        mx = om > mx ? om : mx;
        s2 += __shfl_xor_sync(FULL, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax((unsigned long long *)&out[0], (unsigned long long)mx);
        atomicAdd((unsigned long long *)&out[1], (unsigned long long)s2);
    }
}

int block_row_stats(amgt_bsr *A, cudaStream_t s)
{
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    int64_t *d = nullptr;
    AMGT_TRY(alloc_n(&d, 2, s));
    AMGT_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(int64_t) * 2, s));
    if (A->blc_row > 0)
        AMGT_LAUNCH(row_stats_kernel, grid_for(256, A->blc_row, st->sm_count, 4), 256, 0, s, A->blc_row, A->blcPtr, d);
    const int64_t *h = nullptr;
    int rc = read_back(d, 2, s, &h);
    free_ptr(d, s);
    if (rc) return rc;
    A->max_blc_per_row = (int)h[0];
    const double brow = A->blc_row, avg = brow > 0 ? A->blc_num / brow : 0.0;
    const double var = brow > 0 ? (double)h[1] / brow - avg * avg : 0.0;
    A->stand = var > 0 ? sqrt(var) : 0.0;
    return AMGT_OK;
}

// ---------------------------------------------------------- transpose
__global__ void row_of_block_kernel(int brow, const int *__restrict__ bptr, int *__restrict__ rowid,
                                    int *__restrict__ iota)
{
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;
    for (int b = blockIdx.x * wpc + (threadIdx.x >> 5); b < brow; b += gridDim.x * wpc)
        for (int k = bptr[b] + lane; k < bptr[b + 1]; k += 32) {
            rowid[k] = b;
            iota[k] = k;
        }
}

__global__ void col_hist_kernel(int nblk, const int *__restrict__ bidx, int *__restrict__ hist)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nblk; k += gridDim.x * blockDim.x)
        atomicAdd(&hist[bidx[k]], 1);
}

// out block d takes source block src[d]: row -> column, values transposed
// (and the fp16 shadow with them when aval16 is given).
__global__ void transpose_gather_kernel(int nblk, const int *__restrict__ src, const int *__restrict__ rowid,
                                        const uint16_t *__restrict__ amap, const double *__restrict__ aval,
                                        int *__restrict__ tidx, uint16_t *__restrict__ tmap,
                                        double *__restrict__ tval, const __half *__restrict__ aval16,
                                        __half *__restrict__ tval16, const float *__restrict__ aval32,
                                        float *__restrict__ tval32)
{
    // 16 threads per block: thread e writes entry e of the transposed block
    const long long total = (long long)nblk * 16;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(t >> 4), e = (int)(t & 15);
        const int sidx = src[d];
        const int r = e >> 2, c = e & 3;  // entry (r, c) of the transpose = (c, r) of the source
        tval[t] = aval[(size_t)16 * sidx + 4 * c + r];
        if (aval16) tval16[t] = aval16[(size_t)16 * sidx + 4 * c + r];
        if (aval32) tval32[t] = aval32[(size_t)16 * sidx + 4 * c + r];
        if (e == 0) {
            tidx[d] = rowid[sidx];
            tmap[d] = (uint16_t)bitmap_transpose(amap[sidx]);
        }
    }
}

}  // namespace amgt

using namespace amgt;

static int csr_valid(const amgt_csr *A)
{
    if (!A || A->num_rows < 0 || A->num_cols < 0 || A->num_nonzeros < 0) return 0;
    if (A->num_rows > 0 && !A->i) return 0;
    if (A->num_nonzeros > 0 && (!A->j || !A->data)) return 0;
    return 1;
}

extern "C" {

int amgt_bsr_free(amgt_bsr *A, amgt_stream_t stream)
{
    if (!A) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    tune_forget(A);
    free_ptr(A->blcPtr, s);
    free_ptr(A->blcIdx, s);
    free_ptr(A->blcVal, s);
    free_ptr(A->blcMap, s);
    free_ptr(A->rowPtrbyWarp, s);
    free_ptr(A->rowIdxbyWarp, s);
    free_ptr(A->blcVal_fp32, s);
    free_ptr(A->blcVal_fp16, s);
    free_ptr(A->blcVal_bf16, s);
    memset(A, 0, sizeof(*A));
    return AMGT_OK;
}

int amgt_csr_free(amgt_csr *A, amgt_stream_t stream)
{
    if (!A) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    free_ptr(A->i, s);
    free_ptr(A->j, s);
    free_ptr(A->data, s);
    memset(A, 0, sizeof(*A));
    return AMGT_OK;
}

}  // extern "C"

namespace amgt {

// amgt_csr_to_bsr with an optional host callback `between`, run after the
// count pass is queued and before the host waits for the block count (host
// work that can overlap it; the AMG setup converts the first
// interpolation there, on its own stream).
int csr_to_bsr_impl(const amgt_csr *A, amgt_bsr *out, amgt_stream_t stream, int (*between)(void *), void *ctx,
                    CvtFuse *fuse)
{
    if (!csr_valid(A) || !out) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int m = A->num_rows, n = A->num_cols;
    const int brow = (m + 3) / 4;
    memset(out, 0, sizeof(*out));
    out->row = m;
    out->col = n;
    out->blc_row = brow;
    out->blc_col = (n + 3) / 4;

    int *cnt = nullptr, *large = nullptr;
    unsigned char *slowf = nullptr;  // per block row: left to the warp kernels
    int64_t *stats = nullptr;
    unsigned long long *sorted = nullptr;  // sorted entries of rows of 33..512 entries
    unsigned char *slotb = nullptr;        // per entry of shorter rows: block slot | first-of-column flag
    int rc = AMGT_OK;
    const int64_t *h = nullptr;
    int nb = 0;
    FillExtras fx{nullptr, nullptr, nullptr, nullptr, 0};
    bool all_sorted = false;  // no block row left to the warp or large-row kernels
    static std::atomic<bool> smem_set[64];  // per device: the large-row kernels' shared-memory opt-in
    int dev = 0;
    AMGT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !smem_set[dev]) {
        AMGT_CUDA_TRY(cudaFuncSetAttribute(csr2bsr_large_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           2 * kWin * (int)sizeof(uint32_t)));
        AMGT_CUDA_TRY(cudaFuncSetAttribute(csr2bsr_large_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           2 * kWin * (int)sizeof(uint32_t)));
        smem_set[dev] = true;
    }
    // stats: [0] longest block row, [1] sum of squares, [2] block count,
    // [3] large-row count (int), [4] slow-row count (int)
    if ((rc = alloc_n(&out->blcPtr, brow + 1, s)) || (rc = alloc_n(&cnt, brow + 1, s)) ||
        (rc = alloc_n(&large, 2 * (size_t)brow, s)) || (rc = alloc_n(&stats, 5, s)) ||
        (rc = alloc_n(&sorted, (size_t)A->num_nonzeros, s)) ||
        (rc = alloc_n(&slotb, (size_t)A->num_nonzeros, s)) || (rc = alloc_n(&slowf, (size_t)brow, s)))
        goto fail;
    AMGT_CUDA_TRY(cudaMemsetAsync(stats, 0, sizeof(int64_t) * 5, s));
    AMGT_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * (brow + 1), s));
    if (brow > 0) {
        // slow-row list behind the large-row list (2 brow ints)
        int *slow = large + brow, *nslow = (int *)&stats[4];
        AMGT_LAUNCH(csr2bsr_count_sorted_kernel, grid_for(32 * kStWarps, brow, st->sm_count, 12), 32 * kStWarps, 0,
                    s, m, n, A->i, A->j, brow, cnt, slow, nslow, slowf, stats, slotb);
        AMGT_LAUNCH(csr2bsr_count_kernel, 2 * st->sm_count, 32 * kCvtWarps, 0, s, m, n, A->i, A->j, brow, slow,
                    nslow, cnt, large, stats, st->err, sorted, slotb);
        AMGT_LAUNCH(csr2bsr_large_kernel<false>, 2 * st->sm_count, kLargeThreads, 2 * kWin * sizeof(uint32_t), s,
                    m, n, A->i, A->j, A->data, large, stats, cnt, nullptr, nullptr, nullptr, nullptr, stats);
    }
    if ((rc = exclusive_scan_int(cnt, out->blcPtr, brow + 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemcpyAsync(&stats[2], out->blcPtr + brow, sizeof(int), cudaMemcpyDeviceToDevice, s));
    if (between && (rc = between(ctx))) goto fail;
    if ((rc = read_back(stats, 5, s, &h))) goto fail;
    nb = (int)h[2];
    all_sorted = h[3] == 0 && h[4] == 0;
    out->max_blc_per_row = (int)h[0];
    {
        const double S2 = (double)h[1];
        const double avg = brow ? (double)nb / brow : 0.0;
        double var = brow ? S2 / brow - avg * avg : 0.0;
        out->stand = var > 0 ? sqrt(var) : 0.0;
    }
    if ((rc = check_device_error(s))) goto fail;
    out->blc_num = nb;
    out->nnz = (int)(16LL * nb > 0x7FFFFFFF ? 0x7FFFFFFF : 16LL * nb);  // saturates
    out->avg_nnz = nb ? (double)A->num_nonzeros / nb : 0.0;
    out->csr_nnz = A->num_nonzeros;
    if ((rc = alloc_n(&out->blcIdx, nb, s)) || (rc = alloc_n(&out->blcMap, nb, s)) ||
        (rc = alloc_n(&out->blcVal, (size_t)16 * nb, s)))
        goto fail;
    if (fuse) {
        fuse->fused = false;
        if (all_sorted && brow > 0) {
            fx.l1 = fuse->l1;
            fx.l1_invert = fuse->invert;
            if (fuse->want16 && nb > 0) {
                if ((rc = alloc_n(&out->blcVal_fp16, (size_t)16 * nb, s))) goto fail;
                fx.v16 = reinterpret_cast<__half *>(out->blcVal_fp16);
                fx.flags = reinterpret_cast<unsigned long long *>(fuse->flags);
                if (fuse->want32) {
                    if ((rc = alloc_n(&out->blcVal_fp32, (size_t)16 * nb, s))) goto fail;
                    fx.v32 = out->blcVal_fp32;
                }
            }
            fuse->fused = true;
        }
    }
    if (brow > 0) {
        const int *slow = large + brow, *nslow = (const int *)&stats[4];
        AMGT_LAUNCH(csr2bsr_fill_sorted_kernel, grid_for(8 * kFsWarps, brow, st->sm_count, 16), 32 * kFsWarps, 0, s,
                    m, A->i, A->j,
                    A->data, brow, slowf, out->blcPtr, out->blcIdx, out->blcMap, out->blcVal, slotb, fx);
        AMGT_LAUNCH(csr2bsr_fill_kernel, 2 * st->sm_count, 32 * kCvtWarps, 0, s, m, n, A->i, A->j, A->data, brow,
                    slow, nslow, out->blcPtr, out->blcIdx, out->blcMap, out->blcVal, sorted, slotb, st->err);
        AMGT_LAUNCH(csr2bsr_large_kernel<true>, 2 * st->sm_count, kLargeThreads, 2 * kWin * sizeof(uint32_t), s, m,
                    n, A->i, A->j, A->data, large, stats, nullptr, out->blcPtr, out->blcIdx, out->blcMap, out->blcVal,
                    nullptr);
    }
    free_ptr(cnt, s);
    free_ptr(large, s);
    free_ptr(stats, s);
    free_ptr(sorted, s);
    free_ptr(slotb, s);
    free_ptr(slowf, s);
    return AMGT_OK;
fail:
    free_ptr(cnt, s);
    free_ptr(large, s);
    free_ptr(stats, s);
    free_ptr(sorted, s);
    free_ptr(slotb, s);
    free_ptr(slowf, s);
    amgt_bsr_free(out, stream);
    return rc;
}

}  // namespace amgt

extern "C" {

int amgt_csr_to_bsr(const amgt_csr *A, amgt_bsr *out, amgt_stream_t stream)
{
    return amgt::csr_to_bsr_impl(A, out, stream, nullptr, nullptr);
}

int amgt_bsr_to_csr(const amgt_bsr *A, amgt_csr *out, amgt_stream_t stream)
{
    if (!A || !out || A->row < 0 || (A->blc_row > 0 && !A->blcPtr)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int m = A->row, brow = A->blc_row;
    memset(out, 0, sizeof(*out));
    out->num_rows = m;
    out->num_cols = A->col;
    int *cnt = nullptr;
    int64_t *tot = nullptr;
    const int64_t *h = nullptr;
    int rc = AMGT_OK;
    if ((rc = alloc_n(&out->i, m + 1, s)) || (rc = alloc_n(&cnt, m + 1, s)) || (rc = alloc_n(&tot, 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * (m + 1), s));
    AMGT_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(int64_t), s));
    if (brow > 0)
        AMGT_LAUNCH(bsr2csr_count_kernel, grid_for(8, brow, st->sm_count, 8), 256, 0, s, m, brow, A->blcPtr,
                    A->blcMap, cnt);
    if ((rc = exclusive_scan_int(cnt, out->i, m + 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemcpyAsync(tot, out->i + m, sizeof(int), cudaMemcpyDeviceToDevice, s));
    if ((rc = read_back(tot, 1, s, &h))) goto fail;
    out->num_nonzeros = (int)h[0];
    if ((rc = alloc_n(&out->j, out->num_nonzeros, s)) || (rc = alloc_n(&out->data, out->num_nonzeros, s))) goto fail;
    if (brow > 0)
        AMGT_LAUNCH(bsr2csr_fill_kernel, grid_for(8, brow, st->sm_count, 8), 256, 0, s, m, brow, A->blcPtr, A->blcIdx,
                    A->blcMap, A->blcVal, out->i, out->j, out->data);
    free_ptr(cnt, s);
    free_ptr(tot, s);
    return AMGT_OK;
fail:
    free_ptr(cnt, s);
    free_ptr(tot, s);
    amgt_csr_free(out, stream);
    return rc;
}

int amgt_bsr_balance(amgt_bsr *A, amgt_stream_t stream)
{
    if (!A || (A->blc_row > 0 && !A->blcPtr)) return AMGT_ERR_INVALID;
    if (A->rowPtrbyWarp) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int brow = A->blc_row;
    int *cnt = nullptr;
    int64_t *tot = nullptr;
    const int64_t *h = nullptr;
    int rc = AMGT_OK;
    if ((rc = alloc_n(&cnt, brow + 1, s)) || (rc = alloc_n(&A->rowPtrbyWarp, brow + 1, s)) ||
        (rc = alloc_n(&tot, 1, s)))
        goto fail;
    AMGT_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(int64_t), s));
    AMGT_LAUNCH(seg_count_kernel, grid_for(256, brow + 1, st->sm_count, 8), 256, 0, s, brow, A->blcPtr, cnt);
    if ((rc = exclusive_scan_int(cnt, A->rowPtrbyWarp, brow + 1, s))) goto fail;
    AMGT_CUDA_TRY(cudaMemcpyAsync(tot, A->rowPtrbyWarp + brow, sizeof(int), cudaMemcpyDeviceToDevice, s));
    if ((rc = read_back(tot, 1, s, &h))) goto fail;
    A->warpnum = (int)h[0];
    if ((rc = alloc_n(&A->rowIdxbyWarp, A->warpnum, s))) goto fail;
    if (brow > 0)
        AMGT_LAUNCH(seg_fill_kernel, grid_for(256, brow, st->sm_count, 8), 256, 0, s, brow, A->rowPtrbyWarp,
                    A->rowIdxbyWarp);
    free_ptr(cnt, s);
    free_ptr(tot, s);
    return AMGT_OK;
fail:
    free_ptr(cnt, s);
    free_ptr(tot, s);
    free_ptr(A->rowPtrbyWarp, s);
    free_ptr(A->rowIdxbyWarp, s);
    A->warpnum = 0;
    return rc;
}

int amgt_bsr_make_shadow(amgt_bsr *A, int prec, amgt_stream_t stream)
{
    if (!A || (A->blc_num > 0 && !A->blcVal)) return AMGT_ERR_INVALID;
    if (prec == AMGT_DOUBLE) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = 16LL * A->blc_num;
    const int grid = grid_for(256 * 4, n, st->sm_count, 8);
    switch (prec) {
    case AMGT_FLOAT:
        if (A->blcVal_fp32) return AMGT_OK;
        AMGT_TRY(alloc_n(&A->blcVal_fp32, (size_t)n, s));
        AMGT_LAUNCH(shadow_kernel<AMGT_FLOAT>, grid, 256, 0, s, n, A->blcVal, (void *)A->blcVal_fp32);
        return AMGT_OK;
    case AMGT_HALF:
        if (A->blcVal_fp16) return AMGT_OK;
        AMGT_TRY(alloc_n(&A->blcVal_fp16, (size_t)n, s));
        AMGT_LAUNCH(shadow_kernel<AMGT_HALF>, grid, 256, 0, s, n, A->blcVal, (void *)A->blcVal_fp16);
        return AMGT_OK;
    case AMGT_BF16:
        if (A->blcVal_bf16) return AMGT_OK;
        AMGT_TRY(alloc_n(&A->blcVal_bf16, (size_t)n, s));
        AMGT_LAUNCH(shadow_kernel<AMGT_BF16>, grid, 256, 0, s, n, A->blcVal, (void *)A->blcVal_bf16);
        return AMGT_OK;
    default:
        return AMGT_ERR_INVALID;
    }
}

int amgt_bsr_make_exact(amgt_bsr *A, amgt_stream_t stream)
{
    if (!A || (A->blc_num > 0 && !A->blcVal)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    int64_t *flag = nullptr;
    const int64_t *h = nullptr;
    int rc;
    if ((rc = alloc_n(&flag, 1, s))) return rc;
    bool own16 = false;
    if (!(rc = (cudaMemsetAsync(flag, 0, sizeof(int64_t), s) == cudaSuccess) ? AMGT_OK : AMGT_ERR_CUDA) &&
        !(rc = bsr_exact_check(A, flag, &own16, s, st->sm_count)) && !(rc = read_back(flag, 1, s, &h)))
        rc = bsr_exact_apply(A, h[0], own16, s);
    free_ptr(flag, s);
    return rc;
}

}  // extern "C"

namespace amgt {

int bsr_transpose_impl(const amgt_bsr *A, amgt_bsr *out, amgt_stream_t stream, bool with16, bool with32)
{
    if (!A || !out || (A->blc_row > 0 && !A->blcPtr)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = A->blc_num, brow = A->blc_row, bcol = A->blc_col;
    memset(out, 0, sizeof(*out));
    out->row = A->col;
    out->col = A->row;
    out->blc_row = bcol;
    out->blc_col = brow;
    out->blc_num = nb;
    out->nnz = (int)(16LL * nb > 0x7FFFFFFF ? 0x7FFFFFFF : 16LL * nb);  // saturates
    out->csr_nnz = A->csr_nnz;
    out->avg_nnz = A->avg_nnz;
    int *rowid = nullptr, *iota = nullptr, *keys_in = nullptr, *keys_out = nullptr, *src = nullptr, *hist = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int rc = AMGT_OK;
    int bits = 1;
    while ((1 << bits) <= bcol) ++bits;
    if ((rc = alloc_n(&out->blcPtr, bcol + 1, s)) || (rc = alloc_n(&out->blcIdx, nb, s)) ||
        (rc = alloc_n(&out->blcMap, nb, s)) || (rc = alloc_n(&out->blcVal, (size_t)16 * nb, s)) ||
        (rc = alloc_n(&rowid, nb, s)) || (rc = alloc_n(&iota, nb, s)) || (rc = alloc_n(&keys_out, nb, s)) ||
        (rc = alloc_n(&src, nb, s)) || (rc = alloc_n(&hist, bcol + 1, s)))
        goto fail;
    keys_in = A->blcIdx;
    AMGT_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * (bcol + 1), s));
    if (nb > 0) {
        AMGT_LAUNCH(row_of_block_kernel, grid_for(8, brow, st->sm_count, 8), 256, 0, s, brow, A->blcPtr, rowid, iota);
        AMGT_LAUNCH(col_hist_kernel, grid_for(256, nb, st->sm_count, 8), 256, 0, s, nb, A->blcIdx, hist);
        // stable radix sort by block column keeps block rows ascending inside each column
        AMGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys_in, keys_out, iota, src, nb, 0, bits, s));
        tmp = dev_alloc(tmp_bytes ? tmp_bytes : 16, s);
        if (!tmp) { rc = AMGT_ERR_ALLOC; goto fail; }
        count_launch();
        AMGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys_in, keys_out, iota, src, nb, 0, bits, s));
        const bool g16 = with16 && A->blcVal_fp16, g32 = with32 && A->blcVal_fp32;
        if (g16 && (rc = alloc_n(&out->blcVal_fp16, (size_t)16 * nb, s))) goto fail;
        if (g32 && (rc = alloc_n(&out->blcVal_fp32, (size_t)16 * nb, s))) goto fail;
        AMGT_LAUNCH(transpose_gather_kernel, grid_for(256, 16LL * nb, st->sm_count, 8), 256, 0, s, nb, src, rowid,
                    A->blcMap, A->blcVal, out->blcIdx, out->blcMap, out->blcVal,
                    g16 ? reinterpret_cast<const __half *>(A->blcVal_fp16) : nullptr,
                    g16 ? reinterpret_cast<__half *>(out->blcVal_fp16) : nullptr, g32 ? A->blcVal_fp32 : nullptr,
                    g32 ? out->blcVal_fp32 : nullptr);
    }
    if ((rc = exclusive_scan_int(hist, out->blcPtr, bcol + 1, s))) goto fail;
    free_ptr(rowid, s); free_ptr(iota, s); free_ptr(keys_out, s); free_ptr(src, s); free_ptr(hist, s);
    if (tmp) dev_free(tmp, s);
    return block_row_stats(out, s);
fail:
    free_ptr(rowid, s); free_ptr(iota, s); free_ptr(keys_out, s); free_ptr(src, s); free_ptr(hist, s);
    if (tmp) dev_free(tmp, s);
    amgt_bsr_free(out, stream);
    return rc;
}

}  // namespace amgt

extern "C" {

int amgt_bsr_transpose(const amgt_bsr *A, amgt_bsr *out, amgt_stream_t stream)
{
    return amgt::bsr_transpose_impl(A, out, stream, false, false);
}

}  // extern "C"
