/*
 * amgt_oracle.c - TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of AmgT's mBSR path (conversion, SpMV, SpGEMM, mBSR->CSR)
 * and of the HYPRE problem generators the reference's own tests use.  It is
 * the checker for the CUDA library: only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py load it.  The product never calls it.
 *
 * Parity pins (reference outputs this code is checked against, see
 * tests/golden/):
 *   - structural nnz of A*A for HYPRE's Laplacian generators, from the
 *     reference's SpGEMM regression outputs
 *     (AmgT_HYPRE/src/test/TEST_bench/benchmark_spgemm.saved.lassen:1-60);
 *   - the 7-point 10x10x10 operator HYPRE wrote with ij -printbin
 *     (AmgT_HYPRE/src/test/TEST_ij/data/poisson_10x10x10_np1/IJ.A.i4f8.*):
 *     rows, column order (diagonal first) and values.
 * References below use R = AmgT_HYPRE/src.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off: no fused
 * multiply-add, so the fp64 / fp32 sums are the exact IEEE sequences that
 * the CUDA kernels reproduce with __dmul_rn/__dadd_rn and friends).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EXPORT __attribute__((visibility("default")))

enum { ORC_DOUBLE = 0, ORC_FLOAT = 1, ORC_HALF = 2, ORC_BF16 = 3 };

ORC_EXPORT int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

ORC_EXPORT void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ RNG */
/* Counter-based stream: value k of stream `seed` is the splitmix64
 * finaliser (Steele, Lea & Flood, OOPSLA 2014) of seed * phi + k, so any
 * element can be generated independently (host or device). */
static inline uint64_t orc_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t orc_rand_u64(uint64_t seed, uint64_t k)
{
    return orc_mix64(seed * 0x9E3779B97F4A7C15ull + k + 1);
}

/* uniform in [-1, 1): 53 random bits */
static inline double orc_rand_sym(uint64_t seed, uint64_t k)
{
    return (double)(orc_rand_u64(seed, k) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

ORC_EXPORT void orc_rand_uniform(uint64_t seed, int64_t n, double *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) out[k] = orc_rand_sym(seed, (uint64_t)k);
}

/* standard normal by Box-Muller on two counter draws */
static inline double orc_rand_normal(uint64_t seed, uint64_t k)
{
    double u1 = ((double)(orc_rand_u64(seed, 2 * k) >> 11) + 1.0) / 9007199254740993.0;
    double u2 = (double)(orc_rand_u64(seed, 2 * k + 1) >> 11) / 9007199254740992.0;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* ----------------------------------------------------------- generators */
/* HYPRE's structured generators order unknowns x fastest
 * (row = x + nx*(y + ny*z)) and store the diagonal first, then the other
 * columns ascending (R/test/TEST_ij/data/poisson_10x10x10_np1/IJ.A.i4f8:
 * row 111 = [111, 11, 101, 110, 112, 121, 211]).  All generators below
 * write rows that way.  Capacity: caller passes arrays of n*stencil. */

/* GenerateLaplacian (R/parcsr_ls/par_laplace.c:15, values from
 * R/test/ij_mm.c:1492-1508): 7-point (5-point when nz == 1). */
ORC_EXPORT int64_t orc_gen_laplacian(int nx, int ny, int nz, double cx,
                                     double cy, double cz, int *ia, int *ja,
                                     double *a)
{
    double diag = 0.0;
    if (nx > 1) diag += 2.0 * cx;
    if (ny > 1) diag += 2.0 * cy;
    if (nz > 1) diag += 2.0 * cz;
    const int64_t n = (int64_t)nx * ny * nz;
    /* row lengths first (closed form per row) */
    ia[0] = 0;
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / ((int64_t)nx * ny));
        int len = 1 + (z > 0) + (y > 0) + (x > 0) + (x < nx - 1) + (y < ny - 1) + (z < nz - 1);
        ia[r + 1] = ia[r] + len;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / ((int64_t)nx * ny));
        int64_t p = ia[r];
        const int64_t sxy = (int64_t)nx * ny;
        ja[p] = (int)r; a[p++] = diag;
        if (z > 0) { ja[p] = (int)(r - sxy); a[p++] = -cz; }
        if (y > 0) { ja[p] = (int)(r - nx); a[p++] = -cy; }
        if (x > 0) { ja[p] = (int)(r - 1); a[p++] = -cx; }
        if (x < nx - 1) { ja[p] = (int)(r + 1); a[p++] = -cx; }
        if (y < ny - 1) { ja[p] = (int)(r + nx); a[p++] = -cy; }
        if (z < nz - 1) { ja[p] = (int)(r + sxy); a[p++] = -cz; }
    }
    return ia[n];
}

/* Full box stencil (3 x 3 x 3, or 3 x 3 when nz == 1): GenerateLaplacian27pt
 * (R/parcsr_ls/par_laplace_27pt.c:15; diagonal 26 in 3D, 8 in 2D, off -1,
 * R/test/ij_mm.c:2300-2362) and GenerateLaplacian9pt
 * (R/parcsr_ls/par_laplace_9pt.c:15). */
ORC_EXPORT int64_t orc_gen_box(int nx, int ny, int nz, int *ia, int *ja, double *a)
{
    const double diag = (nz > 1) ? 26.0 : ((ny > 1) ? 8.0 : 2.0);
    const int64_t n = (int64_t)nx * ny * nz, sxy = (int64_t)nx * ny;
    ia[0] = 0;
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int lx = 1 + (x > 0) + (x < nx - 1), ly = 1 + (y > 0) + (y < ny - 1),
            lz = 1 + (z > 0) + (z < nz - 1);
        ia[r + 1] = ia[r] + lx * ly * lz;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int64_t p = ia[r];
        ja[p] = (int)r; a[p++] = diag;
        for (int dz = -1; dz <= 1; ++dz) {
            if (z + dz < 0 || z + dz >= nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                if (y + dy < 0 || y + dy >= ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    if (x + dx < 0 || x + dx >= nx) continue;
                    if (!dx && !dy && !dz) continue;
                    ja[p] = (int)(r + dx + (int64_t)dy * nx + (int64_t)dz * sxy);
                    a[p++] = -1.0;
                }
            }
        }
    }
    return ia[n];
}

/* 27-point variable-coefficient diffusion (no reference counterpart; the
 * mixed-precision workload).  Node coefficient k = exp(sigma * N(0,1)) with
 * the exponent clipped to +-ln(ratio)/2, so max/min <= ratio.  Coupling of
 * neighbours i, j at offset d: -w(d) * 2 k_i k_j / (k_i + k_j) with
 * w = 1 (face), 1/2 (edge), 1/4 (corner).  Diagonal = sum over all 26
 * offsets of w * harmonic mean, an out-of-domain neighbour counting with
 * k_j = k_i (Dirichlet).  Symmetric, weakly diagonally dominant, strictly
 * on the boundary: SPD. */
ORC_EXPORT int64_t orc_gen_varcoef27(int nx, int ny, int nz, uint64_t seed,
                                     double sigma, double ratio, int *ia,
                                     int *ja, double *a)
{
    const int64_t n = (int64_t)nx * ny * nz, sxy = (int64_t)nx * ny;
    const double clip = 0.5 * log(ratio);
    double *k = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        double e = sigma * orc_rand_normal(seed, (uint64_t)r);
        if (e > clip) e = clip;
        if (e < -clip) e = -clip;
        k[r] = exp(e);
    }
    ia[0] = 0;
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int lx = 1 + (x > 0) + (x < nx - 1), ly = 1 + (y > 0) + (y < ny - 1),
            lz = 1 + (z > 0) + (z < nz - 1);
        ia[r + 1] = ia[r] + lx * ly * lz;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int64_t p = ia[r];
        int64_t pd = p++;
        double diag = 0.0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int m = (dx != 0) + (dy != 0) + (dz != 0);
                    if (!m) continue;
                    double w = (m == 1) ? 1.0 : ((m == 2) ? 0.5 : 0.25);
                    int inside = x + dx >= 0 && x + dx < nx && y + dy >= 0 &&
                                 y + dy < ny && z + dz >= 0 && z + dz < nz;
                    int64_t c = r + dx + (int64_t)dy * nx + (int64_t)dz * sxy;
                    double kj = inside ? k[c] : k[r];
                    double h = w * 2.0 * k[r] * kj / (k[r] + kj);
                    diag += h;
                    if (inside) { ja[p] = (int)c; a[p++] = -h; }
                }
        ja[pd] = (int)r;
        a[pd] = diag;
    }
    free(k);
    return ia[n];
}

/* 1-D linear interpolation weights of fine point i: up to 2 pairs */
static int orc_interp_1d(int i, int nfine, int ncoarse, int *idx, double *w)
{
    if (nfine == 1) { idx[0] = 0; w[0] = 1.0; return 1; }
    if ((i & 1) == 0) { idx[0] = i / 2; w[0] = 1.0; return 1; }
    idx[0] = (i - 1) / 2; w[0] = 0.5;
    if ((i + 1) / 2 < ncoarse) { idx[1] = (i + 1) / 2; w[1] = 0.5; return 2; }
    return 1;
}

/* Linear interpolation between vertex-centred grids, tensor product over
 * the dimensions with extent > 1: coarse point j sits on fine point 2j,
 * ncx = ceil(nx/2); fine odd points take 1/2 from each coarse neighbour that
 * exists.  P is (nx*ny*nz) x (ncx*ncy*ncz), rows sorted.  Returns nnz;
 * ia/ja/a need capacity n*8.  *nc_out = coarse size. */
ORC_EXPORT int64_t orc_gen_interp(int nx, int ny, int nz, int *ia, int *ja,
                                  double *a, int *ncx_out, int *ncy_out,
                                  int *ncz_out)
{
    const int ncx = (nx > 1) ? (nx + 1) / 2 : 1, ncy = (ny > 1) ? (ny + 1) / 2 : 1,
              ncz = (nz > 1) ? (nz + 1) / 2 : 1;
    *ncx_out = ncx; *ncy_out = ncy; *ncz_out = ncz;
    const int64_t n = (int64_t)nx * ny * nz, sxy = (int64_t)nx * ny;
    ia[0] = 0;
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int c[3], w0[2];
        double w1[2];
        c[0] = orc_interp_1d(x, nx, ncx, w0, w1);
        c[1] = orc_interp_1d(y, ny, ncy, w0, w1);
        c[2] = orc_interp_1d(z, nz, ncz, w0, w1);
        ia[r + 1] = ia[r] + c[0] * c[1] * c[2];
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        int x = (int)(r % nx), y = (int)((r / nx) % ny), z = (int)(r / sxy);
        int ix[2], iy[2], iz[2];
        double wx[2], wy[2], wz[2];
        int cxn = orc_interp_1d(x, nx, ncx, ix, wx);
        int cyn = orc_interp_1d(y, ny, ncy, iy, wy);
        int czn = orc_interp_1d(z, nz, ncz, iz, wz);
        int64_t p = ia[r];
        for (int c = 0; c < czn; ++c)
            for (int b = 0; b < cyn; ++b)
                for (int q = 0; q < cxn; ++q) {
                    ja[p] = ix[q] + ncx * (iy[b] + ncy * iz[c]);
                    a[p++] = wx[q] * wy[b] * wz[c];
                }
    }
    return ia[n];
}

/* ------------------------------------------------------ rounding (IEEE) */
/* Round a double to a binary format with `mant` stored mantissa bits and
 * `ebits` exponent bits, round-to-nearest-even, with subnormals and
 * overflow to infinity (IEEE 754-2008 section 4.3.1).  Used for the fp16
 * (mant 10, ebits 5) and bf16 (mant 7, ebits 8) value shadows. */
static uint16_t orc_round_small(double d, int mant, int ebits)
{
    uint64_t u;
    memcpy(&u, &d, 8);
    const uint16_t sign = (uint16_t)((u >> 63) << 15);
    const int exp = (int)((u >> 52) & 0x7FF);
    const uint64_t frac = u & 0xFFFFFFFFFFFFFull;
    const int bias = (1 << (ebits - 1)) - 1, emax_field = (1 << ebits) - 1;
    const uint16_t inf = (uint16_t)(emax_field << mant);
    if (exp == 0x7FF) return sign | inf | (frac ? (uint16_t)(1u << (mant - 1)) : 0);
    if (exp == 0) return sign; /* fp64 subnormal: far below either format */
    const int e = exp - 1023;
    if (e > bias) return sign | inf;
    const uint64_t sig = frac | (1ull << 52);
    const int emin = 1 - bias;
    int shift = 52 - mant + ((e < emin) ? (emin - e) : 0);
    if (shift >= 64) return sign;
    uint64_t q = sig >> shift;
    const uint64_t rem = sig & ((1ull << shift) - 1), halfway = 1ull << (shift - 1);
    if (rem > halfway || (rem == halfway && (q & 1))) ++q;
    if (e >= emin) {
        int fe = e + bias;
        if (q == (1ull << (mant + 1))) { q >>= 1; ++fe; }
        if (fe >= emax_field) return sign | inf;
        return sign | (uint16_t)(fe << mant) | (uint16_t)(q & ((1u << mant) - 1));
    }
    return sign | (uint16_t)q; /* subnormal; q == 2^mant becomes the min normal */
}

static double orc_small_to_double(uint16_t h, int mant, int ebits)
{
    const int bias = (1 << (ebits - 1)) - 1, emax_field = (1 << ebits) - 1;
    const int sign = h >> 15, fe = (h >> mant) & emax_field, fr = h & ((1 << mant) - 1);
    double v;
    if (fe == emax_field) v = fr ? NAN : INFINITY;
    else if (fe == 0) v = ldexp((double)fr, 1 - bias - mant);
    else v = ldexp((double)(fr | (1 << mant)), fe - bias - mant);
    return sign ? -v : v;
}

ORC_EXPORT uint16_t orc_to_half(double d) { return orc_round_small(d, 10, 5); }
ORC_EXPORT uint16_t orc_to_bf16(double d) { return orc_round_small(d, 7, 8); }
ORC_EXPORT double orc_half_to_double(uint16_t h) { return orc_small_to_double(h, 10, 5); }
ORC_EXPORT double orc_bf16_to_double(uint16_t h) { return orc_small_to_double(h, 7, 8); }

/* value of a stored block entry as the arithmetic of `prec` sees it */
static inline float orc_lowp(double v, int prec)
{
    switch (prec) {
    case ORC_HALF: return (float)orc_small_to_double(orc_round_small(v, 10, 5), 10, 5);
    case ORC_BF16: return (float)orc_small_to_double(orc_round_small(v, 7, 8), 7, 8);
    default: return (float)v;
    }
}

ORC_EXPORT void orc_make_shadow(int prec, int64_t n, const double *v, void *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (prec == ORC_FLOAT) ((float *)out)[i] = (float)v[i];
        else if (prec == ORC_HALF) ((uint16_t *)out)[i] = orc_round_small(v[i], 10, 5);
        else ((uint16_t *)out)[i] = orc_round_small(v[i], 7, 8);
    }
}

/* ---------------------------------------------------------- CSR -> mBSR */
/* Semantics of CSR2BSR_GPU (R/seq_mv/csr_matvec_device.c:1201-1267):
 * block row b covers CSR rows 4b..4b+3; an entry (r, c) lands in block
 * column c/4 at position (r%4)*4 + c%4 of the row-major 16-value block and
 * sets that bit of the block's bitmap (csr2bsr_getidx, :830-948); block
 * columns ascend (the rank sort at :917-927); missing values are zero
 * (cudaMemset at :1252).  stand = sqrt(sum (len - avg)^2 / brow) (getStand,
 * :638-671, and :1245-1249); avg_nnz = nnz / blocks (:1236). */
typedef struct { int key; uint16_t map; } orc_kv;

static int orc_kv_cmp(const void *a, const void *b)
{
    int x = ((const orc_kv *)a)->key, y = ((const orc_kv *)b)->key;
    return (x > y) - (x < y);
}

/* sort (key, map) pairs by key and merge equal keys with OR; returns count */
static int orc_unique_or(orc_kv *kv, int n)
{
    if (n <= 1) return n;
    /* insertion sort for short lists, qsort otherwise */
    if (n <= 32) {
        for (int i = 1; i < n; ++i) {
            orc_kv t = kv[i];
            int j = i - 1;
            while (j >= 0 && kv[j].key > t.key) { kv[j + 1] = kv[j]; --j; }
            kv[j + 1] = t;
        }
    } else {
        qsort(kv, (size_t)n, sizeof(orc_kv), orc_kv_cmp);
    }
    int m = 0;
    for (int i = 0; i < n; ++i) {
        if (m > 0 && kv[m - 1].key == kv[i].key) kv[m - 1].map |= kv[i].map;
        else kv[m++] = kv[i];
    }
    return m;
}

/* pass 1: blocks per block row into bptr[1..brow] (then scanned); returns
 * the block count and the longest block row */
ORC_EXPORT int64_t orc_csr2bsr_count(int m, int n, const int *ia, const int *ja,
                                     int *bptr, int *max_row)
{
    (void)n;
    const int brow = (m + 3) / 4;
    int mx = 0;
#pragma omp parallel reduction(max : mx)
    {
        int cap = 256;
        orc_kv *kv = (orc_kv *)malloc(sizeof(orc_kv) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int b = 0; b < brow; ++b) {
            int r0 = 4 * b, r1 = (4 * b + 4 < m) ? 4 * b + 4 : m;
            int len = ia[r1] - ia[r0];
            if (len > cap) { cap = 2 * len; kv = (orc_kv *)realloc(kv, sizeof(orc_kv) * (size_t)cap); }
            int t = 0;
            for (int r = r0; r < r1; ++r)
                for (int p = ia[r]; p < ia[r + 1]; ++p) {
                    kv[t].key = ja[p] >> 2;
                    kv[t].map = (uint16_t)(1u << ((r & 3) * 4 + (ja[p] & 3)));
                    ++t;
                }
            int u = orc_unique_or(kv, t);
            bptr[b + 1] = u;
            if (u > mx) mx = u;
        }
        free(kv);
    }
    bptr[0] = 0;
    for (int b = 0; b < brow; ++b) bptr[b + 1] += bptr[b];
    if (max_row) *max_row = mx;
    return bptr[brow];
}

/* pass 2: block columns, bitmaps, zero-padded values, stand, avg_nnz */
ORC_EXPORT void orc_csr2bsr_fill(int m, int n, const int *ia, const int *ja,
                                 const double *a, const int *bptr, int *bidx,
                                 uint16_t *bmap, double *bval, double *stand,
                                 double *avg_nnz)
{
    (void)n;
    const int brow = (m + 3) / 4;
#pragma omp parallel
    {
        int cap = 256;
        orc_kv *kv = (orc_kv *)malloc(sizeof(orc_kv) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int b = 0; b < brow; ++b) {
            int r0 = 4 * b, r1 = (4 * b + 4 < m) ? 4 * b + 4 : m;
            int len = ia[r1] - ia[r0];
            if (len > cap) { cap = 2 * len; kv = (orc_kv *)realloc(kv, sizeof(orc_kv) * (size_t)cap); }
            int t = 0;
            for (int r = r0; r < r1; ++r)
                for (int p = ia[r]; p < ia[r + 1]; ++p) {
                    kv[t].key = ja[p] >> 2;
                    kv[t].map = (uint16_t)(1u << ((r & 3) * 4 + (ja[p] & 3)));
                    ++t;
                }
            int u = orc_unique_or(kv, t);
            int base = bptr[b];
            for (int k = 0; k < u; ++k) {
                bidx[base + k] = kv[k].key;
                bmap[base + k] = kv[k].map;
            }
            if (bval) {
                memset(bval + (size_t)16 * base, 0, sizeof(double) * 16 * (size_t)u);
                for (int r = r0; r < r1; ++r)
                    for (int p = ia[r]; p < ia[r + 1]; ++p) {
                        int key = ja[p] >> 2, lo = base, hi = base + u - 1;
                        while (lo < hi) {
                            int mid = (lo + hi) >> 1;
                            if (bidx[mid] < key) lo = mid + 1; else hi = mid;
                        }
                        bval[(size_t)16 * lo + (r & 3) * 4 + (ja[p] & 3)] = a[p];
                    }
            }
        }
        free(kv);
    }
    const double nb = (double)bptr[brow];
    const double avg = brow ? nb / brow : 0.0;
    double s = 0.0;
    for (int b = 0; b < brow; ++b) {
        double d = (double)(bptr[b + 1] - bptr[b]) - avg;
        s += d * d;
    }
    if (stand) *stand = brow ? sqrt(s / brow) : 0.0;
    if (avg_nnz) *avg_nnz = nb > 0 ? (double)ia[m] / nb : 0.0;
}

/* ---------------------------------------------------------- mBSR -> CSR */
/* Semantics of bsr2csr_get_ptr / bsr2csr_get_idx_val
 * (R/seq_mv/csr_spgemm_device.c:1344-1440): CSR row 4b+r holds, for each
 * block of block row b in order, the set bits of nibble r of the bitmap as
 * columns 4*bcol + c (ascending), with the stored value. */
ORC_EXPORT int64_t orc_bsr2csr_count(int m, const int *bptr, const uint16_t *bmap, int *ia)
{
    const int brow = (m + 3) / 4;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < brow; ++b) {
        int cnt[4] = {0, 0, 0, 0};
        for (int k = bptr[b]; k < bptr[b + 1]; ++k)
            for (int r = 0; r < 4; ++r) cnt[r] += __builtin_popcount((bmap[k] >> (4 * r)) & 0xF);
        for (int r = 0; r < 4 && 4 * b + r < m; ++r) ia[4 * b + r + 1] = cnt[r];
    }
    ia[0] = 0;
    for (int r = 0; r < m; ++r) ia[r + 1] += ia[r];
    return ia[m];
}

ORC_EXPORT void orc_bsr2csr_fill(int m, const int *bptr, const int *bidx,
                                 const uint16_t *bmap, const double *bval,
                                 const int *ia, int *ja, double *a)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        int b = r >> 2, q = r & 3, p = ia[r];
        for (int k = bptr[b]; k < bptr[b + 1]; ++k) {
            unsigned nib = (bmap[k] >> (4 * q)) & 0xF;
            for (int c = 0; c < 4; ++c)
                if (nib & (1u << c)) {
                    ja[p] = 4 * bidx[k] + c;
                    if (a) a[p] = bval[(size_t)16 * k + 4 * q + c];
                    ++p;
                }
        }
    }
}

/* ----------------------------------------------------------------- SpMV */
/* y = alpha * A * x + beta * y on mBSR (spmv_amgT_fp64,
 * R/seq_mv/csr_matvec_device.c:1302-1411: y scaled by beta then
 * y += alpha * (A x), :1322-1326 and :487).  Per scalar row: blocks in
 * stored order, columns ascending, one running sum.  Reduced precisions:
 * values rounded to the format, x rounded to fp32, fp32 products and sum,
 * then combined in fp64.  The kernels sum in a different (fixed) order, so
 * tests compare with an error bound, not bit for bit.  Columns past
 * n (last block column when n % 4 != 0) hold zero values and are skipped
 * (the reference reads x out of bounds there, :474-475). */
ORC_EXPORT void orc_bsr_spmv(int prec, int m, int n, const int *bptr,
                             const int *bidx, const double *bval, double alpha,
                             const double *x, double beta, double *y)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        const int b = r >> 2, q = r & 3;
        double t = 0.0;
        float tf = 0.0f;
        for (int k = bptr[b]; k < bptr[b + 1]; ++k) {
            const double *v = bval + (size_t)16 * k + 4 * q;
            for (int c = 0; c < 4; ++c) {
                int col = 4 * bidx[k] + c;
                if (col >= n) continue;
                if (prec == ORC_DOUBLE) t += v[c] * x[col];
                else tf += orc_lowp(v[c], prec) * (float)x[col];
            }
        }
        if (prec != ORC_DOUBLE) t = (double)tf;
        y[r] = (beta == 0.0) ? alpha * t : alpha * t + beta * y[r];
    }
}

/* Row-wise error bound companion: s[r] = |alpha| * sum |a_rc| |x_c| +
 * |beta| |y_r| (used to scale the SpMV tolerance). */
ORC_EXPORT void orc_bsr_spmv_absbound(int m, int n, const int *bptr, const int *bidx,
                                      const double *bval, double alpha,
                                      const double *x, double beta,
                                      const double *y, double *s)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        const int b = r >> 2, q = r & 3;
        double t = 0.0;
        for (int k = bptr[b]; k < bptr[b + 1]; ++k)
            for (int c = 0; c < 4; ++c) {
                int col = 4 * bidx[k] + c;
                if (col < n) t += fabs(bval[(size_t)16 * k + 4 * q + c] * x[col]);
            }
        s[r] = fabs(alpha) * t + fabs(beta) * fabs(y[r]);
    }
}

/* --------------------------------------------------------------- SpGEMM */
/* bitMatrixMul (R/seq_mv/csr_spgemm_device.c:189-205) with
 * Bitmap_col_x_row (R/seq_mv/seq_mv.h:149): OR over k of the outer product
 * of column k of a and row k of b; bit r*4+c = entry (r, c). */
static inline uint16_t orc_bitmul(uint16_t a, uint16_t b)
{
    unsigned res = 0;
    for (int k = 0; k < 4; ++k) {
        unsigned colk = (a >> k) & 0x1111u; /* bits r*4 */
        unsigned rowk = (b >> (4 * k)) & 0xFu;
        res |= (colk * 0xFu) & (rowk * 0x1111u);
    }
    return (uint16_t)res;
}

ORC_EXPORT uint16_t orc_bitmatmul(uint16_t a, uint16_t b) { return orc_bitmul(a, b); }

/* Symbolic (symbolic_spgemm_step1/2, :206-752): C block (I, J) exists iff
 * some A block (I, K) and B block (K, J) have a non-zero bitmap product;
 * C's bitmap is the OR of those products (numeric_spgemm_hybrid
 * `mapC |=`, :1219, :1322).  Block columns ascend.  Pass 1 counts C blocks
 * per block row into cptr (scanned) and returns the total; csr_nnz (if not
 * NULL) receives the number of set bits (CSR nonzeros of C). */
ORC_EXPORT int64_t orc_spgemm_count(int brA, const int *aptr, const int *aidx,
                                    const uint16_t *amap, int bcB, const int *bptr,
                                    const int *bidx, const uint16_t *bmap, int *cptr,
                                    int64_t *csr_nnz)
{
    int64_t total = 0, bits = 0;
#pragma omp parallel reduction(+ : total, bits)
    {
        int *mark = (int *)malloc(sizeof(int) * (size_t)(bcB > 0 ? bcB : 1));
        uint16_t *acc = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(bcB > 0 ? bcB : 1));
        int *list = (int *)malloc(sizeof(int) * (size_t)(bcB > 0 ? bcB : 1));
        for (int j = 0; j < bcB; ++j) mark[j] = -1;
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < brA; ++i) {
            int cnt = 0;
            for (int p = aptr[i]; p < aptr[i + 1]; ++p) {
                int k = aidx[p];
                for (int q = bptr[k]; q < bptr[k + 1]; ++q) {
                    uint16_t mc = orc_bitmul(amap[p], bmap[q]);
                    if (!mc) continue;
                    int j = bidx[q];
                    if (mark[j] != i) { mark[j] = i; acc[j] = 0; list[cnt++] = j; }
                    acc[j] |= mc;
                }
            }
            for (int t = 0; t < cnt; ++t) { bits += __builtin_popcount(acc[list[t]]); }
            if (cptr) cptr[i + 1] = cnt;
            total += cnt;
        }
        free(mark); free(acc); free(list);
    }
    if (cptr) {
        cptr[0] = 0;
        for (int i = 0; i < brA; ++i) cptr[i + 1] += cptr[i];
    }
    if (csr_nnz) *csr_nnz = bits;
    return total;
}

static int orc_int_cmp(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Pass 2 + numeric (numeric_spgemm_hybrid, :1142-1342, scalar branch
 * :1289-1339): for each A block of the row in stored order, for each B
 * block of B's row K in stored order with a non-zero bitmap product, the
 * 4x4 product entry (r, c) = sum over k ascending of a[r][k] * b[k][c],
 * taking only terms whose A bit and B bit are set, started from zero; it is
 * added to C(r, c) only where the product bitmap has the bit.  DOUBLE in
 * fp64; FLOAT / HALF / BF16 with values rounded to the format and fp32
 * products, sums and C accumulators, C values returned as fp64 (exact) and
 * as the format's shadow (cshadow, may be NULL).
 *
 * contract (DOUBLE only): each product entry is the fused multiply-add
 * chain t = fma(a[r][k], b[k][c], t) over k ascending, started from zero.
 * That is the reference's own fp64 arithmetic: its scalar branch writes
 * `temp_valC[ii*4+kk] += a * b` (:1317), which nvcc contracts into an FMA
 * (its build passes no --fmad=false), and its tensor-core branch for A
 * blocks of >= 10 stored entries (:1173-1262, mma.m8n8k4.f64) takes every
 * k term, stored or not; a term whose A or B value is an unstored zero
 * leaves an FMA chain unchanged for finite values, so both branches give
 * this chain as long as the m8n8k4 product rounds like a k-ordered chain
 * (the PTX description of the f64 mma fixes no order; the tests that use
 * this variant against the tensor-core branch's blocks allow 1e-12
 * relative).  contract = 0: separate multiply and add (the arithmetic the
 * fp32 form keeps). */
static void orc_spgemm_fill_impl(int prec, int contract, int brA, const int *aptr, const int *aidx,
                                 const uint16_t *amap, const double *aval, int bcB,
                                 const int *bptr, const int *bidx, const uint16_t *bmap,
                                 const double *bval, const int *cptr, int *cidx,
                                 uint16_t *cmap, double *cval, void *cshadow)
{
#pragma omp parallel
    {
        int *pos = (int *)malloc(sizeof(int) * (size_t)(bcB > 0 ? bcB : 1));
        int *mark = (int *)malloc(sizeof(int) * (size_t)(bcB > 0 ? bcB : 1));
        for (int j = 0; j < bcB; ++j) mark[j] = -1;
        int cap = 1024;
        double *accd = (double *)malloc(sizeof(double) * 16 * (size_t)cap);
        float *accf = (float *)malloc(sizeof(float) * 16 * (size_t)cap);
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < brA; ++i) {
            const int base = cptr[i], len = cptr[i + 1] - cptr[i];
            /* pattern */
            int cnt = 0;
            for (int p = aptr[i]; p < aptr[i + 1]; ++p) {
                int k = aidx[p];
                for (int q = bptr[k]; q < bptr[k + 1]; ++q) {
                    uint16_t mc = orc_bitmul(amap[p], bmap[q]);
                    if (!mc) continue;
                    int j = bidx[q];
                    if (mark[j] != i) { mark[j] = i; cidx[base + cnt++] = j; }
                }
            }
            (void)len;
            qsort(cidx + base, (size_t)cnt, sizeof(int), orc_int_cmp);
            for (int t = 0; t < cnt; ++t) { pos[cidx[base + t]] = t; cmap[base + t] = 0; }
            if (cnt > cap) {
                cap = 2 * cnt;
                accd = (double *)realloc(accd, sizeof(double) * 16 * (size_t)cap);
                accf = (float *)realloc(accf, sizeof(float) * 16 * (size_t)cap);
            }
            memset(accd, 0, sizeof(double) * 16 * (size_t)cnt);
            memset(accf, 0, sizeof(float) * 16 * (size_t)cnt);
            /* numeric */
            for (int p = aptr[i]; p < aptr[i + 1]; ++p) {
                const int k = aidx[p];
                const uint16_t ma = amap[p];
                const double *av = aval + (size_t)16 * p;
                float af[16];
                if (prec != ORC_DOUBLE)
                    for (int e = 0; e < 16; ++e) af[e] = orc_lowp(av[e], prec);
                for (int q = bptr[k]; q < bptr[k + 1]; ++q) {
                    const uint16_t mb = bmap[q];
                    const uint16_t mc = orc_bitmul(ma, mb);
                    if (!mc) continue;
                    const int t = pos[bidx[q]];
                    cmap[base + t] |= mc;
                    const double *bv = bval + (size_t)16 * q;
                    if (prec == ORC_DOUBLE) {
                        for (int r = 0; r < 4; ++r)
                            for (int c = 0; c < 4; ++c) {
                                if (!(mc & (1u << (4 * r + c)))) continue;
                                double s = 0.0;
                                for (int kk = 0; kk < 4; ++kk)
                                    if ((ma & (1u << (4 * r + kk))) && (mb & (1u << (4 * kk + c)))) {
                                        if (contract) s = fma(av[4 * r + kk], bv[4 * kk + c], s);
                                        else s = s + av[4 * r + kk] * bv[4 * kk + c];
                                    }
                                accd[16 * t + 4 * r + c] += s;
                            }
                    } else {
                        float bf[16];
                        for (int e = 0; e < 16; ++e) bf[e] = orc_lowp(bv[e], prec);
                        for (int r = 0; r < 4; ++r)
                            for (int c = 0; c < 4; ++c) {
                                if (!(mc & (1u << (4 * r + c)))) continue;
                                float s = 0.0f;
                                for (int kk = 0; kk < 4; ++kk)
                                    if ((ma & (1u << (4 * r + kk))) && (mb & (1u << (4 * kk + c))))
                                        s = s + af[4 * r + kk] * bf[4 * kk + c];
                                accf[16 * t + 4 * r + c] += s;
                            }
                    }
                }
            }
            for (int t = 0; t < cnt; ++t)
                for (int e = 0; e < 16; ++e) {
                    size_t o = (size_t)16 * (base + t) + e;
                    if (prec == ORC_DOUBLE) {
                        cval[o] = accd[16 * t + e];
                    } else {
                        float f = accf[16 * t + e];
                        cval[o] = (double)f;
                        if (cshadow) {
                            if (prec == ORC_FLOAT) ((float *)cshadow)[o] = f;
                            else if (prec == ORC_HALF) ((uint16_t *)cshadow)[o] = orc_round_small((double)f, 10, 5);
                            else ((uint16_t *)cshadow)[o] = orc_round_small((double)f, 7, 8);
                        }
                    }
                }
        }
        free(pos); free(mark); free(accd); free(accf);
    }
}

ORC_EXPORT void orc_spgemm_fill(int prec, int brA, const int *aptr, const int *aidx,
                                const uint16_t *amap, const double *aval, int bcB,
                                const int *bptr, const int *bidx, const uint16_t *bmap,
                                const double *bval, const int *cptr, int *cidx,
                                uint16_t *cmap, double *cval, void *cshadow)
{
    orc_spgemm_fill_impl(prec, 0, brA, aptr, aidx, amap, aval, bcB, bptr, bidx, bmap, bval, cptr, cidx, cmap, cval,
                         cshadow);
}

/* The same with the reference's fp64 contraction (contract = 1 above). */
ORC_EXPORT void orc_spgemm_fill_fma(int prec, int brA, const int *aptr, const int *aidx,
                                    const uint16_t *amap, const double *aval, int bcB,
                                    const int *bptr, const int *bidx, const uint16_t *bmap,
                                    const double *bval, const int *cptr, int *cidx,
                                    uint16_t *cmap, double *cval, void *cshadow)
{
    orc_spgemm_fill_impl(prec, 1, brA, aptr, aidx, amap, aval, bcB, bptr, bidx, bmap, bval, cptr, cidx, cmap, cval,
                         cshadow);
}

/* ------------------------------------------------------------ transpose */
/* A^T in mBSR: block (I, J) becomes (J, I) with values and bitmap
 * transposed inside the block; block columns ascend.  out arrays sized
 * like A's; tptr has bcA + 1 entries. */
ORC_EXPORT void orc_bsr_transpose(int brA, int bcA, const int *aptr, const int *aidx,
                                  const uint16_t *amap, const double *aval, int *tptr,
                                  int *tidx, uint16_t *tmap, double *tval)
{
    memset(tptr, 0, sizeof(int) * (size_t)(bcA + 1));
    for (int i = 0; i < brA; ++i)
        for (int p = aptr[i]; p < aptr[i + 1]; ++p) tptr[aidx[p] + 1]++;
    for (int j = 0; j < bcA; ++j) tptr[j + 1] += tptr[j];
    int *fill = (int *)malloc(sizeof(int) * (size_t)(bcA > 0 ? bcA : 1));
    memcpy(fill, tptr, sizeof(int) * (size_t)bcA);
    for (int i = 0; i < brA; ++i) /* rows in order: block columns of A^T ascend */
        for (int p = aptr[i]; p < aptr[i + 1]; ++p) {
            int j = aidx[p], d = fill[j]++;
            tidx[d] = i;
            unsigned m = amap[p], t = 0;
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c)
                    if (m & (1u << (4 * r + c))) t |= 1u << (4 * c + r);
            tmap[d] = (uint16_t)t;
            if (aval && tval)
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c)
                        tval[(size_t)16 * d + 4 * c + r] = aval[(size_t)16 * p + 4 * r + c];
        }
    free(fill);
}

/* ------------------------------------------------------------------ AMG */
/* CPU restatement of the setup + solve that drives the two hooks
 * (BoomerAMG-PCG with a V(1,1) l1-Jacobi cycle): Galerkin products
 * A_{l+1} = P_l^T (A_l P_l) on mBSR (hypre_ParCSRMatrixRAPKT,
 * R/parcsr_mv/par_csr_triplemat_device.c:630-905), l1 norms (option 1,
 * R/parcsr_ls/ams.c:627-636), the cycle of R/parcsr_ls/par_cycle.c:678-751
 * with relax 18 (R/parcsr_ls/par_relax.c:1178-1260), a dense inverse on the
 * coarsest level, and PCG with ||r||/||b|| stopping (R/krylov/pcg.c).  All
 * fp64.  Interpolation operators are inputs. */
typedef struct {
    int n;
    int *bptr, *bidx;
    uint16_t *bmap;
    double *bval;
    int nblk;
    /* transfer to the next level */
    int pn;                               /* coarse size */
    int *pptr, *pidx, *rptr, *ridx;
    uint16_t *pmap, *rmap;
    double *pval, *rval;
    double *inv_l1, *f, *u, *t, *s;
} orc_level;

typedef struct {
    int L;
    orc_level *lv;
    double *cinv; /* dense inverse of the coarsest operator */
    double w;
    double *r, *z, *p, *q;
} orc_amg;

static void orc_csr_to_level(int m, int n, const int *ia, const int *ja, const double *a, int **bptr, int **bidx,
                             uint16_t **bmap, double **bval, int *nblk)
{
    const int brow = (m + 3) / 4;
    *bptr = (int *)calloc((size_t)brow + 1, sizeof(int));
    int mx;
    int64_t nb = orc_csr2bsr_count(m, n, ia, ja, *bptr, &mx);
    *bidx = (int *)malloc(sizeof(int) * (size_t)(nb ? nb : 1));
    *bmap = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(nb ? nb : 1));
    *bval = (double *)malloc(sizeof(double) * 16 * (size_t)(nb ? nb : 1));
    double st, av;
    orc_csr2bsr_fill(m, n, ia, ja, a, *bptr, *bidx, *bmap, *bval, &st, &av);
    *nblk = (int)nb;
}

/* dense inverse (Cholesky, then Gauss-Jordan fallback) */
static int orc_invert(int n, double *A)
{
    double *L = (double *)malloc(sizeof(double) * (size_t)n * n);
    memcpy(L, A, sizeof(double) * (size_t)n * n);
    int spd = 1;
    for (int j = 0; j < n && spd; ++j) {
        double d = L[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(d > 0.0)) { spd = 0; break; }
        d = sqrt(d);
        L[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = L[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = s / d;
        }
    }
    if (spd) {
        double *Li = (double *)calloc((size_t)n * n, sizeof(double));
        for (int j = 0; j < n; ++j) {
            Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
            for (int i = j + 1; i < n; ++i) {
                double s = 0.0;
                for (int k = j; k < i; ++k) s -= L[(size_t)i * n + k] * Li[(size_t)k * n + j];
                Li[(size_t)i * n + j] = s / L[(size_t)i * n + i];
            }
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int k = (i > j ? i : j); k < n; ++k) s += Li[(size_t)k * n + i] * Li[(size_t)k * n + j];
                A[(size_t)i * n + j] = s;
            }
        free(Li);
        free(L);
        return 0;
    }
    free(L);
    return -1;
}

ORC_EXPORT void *orc_amg_setup(int n, const int *ia, const int *ja, const double *a, int nP, const int *pm,
                               const int *pn, const int *const *pia, const int *const *pja,
                               const double *const *pa, double w)
{
    orc_amg *h = (orc_amg *)calloc(1, sizeof(orc_amg));
    h->L = nP + 1;
    h->w = w;
    h->lv = (orc_level *)calloc((size_t)h->L, sizeof(orc_level));
    orc_level *lv = h->lv;
    lv[0].n = n;
    orc_csr_to_level(n, n, ia, ja, a, &lv[0].bptr, &lv[0].bidx, &lv[0].bmap, &lv[0].bval, &lv[0].nblk);
    for (int l = 0; l < h->L - 1; ++l) {
        orc_level *v = &lv[l], *c = &lv[l + 1];
        (void)pm;
        v->pn = pn[l];
        int pnb;
        orc_csr_to_level(v->n, pn[l], pia[l], pja[l], pa[l], &v->pptr, &v->pidx, &v->pmap, &v->pval, &pnb);
        const int pbc = (pn[l] + 3) / 4, pbr = (v->n + 3) / 4;
        v->rptr = (int *)calloc((size_t)pbc + 1, sizeof(int));
        v->ridx = (int *)malloc(sizeof(int) * (size_t)(pnb ? pnb : 1));
        v->rmap = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(pnb ? pnb : 1));
        v->rval = (double *)malloc(sizeof(double) * 16 * (size_t)(pnb ? pnb : 1));
        orc_bsr_transpose(pbr, pbc, v->pptr, v->pidx, v->pmap, v->pval, v->rptr, v->ridx, v->rmap, v->rval);
        /* AP = A P */
        const int abr = (v->n + 3) / 4;
        int *apptr = (int *)calloc((size_t)abr + 1, sizeof(int));
        int64_t bits;
        int64_t apn = orc_spgemm_count(abr, v->bptr, v->bidx, v->bmap, pbc, v->pptr, v->pidx, v->pmap, apptr, &bits);
        int *apidx = (int *)malloc(sizeof(int) * (size_t)(apn ? apn : 1));
        uint16_t *apmap = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(apn ? apn : 1));
        double *apval = (double *)malloc(sizeof(double) * 16 * (size_t)(apn ? apn : 1));
        orc_spgemm_fill_fma(ORC_DOUBLE, abr, v->bptr, v->bidx, v->bmap, v->bval, pbc, v->pptr, v->pidx, v->pmap, v->pval,
                        apptr, apidx, apmap, apval, NULL);
        /* RAP = R AP */
        c->n = pn[l];
        c->bptr = (int *)calloc((size_t)pbc + 1, sizeof(int));
        int64_t cn = orc_spgemm_count(pbc, v->rptr, v->ridx, v->rmap, pbc, apptr, apidx, apmap, c->bptr, &bits);
        c->nblk = (int)cn;
        c->bidx = (int *)malloc(sizeof(int) * (size_t)(cn ? cn : 1));
        c->bmap = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(cn ? cn : 1));
        c->bval = (double *)malloc(sizeof(double) * 16 * (size_t)(cn ? cn : 1));
        orc_spgemm_fill_fma(ORC_DOUBLE, pbc, v->rptr, v->ridx, v->rmap, v->rval, pbc, apptr, apidx, apmap, apval, c->bptr,
                        c->bidx, c->bmap, c->bval, NULL);
        free(apptr); free(apidx); free(apmap); free(apval);
    }
    for (int l = 0; l < h->L; ++l) {
        orc_level *v = &lv[l];
        v->inv_l1 = (double *)malloc(sizeof(double) * (size_t)v->n);
        for (int r = 0; r < v->n; ++r) {
            const int b = r >> 2, q = r & 3;
            double s = 0.0;
            for (int k = v->bptr[b]; k < v->bptr[b + 1]; ++k)
                for (int c = 0; c < 4; ++c) s += fabs(v->bval[(size_t)16 * k + 4 * q + c]);
            v->inv_l1[r] = s != 0.0 ? 1.0 / s : 0.0;
        }
        v->f = (double *)calloc((size_t)v->n, sizeof(double));
        v->u = (double *)calloc((size_t)v->n, sizeof(double));
        v->t = (double *)calloc((size_t)v->n, sizeof(double));
        v->s = (double *)calloc((size_t)v->n, sizeof(double));
    }
    orc_level *c = &lv[h->L - 1];
    h->cinv = (double *)calloc((size_t)c->n * c->n, sizeof(double));
    for (int r = 0; r < c->n; ++r) {
        const int b = r >> 2, q = r & 3;
        for (int k = c->bptr[b]; k < c->bptr[b + 1]; ++k)
            for (int cc = 0; cc < 4; ++cc) {
                const int col = 4 * c->bidx[k] + cc;
                if (col < c->n) h->cinv[(size_t)r * c->n + col] = c->bval[(size_t)16 * k + 4 * q + cc];
            }
    }
    orc_invert(c->n, h->cinv);
    h->r = (double *)calloc((size_t)n, sizeof(double));
    h->z = (double *)calloc((size_t)n, sizeof(double));
    h->p = (double *)calloc((size_t)n, sizeof(double));
    h->q = (double *)calloc((size_t)n, sizeof(double));
    return h;
}

ORC_EXPORT int orc_amg_num_levels(void *hv) { return ((orc_amg *)hv)->L; }

ORC_EXPORT int orc_amg_level_size(void *hv, int l, int *nblk)
{
    orc_amg *h = (orc_amg *)hv;
    if (nblk) *nblk = h->lv[l].nblk;
    return h->lv[l].n;
}

/* out = f - A u (resid) or u + w (f - A u) ./ l1 (jacobi) */
static void orc_level_apply(const orc_level *v, const double *f, const double *u, double *out, int jacobi, double w)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < v->n; ++r) {
        const int b = r >> 2, q = r & 3;
        double t = 0.0;
        for (int k = v->bptr[b]; k < v->bptr[b + 1]; ++k) {
            const double *val = v->bval + (size_t)16 * k + 4 * q;
            for (int c = 0; c < 4; ++c) {
                const int col = 4 * v->bidx[k] + c;
                if (col < v->n) t += val[c] * u[col];
            }
        }
        out[r] = jacobi ? u[r] + w * (f[r] - t) * v->inv_l1[r] : f[r] - t;
    }
}

static void orc_cycle(orc_amg *h, const double *rhs, double *out)
{
    orc_level *lv = h->lv;
    const int L = h->L;
    for (int l = 0; l < L - 1; ++l) {
        orc_level *v = &lv[l];
        const double *f = l == 0 ? rhs : v->f;
        for (int r = 0; r < v->n; ++r) v->u[r] = h->w * f[r] * v->inv_l1[r];
        orc_level_apply(v, f, v->u, v->t, 0, h->w);
        orc_bsr_spmv(ORC_DOUBLE, v->pn, v->n, v->rptr, v->ridx, v->rval, 1.0, v->t, 0.0, lv[l + 1].f);
    }
    orc_level *c = &lv[L - 1];
    const double *fc = L == 1 ? rhs : c->f;
    double *uc = L == 1 ? out : c->s;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < c->n; ++r) {
        double s = 0.0;
        for (int j = 0; j < c->n; ++j) s += h->cinv[(size_t)r * c->n + j] * fc[j];
        uc[r] = s;
    }
    for (int l = L - 2; l >= 0; --l) {
        orc_level *v = &lv[l];
        const double *f = l == 0 ? rhs : v->f;
        double *o = l == 0 ? out : v->s;
        orc_bsr_spmv(ORC_DOUBLE, v->n, v->pn, v->pptr, v->pidx, v->pval, 1.0, lv[l + 1].s, 1.0, v->u);
        orc_level_apply(v, f, v->u, o, 1, h->w);
    }
}

static double orc_dot(int n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* PCG; hist receives ||r||/||b|| per iteration (entry 0 = initial), cap
 * maxit + 1 entries.  Returns the iteration count. */
ORC_EXPORT int orc_amg_solve(void *hv, const double *b, double *x, double tol, int maxit, double *hist,
                             double *relres)
{
    orc_amg *h = (orc_amg *)hv;
    orc_level *v0 = &h->lv[0];
    const int n = v0->n;
    orc_level_apply(v0, b, x, h->r, 0, 0.0);
    const double bb = orc_dot(n, b, b);
    double rr = orc_dot(n, h->r, h->r);
    double rel = bb > 0 ? sqrt(rr / bb) : 0.0;
    if (hist) hist[0] = rel;
    int it = 0;
    if (rel > tol) {
        orc_cycle(h, h->r, h->z);
        double rz = orc_dot(n, h->r, h->z);
        memcpy(h->p, h->z, sizeof(double) * (size_t)n);
        for (it = 1; it <= maxit; ++it) {
            /* q = A p */
#pragma omp parallel for schedule(static)
            for (int r = 0; r < n; ++r) {
                const int bb4 = r >> 2, q = r & 3;
                double t = 0.0;
                for (int k = v0->bptr[bb4]; k < v0->bptr[bb4 + 1]; ++k)
                    for (int c = 0; c < 4; ++c) {
                        const int col = 4 * v0->bidx[k] + c;
                        if (col < n) t += v0->bval[(size_t)16 * k + 4 * q + c] * h->p[col];
                    }
                h->q[r] = t;
            }
            const double pq = orc_dot(n, h->p, h->q);
            const double alpha = pq != 0.0 ? rz / pq : 0.0;
            for (int i = 0; i < n; ++i) {
                x[i] += alpha * h->p[i];
                h->r[i] -= alpha * h->q[i];
            }
            rr = orc_dot(n, h->r, h->r);
            rel = sqrt(rr / bb);
            if (hist) hist[it] = rel;
            if (rel <= tol) break;
            orc_cycle(h, h->r, h->z);
            const double rz_new = orc_dot(n, h->r, h->z);
            const double beta = rz != 0.0 ? rz_new / rz : 0.0;
            rz = rz_new;
            for (int i = 0; i < n; ++i) h->p[i] = h->z[i] + beta * h->p[i];
        }
        if (it > maxit) it = maxit;
    }
    if (relres) *relres = rel;
    return it;
}

ORC_EXPORT void orc_amg_free(void *hv)
{
    orc_amg *h = (orc_amg *)hv;
    if (!h) return;
    for (int l = 0; l < h->L; ++l) {
        orc_level *v = &h->lv[l];
        free(v->bptr); free(v->bidx); free(v->bmap); free(v->bval);
        free(v->pptr); free(v->pidx); free(v->pmap); free(v->pval);
        free(v->rptr); free(v->ridx); free(v->rmap); free(v->rval);
        free(v->inv_l1); free(v->f); free(v->u); free(v->t); free(v->s);
    }
    free(h->lv); free(h->cinv); free(h->r); free(h->z); free(h->p); free(h->q);
    free(h);
}
