// The learned precision / strength-threshold policy: per-level features of
// an mBSR operator, structured (semi)coarsening interpolation, and a small
// MLP (16 -> 64 -> 64 -> 4, fp32, ReLU) with forward, backward and Adam
// kernels written here.  No reference counterpart: AmgT fixes the level ->
// precision table (get_calculationPrecison, AmgT_HYPRE/src/seq_mv/
// csr_spgemm_device.c:1847-1862) and BoomerAMG takes theta as a parameter
// (HYPRE_BoomerAMGSetStrongThreshold).
//
// MLP parameters, one fp32 array: W1 [64 x 16], b1 [64], W2 [64 x 64],
// b2 [64], W3 [4 x 64], b3 [4] (row-major, out x in).  Output 0 is theta's
// logit (theta = sigmoid), outputs 1 .. 3 the logits of the level's
// precision (fp64, fp32, fp16).  Loss per sample: (sigmoid(o0) - theta*)^2
// + cross-entropy(softmax(o1..3), class*).  One warp per sample; hidden
// unit j lives in lane j % 32 (units j and j + 32).  Gradients are written
// per sample and summed over the batch in a fixed order (deterministic).
#include <cmath>
#include <vector>

#include "amgt_internal.cuh"

namespace amgt {

constexpr int kIn = AMGT_MLP_IN, kHid = AMGT_MLP_HIDDEN, kOut = AMGT_MLP_OUT;
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kOut * kHid, kNParam = oB3 + kOut;
static_assert(kNParam == AMGT_MLP_NPARAM, "parameter layout");
static_assert(kHid == 64 && kIn <= 32 && kOut == 4, "warp layout: two hidden units per lane");

// forward of one sample in one warp; h1, h2: this lane's units (j, j + 32)
__device__ __forceinline__ void mlp_fwd_warp(const float *__restrict__ P, const float *__restrict__ x, int lane,
                                             float h1[2], float h2[2], float o[4])
{
    const float xi = lane < kIn ? x[lane] : 0.0f;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int j = lane + 32 * u;
        float z = P[oB1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i) z = fmaf(P[oW1 + j * kIn + i], __shfl_sync(FULL, xi, i), z);
        h1[u] = fmaxf(z, 0.0f);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int j = lane + 32 * u;
        float z = P[oB2 + j];
#pragma unroll 8
        for (int i = 0; i < 32; ++i) z = fmaf(P[oW2 + j * kHid + i], __shfl_sync(FULL, h1[0], i), z);
#pragma unroll 8
        for (int i = 0; i < 32; ++i) z = fmaf(P[oW2 + j * kHid + 32 + i], __shfl_sync(FULL, h1[1], i), z);
        h2[u] = fmaxf(z, 0.0f);
    }
#pragma unroll
    for (int k = 0; k < kOut; ++k) {
        float s = P[oW3 + k * kHid + lane] * h2[0] + P[oW3 + k * kHid + lane + 32] * h2[1];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
        o[k] = s + P[oB3 + k];
    }
}

__global__ void mlp_forward_kernel(const float *__restrict__ P, int n, const float *__restrict__ X,
                                   float *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    for (int smp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; smp < n; smp += (gridDim.x * blockDim.x) >> 5) {
        float h1[2], h2[2], o[4];
        mlp_fwd_warp(P, X + (long long)smp * kIn, lane, h1, h2, o);
        if (lane < kOut) out[(long long)smp * kOut + lane] = o[lane];
    }
}

// per-sample gradient of the loss (row smp of G) and the loss (loss[smp]);
// samples idx[k0 .. k0 + nb - 1] (idx NULL: k0 ..)
__global__ void mlp_grad_kernel(const float *__restrict__ P, const float *__restrict__ X,
                                const float *__restrict__ T, const int *__restrict__ idx, int k0, int nb,
                                float *__restrict__ G, float *__restrict__ loss)
{
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nb; t += (gridDim.x * blockDim.x) >> 5) {
        const int smp = idx ? idx[k0 + t] : k0 + t;
        const float *x = X + (long long)smp * kIn;
        float h1[2], h2[2], o[4];
        mlp_fwd_warp(P, x, lane, h1, h2, o);
        // output gradient
        const float th = T[2 * smp], cls = T[2 * smp + 1];
        const float sg = 1.0f / (1.0f + expf(-o[0]));
        const float m = fmaxf(o[1], fmaxf(o[2], o[3]));
        const float e1 = expf(o[1] - m), e2 = expf(o[2] - m), e3 = expf(o[3] - m), es = e1 + e2 + e3;
        const int c = (int)cls;
        float dO[4];
        dO[0] = 2.0f * (sg - th) * sg * (1.0f - sg);
        dO[1] = e1 / es - (c == 0 ? 1.0f : 0.0f);
        dO[2] = e2 / es - (c == 1 ? 1.0f : 0.0f);
        dO[3] = e3 / es - (c == 2 ? 1.0f : 0.0f);
        float *g = G + (long long)t * kNParam;
        if (lane == 0) {
            const float pc = (c == 0 ? e1 : c == 1 ? e2 : e3) / es;
            loss[t] = (sg - th) * (sg - th) - logf(fmaxf(pc, 1e-30f));
        }
        // layer 3
        float dh2[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int i = lane + 32 * u;
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < kOut; ++k) {
                g[oW3 + k * kHid + i] = dO[k] * h2[u];
                s = fmaf(P[oW3 + k * kHid + i], dO[k], s);
            }
            dh2[u] = h2[u] > 0.0f ? s : 0.0f;
        }
        if (lane < kOut) g[oB3 + lane] = dO[lane];
        // layer 2: dW2[j][i] = dh2_j h1_i; dh1_i = sum_j W2[j][i] dh2_j
        float dh1[2] = {0.0f, 0.0f};
#pragma unroll
        for (int half = 0; half < 2; ++half)
            for (int jj = 0; jj < 32; ++jj) {
                const int j = 32 * half + jj;
                const float dj = __shfl_sync(FULL, dh2[half], jj);
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = lane + 32 * u;
                    g[oW2 + j * kHid + i] = dj * h1[u];
                    dh1[u] = fmaf(P[oW2 + j * kHid + i], dj, dh1[u]);
                }
            }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int j = lane + 32 * u;
            g[oB2 + j] = dh2[u];
            dh1[u] = h1[u] > 0.0f ? dh1[u] : 0.0f;
            g[oB1 + j] = dh1[u];
        }
        // layer 1: dW1[j][i] = dh1_j x_i
        const float xi = lane < kIn ? x[lane] : 0.0f;
#pragma unroll
        for (int half = 0; half < 2; ++half)
            for (int jj = 0; jj < 32; ++jj) {
                const float dj = __shfl_sync(FULL, dh1[half], jj);
                if (lane < kIn) g[oW1 + (32 * half + jj) * kIn + lane] = dj * xi;
            }
    }
}

// grad[p] = (1/nb) sum over t of G[t][p]; lossm = mean loss (fixed order)
__global__ void mlp_reduce_kernel(int nb, const float *__restrict__ G, const float *__restrict__ loss,
                                  float *__restrict__ grad, float *__restrict__ lossm)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kNParam; p += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int t = 0; t < nb; ++t) s += G[(long long)t * kNParam + p];
        grad[p] = s / (float)nb;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && lossm) {
        float s = 0.0f;
        for (int t = 0; t < nb; ++t) s += loss[t];
        *lossm = s / (float)nb;
    }
}

__global__ void mlp_adam_kernel(float *__restrict__ P, const float *__restrict__ grad, float *__restrict__ m,
                                float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kNParam; p += gridDim.x * blockDim.x) {
        const float g = grad[p];
        const float mm = b1 * m[p] + (1.0f - b1) * g, vv = b2 * v[p] + (1.0f - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        P[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// --------------------------------------------------------------- features
// Per scalar row of an mBSR operator (fp64 values, bitmaps for presence):
// diagonal d, off-diagonal |.| sum and max, row sum, positive off-diagonal
// count, and the |.| of the couplings along each grid axis (an entry whose
// column offset decodes to (dx, dy, dz) on the level's nx x ny x nz grid
// adds to every axis it moves along).  Per-CTA partials, reduced in order.
enum { F_DD = 0, F_DDMIN, F_RS, F_RS2, F_NPOS, F_NOFF, F_SX, F_SY, F_SZ, F_OFFMAX, F_ROWS, F_MIX, F_NP };

__device__ __forceinline__ void decode_offset(long long off, int nx, int ny, int *dx, int *dy, int *dz)
{
    const long long sxy = (long long)nx * ny;
    long long z = 0, y = 0;
    if (sxy > 0) {
        z = off >= 0 ? (off + sxy / 2) / sxy : -((-off + sxy / 2) / sxy);
        off -= z * sxy;
    }
    if (nx > 0) {
        y = off >= 0 ? (off + nx / 2) / nx : -((-off + nx / 2) / nx);
        off -= y * nx;
    }
    *dx = (int)off;
    *dy = (int)y;
    *dz = (int)z;
}

__global__ void __launch_bounds__(256) features_kernel(int m, const int *__restrict__ ptr, const int *__restrict__ idx,
                                                      const double *__restrict__ val, const uint16_t *__restrict__ map,
                                                      int nx, int ny, double *__restrict__ part)
{
    __shared__ double sh[F_NP][8];
    double acc[F_NP];
#pragma unroll
    for (int k = 0; k < F_NP; ++k) acc[k] = 0.0;
    acc[F_DDMIN] = 1e300;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        const int b = row >> 2, q = row & 3;
        double d = 0.0, off = 0.0, omax = 0.0, rs = 0.0, sx = 0.0, sy = 0.0, sz = 0.0, mix = 0.0;
        int npos = 0, noff = 0;
        for (int k = ptr[b]; k < ptr[b + 1]; ++k) {
            const unsigned mk = map[k];
            for (int c = 0; c < 4; ++c) {
                if (!((mk >> (4 * q + c)) & 1u)) continue;
                const long long col = 4LL * idx[k] + c;
                const double a = val[16LL * k + 4 * q + c];
                rs += a;
                if (col == row) {
                    d = a;
                    continue;
                }
                const double aa = fabs(a);
                off += aa;
                omax = fmax(omax, aa);
                npos += a > 0.0;
                ++noff;
                int dx, dy, dz;
                decode_offset(col - row, nx, ny, &dx, &dy, &dz);
                if (dx) sx += aa;
                if (dy) sy += aa;
                if (dz) sz += aa;
                if ((dx != 0) + (dy != 0) + (dz != 0) > 1) mix += aa;
            }
        }
        const double ad = fabs(d) > 0.0 ? fabs(d) : 1.0;
        const double dd = off > 0.0 ? fabs(d) / off : 10.0;
        acc[F_DD] += fmin(dd, 10.0);
        acc[F_DDMIN] = fmin(acc[F_DDMIN], fmin(dd, 10.0));
        acc[F_RS] += rs / ad;
        acc[F_RS2] += (rs / ad) * (rs / ad);
        acc[F_NPOS] += npos;
        acc[F_NOFF] += noff;
        acc[F_SX] += sx / ad;
        acc[F_SY] += sy / ad;
        acc[F_SZ] += sz / ad;
        acc[F_OFFMAX] += omax / ad;
        acc[F_ROWS] += 1.0;
        acc[F_MIX] += mix / ad;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < F_NP; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(FULL, v, o);
            v = (k == F_DDMIN) ? fmin(v, u) : v + u;
        }
        if (lane == 0) sh[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < F_NP) {
        const int k = threadIdx.x;
        double v = sh[k][0];
        for (int i = 1; i < 8; ++i) v = (k == F_DDMIN) ? fmin(v, sh[k][i]) : v + sh[k][i];
        part[(long long)blockIdx.x * F_NP + k] = v;
    }
}

__global__ void features_final_kernel(int np, const double *__restrict__ part, double *__restrict__ out)
{
    if (threadIdx.x >= F_NP) return;
    const int k = threadIdx.x;
    double v = (k == F_DDMIN) ? 1e300 : 0.0;
    for (int i = 0; i < np; ++i) v = (k == F_DDMIN) ? fmin(v, part[(long long)i * F_NP + k]) : v + part[(long long)i * F_NP + k];
    out[k] = v;
}

// ------------------------------------------------ structured interpolation
// Linear interpolation between vertex-centred grids along the axes with
// c[d] = 1 (coarse j on fine 2j; odd fine points take 1/2 of both
// neighbours), identity along the others: P = Px (x) Py (x) Pz.
__device__ __forceinline__ int axis_terms(int i, int nf, int nc, int coarsen, int cidx[2], double w[2])
{
    if (!coarsen || nf == 1) {
        cidx[0] = coarsen ? 0 : i;
        w[0] = 1.0;
        return 1;
    }
    if ((i & 1) == 0) {
        cidx[0] = i >> 1;
        w[0] = 1.0;
        return 1;
    }
    cidx[0] = (i - 1) >> 1;
    w[0] = 0.5;
    if (((i + 1) >> 1) < nc) {
        cidx[1] = (i + 1) >> 1;
        w[1] = 0.5;
        return 2;
    }
    return 1;
}

struct InterpGeo {
    int nx, ny, nz, cx, cy, cz, ncx, ncy, ncz;
};

__global__ void interp_count_kernel(InterpGeo g, int *__restrict__ cnt)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(r % g.nx), y = (int)((r / g.nx) % g.ny), z = (int)(r / ((long long)g.nx * g.ny));
        int ci[2];
        double w[2];
        cnt[r] = axis_terms(x, g.nx, g.ncx, g.cx, ci, w) * axis_terms(y, g.ny, g.ncy, g.cy, ci, w) *
                 axis_terms(z, g.nz, g.ncz, g.cz, ci, w);
    }
}

__global__ void interp_fill_kernel(InterpGeo g, const int *__restrict__ ia, int *__restrict__ ja,
                                   double *__restrict__ a)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(r % g.nx), y = (int)((r / g.nx) % g.ny), z = (int)(r / ((long long)g.nx * g.ny));
        int cxi[2], cyi[2], czi[2];
        double wx[2], wy[2], wz[2];
        const int kx = axis_terms(x, g.nx, g.ncx, g.cx, cxi, wx), ky = axis_terms(y, g.ny, g.ncy, g.cy, cyi, wy),
                  kz = axis_terms(z, g.nz, g.ncz, g.cz, czi, wz);
        int e = ia[r];
        for (int c = 0; c < kz; ++c)  // columns ascend: z, then y, then x
            for (int b = 0; b < ky; ++b)
                for (int q = 0; q < kx; ++q) {
                    ja[e] = cxi[q] + g.ncx * (cyi[b] + g.ncy * czi[c]);
                    a[e] = wx[q] * wy[b] * wz[c];
                    ++e;
                }
    }
}

// ------------------------------------------- rotated anisotropic diffusion
// -div(K grad u) on an nx x ny (x nz) grid, K = R(angle) diag(1, eps) R^T in
// the x-y plane and 1 along z, Dirichlet boundary, unit spacing: the
// 9-point x-y stencil of -a u_xx - 2 b u_xy - c u_yy (a = cos^2 + eps sin^2,
// c = sin^2 + eps cos^2, b = (1 - eps) cos sin; the mixed term by central
// differences, -b/2 on the (1,1) / (-1,-1) diagonals and +b/2 on the others)
// plus -u_zz.  Rows: diagonal first, then columns ascending.
struct AnisoGeo {
    int nx, ny, nz;
    double a, b, c;
};

__device__ __forceinline__ int aniso_row(const AnisoGeo &g, long long r, int *cols, double *vals)
{
    const int x = (int)(r % g.nx), y = (int)((r / g.nx) % g.ny), z = (int)(r / ((long long)g.nx * g.ny));
    int k = 0;
    cols[k] = (int)r;
    vals[k++] = 2.0 * g.a + 2.0 * g.c + (g.nz > 1 ? 2.0 : 0.0);
    const long long sxy = (long long)g.nx * g.ny;
    // ascending column order: z-1; y-1 (x-1, x, x+1); y (x-1, x+1); y+1 (...); z+1
    if (z > 0) { cols[k] = (int)(r - sxy); vals[k++] = -1.0; }
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            if (x + dx < 0 || x + dx >= g.nx || y + dy < 0 || y + dy >= g.ny) continue;
            double v;
            if (dy == 0) v = -g.a;
            else if (dx == 0) v = -g.c;
            else v = (dx == dy) ? -0.5 * g.b : 0.5 * g.b;
            if (v == 0.0) continue;
            cols[k] = (int)(r + dx + (long long)dy * g.nx);
            vals[k++] = v;
        }
    if (z + 1 < g.nz) { cols[k] = (int)(r + sxy); vals[k++] = -1.0; }
    return k;
}

__global__ void aniso_count_kernel(AnisoGeo g, int *__restrict__ cnt)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    int cols[11];
    double vals[11];
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
        cnt[r] = aniso_row(g, r, cols, vals);
}

__global__ void aniso_fill_kernel(AnisoGeo g, const int *__restrict__ ia, int *__restrict__ ja,
                                  double *__restrict__ a)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    int cols[11];
    double vals[11];
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const int k = aniso_row(g, r, cols, vals);
        for (int e = 0; e < k; ++e) {
            ja[ia[r] + e] = cols[e];
            a[ia[r] + e] = vals[e];
        }
    }
}

}  // namespace amgt

using namespace amgt;

extern "C" {

int amgt_aniso_problem(const int *dims, double eps, double angle, amgt_csr *A, amgt_stream_t stream)
{
    if (!dims || !A || dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || !(eps > 0.0)) return AMGT_ERR_INVALID;
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    if (n * 11 > 0x7fffffffLL) return AMGT_ERR_TOO_LARGE;
    const double cs = std::cos(angle), sn = std::sin(angle);
    AnisoGeo g{dims[0], dims[1], dims[2], cs * cs + eps * sn * sn, (1.0 - eps) * cs * sn, sn * sn + eps * cs * cs};
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    memset(A, 0, sizeof(*A));
    int *cnt = nullptr;
    int64_t *tot = nullptr;
    const int64_t *h = nullptr;
    int rc = AMGT_OK;
    const int grid = grid_for(256, n, st->sm_count, 8);
    if ((rc = alloc_n(&A->i, (size_t)n + 1, s)) || (rc = alloc_n(&cnt, (size_t)n + 1, s)) ||
        (rc = alloc_n(&tot, 1, s)))
        goto fail;
    if (cudaMemsetAsync(cnt + n, 0, sizeof(int), s) != cudaSuccess || cudaMemsetAsync(tot, 0, 8, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    count_launch();
    aniso_count_kernel<<<grid, 256, 0, s>>>(g, cnt);
    if ((rc = exclusive_scan_int(cnt, A->i, (int)n + 1, s))) goto fail;
    if (cudaMemcpyAsync(tot, A->i + n, sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    if ((rc = read_back(tot, 1, s, &h))) goto fail;
    A->num_rows = A->num_cols = (int)n;
    A->num_nonzeros = (int)h[0];
    if ((rc = alloc_n(&A->j, (size_t)A->num_nonzeros, s)) || (rc = alloc_n(&A->data, (size_t)A->num_nonzeros, s)))
        goto fail;
    count_launch();
    aniso_fill_kernel<<<grid, 256, 0, s>>>(g, A->i, A->j, A->data);
    if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
fail:
    free_ptr(cnt, s);
    free_ptr(tot, s);
    if (rc) amgt_csr_free(A, stream);
    return rc;
}

int amgt_level_features(const amgt_bsr *A, int level, const int *dims, float *out, amgt_stream_t stream)
{
    if (!A || !out || !dims || A->row <= 0 || !A->blcPtr || !A->blcVal || !A->blcMap) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = grid_for(256, A->row, st->sm_count, 4);
    double *part = nullptr;
    AMGT_TRY(alloc_n(&part, (size_t)grid * F_NP + 16, s));
    int64_t *res = reinterpret_cast<int64_t *>(part + (size_t)grid * F_NP);
    count_launch();
    features_kernel<<<grid, 256, 0, s>>>(A->row, A->blcPtr, A->blcIdx, A->blcVal, A->blcMap, dims[0], dims[1], part);
    count_launch();
    features_final_kernel<<<1, 32, 0, s>>>(grid, part, reinterpret_cast<double *>(res));
    if (cudaGetLastError() != cudaSuccess) {
        free_ptr(part, s);
        return AMGT_ERR_CUDA;
    }
    const int64_t *h = nullptr;
    const int rc = read_back(res, F_NP, s, &h);
    double f[F_NP];
    if (rc == AMGT_OK) memcpy(f, h, sizeof(f));
    free_ptr(part, s);
    if (rc) return rc;
    const double rows = f[F_ROWS] > 0 ? f[F_ROWS] : 1.0;
    const double nnz = (double)A->csr_nnz;
    const double rsm = f[F_RS] / rows;
    const double st_sum = f[F_SX] + f[F_SY] + f[F_SZ];
    const double den = st_sum > 0 ? st_sum : 1.0;
    double v[AMGT_MLP_IN];
    v[0] = std::log10((double)A->row);
    v[1] = nnz / rows / 10.0;
    v[2] = A->blc_num > 0 ? nnz / (16.0 * A->blc_num) : 0.0;
    v[3] = f[F_DD] / rows;
    v[4] = f[F_DDMIN];
    v[5] = rsm;
    v[6] = std::sqrt(std::max(0.0, f[F_RS2] / rows - rsm * rsm));
    v[7] = f[F_NOFF] > 0 ? f[F_NPOS] / f[F_NOFF] : 0.0;
    v[8] = f[F_SX] / den;
    v[9] = f[F_SY] / den;
    v[10] = f[F_SZ] / den;
    v[11] = f[F_MIX] / den;
    v[12] = f[F_OFFMAX] / rows;
    v[13] = level / 10.0;
    v[14] = dims[2] > 1 ? 1.0 : 0.0;
    v[15] = 1.0;
    for (int k = 0; k < AMGT_MLP_IN; ++k) out[k] = (float)v[k];
    return AMGT_OK;
}

int amgt_structured_interp(const int *dims, const int *coarsen, amgt_csr *P, int *cdims, amgt_stream_t stream)
{
    if (!dims || !coarsen || !P || !cdims || dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return AMGT_ERR_INVALID;
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    if (n > 0x3fffffffLL) return AMGT_ERR_TOO_LARGE;
    InterpGeo g{dims[0], dims[1], dims[2], coarsen[0] && dims[0] > 1, coarsen[1] && dims[1] > 1,
                coarsen[2] && dims[2] > 1, 0, 0, 0};
    g.ncx = g.cx ? (g.nx + 1) / 2 : g.nx;
    g.ncy = g.cy ? (g.ny + 1) / 2 : g.ny;
    g.ncz = g.cz ? (g.nz + 1) / 2 : g.nz;
    cdims[0] = g.ncx;
    cdims[1] = g.ncy;
    cdims[2] = g.ncz;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    memset(P, 0, sizeof(*P));
    int *cnt = nullptr;
    int64_t *tot = nullptr;
    const int64_t *h = nullptr;
    int rc = AMGT_OK;
    const int grid = grid_for(256, n, st->sm_count, 8);
    if ((rc = alloc_n(&P->i, (size_t)n + 1, s)) || (rc = alloc_n(&cnt, (size_t)n + 1, s)) ||
        (rc = alloc_n(&tot, 1, s)))
        goto fail;
    if (cudaMemsetAsync(cnt + n, 0, sizeof(int), s) != cudaSuccess || cudaMemsetAsync(tot, 0, 8, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    count_launch();
    interp_count_kernel<<<grid, 256, 0, s>>>(g, cnt);
    if ((rc = exclusive_scan_int(cnt, P->i, (int)n + 1, s))) goto fail;
    if (cudaMemcpyAsync(tot, P->i + n, sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto fail;
    }
    if ((rc = read_back(tot, 1, s, &h))) goto fail;
    P->num_rows = (int)n;
    P->num_cols = g.ncx * g.ncy * g.ncz;
    P->num_nonzeros = (int)h[0];
    if ((rc = alloc_n(&P->j, (size_t)P->num_nonzeros, s)) || (rc = alloc_n(&P->data, (size_t)P->num_nonzeros, s)))
        goto fail;
    count_launch();
    interp_fill_kernel<<<grid, 256, 0, s>>>(g, P->i, P->j, P->data);
    if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
fail:
    free_ptr(cnt, s);
    free_ptr(tot, s);
    if (rc) amgt_csr_free(P, stream);
    return rc;
}

int amgt_mlp_forward(const float *params, int n, const float *X, float *out, amgt_stream_t stream)
{
    if (!params || n < 0 || (n > 0 && (!X || !out))) return AMGT_ERR_INVALID;
    if (n == 0) return AMGT_OK;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    AMGT_LAUNCH(mlp_forward_kernel, grid_for(8, n, st->sm_count, 8), 256, 0, (cudaStream_t)stream, params, n, X, out);
    return AMGT_OK;
}

int amgt_mlp_grad(const float *params, int n, const float *X, const float *T, float *grad, float *loss,
                  amgt_stream_t stream)
{
    if (!params || n < 1 || !X || !T || !grad) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    float *G = nullptr, *ls = nullptr;
    int rc = AMGT_OK;
    if ((rc = alloc_n(&G, (size_t)n * kNParam, s)) || (rc = alloc_n(&ls, (size_t)n, s))) goto done;
    count_launch();
    mlp_grad_kernel<<<grid_for(8, n, st->sm_count, 8), 256, 0, s>>>(params, X, T, nullptr, 0, n, G, ls);
    count_launch();
    mlp_reduce_kernel<<<grid_for(256, kNParam, st->sm_count, 1), 256, 0, s>>>(n, G, ls, grad, loss);
    if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
done:
    free_ptr(G, s);
    free_ptr(ls, s);
    return rc;
}

int amgt_mlp_train(float *params, int n, const float *X, const float *T, int epochs, int batch, float lr,
                   unsigned seed, float *loss_hist, amgt_stream_t stream)
{
    if (!params || n < 1 || !X || !T || epochs < 0 || batch < 1 || !(lr > 0.0f)) return AMGT_ERR_INVALID;
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    cudaStream_t s = (cudaStream_t)stream;
    const int nb_max = std::min(batch, n);
    float *G = nullptr, *ls = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *lossm = nullptr;
    int *idx = nullptr;
    int rc = AMGT_OK;
    std::vector<int> perm(n);
    if ((rc = alloc_n(&G, (size_t)nb_max * kNParam, s)) || (rc = alloc_n(&ls, (size_t)nb_max, s)) ||
        (rc = alloc_n(&grad, (size_t)kNParam, s)) || (rc = alloc_n(&m, (size_t)kNParam, s)) ||
        (rc = alloc_n(&v, (size_t)kNParam, s)) || (rc = alloc_n(&idx, (size_t)n, s)) ||
        (rc = alloc_n(&lossm, (size_t)std::max(1, epochs), s)))
        goto done;
    if (cudaMemsetAsync(m, 0, sizeof(float) * kNParam, s) != cudaSuccess ||
        cudaMemsetAsync(v, 0, sizeof(float) * kNParam, s) != cudaSuccess) {
        rc = AMGT_ERR_CUDA;
        goto done;
    }
    {
        uint64_t state = 0x9E3779B97F4A7C15ull * (seed + 1);
        auto next = [&]() {  // splitmix64
            uint64_t z = (state += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return z ^ (z >> 31);
        };
        int step = 0;
        const float b1 = 0.9f, b2 = 0.999f;
        for (int ep = 0; ep < epochs && !rc; ++ep) {
            for (int i = 0; i < n; ++i) perm[i] = i;
            for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (uint64_t)(i + 1)]);
            // the permutation is consumed by this epoch's launches before the
            // next one overwrites it (pageable copy: complete on return)
            if (cudaMemcpyAsync(idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s) != cudaSuccess) {
                rc = AMGT_ERR_CUDA;
                break;
            }
            for (int k0 = 0; k0 < n && !rc; k0 += nb_max) {
                const int nb = std::min(nb_max, n - k0);
                ++step;
                const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
                count_launch();
                mlp_grad_kernel<<<grid_for(8, nb, st->sm_count, 8), 256, 0, s>>>(params, X, T, idx, k0, nb, G, ls);
                count_launch();
                mlp_reduce_kernel<<<grid_for(256, kNParam, st->sm_count, 1), 256, 0, s>>>(
                    nb, G, ls, grad, (k0 + nb >= n) ? lossm + ep : nullptr);
                count_launch();
                mlp_adam_kernel<<<grid_for(256, kNParam, st->sm_count, 1), 256, 0, s>>>(params, grad, m, v, lr, b1, b2,
                                                                                       1e-8f, c1, c2);
                if (cudaGetLastError() != cudaSuccess) rc = AMGT_ERR_CUDA;
            }
            if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = AMGT_ERR_CUDA;  // perm is rewritten next epoch
        }
        if (!rc && loss_hist && epochs > 0 &&
            cudaMemcpy(loss_hist, lossm, sizeof(float) * epochs, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = AMGT_ERR_CUDA;
    }
done:
    free_ptr(G, s);
    free_ptr(ls, s);
    free_ptr(grad, s);
    free_ptr(m, s);
    free_ptr(v, s);
    free_ptr(idx, s);
    free_ptr(lossm, s);
    return rc;
}

}  // extern "C"
