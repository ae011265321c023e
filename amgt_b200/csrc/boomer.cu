// BoomerAMG's setup on the host, restated for one process and one function
// per unknown: the settings the headline configurations name (HMIS
// coarsening, strength threshold theta, extended+i interpolation truncated
// to P_max entries per row; PMIS as an option) and, for a whole hierarchy,
// the Galerkin products in the order and arithmetic of HYPRE's host setup.
// HYPRE 2.31 runs HMIS on the host even in GPU builds
// (R/parcsr_ls/par_coarsen.c:2845-2865).  Two users: amgt_boomer_interp
// coarsens one GPU level at a time for amgt_amg_setup_adaptive (copy A_l
// down, coarsen, upload P_l), and amgt_boomer_hierarchy_host builds every
// P_l as HYPRE's CPU BoomerAMG would, for amgt_amg_setup.
//
// Steps, each restating HYPRE's semantics (R = AmgT_HYPRE/src):
//   strength   i depends on j (j != i) when a_ij < theta * min_k a_ik for
//              a_ii >= 0 (a_ij > theta * max_k a_ik for a_ii < 0); a row
//              whose |row sum| exceeds max_row_sum * |a_ii| (max_row_sum
//              < 1) has no strong couplings (hypre_BoomerAMGCreateSHost,
//              R/parcsr_ls/par_strength.c).
//   first pass Ruge-Stueben's first colouring pass (hypre_BoomerAMGCoarsenRuge
//              with coarsen type 10 -> 11, par_coarsen.c:911-1391): measure =
//              number of points that depend on a point; repeatedly the oldest
//              point of the largest measure becomes C, the points depending on
//              it F, measures updated; points nobody depends on are marked Z.
//   PMIS       hypre_BoomerAMGCoarsenPMISHost (par_coarsen.c:2101-2815), after
//              the first pass (CF_init = 1, HMIS) or alone (coarsen type 8):
//              measures get a uniform (0, 1) draw each (Park and Miller's
//              minimal standard generator, seed 2747, rows in order); a point
//              that depends on a C point is F; the rest choose C points as
//              independent sets of locally largest measure until every point
//              is decided.
//   ext+i      hypre_BoomerAMGBuildExtPIInterpHost (par_lr_interp.c:1025):
//              F point i interpolates from C_i-hat = strong C neighbours and
//              the strong C neighbours of its strong F neighbours; a strong F
//              neighbour's coupling is distributed over C_i-hat and i itself
//              in proportion to its own couplings of the opposite sign to its
//              diagonal; weak couplings go to the diagonal; w = -sum / diag.
//   truncation hypre_ParCSRMatrixTruncate with P_max entries
//              (R/parcsr_mv/par_csr_matrix.c:2866-3240) once P is complete:
//              rows longer than P_max are sorted by |w| descending (the
//              quicksort of Kernighan and Ritchie, as hypre_qsort2_abs does,
//              so ties fall the same way), the first P_max kept and rescaled
//              to the row's former sum.
//   Galerkin   hypre_BoomerAMGBuildCoarseOperatorKT (par_rap.c:30), the
//              product of HYPRE's host setup: row by row, R A first, then
//              (R A) P; the next level reads the result in this order.
// Rows are read in their stored order with the diagonal first (HYPRE's
// storage): the order decides which of equal-magnitude weights truncation
// keeps, so the whole-hierarchy builder keeps HYPRE's order level to level.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "amgt_internal.cuh"

namespace amgt {
namespace {

constexpr int C_PT = 1, F_PT = -1, Z_PT = -2, SF_PT = -3, UNDECIDED = 0;

struct Strength {
    std::vector<int> si, sj;  // strong off-diagonal couplings, A's row order
};

// Rows must hold their diagonal first.  Rows in parallel (OpenMP): a count
// pass, then each row's strong columns in its own place, in row order.
static int strong_row(int i, const int *ia, const int *ja, const double *a, double theta, double max_row_sum,
                      int *out)
{
    const int b = ia[i], e = ia[i + 1];
    if (!(b < e && ja[b] == i)) return 0;
    const double diag = a[b];
    double scale = 0.0, rsum = diag;
    for (int k = b + 1; k < e; ++k) {
        scale = diag < 0 ? std::max(scale, a[k]) : std::min(scale, a[k]);
        rsum += a[k];
    }
    const bool all_weak = std::fabs(rsum) > std::fabs(diag) * max_row_sum && max_row_sum < 1.0;
    if (all_weak) return 0;
    int cnt = 0;
    for (int k = b + 1; k < e; ++k) {
        const bool strong = diag < 0 ? !(a[k] <= theta * scale) : !(a[k] >= theta * scale);
        if (strong) {
            if (out) out[cnt] = ja[k];
            ++cnt;
        }
    }
    return cnt;
}

Strength strength(int n, const int *ia, const int *ja, const double *a, double theta, double max_row_sum)
{
    Strength S;
    S.si.assign(n + 1, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) S.si[i + 1] = strong_row(i, ia, ja, a, theta, max_row_sum, nullptr);
    for (int i = 0; i < n; ++i) S.si[i + 1] += S.si[i];
    S.sj.resize(S.si[n]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) strong_row(i, ia, ja, a, theta, max_row_sum, S.sj.data() + S.si[i]);
    return S;
}

// Buckets of points by measure, each a FIFO list (points enter at the tail,
// the head is taken): HYPRE's list of lists (amg_linklist.c).
struct Buckets {
    std::vector<int> head, tail, next, prev;
    int top = -1;  // largest non-empty measure
    Buckets(int n, int maxm) : head(maxm + 2, -1), tail(maxm + 2, -1), next(n, -1), prev(n, -1) {}
    void grow(int m)
    {
        if (m >= (int)head.size()) {
            head.resize(m + 2, -1);
            tail.resize(m + 2, -1);
        }
    }
    void enter(int m, int i)
    {
        grow(m);
        prev[i] = tail[m];
        next[i] = -1;
        if (tail[m] >= 0) next[tail[m]] = i;
        else head[m] = i;
        tail[m] = i;
        top = std::max(top, m);
    }
    void remove(int m, int i)
    {
        if (prev[i] >= 0) next[prev[i]] = next[i];
        else head[m] = next[i];
        if (next[i] >= 0) prev[next[i]] = prev[i];
        else tail[m] = prev[i];
        prev[i] = next[i] = -1;
        while (top >= 0 && head[top] < 0) --top;
    }
    int first() const { return top >= 0 ? head[top] : -1; }
};

// Ruge-Stueben first pass (coarsen type 11: Z for unneeded points).
void first_pass(int n, const Strength &S, std::vector<int> &cf)
{
    // S^T: the points that depend on each point, ascending
    std::vector<int> ti(n + 1, 0), tj(S.sj.size());
    for (int j : S.sj) ++ti[j + 1];
    for (int i = 0; i < n; ++i) ti[i + 1] += ti[i];
    {
        std::vector<int> fill(ti.begin(), ti.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = S.si[i]; k < S.si[i + 1]; ++k) tj[fill[S.sj[k]]++] = i;
    }
    std::vector<int> meas(n);
    int maxm = 0;
    for (int i = 0; i < n; ++i) {
        meas[i] = ti[i + 1] - ti[i];
        maxm = std::max(maxm, meas[i]);
    }
    cf.assign(n, UNDECIDED);
    int left = 0;
    for (int j = 0; j < n; ++j) {
        if (S.si[j + 1] - S.si[j] == 0) {
            cf[j] = SF_PT;
            meas[j] = 0;
        } else {
            ++left;
        }
    }
    Buckets L(n, maxm + n / 2 + 8);
    for (int j = 0; j < n; ++j) {
        if (cf[j] == SF_PT) continue;
        if (meas[j] > 0) {
            L.enter(meas[j], j);
        } else {
            cf[j] = Z_PT;
            for (int k = S.si[j]; k < S.si[j + 1]; ++k) {
                const int nb = S.sj[k];
                if (cf[nb] == SF_PT) continue;
                if (nb < j) {
                    if (meas[nb] > 0) L.remove(meas[nb], nb);
                    L.enter(++meas[nb], nb);
                } else {
                    ++meas[nb];
                }
            }
            --left;
        }
    }
    while (left > 0) {
        const int c = L.first();
        if (c < 0) break;  // nothing left on the lists
        cf[c] = C_PT;
        L.remove(meas[c], c);
        meas[c] = 0;
        --left;
        for (int t = ti[c]; t < ti[c + 1]; ++t) {
            const int nb = tj[t];
            if (cf[nb] != UNDECIDED) continue;
            cf[nb] = F_PT;
            L.remove(meas[nb], nb);
            --left;
            for (int k = S.si[nb]; k < S.si[nb + 1]; ++k) {
                const int n2 = S.sj[k];
                if (cf[n2] != UNDECIDED) continue;
                L.remove(meas[n2], n2);
                L.enter(++meas[n2], n2);
            }
        }
        for (int k = S.si[c]; k < S.si[c + 1]; ++k) {
            const int nb = S.sj[k];
            if (cf[nb] != UNDECIDED) continue;
            L.remove(meas[nb], nb);
            if (--meas[nb] > 0) {
                L.enter(meas[nb], nb);
            } else {
                cf[nb] = F_PT;
                --left;
                for (int k2 = S.si[nb]; k2 < S.si[nb + 1]; ++k2) {
                    const int n2 = S.sj[k2];
                    if (cf[n2] != UNDECIDED) continue;
                    L.remove(meas[n2], n2);
                    L.enter(++meas[n2], n2);
                }
            }
        }
    }
}

// Park and Miller's minimal standard generator (multiplier 16807, modulus
// 2^31 - 1, Schrage's decomposition), as HYPRE seeds and draws it.
struct MinStd {
    long long seed;
    explicit MinStd(long long s) : seed(s < 1 ? 1 : (s >= 2147483647LL ? 2147483646LL : s)) {}
    double next()
    {
        const long long a = 16807, m = 2147483647LL, q = 127773, r = 2836;
        const long long hi = seed / q, lo = seed % q;
        const long long t = a * lo - r * hi;
        seed = t > 0 ? t : t + m;
        return (double)seed / (double)m;
    }
};

// PMIS (hypre_BoomerAMGCoarsenPMISHost): with cf_init, after the first
// pass (CF_init = 1, HMIS); without, from scratch (CF_init = 0, coarsen
// type 8, BoomerAMG's GPU default).
void pmis(int n, const Strength &S, std::vector<int> &cf, bool cf_init)
{
    std::vector<double> meas(n, 0.0);
    for (int j : S.sj) meas[j] += 1.0;
    MinStd rng(2747);
    for (int i = 0; i < n; ++i) meas[i] += rng.next();
    std::vector<int> graph;
    graph.reserve(n);
    if (!cf_init) {
        cf.assign(n, UNDECIDED);
        for (int i = 0; i < n; ++i)
            if (S.si[i + 1] == S.si[i]) cf[i] = SF_PT;  // no strong coupling: an isolated fine point
    }
    for (int i = 0; i < n; ++i) {
        if (cf[i] == SF_PT) {
            meas[i] = 0.0;
            continue;
        }
        if (cf[i] == F_PT) cf[i] = UNDECIDED;
        if (cf[i] == Z_PT) {
            if (meas[i] >= 1.0 || S.si[i + 1] - S.si[i] > 0) {
                cf[i] = UNDECIDED;
                graph.push_back(i);
            } else {
                cf[i] = F_PT;
            }
        } else {
            graph.push_back(i);
        }
    }
    // The loops over the graph run in parallel (OpenMP), as HYPRE's do: the
    // independent-set pass only clears marks (every writer writes 0), and the
    // C/F pass reads marks that stay > 0 for the set's points and <= 0 for
    // the others whichever thread writes first, so the result is the
    // sequential one.
    int iter = 0;
    while (!graph.empty()) {
        const int gn = (int)graph.size();
        if (!cf_init || iter > 0) {
#pragma omp parallel for schedule(static)
            for (int g = 0; g < gn; ++g) {
                const int i = graph[g];
                if (meas[i] > 1.0) cf[i] = 1;
            }
#pragma omp parallel for schedule(static)
            for (int g = 0; g < gn; ++g) {
                const int i = graph[g];
                if (!(meas[i] > 1.0)) continue;
                for (int k = S.si[i]; k < S.si[i + 1]; ++k) {
                    const int j = S.sj[k];
                    if (!(meas[j] > 1.0)) continue;
                    if (meas[i] > meas[j]) cf[j] = 0;
                    else if (meas[j] > meas[i]) cf[i] = 0;
                }
            }
        }
        ++iter;
#pragma omp parallel for schedule(static)
        for (int g = 0; g < gn; ++g) {
            const int i = graph[g];
            if (meas[i] < 1.0) cf[i] = F_PT;
            if (cf[i] > 0) {
                cf[i] = C_PT;
            } else {
                for (int k = S.si[i]; k < S.si[i + 1]; ++k)
                    if (cf[S.sj[k]] > 0) cf[i] = F_PT;
            }
        }
        std::vector<int> keep;
        keep.reserve(graph.size());
        for (int i : graph) {
            if (cf[i] != 0) meas[i] = 0.0;
            else keep.push_back(i);
        }
        if (keep.size() == graph.size() && iter > 1) break;  // no progress (cannot happen for finite measures)
        graph.swap(keep);
    }
}

// quicksort of Kernighan and Ritchie on |w| descending, moving columns along
void qsort_abs_desc(int *v, double *w, int left, int right)
{
    if (left >= right) return;
    auto swap2 = [&](int i, int j) {
        std::swap(v[i], v[j]);
        std::swap(w[i], w[j]);
    };
    swap2(left, (left + right) / 2);
    int last = left;
    for (int i = left + 1; i <= right; ++i)
        if (std::fabs(w[i]) > std::fabs(w[left])) swap2(++last, i);
    swap2(left, last);
    qsort_abs_desc(v, w, left, last - 1);
    qsort_abs_desc(v, w, last + 1, right);
}

struct ExtI {
    const int *ia, *ja;
    const double *a;
    const Strength *S;
    const int *cf, *f2c;
};

// Row i of ext+i (hypre_BoomerAMGBuildExtPIInterpHost, par_lr_interp.c:
// 1520-1760): C_i-hat in discovery order at positions row0, row0 + 1, ...
// of (pj, pa) and, when pj is given, the weights; returns the row's length.
// marker and strong_f are the calling thread's (marker >= row0: position of
// a C_i-hat point; strong_f: this row's mark of its strong F neighbours,
// unique per row).
int ext_i_row(const ExtI &E, int i, int *marker, int &strong_f, int row0, int *pj, double *pa)
{
    const int *ia = E.ia, *ja = E.ja, *cf = E.cf, *f2c = E.f2c;
    const double *a = E.a;
    const Strength &S = *E.S;
    int len = 0;
    if (cf[i] >= 0) {
        if (pj) {
            pj[row0] = f2c[i];
            pa[row0] = 1.0;
        }
        return 1;
    }
    if (cf[i] == SF_PT) return 0;
    --strong_f;
    auto add = [&](int c) {
        if (marker[c] < row0) {
            marker[c] = row0 + len;
            if (pj) {
                pj[row0 + len] = f2c[c];
                pa[row0 + len] = 0.0;
            }
            ++len;
        }
    };
    for (int k = S.si[i]; k < S.si[i + 1]; ++k) {
        const int i1 = S.sj[k];
        if (cf[i1] >= 0) {
            add(i1);
        } else if (cf[i1] != SF_PT) {
            marker[i1] = strong_f;
            for (int kk = S.si[i1]; kk < S.si[i1 + 1]; ++kk) {
                const int k1 = S.sj[kk];
                if (cf[k1] >= 0) add(k1);
            }
        }
    }
    if (pj) {
        double diag = a[ia[i]];
        for (int k = ia[i] + 1; k < ia[i + 1]; ++k) {
            const int i1 = ja[k];
            if (marker[i1] >= row0) {
                pa[marker[i1]] += a[k];
            } else if (marker[i1] == strong_f) {
                double sum = 0.0;
                const int sgn = a[ia[i1]] < 0 ? -1 : 1;
                for (int k2 = ia[i1] + 1; k2 < ia[i1 + 1]; ++k2) {
                    const int i2 = ja[k2];
                    if ((marker[i2] >= row0 || i2 == i) && sgn * a[k2] < 0) sum += a[k2];
                }
                if (sum != 0.0) {
                    const double dist = a[k] / sum;
                    for (int k2 = ia[i1] + 1; k2 < ia[i1 + 1]; ++k2) {
                        const int i2 = ja[k2];
                        if (marker[i2] >= row0 && sgn * a[k2] < 0) pa[marker[i2]] += dist * a[k2];
                        if (i2 == i && sgn * a[k2] < 0) diag += dist * a[k2];
                    }
                } else {
                    diag += a[k];
                }
            } else if (cf[i1] != SF_PT) {
                diag += a[k];
            }
        }
        if (diag != 0.0)
            for (int k = row0; k < row0 + len; ++k) pa[k] /= -diag;
    }
    --strong_f;
    return len;
}

// P_max truncation of one row (hypre_ParCSRMatrixTruncate's max_elmts
// branch, par_csr_matrix.c:3100-3215): rows longer than p_max sorted by
// |w| descending, the first p_max kept and rescaled to the former row sum;
// returns the kept length.
int truncate_row(int *pj, double *pa, int len, int p_max)
{
    if (p_max <= 0 || len <= p_max) return len;
    double rsum = 0.0;
    for (int k = 0; k < len; ++k) rsum += pa[k];
    qsort_abs_desc(pj, pa, 0, len - 1);
    double scale = 0.0;
    for (int k = 0; k < p_max; ++k) scale += pa[k];
    if (scale != 0.0 && scale != rsum) {
        const double f = rsum / scale;
        for (int k = 0; k < p_max; ++k) pa[k] *= f;
    }
    return p_max;
}

}  // namespace

// Coarsening and ext+i interpolation of one level (host arrays; rows with
// the diagonal first).  cf: C (1) / F (-1) per row; P in CSR, columns in
// coarse numbering (C points in row order).
int boomer_level(int n, const int *ia, const int *ja, const double *a, const amgt_boomer_params &prm,
                 std::vector<int> &cf, std::vector<int> &pi, std::vector<int> &pj, std::vector<double> &pa)
{
    const int p_max = prm.p_max;
    const Strength S = strength(n, ia, ja, a, prm.theta, prm.max_row_sum);
    if (prm.coarsen_type == 10) first_pass(n, S, cf);
    pmis(n, S, cf, prm.coarsen_type == 10);
    std::vector<int> f2c(n, -1);
    int nc = 0;
    for (int i = 0; i < n; ++i)
        if (cf[i] >= 0) f2c[i] = nc++;
    // ext+i row by row, rows in parallel (OpenMP, contiguous row ranges per
    // thread, so that a thread's row starts increase): a count pass sizes
    // every row, then each row is built and truncated in its own place and
    // the rows are compacted
    pi.assign(n + 1, 0);
    std::vector<int> keep(n, 0);
    const ExtI E{ia, ja, a, &S, cf.data(), f2c.data()};
#pragma omp parallel
    {
        std::vector<int> marker(n, -1);
        int strong_f = -2, vpos = 0;  // vpos: the thread's running row start, so that markers stay below it
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            pi[i + 1] = ext_i_row(E, i, marker.data(), strong_f, vpos, nullptr, nullptr);
            vpos += pi[i + 1];
        }
    }
    for (int i = 0; i < n; ++i) pi[i + 1] += pi[i];
    std::vector<int> tj(pi[n]);
    std::vector<double> ta(pi[n]);
#pragma omp parallel
    {
        std::vector<int> marker(n, -1);
        int strong_f = -2;
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            const int row0 = pi[i];
            const int len = ext_i_row(E, i, marker.data(), strong_f, row0, tj.data(), ta.data());
            keep[i] = truncate_row(tj.data() + row0, ta.data() + row0, len, p_max);
        }
    }
    // compaction: the kept entries of each row, in place order
    std::vector<int> out(n + 1, 0);
    for (int i = 0; i < n; ++i) out[i + 1] = out[i] + keep[i];
    pj.resize(out[n]);
    pa.resize(out[n]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < keep[i]; ++k) {
            pj[out[i] + k] = tj[pi[i] + k];
            pa[out[i] + k] = ta[pi[i] + k];
        }
    pi.swap(out);
    return nc;
}

namespace {

struct HostCsr {
    int rows = 0, cols = 0;
    std::vector<int> i, j;
    std::vector<double> a;
};

// hypre_CSRMatrixTransposeHost (seq_mv/csr_matop.c:1043): a counting sort
// by column, so row c of the transpose lists the rows holding column c in
// ascending order.
HostCsr transpose(const HostCsr &A)
{
    HostCsr T;
    T.rows = A.cols;
    T.cols = A.rows;
    T.i.assign(A.cols + 1, 0);
    for (int c : A.j) ++T.i[c + 1];
    for (int c = 0; c < A.cols; ++c) T.i[c + 1] += T.i[c];
    T.j.resize(A.j.size());
    T.a.resize(A.a.size());
    std::vector<int> fill(T.i.begin(), T.i.end() - 1);
    for (int r = 0; r < A.rows; ++r)
        for (int k = A.i[r]; k < A.i[r + 1]; ++k) {
            const int p = fill[A.j[k]]++;
            T.j[p] = r;
            T.a[p] = A.a[k];
        }
    return T;
}

// hypre_BoomerAMGBuildCoarseOperatorKT (parcsr_ls/par_rap.c:30), one
// process: the Galerkin product BoomerAMG's host setup forms (the
// modularised hypre_ParCSRMatrixRAPKT only runs on the device,
// par_amg.c:304-316).  R = P^T by the counting-sort transpose
// (hypre_CSRMatrixTransposeHost, seq_mv/csr_matop.c:1043: row c lists the
// fine rows of column c ascending).  Row ic: first row ic of R A (for each
// fine row i1 of R's row, for each entry of A's row i1 in stored order; a
// column enters where first met with r*a, later products added), then
// row ic of (R A) P (for each entry of that RA row in the order met, for
// each entry of P's row; the diagonal stored first).  Plain multiply, then
// add (par_rap.c:1700-1880).
// Row ic of (R A) P into (cj, ca) at row0 (count only when cj is null);
// returns its length.  a_stamp/a_pos/p_mark/ra_* are the calling thread's.
static int rap_row(const HostCsr &R, const HostCsr &A, const HostCsr &P, int ic, int row0, int *a_stamp,
                   int *a_pos, int *p_mark, std::vector<int> &ra_j, std::vector<double> &ra_a, int *cj, double *ca)
{
    int len = 1;  // the diagonal first
    p_mark[ic] = row0;
    if (cj) {
        cj[row0] = ic;
        ca[row0] = 0.0;
    }
    ra_j.clear();
    ra_a.clear();
    for (int kr = R.i[ic]; kr < R.i[ic + 1]; ++kr) {
        const int i1 = R.j[kr];
        const double r = R.a[kr];
        for (int ka = A.i[i1]; ka < A.i[i1 + 1]; ++ka) {
            const int i2 = A.j[ka];
            const double ra = r * A.a[ka];
            if (a_stamp[i2] != ic) {
                a_stamp[i2] = ic;
                a_pos[i2] = (int)ra_j.size();
                ra_j.push_back(i2);
                ra_a.push_back(ra);
            } else {
                ra_a[a_pos[i2]] += ra;
            }
        }
    }
    for (size_t t = 0; t < ra_j.size(); ++t) {
        const int i1 = ra_j[t];
        const double ra = ra_a[t];
        for (int kp = P.i[i1]; kp < P.i[i1 + 1]; ++kp) {
            const int i3 = P.j[kp];
            if (p_mark[i3] < row0) {
                p_mark[i3] = row0 + len;
                if (cj) {
                    cj[row0 + len] = i3;
                    ca[row0 + len] = ra * P.a[kp];
                }
                ++len;
            } else if (cj) {
                ca[p_mark[i3]] += ra * P.a[kp];
            }
        }
    }
    return len;
}

HostCsr rap_kt(const HostCsr &A, const HostCsr &P)
{
    const HostCsr R = transpose(P);
    const int nc = P.cols;
    HostCsr C;
    C.rows = C.cols = nc;
    C.i.assign(nc + 1, 0);
    // rows in parallel (OpenMP, contiguous ranges per thread): a count
    // pass, then every row in its own place
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel
        {
            std::vector<int> a_stamp(A.cols, -1), a_pos(A.cols, 0), p_mark(nc, -1);
            std::vector<int> ra_j;
            std::vector<double> ra_a;
            int vpos = 0;  // count pass: the thread's running row start
#pragma omp for schedule(static)
            for (int ic = 0; ic < nc; ++ic) {
                if (pass == 0) {
                    const int len = rap_row(R, A, P, ic, vpos, a_stamp.data(), a_pos.data(), p_mark.data(), ra_j,
                                            ra_a, nullptr, nullptr);
                    C.i[ic + 1] = len;
                    vpos += len;
                } else {
                    rap_row(R, A, P, ic, C.i[ic], a_stamp.data(), a_pos.data(), p_mark.data(), ra_j, ra_a,
                            C.j.data(), C.a.data());
                }
            }
        }
        if (pass == 0) {
            for (int ic = 0; ic < nc; ++ic) C.i[ic + 1] += C.i[ic];
            C.j.resize(C.i[nc]);
            C.a.resize(C.i[nc]);
        }
    }
    return C;
}

}  // namespace

// The whole hierarchy as HYPRE's CPU BoomerAMG builds it on one process
// (hypre_BoomerAMGSetup, par_amg_setup.c): per level strength, HMIS and
// ext+i with truncation (boomer_level), then A_{l+1} = (P^T A_l) P as
// hypre_BoomerAMGBuildCoarseOperatorKT forms it (rap_kt).  A_{l+1} keeps the product's column order
// (diagonal first, then as met), which the next level's strength, HMIS and
// ext+i read in that order -- the order that decides the truncation's ties.
// Coarsening stops, as par_amg_setup.c:1671 and 3177 do, when a level has
// no coarse point or no fine point, when a coarse level has at most
// max_coarse rows, or at max_levels levels.  A coarse level of at least 3/4
// of its fine level switches HYPRE to CLJP coarsening
// (par_amg_setup.c:3166-3169), which is not built here:
// AMGT_ERR_UNSUPPORTED.
int boomer_hierarchy(const HostCsr &A0, const amgt_boomer_params &p, int max_levels, int max_coarse,
                     std::vector<HostCsr> &As, std::vector<HostCsr> &Ps)
{
    As.assign(1, A0);
    Ps.clear();
    while ((int)As.size() < max_levels && As.back().rows > max_coarse) {
        const HostCsr &A = As.back();
        std::vector<int> cf;
        HostCsr P;
        P.rows = A.rows;
        P.cols = boomer_level(A.rows, A.i.data(), A.j.data(), A.a.data(), p, cf, P.i, P.j, P.a);
        if (P.cols == 0 || P.cols == A.rows) break;
        if (P.cols >= 0.75 * A.rows && (int)As.size() + 1 < max_levels && P.cols > max_coarse)
            return AMGT_ERR_UNSUPPORTED;  // HYPRE would continue with CLJP
        HostCsr C = rap_kt(A, P);
        Ps.push_back(std::move(P));
        As.push_back(std::move(C));
    }
    return AMGT_OK;
}

}  // namespace amgt

using namespace amgt;

extern "C" {

int amgt_boomer_coarsen_host(int n, const int *ia, const int *ja, const double *a, const amgt_boomer_params *prm,
                             int *cf_marker, amgt_csr *P)
{
    if (n <= 0 || !ia || !ja || !a || !P) return AMGT_ERR_INVALID;
    amgt_boomer_params d;
    amgt_boomer_default_params(&d);
    const amgt_boomer_params &p = prm ? *prm : d;
    if (!(p.theta >= 0.0) || p.p_max < 0 || (p.coarsen_type != 10 && p.coarsen_type != 8)) return AMGT_ERR_INVALID;
    for (int i = 0; i < n; ++i)
        if (ia[i] > ia[i + 1] || (ia[i] < ia[i + 1] && ja[ia[i]] != i)) return AMGT_ERR_INVALID;  // diagonal first
    std::vector<int> cf, pi, pj;
    std::vector<double> pa;
    const int nc = boomer_level(n, ia, ja, a, p, cf, pi, pj, pa);
    memset(P, 0, sizeof(*P));
    P->num_rows = n;
    P->num_cols = nc;
    P->num_nonzeros = (int)pj.size();
    P->i = static_cast<int *>(malloc(sizeof(int) * (n + 1)));
    P->j = static_cast<int *>(malloc(sizeof(int) * std::max<size_t>(1, pj.size())));
    P->data = static_cast<double *>(malloc(sizeof(double) * std::max<size_t>(1, pa.size())));
    if (!P->i || !P->j || !P->data) {
        amgt_boomer_free_host(P);
        return AMGT_ERR_ALLOC;
    }
    memcpy(P->i, pi.data(), sizeof(int) * (n + 1));
    if (!pj.empty()) {
        memcpy(P->j, pj.data(), sizeof(int) * pj.size());
        memcpy(P->data, pa.data(), sizeof(double) * pa.size());
    }
    if (cf_marker) memcpy(cf_marker, cf.data(), sizeof(int) * n);
    return AMGT_OK;
}

int amgt_boomer_interp(const amgt_bsr *A, const amgt_boomer_params *prm, amgt_csr *P, int *cf_marker,
                       amgt_stream_t stream)
{
    if (!A || !P || A->row <= 0 || A->row != A->col) return AMGT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    amgt_csr C{};
    AMGT_TRY(amgt_bsr_to_csr(A, &C, stream));
    const int n = C.num_rows;
    std::vector<int> ia(n + 1), ja(C.num_nonzeros);
    std::vector<double> a(C.num_nonzeros);
    cudaError_t e = cudaMemcpyAsync(ia.data(), C.i, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && C.num_nonzeros > 0)
        e = cudaMemcpyAsync(ja.data(), C.j, sizeof(int) * C.num_nonzeros, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && C.num_nonzeros > 0)
        e = cudaMemcpyAsync(a.data(), C.data, sizeof(double) * C.num_nonzeros, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    amgt_csr_free(&C, stream);
    AMGT_CUDA_TRY(e);
    // HYPRE's storage: the diagonal first, the other columns ascending
    for (int i = 0; i < n; ++i) {
        int d = -1;
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] == i) d = k;
        if (d < 0) return AMGT_ERR_INVALID;  // no stored diagonal
        for (int k = d; k > ia[i]; --k) {
            std::swap(ja[k], ja[k - 1]);
            std::swap(a[k], a[k - 1]);
        }
    }
    amgt_csr H{};
    AMGT_TRY(amgt_boomer_coarsen_host(n, ia.data(), ja.data(), a.data(), prm, cf_marker, &H));
    memset(P, 0, sizeof(*P));
    int rc = AMGT_OK;
    if ((rc = alloc_n(&P->i, (size_t)n + 1, s)) || (rc = alloc_n(&P->j, (size_t)H.num_nonzeros, s)) ||
        (rc = alloc_n(&P->data, (size_t)H.num_nonzeros, s))) {
        amgt_csr_free(P, stream);
        amgt_boomer_free_host(&H);
        return rc;
    }
    P->num_rows = n;
    P->num_cols = H.num_cols;
    P->num_nonzeros = H.num_nonzeros;
    e = cudaMemcpyAsync(P->i, H.i, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && H.num_nonzeros > 0)
        e = cudaMemcpyAsync(P->j, H.j, sizeof(int) * H.num_nonzeros, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && H.num_nonzeros > 0)
        e = cudaMemcpyAsync(P->data, H.data, sizeof(double) * H.num_nonzeros, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host arrays are freed next
    amgt_boomer_free_host(&H);
    if (e != cudaSuccess) {
        amgt_csr_free(P, stream);
        AMGT_CUDA_TRY(e);
    }
    return AMGT_OK;
}

int amgt_boomer_free_host(amgt_csr *P)
{
    if (!P) return AMGT_ERR_INVALID;
    free(P->i);
    free(P->j);
    free(P->data);
    memset(P, 0, sizeof(*P));
    return AMGT_OK;
}

void amgt_boomer_default_params(amgt_boomer_params *p)
{
    if (!p) return;
    p->theta = 0.25;
    p->max_row_sum = 1.0;
    p->p_max = 4;
    p->coarsen_type = 10;
}

struct amgt_boomer_hier {
    std::vector<HostCsr> A, P;
};

int amgt_boomer_hierarchy_host(int n, const int *ia, const int *ja, const double *a, const amgt_boomer_params *prm,
                               int max_levels, int max_coarse, amgt_boomer_hier **out)
{
    if (!out) return AMGT_ERR_INVALID;
    *out = nullptr;
    if (n <= 0 || !ia || !ja || !a || max_levels < 1 || max_coarse < 1) return AMGT_ERR_INVALID;
    amgt_boomer_params d;
    amgt_boomer_default_params(&d);
    const amgt_boomer_params &p = prm ? *prm : d;
    if (!(p.theta >= 0.0) || p.p_max < 0 || (p.coarsen_type != 10 && p.coarsen_type != 8)) return AMGT_ERR_INVALID;
    if (ia[0] != 0) return AMGT_ERR_INVALID;
    for (int i = 0; i < n; ++i) {
        if (ia[i] > ia[i + 1] || ia[i] == ia[i + 1] || ja[ia[i]] != i) return AMGT_ERR_INVALID;  // diagonal first
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] < 0 || ja[k] >= n) return AMGT_ERR_INVALID;
    }
    HostCsr A0;
    A0.rows = A0.cols = n;
    A0.i.assign(ia, ia + n + 1);
    A0.j.assign(ja, ja + ia[n]);
    A0.a.assign(a, a + ia[n]);
    amgt_boomer_hier *h = new (std::nothrow) amgt_boomer_hier;
    if (!h) return AMGT_ERR_ALLOC;
    int rc;
    try {
        rc = boomer_hierarchy(A0, p, max_levels, max_coarse, h->A, h->P);
    } catch (const std::bad_alloc &) {
        rc = AMGT_ERR_ALLOC;
    }
    if (rc != AMGT_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return AMGT_OK;
}

int amgt_boomer_hierarchy_levels(const amgt_boomer_hier *h) { return h ? (int)h->A.size() : 0; }

int amgt_boomer_hierarchy_level(const amgt_boomer_hier *h, int l, amgt_csr *A, amgt_csr *P)
{
    if (!h || l < 0 || l >= (int)h->A.size()) return AMGT_ERR_INVALID;
    auto view = [](const HostCsr &M, amgt_csr *v) {
        v->num_rows = M.rows;
        v->num_cols = M.cols;
        v->num_nonzeros = (int)M.j.size();
        v->i = const_cast<int *>(M.i.data());
        v->j = const_cast<int *>(M.j.data());
        v->data = const_cast<double *>(M.a.data());
    };
    if (A) view(h->A[l], A);
    if (P) {
        memset(P, 0, sizeof(*P));
        if (l < (int)h->P.size()) view(h->P[l], P);
    }
    return AMGT_OK;
}

void amgt_boomer_hierarchy_free(amgt_boomer_hier *h) { delete h; }

}  // extern "C"
