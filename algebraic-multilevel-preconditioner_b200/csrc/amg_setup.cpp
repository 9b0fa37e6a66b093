// Host setup of the AMG local solver (--local-approx amg): the hierarchy of one local matrix, as
// the reference's AMGCL setup builds it (src/linalg/inexact_solver.cpp:45-178, builtin backend,
// default parameters), for callers without Python (the C++ drop-in builds each rank's hierarchy
// with it).  The same algorithms as s2l_b200/amg.py, with the same arithmetic and order, so both
// give identical hierarchies:
//   smoothed aggregation: strength eps^2 a_ii a_jj < a_ij^2 (eps = 0.08f, halved per level), plain
//     aggregation in row order, tentative P = 1 smoothed with omega = 2/3 on the filtered matrix;
//   Ruge-Stuben: negative strong couplings (0.25), C/F splitting by decreasing measure in AMGCL's
//     bucket order, direct interpolation truncated at 0.2 and rescaled;
//   R = P^T, coarse operator R (A P) by row-wise products that drop exact zeros;
//   levels while a level has more than coarse_enough rows, the last one kept dense.
// No device is used.
#include "s2l_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <new>
#include <vector>

namespace {

// Every step runs in the precision Real of the setup: double, or float for the reference's
// --local-precision single (AMGCL's builtin<float> backend computes its whole setup in float).
template <typename Real>
struct CsrT {
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<Real> v;
};
using Csr = CsrT<double>;

template <typename Real, typename From>
CsrT<Real> convert(const CsrT<From>& A)
{
    CsrT<Real> B;
    B.rows = A.rows;
    B.cols = A.cols;
    B.rp = A.rp;
    B.ci = A.ci;
    B.v.assign(A.v.begin(), A.v.end());
    return B;
}

constexpr int kUndef = -1, kRemoved = -2;
// AMGCL detail::eps<Real>(1): twice the machine epsilon of the precision
template <typename Real>
constexpr Real tiny()
{
    return Real(2) * std::numeric_limits<Real>::epsilon();
}

// C = A B (rows of A times B), accumulated in A's row order then B's, exact zeros dropped, columns
// sorted
template <typename Real>
CsrT<Real> product(const CsrT<Real>& A, const CsrT<Real>& B)
{
    CsrT<Real> C;
    C.rows = A.rows;
    C.cols = B.cols;
    C.rp.assign((size_t)A.rows + 1, 0);
    std::vector<Real> sums((size_t)B.cols, Real(0));
    std::vector<int64_t> mark((size_t)B.cols, -1);
    std::vector<int32_t> cols;
    for (int64_t i = 0; i < A.rows; ++i) {
        cols.clear();
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t k = A.ci[e];
            const Real a = A.v[e];
            for (int64_t f = B.rp[k]; f < B.rp[k + 1]; ++f) {
                const int32_t j = B.ci[f];
                sums[j] += a * B.v[f];
                if (mark[j] != i) {
                    mark[j] = i;
                    cols.push_back(j);
                }
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int32_t j : cols) {
            if (sums[j] != Real(0)) {
                C.ci.push_back(j);
                C.v.push_back(sums[j]);
            }
            sums[j] = Real(0);
        }
        C.rp[i + 1] = (int64_t)C.ci.size();
    }
    return C;
}

template <typename Real>
CsrT<Real> transpose(const CsrT<Real>& P)
{
    CsrT<Real> R;
    R.rows = P.cols;
    R.cols = P.rows;
    R.rp.assign((size_t)P.cols + 1, 0);
    for (int32_t c : P.ci) ++R.rp[c + 1];
    for (int64_t k = 0; k < P.cols; ++k) R.rp[k + 1] += R.rp[k];
    R.ci.resize(P.ci.size());
    R.v.resize(P.v.size());
    std::vector<int64_t> fill(R.rp.begin(), R.rp.end() - 1);
    for (int64_t i = 0; i < P.rows; ++i)
        for (int64_t e = P.rp[i]; e < P.rp[i + 1]; ++e) {
            const int64_t q = fill[P.ci[e]]++;
            R.ci[q] = (int32_t)i;
            R.v[q] = P.v[e];
        }
    return R;
}

// ---------------------------------------------------------------- smoothed aggregation
// P of one level, false when no row has a strong connection
template <typename Real>
bool sa_transfer(const CsrT<Real>& A, float eps, CsrT<Real>& P)
{
    const int64_t n = A.rows;
    const Real eps2 = (Real)(eps * eps);  // the product of two floats, in float
    std::vector<Real> dia((size_t)n, Real(0));
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e)
            if (A.ci[e] == i) dia[i] = A.v[e];
    std::vector<char> strong(A.ci.size(), 0);
    std::vector<int> aid((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        bool any = false;
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t c = A.ci[e];
            const Real v = A.v[e];
            strong[e] = c != i && (eps2 * dia[i]) * dia[c] < v * v;
            any = any || strong[e];
        }
        aid[i] = any ? kUndef : kRemoved;
    }
    int count = 0;
    std::vector<int32_t> neib;
    for (int64_t i = 0; i < n; ++i) {
        if (aid[i] != kUndef) continue;
        const int cur = count++;
        aid[i] = cur;
        neib.clear();
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t c = A.ci[e];
            if (strong[e] && aid[c] != kRemoved) {
                aid[c] = cur;
                neib.push_back(c);
            }
        }
        for (int32_t c : neib)
            for (int64_t e = A.rp[c]; e < A.rp[c + 1]; ++e)
                if (strong[e] && aid[A.ci[e]] == kUndef) aid[A.ci[e]] = cur;
    }
    if (count == 0) return false;
    // aggregates emptied by later ones: renumber without gaps
    std::vector<int> newid((size_t)count, 0);
    for (int a : aid)
        if (a >= 0) newid[a] = 1;
    int used = 0;
    for (int k = 0; k < count; ++k) newid[k] = newid[k] ? used++ : -1;
    for (int& a : aid)
        if (a >= 0) a = newid[a];
    count = used;
    // P(i, :) = sum over the strong and diagonal entries of row i, in order, of
    // ((1 - omega) on the diagonal, -omega a_ij / d_F(i) elsewhere) P0(j, :)
    const Real omega = Real(1) * Real(2.0 / 3.0);
    P = CsrT<Real>();
    P.rows = n;
    P.cols = count;
    P.rp.assign((size_t)n + 1, 0);
    std::vector<std::pair<int32_t, Real>> acc;
    for (int64_t i = 0; i < n; ++i) {
        Real df = Real(0);  // filtered diagonal: the diagonal plus the weak entries
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e)
            if (!strong[e]) df += A.v[e];
        const Real scale = df != Real(0) ? -omega * (Real(1) / df) : Real(0);
        acc.clear();
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t c = A.ci[e];
            const bool diag = c == i;
            if (!(diag || strong[e]) || aid[c] < 0) continue;
            const Real val = diag ? Real(1) - omega : scale * A.v[e];
            const int32_t t = aid[c];
            auto it = std::find_if(acc.begin(), acc.end(), [t](const std::pair<int32_t, Real>& p) { return p.first == t; });
            if (it == acc.end()) acc.emplace_back(t, val);
            else it->second = it->second + val;
        }
        std::sort(acc.begin(), acc.end());
        for (const auto& p : acc) {
            P.ci.push_back(p.first);
            P.v.push_back(p.second);
        }
        P.rp[i + 1] = (int64_t)P.ci.size();
    }
    return true;
}

// ---------------------------------------------------------------- Ruge-Stuben
enum : char { kU = 0, kF = 1, kC = 2 };

template <typename Real>
bool rs_transfer(const CsrT<Real>& A, CsrT<Real>& P)
{
    const int64_t n = A.rows;
    const Real eps_str = (Real)0.25f, eps_tr = (Real)0.2f;
    const Real kTiny = tiny<Real>();
    std::vector<char> strong(A.ci.size(), 0), cf((size_t)n, kU);
    for (int64_t i = 0; i < n; ++i) {
        Real amin = Real(0);
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e)
            if (A.ci[e] != i) amin = std::min(amin, A.v[e]);
        if (std::fabs(amin) < kTiny) {
            cf[i] = kF;
            continue;
        }
        const Real thr = amin * eps_str;
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) strong[e] = A.ci[e] != i && A.v[e] < thr;
    }
    // transposed strength graph: for column c, the rows depending strongly on it, by row
    std::vector<int64_t> tp((size_t)n + 1, 0);
    for (size_t e = 0; e < A.ci.size(); ++e)
        if (strong[e]) ++tp[A.ci[e] + 1];
    for (int64_t i = 0; i < n; ++i) tp[i + 1] += tp[i];
    std::vector<int32_t> tcol((size_t)tp[n]);
    {
        std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e)
                if (strong[e]) tcol[fill[A.ci[e]]++] = (int32_t)i;
    }
    // C/F splitting by decreasing measure, in groups of equal measure
    std::vector<int64_t> lam((size_t)n, 0);
    int64_t lmax = 0;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t q = tp[i]; q < tp[i + 1]; ++q) lam[i] += cf[tcol[q]] == kU ? 1 : 2;
        lmax = std::max(lmax, lam[i]);
    }
    const int64_t size = std::max(n, lmax + 1);
    std::vector<int64_t> ptr((size_t)size + 1, 0), cnt((size_t)size, 0), i2n((size_t)n), n2i((size_t)n);
    for (int64_t i = 0; i < n; ++i) ++ptr[lam[i] + 1];
    for (int64_t k = 0; k < size; ++k) ptr[k + 1] += ptr[k];
    for (int64_t i = 0; i < n; ++i) {
        const int64_t pos = ptr[lam[i]] + cnt[lam[i]]++;
        i2n[pos] = i;
        n2i[i] = pos;
    }
    auto move = [&](int64_t x, int64_t old_pos, int64_t new_pos) {
        const int64_t y = i2n[new_pos];
        n2i[x] = new_pos;
        n2i[y] = old_pos;
        i2n[old_pos] = y;
        i2n[new_pos] = x;
    };
    for (int64_t top = n - 1; top >= 0; --top) {
        const int64_t i = i2n[top];
        const int64_t li = lam[i];
        if (li == 0) {
            for (auto& m : cf)
                if (m == kU) m = kC;
            break;
        }
        --cnt[li];
        if (cf[i] == kF) continue;
        cf[i] = kC;
        for (int64_t q = tp[i]; q < tp[i + 1]; ++q) {
            const int32_t c = tcol[q];
            if (cf[c] != kU) continue;
            cf[c] = kF;
            for (int64_t e = A.rp[c]; e < A.rp[c + 1]; ++e) {  // what c depends on rises by one
                if (!strong[e]) continue;
                const int32_t a = A.ci[e];
                const int64_t la = lam[a];
                if (cf[a] != kU || la + 1 >= n) continue;
                move(a, n2i[a], ptr[la] + cnt[la] - 1);
                --cnt[la];
                ++cnt[la + 1];
                ptr[la + 1] = ptr[la] + cnt[la];
                lam[a] = la + 1;
            }
        }
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {  // what i depends on drops by one
            if (!strong[e]) continue;
            const int32_t c = A.ci[e];
            const int64_t lc = lam[c];
            if (cf[c] != kU || lc == 0) continue;
            move(c, n2i[c], ptr[lc]);
            --cnt[lc];
            ++cnt[lc - 1];
            ++ptr[lc];
            lam[c] = lc - 1;
        }
    }
    std::vector<int32_t> cidx((size_t)n, 0);
    int32_t nc = 0;
    for (int64_t i = 0; i < n; ++i)
        if (cf[i] == kC) cidx[i] = nc++;
    if (nc == 0) return false;
    // direct interpolation with truncation
    P = CsrT<Real>();
    P.rows = n;
    P.cols = nc;
    P.rp.assign((size_t)n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        if (cf[i] == kC) {
            P.ci.push_back(cidx[i]);
            P.v.push_back(Real(1));
            P.rp[i + 1] = (int64_t)P.ci.size();
            continue;
        }
        Real lo = Real(0), hi = Real(0);
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e)
            if (strong[e] && cf[A.ci[e]] == kC) {
                lo = std::min(lo, A.v[e]);
                hi = std::max(hi, A.v[e]);
            }
        lo *= eps_tr;
        hi *= eps_tr;
        Real dia = 0, a_num = 0, a_den = 0, b_num = 0, b_den = 0, d_neg = 0, d_pos = 0;
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t c = A.ci[e];
            const Real v = A.v[e];
            if (c == i) {
                dia = v;
                continue;
            }
            const bool sc = strong[e] && cf[c] == kC;
            if (v < Real(0)) {
                a_num += v;
                if (sc) {
                    a_den += v;
                    if (lo < v) d_neg += v;
                }
            } else {
                b_num += v;
                if (sc) {
                    b_den += v;
                    if (v < hi) d_pos += v;
                }
            }
        }
        const Real cf_neg = std::fabs(a_den - d_neg) > kTiny ? std::fabs(a_den) / std::fabs(a_den - d_neg) : Real(1);
        const Real cf_pos = std::fabs(b_den - d_pos) > kTiny ? std::fabs(b_den) / std::fabs(b_den - d_pos) : Real(1);
        if (Real(0) < b_num && std::fabs(b_den) < kTiny) dia += b_num;
        const Real alpha =
            std::fabs(a_den) > kTiny ? -cf_neg * std::fabs(a_num) / (std::fabs(dia) * std::fabs(a_den)) : Real(0);
        const Real beta =
            std::fabs(b_den) > kTiny ? -cf_pos * std::fabs(b_num) / (std::fabs(dia) * std::fabs(b_den)) : Real(0);
        for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) {
            const int32_t c = A.ci[e];
            const Real v = A.v[e];
            if (!(strong[e] && cf[c] == kC) || (lo <= v && v <= hi)) continue;
            P.ci.push_back(cidx[c]);
            P.v.push_back((v < Real(0) ? alpha : beta) * v);
        }
        P.rp[i + 1] = (int64_t)P.ci.size();
    }
    return true;
}

int read_csr(int64_t n, const int64_t* rp, const int32_t* ci, const double* v, Csr& A)
{
    if (n <= 0 || n > INT32_MAX || !rp || !ci || !v || rp[0] != 0) return S2L_ERR_BADARG;
    for (int64_t i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i]) return S2L_ERR_BADARG;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
            if (ci[e] < 0 || ci[e] >= n || (e > rp[i] && ci[e] <= ci[e - 1]) || !std::isfinite(v[e]))
                return S2L_ERR_BADARG;
    A.rows = A.cols = n;
    A.rp.assign(rp, rp + n + 1);
    A.ci.assign(ci, ci + rp[n]);
    A.v.assign(v, v + rp[n]);
    return S2L_OK;
}

}  // namespace

struct s2l_amg {
    std::vector<Csr> A, P, R;  // P[l].rows == 0: a last level without a coarser one
    int64_t n_coarse = 0;
    std::vector<double> coarse;  // row-major
    bool single = false;         // computed in float (every value exactly a float)
};

namespace {

template <typename Real>
void finish_coarse(s2l_amg& h, const CsrT<Real>& C)
{
    h.n_coarse = C.rows;
    h.coarse.assign((size_t)(C.rows * C.rows), 0.0);
    for (int64_t i = 0; i < C.rows; ++i)
        for (int64_t e = C.rp[i]; e < C.rp[i + 1]; ++e) h.coarse[(size_t)(i * C.rows + C.ci[e])] = (double)C.v[e];
}

// the levels of A in precision Real (AMGCL's amg constructor): transfer operators while a level
// has more than coarse_enough rows, the last level kept dense
template <typename Real>
void build_levels(CsrT<Real> A, int coarse_enough, int coarsening, s2l_amg& h)
{
    float eps = 0.08f;
    bool have = true, direct = true;
    while (have && A.rows > coarse_enough) {
        CsrT<Real> P;
        const bool ok = coarsening == S2L_AMG_RS ? rs_transfer(A, P) : sa_transfer(A, eps, P);
        eps = eps * 0.5f;
        h.A.push_back(convert<double>(A));
        if (!ok) {  // nothing to coarsen: the last level is smoothed only
            h.P.emplace_back();
            h.R.emplace_back();
            have = false;
            direct = false;
            break;
        }
        CsrT<Real> R = transpose(P);
        A = product(R, product(A, P));
        h.P.push_back(convert<double>(P));
        h.R.push_back(convert<double>(R));
    }
    if (direct) finish_coarse(h, A);
}

// new values on the kept transfer operators of `old` (AMGCL's rebuild), in old's precision
template <typename Real>
void rebuild_levels(const s2l_amg& old, CsrT<Real> A, s2l_amg& h)
{
    bool direct = true;
    for (size_t l = 0; l < old.A.size(); ++l) {
        h.A.push_back(convert<double>(A));
        h.P.push_back(old.P[l]);
        h.R.push_back(old.R[l]);
        if (old.P[l].rows == 0) {
            direct = false;
            break;
        }
        A = product(convert<Real>(old.R[l]), product(A, convert<Real>(old.P[l])));
    }
    if (direct && old.n_coarse > 0) finish_coarse(h, A);
}

}  // namespace

extern "C" {

int s2l_amg_build(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, int coarse_enough,
                  int coarsening, s2l_amg** out)
{
    if (!out) return S2L_ERR_BADARG;
    *out = nullptr;
    const bool single = (coarsening & S2L_AMG_SINGLE) != 0;
    coarsening &= ~S2L_AMG_SINGLE;
    if (coarse_enough < 1 || (coarsening != S2L_AMG_SA && coarsening != S2L_AMG_RS)) return S2L_ERR_BADARG;
    Csr A;
    const int rc = read_csr(n, rowptr, col, val, A);
    if (rc != S2L_OK) return rc;
    std::unique_ptr<s2l_amg> h(new (std::nothrow) s2l_amg());
    if (!h) return S2L_ERR_OOM;
    h->single = single;
    try {
        if (single) build_levels(convert<float>(A), coarse_enough, coarsening, *h);
        else build_levels(A, coarse_enough, coarsening, *h);
    } catch (const std::bad_alloc&) {
        return S2L_ERR_OOM;
    }
    *out = h.release();
    return S2L_OK;
}

int s2l_amg_rebuild(const s2l_amg* old, const int64_t* rowptr, const int32_t* col, const double* val, s2l_amg** out)
{
    if (!old || !out) return S2L_ERR_BADARG;
    *out = nullptr;
    const int64_t n = old->A.empty() ? old->n_coarse : old->A[0].rows;
    Csr A;
    const int rc = read_csr(n, rowptr, col, val, A);
    if (rc != S2L_OK) return rc;
    if (!old->A.empty()) {  // the same pattern as the level it replaces
        if (A.rp != old->A[0].rp || A.ci != old->A[0].ci) return S2L_ERR_BADARG;
    }
    std::unique_ptr<s2l_amg> h(new (std::nothrow) s2l_amg());
    if (!h) return S2L_ERR_OOM;
    h->single = old->single;
    try {
        if (old->single) rebuild_levels(*old, convert<float>(A), *h);
        else rebuild_levels(*old, A, *h);
    } catch (const std::bad_alloc&) {
        return S2L_ERR_OOM;
    }
    *out = h.release();
    return S2L_OK;
}

int s2l_amg_shape(const s2l_amg* h, int* nlev, int64_t* n_coarse)
{
    if (!h || !nlev || !n_coarse) return S2L_ERR_BADARG;
    *nlev = (int)h->A.size();
    *n_coarse = h->n_coarse;
    return S2L_OK;
}

int s2l_amg_matrix(const s2l_amg* h, int level, int which, int64_t* rows, int64_t* cols, const int64_t** rowptr,
                   const int32_t** col, const double** val)
{
    if (!h || !rows || !cols || !rowptr || !col || !val || level < 0 || level >= (int)h->A.size() || which < 0 ||
        which > 2)
        return S2L_ERR_BADARG;
    const Csr& M = which == 0 ? h->A[level] : (which == 1 ? h->P[level] : h->R[level]);
    *rows = M.rows;
    *cols = M.cols;
    *rowptr = M.rows ? M.rp.data() : nullptr;
    *col = M.ci.empty() ? nullptr : M.ci.data();
    *val = M.v.empty() ? nullptr : M.v.data();
    return S2L_OK;
}

int s2l_amg_coarse(const s2l_amg* h, const double** dense)
{
    if (!h || !dense) return S2L_ERR_BADARG;
    *dense = h->n_coarse ? h->coarse.data() : nullptr;
    return S2L_OK;
}

int s2l_amg_free(s2l_amg* h)
{
    delete h;
    return S2L_OK;
}

}  // extern "C"
