// Numeric refactorization of the local factors on their kept patterns, and the refresh of the
// coarse matrix, on the device (s2l_gpu_refactor).
//
// The reference's UpdateLevel::Refactorize (include/preconditioner/preconditioner.hpp:15-30,
// src/preconditioner/two_level_schwarz.cpp:30-41): refill A_ii with the new values
// (Subdomain::refillValues, src/partition/subdomain.cpp:107-127), numeric factorization with the
// symbolic analysis kept (LocalSolver::refactorize, src/linalg/local_solver.cpp:111-118), and
// A_00 = W^T A W with the old coarse basis (CoarseSpace::refresh,
// src/preconditioner/coarse_space.cpp:95-105, 186-206).
//
// Work split of one subdomain with solve split T (rows [0, T) sparse, [T, n) dense tail):
//  1. fill: F = 0, then the entries of P_in A_ii Q at their positions in the factor pattern;
//  2. sparse columns j < T, left-looking, one CTA per subdomain walking the columns' dependency
//     levels (a column needs the columns k of its U part, or of its row of L for L L^T), one
//     warp per column, its k in increasing order, the lanes over the rows of column k;
//  3. tail columns j >= T: the same updates from the sparse columns only (k < T), one warp per
//     column, all columns independent; the tail block of F then holds the Schur complement S;
//  4. S gathered dense (the caller factorizes it with cuSOLVER and inverts its triangles for the
//     solve's dense tails).
// Every column is reduced by one warp in a fixed order, so the result does not depend on timing.
#include "s2l_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

namespace cg = cooperative_groups;

namespace {

// position of row i in the column [c0, c1) of F (rows increasing); the pattern is closed under
// elimination, so the row is there
__device__ __forceinline__ int64_t find_row(const int32_t* __restrict__ fri, int64_t c0, int64_t c1, int i)
{
    int64_t lo = c0, hi = c1 - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(fri + mid) < i) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void set_err(int* err, int code)
{
    atomicCAS(err, 0, code);
}

// dest[off(row of s)] -= F[s] m for the positions s in [b, e), the warp's lanes over s, four
// positions per lane in flight (sources and targets are different columns, targets distinct rows)
template <typename Off>
__device__ __forceinline__ void scatter_segment(const double* __restrict__ F, const int32_t* __restrict__ fri,
                                                int64_t b, int64_t e, double m, double* dest, Off off, int lane)
{
    for (int64_t s = b + lane; s < e; s += 128) {
        int i[4];
        double v[4], t[4];
        int64_t o[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t q = s + 32 * u;
            ok[u] = q < e;
            i[u] = ok[u] ? fri[q] : 0;
            v[u] = ok[u] ? F[q] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) o[u] = ok[u] ? off(i[u]) : 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) t[u] = ok[u] ? dest[o[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (ok[u]) dest[o[u]] = t[u] - v[u] * m;
    }
}

// Where a row lands in column j (offsets from the column's first position): rows >= T (the tail
// rows, where the long coupling segments land) through the warp's map, filled here; rows < T by
// binary search among the column's rows < T.
struct ColumnView {
    int64_t c0, c1, cT;
    int T;
    const int32_t* fri;
    const uint16_t* map;
    __device__ int64_t operator()(int i) const
    {
        return i >= T ? (int64_t)map[i - T] : find_row(fri, c0, cT, i) - c0;
    }
};

__device__ ColumnView column_view(const RefactorArgs& a, int64_t gj, int T, uint16_t* map, int lane)
{
    ColumnView cv;
    cv.c0 = a.fcp[gj];
    cv.c1 = a.fcp[gj + 1];
    cv.cT = T > 0 ? find_row(a.fri, cv.c0, cv.c1 + 1, T) : cv.c0;  // c1 when every row is < T
    cv.T = T;
    cv.fri = a.fri;
    cv.map = map;
    for (int64_t p = cv.cT + lane; p < cv.c1; p += 32) map[a.fri[p] - T] = (uint16_t)(p - cv.c0);
    __syncwarp();
    return cv;
}

// Updates of local column j (global column gj = loc + j) by the finished columns k < klimit, one warp.
// LU: U(k, j) = x(k) in increasing k, x(rows > k of L(:, k)) -= L(:, k) U(k, j).
// L L^T: x(rows >= j of L(:, k)) -= L(:, k) L(j, k) over the entries L(j, k) of row j.
__device__ void update_column(const RefactorArgs& a, int64_t loc, int64_t fb, int64_t gj, int klimit, int T,
                              uint16_t* map, int lane)
{
    double* __restrict__ F = a.F;
    const ColumnView cv = column_view(a, gj, T, map, lane);
    double* col = F + cv.c0;
    if (a.fllt[gj]) {
        const int64_t r1 = a.frp[gj + 1];
        for (int64_t t = a.frp[gj]; t < r1; ++t) {
            const int k = a.frk[t];
            if (k >= klimit) break;
            const int64_t p = fb + a.frpos[t];
            scatter_segment(F, a.fri, p, a.fcp[loc + k + 1], F[p], col, cv, lane);
            __syncwarp();
        }
    } else {
        const int64_t u1 = cv.c0 + a.fdg[gj];
        for (int64_t t = cv.c0; t < u1; ++t) {
            const int k = a.fri[t];
            if (k >= klimit) break;
            const double u = F[t];  // final: every update from a smaller k is done
            const int64_t gk = loc + k;
            if (u != 0.0) scatter_segment(F, a.fri, a.fcp[gk] + a.fdg[gk] + 1, a.fcp[gk + 1], u, col, cv, lane);
            __syncwarp();
        }
    }
}

// offset of row i in the column whose full row map is m (every row of the subdomain)
struct FullMap {
    const uint16_t* m;
    __device__ int64_t operator()(int i) const { return m[i]; }
};

// The same for one column with every warp of the CTA.  The sum over k is split: for LU the part
// of U(:, j) (rows < j, a sequential triangular solve) is done by warp 0 first; then the updates of
// rows >= j, independent over k, go round-robin to the warps, each into its own partial column
// (part), which are added in a fixed order at the end.  Rows are located through one map of the
// whole column in shared memory (cmap, a row of the subdomain -> offset).  Every thread of the
// CTA calls this.
__device__ void update_column_coop(const RefactorArgs& a, int64_t loc, int64_t fb, int64_t gj, int j,
                                   uint16_t* cmap, double* part, int gw, int nw, int lane, cg::cluster_group& cl)
{
    double* __restrict__ F = a.F;
    const int64_t c0 = a.fcp[gj], c1 = a.fcp[gj + 1];
    const int64_t len = c1 - c0;
    for (int64_t p = c0 + threadIdx.x; p < c1; p += blockDim.x) cmap[a.fri[p]] = (uint16_t)(p - c0);
    const FullMap fm{cmap};
    double* mine = part + (size_t)gw * a.maxcol;
    for (int64_t q = lane; q < len; q += 32) mine[q] = 0.0;
    cl.sync();  // every CTA's column map is complete
    const bool llt = a.fllt[gj];
    const int64_t u0 = c0, u1 = c0 + a.fdg[gj];
    if (!llt && gw == 0) {
        // U(:, j): the rows < j of the segments, in increasing k
        for (int64_t t = u0; t < u1; ++t) {
            const int k = a.fri[t];
            const double u = F[t];
            const int64_t gk = loc + k;
            const int64_t b = a.fcp[gk] + a.fdg[gk] + 1, e = a.fcp[gk + 1];
            const int64_t ej = find_row(a.fri, b, e + 1, j);  // first row >= j
            if (u != 0.0) scatter_segment(F, a.fri, b, ej, u, F + c0, fm, lane);
            __syncwarp();
        }
    }
    cl.sync();
    if (llt) {
        const int64_t r0 = a.frp[gj], r1 = a.frp[gj + 1];
        for (int64_t t = r0 + gw; t < r1; t += nw) {
            const int k = a.frk[t];
            const int64_t p = fb + a.frpos[t];
            scatter_segment(F, a.fri, p, a.fcp[loc + k + 1], F[p], mine, fm, lane);
            __syncwarp();
        }
    } else {
        for (int64_t t = u0 + gw; t < u1; t += nw) {
            const int k = a.fri[t];
            const double u = F[t];
            const int64_t gk = loc + k;
            const int64_t b = a.fcp[gk] + a.fdg[gk] + 1, e = a.fcp[gk + 1];
            const int64_t ej = find_row(a.fri, b, e + 1, j);
            if (u != 0.0) scatter_segment(F, a.fri, ej, e, u, mine, fm, lane);
            __syncwarp();
        }
    }
    cl.sync();
    const int64_t stride = (int64_t)cl.num_blocks() * blockDim.x;
    for (int64_t q = (int64_t)cl.block_rank() * blockDim.x + threadIdx.x; q < len; q += stride) {
        double sum = 0.0;
        for (int w = 0; w < nw; ++w) sum += part[(size_t)w * a.maxcol + q];
        F[c0 + q] += sum;
    }
    cl.sync();
}

// pivot of column gj: LU divides the strict lower part by U(j, j); L L^T takes the square root of
// the diagonal and divides the rows below by it.  LU keeps the setup's pivot order, so a pivot that
// has become small against the entries below it (a multiplier |L(i, j)| > 1 / pivot_tol) is
// reported (error 4): the kept order no longer suits the values and the caller should rebuild.
__device__ void finish_column(const RefactorArgs& a, int64_t gj, int lane)
{
    double* __restrict__ F = a.F;
    const int64_t c0 = a.fcp[gj], c1 = a.fcp[gj + 1];
    const int64_t pd = c0 + a.fdg[gj];
    const double d = F[pd];
    __syncwarp();
    if (a.fllt[gj]) {
        if (!(d > 0.0) || !isfinite(d)) {
            if (lane == 0) set_err(a.err, 1);
            return;
        }
        const double r = sqrt(d);
        const double ri = 1.0 / r;
        if (lane == 0) F[pd] = r;
        for (int64_t s = pd + 1 + lane; s < c1; s += 32) F[s] *= ri;
    } else {
        if (d == 0.0 || !isfinite(d)) {
            if (lane == 0) set_err(a.err, 1);
            return;
        }
        if (a.pivot_tol > 0.0) {
            double mx = 0.0;
            for (int64_t s = pd + 1 + lane; s < c1; s += 32) mx = fmax(mx, fabs(F[s]));
            for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0 && a.pivot_tol * mx > fabs(d)) set_err(a.err, 4);
        }
        const double di = 1.0 / d;
        for (int64_t s = pd + 1 + lane; s < c1; s += 32) F[s] *= di;
    }
    __syncwarp();
}

__global__ void fill_kernel(int64_t count, const int64_t* __restrict__ src, const int64_t* __restrict__ dst,
                            const double* __restrict__ val, double* __restrict__ F)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x)
        F[dst[e]] = val[src[e]];
}

// one CTA per subdomain: the sparse columns level by level
__global__ void __launch_bounds__(1024, 1) sparse_columns_kernel(const RefactorArgs a)
{
    extern __shared__ uint16_t rmap[];
    cg::cluster_group cl = cg::this_cluster();
    const int cs = (int)cl.num_blocks();
    const int sid = blockIdx.x / cs;
    const int64_t loc = a.subs[sid].loc_off, fb = a.fbase[sid];
    const int T = a.subs[sid].T;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = cs * (int)(blockDim.x >> 5);                        // warps of the cluster
    const int gw = (int)cl.block_rank() * (int)(blockDim.x >> 5) + wid;  // this warp among them
    uint16_t* map = rmap + (size_t)wid * a.smax;
    double* part = a.part + (size_t)sid * nw * a.maxcol;
    // Control flow is the same in every CTA of the cluster, so every thread reaches every
    // cluster barrier; a failed pivot only sets the error word (every loop is bounded).
    for (int lv = a.lv_first[sid]; lv < a.lv_first[sid + 1]; ++lv) {
        const int64_t e0 = a.lv_off[lv], e1 = a.lv_off[lv + 1];
        if (e1 - e0 <= nw / 4) {
            // few columns (the chains near the top of the sparse part): each with the whole cluster
            for (int64_t c = e0; c < e1; ++c) {
                const int j = a.lv_col[c];
                update_column_coop(a, loc, fb, loc + j, j, rmap, part, gw, nw, lane, cl);
                if (gw == 0) finish_column(a, loc + j, lane);
                cl.sync();
            }
        } else {
            for (int64_t c = e0 + gw; c < e1; c += nw) {
                const int j = a.lv_col[c];
                update_column(a, loc, fb, loc + j, j, T, map, lane);
                finish_column(a, loc + j, lane);
            }
        }
        cl.sync();
    }
}

// The multipliers of an LU dense tail factored without pivoting (column-major S^T = L' U', L' in
// the strict lower part): error 4 when one exceeds 1 / tol in magnitude (a pivot that is small
// against its row of S).
__global__ void __launch_bounds__(256) tail_growth_kernel(const double* __restrict__ S, int s, double tol,
                                                          int* err)
{
    const int64_t total = (int64_t)s * s;
    bool bad = false;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / s, i = e - j * s;  // column-major: row i of column j
        if (i > j && tol * fabs(S[e]) > 1.0) bad = true;
    }
    if (bad) set_err(err, 4);
}

// one warp per tail column: the updates from the sparse columns (k < T)
__global__ void __launch_bounds__(256) tail_columns_kernel(const RefactorArgs a)
{
    extern __shared__ uint16_t rmap[];
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= a.ntc) return;
    const int sid = a.tc_sub[w];
    const DevSub& d = a.subs[sid];
    update_column(a, d.loc_off, a.fbase[sid], d.loc_off + a.tc_col[w], d.T, d.T,
                  rmap + (size_t)(threadIdx.x >> 5) * a.smax, lane);
}

// one warp per tail column: its rows >= T into the dense tail (mirrored for L L^T)
__global__ void __launch_bounds__(256) gather_tails_kernel(const RefactorArgs a)
{
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= a.ntc) return;
    const int sid = a.tc_sub[w];
    const DevSub& d = a.subs[sid];
    const int T = d.T, s = d.n_local - T;
    const int j = a.tc_col[w];
    const int64_t gj = d.loc_off + j;
    double* S = a.S + d.d_off;
    const bool llt = a.fllt[gj];
    for (int64_t p = a.fcp[gj] + lane; p < a.fcp[gj + 1]; p += 32) {
        const int i = a.fri[p];
        if (i < T) continue;
        const double v = a.F[p];
        S[(int64_t)(i - T) * s + (j - T)] = v;
        if (llt && i != j) S[(int64_t)(j - T) * s + (i - T)] = v;
    }
}

// The solve's dense tail inverses from inverted triangles (row-major views of column-major
// results): S holds the inverted upper triangle (column-major), i.e. row-major lower part with the
// diagonal = Lt^-1; B (LU only) holds the inverted unit lower triangle, row-major strict upper part
// = Ut^-1 with a unit diagonal; for L L^T Ut^-1 = (Lt^-1)^T.  The other triangles are 0.
template <typename Real>
__global__ void tail_inverses_kernel(const double* __restrict__ S, const double* __restrict__ B, int s, int llt,
                                     Real* __restrict__ linv, Real* __restrict__ uinv)
{
    const int64_t total = (int64_t)s * s;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / s), c = (int)(e % s);
        linv[e] = (Real)(c <= r ? S[e] : 0.0);
        double u;
        if (llt) u = c >= r ? S[(int64_t)c * s + r] : 0.0;
        else u = c > r ? B[e] : (c == r ? 1.0 : 0.0);
        uinv[e] = (Real)u;
    }
}

__global__ void identity_kernel(double* M, int s)
{
    const int64_t total = (int64_t)s * s;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
        M[e] = (e / s == e % s) ? 1.0 : 0.0;
}

// packed sweep values: one warp per (subdomain, sweep warp) walking its tasks in the layout of
// the sweep; entry value = F(src) / diagonal of its row (padding 0, chain-block rows skipped)
template <typename Real>
__global__ void __launch_bounds__(256) sweep_values_kernel(int nsub, const int64_t* __restrict__ fbase,
                                                           const double* __restrict__ F,
                                                           const int64_t* __restrict__ wtask,
                                                           const int64_t* __restrict__ wslot,
                                                           const int64_t* __restrict__ went,
                                                           const uint32_t* __restrict__ thdr,
                                                           const int32_t* __restrict__ tslot,
                                                           const int32_t* __restrict__ src,
                                                           const DevSub* __restrict__ subs,
                                                           const int32_t* __restrict__ dsrc, Real* __restrict__ val)
{
    const int64_t wi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (wi >= (int64_t)nsub * S2L_SWEEP_WARPS) return;
    const int sid = (int)(wi / S2L_SWEEP_WARPS);
    const int64_t fb = fbase[sid], lo = subs[sid].loc_off;
    int64_t so = wslot[wi], eo = went[wi];
    for (int64_t t = wtask[wi]; t < wtask[wi + 1]; ++t) {
        const uint32_t h = thdr[t];
        const int C = (int)(h & 0xFFFFu), gl2 = (int)((h >> 16) & 7u), R = (int)((h >> 19) & 31u) + 1;
        const int k = lane >> gl2;
        double di = 0.0;  // 1 / diagonal of the lane's row, in FP64 as at setup
        if (k < R) {
            const int32_t q = dsrc[lo + tslot[so + k]];
            di = q >= 0 ? 1.0 / F[fb + q] : 1.0;
        }
        so += R;
        for (int c = 0; c < C; ++c) {
            const int64_t e = eo + (int64_t)c * 32 + lane;
            const int32_t p = src[e];
            if (p >= 0) val[e] = (Real)(F[fb + p] * di);
            else if (p == -1) val[e] = Real(0);
        }
        eo += (int64_t)C * 32;
    }
}

// 1 / diagonal per slot (1 where the source is -1: unit diagonals, chain-block rows, tail rows)
template <typename Real>
__global__ void dinv_kernel(int nsub, const DevSub* __restrict__ subs, const int64_t* __restrict__ fbase,
                            const double* __restrict__ F, const int32_t* __restrict__ dsrc, Real* __restrict__ dinv)
{
    const int sid = blockIdx.y;
    const DevSub& d = subs[sid];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.n_local; p += gridDim.x * blockDim.x) {
        const int32_t q = dsrc[d.loc_off + p];
        dinv[d.loc_off + p] = q >= 0 ? (Real)(1.0 / F[fbase[sid] + q]) : Real(1);
    }
}

// chain blocks: W from F, W^-1 by forward substitution (as at setup), and the rewritten rows
// sum_b W^-1(a, b) M(B[b], c); one warp per block
template <typename Real>
__global__ void __launch_bounds__(256) blocks_kernel(int64_t nblocks, const int64_t* __restrict__ boff,
                                                     const int64_t* __restrict__ bioff,
                                                     const int64_t* __restrict__ wsrc,
                                                     const int64_t* __restrict__ be_off,
                                                     const int64_t* __restrict__ be_pos,
                                                     const uint8_t* __restrict__ be_row,
                                                     const int64_t* __restrict__ be_cp,
                                                     const uint8_t* __restrict__ bc_b,
                                                     const int64_t* __restrict__ bc_pos, const double* __restrict__ F,
                                                     Real* __restrict__ binv, Real* __restrict__ val)
{
    __shared__ double wsh[8][S2L_CHAIN_MAX * (S2L_CHAIN_MAX + 1) / 2 * 2];
    const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, wl = (threadIdx.x >> 5) & 7;
    if (b >= nblocks) return;
    const int k = (int)(boff[b + 1] - boff[b]);
    const int np = k * (k + 1) / 2;
    double* W = wsh[wl];
    double* Wi = W + np;
    const int64_t io = bioff[b];
    for (int e = lane; e < np; e += 32) {
        int i = 0;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        const int j = e - i * (i + 1) / 2;
        const int64_t q = wsrc[io + e];
        W[e] = q >= 0 ? F[q] : (i == j ? 1.0 : 0.0);
    }
    __syncwarp();
    if (lane == 0) {
        // Wi = W^-1, column by column (lower, packed row-major)
        for (int j = 0; j < k; ++j)
            for (int i = j; i < k; ++i) {
                double v = i == j ? 1.0 : 0.0;
                for (int q = j; q < i; ++q) v -= W[i * (i + 1) / 2 + q] * Wi[q * (q + 1) / 2 + j];
                Wi[i * (i + 1) / 2 + j] = v / W[i * (i + 1) / 2 + i];
            }
    }
    __syncwarp();
    for (int e = lane; e < np; e += 32) binv[io + e] = (Real)Wi[e];
    for (int64_t e = be_off[b] + lane; e < be_off[b + 1]; e += 32) {
        const int arow = be_row[e];
        double v = 0.0;
        for (int64_t c = be_cp[e]; c < be_cp[e + 1]; ++c) v += Wi[arow * (arow + 1) / 2 + bc_b[c]] * F[bc_pos[c]];
        val[be_pos[e]] = (Real)v;
    }
}

template <typename Real>
__global__ void gather_values_kernel(int64_t count, const int64_t* __restrict__ src, const double* __restrict__ F,
                                     Real* __restrict__ out)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = (Real)F[src[e]];
}

// A 1 in row order (the same summation order as the host's)
__global__ void row_sums_kernel(int64_t n, const int32_t* __restrict__ rp, const double* __restrict__ v,
                                double* __restrict__ out)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t e = rp[r]; e < rp[r + 1]; ++e) s += v[e];
        out[r] = s;
    }
}

// Y (n0 x 16 interleaved) = columns c0 .. c0 + 15 of the identity
__global__ void unit_block_kernel(int64_t n0, int c0, double* Y)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n0 * 16; e += (int64_t)gridDim.x * blockDim.x)
        Y[e] = (e / 16 == c0 + e % 16) ? 1.0 : 0.0;
}

// E(:, c0 + r) = C(:, r) for the columns inside [0, n0) (E row-major)
__global__ void scatter_columns_kernel(int64_t n0, int c0, const double* C, double* E)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n0 * 16; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = e / 16;
        const int col = c0 + (int)(e % 16);
        if (col < n0) E[row * n0 + col] = C[e];
    }
}

// Coarse matrix E = W^T A W for a boolean partition of unity, where column (i, a) of W is
// V_i(:, a) on the owned rows of subdomain i.  Step 1, per row r: for every subdomain i owning a
// column of the row, u_{r,i} = sum over the entries (r, c), c owned by i, of A(r, c) V_i(c, :).
__global__ void __launch_bounds__(256) coarse_z_kernel(int64_t n, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci, const double* __restrict__ v,
                                                       const int32_t* __restrict__ owner,
                                                       const int64_t* __restrict__ rs_ptr,
                                                       const int32_t* __restrict__ rs_sub,
                                                       const int64_t* __restrict__ rs_zoff,
                                                       const DevSub* __restrict__ subs, const double* __restrict__ V,
                                                       double* __restrict__ Z)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s0 = rs_ptr[r], s1 = rs_ptr[r + 1];
        for (int64_t q = s0; q < s1; ++q) {
            const int m = subs[rs_sub[q]].m;
            for (int a = 0; a < m; ++a) Z[rs_zoff[q] + a] = 0.0;
        }
        for (int32_t e = rp[r]; e < rp[r + 1]; ++e) {
            const int c = ci[e];
            const int i = owner[c];
            int64_t q = s0;
            while (q + 1 < s1 && rs_sub[q] != i) ++q;
            const DevSub& d = subs[i];
            const double* vr = V + d.v_off + (int64_t)(c - d.begin) * d.m;
            double* z = Z + rs_zoff[q];
            const double av = v[e];
            for (int a = 0; a < d.m; ++a) z[a] += av * vr[a];
        }
    }
}

// Step 2, one CTA per pair (j, i) of subdomains that meet in a row:
// E(c_off_j + b, c_off_i + a) = sum over the owned rows r of j with a slot for i of V_j(r, b) u_{r,i}(a)
__global__ void __launch_bounds__(256) coarse_pairs_kernel(const int32_t* __restrict__ pair_j,
                                                           const int32_t* __restrict__ pair_i,
                                                           const int64_t* __restrict__ pair_ptr,
                                                           const int32_t* __restrict__ pair_rl,
                                                           const int64_t* __restrict__ pair_zoff,
                                                           const DevSub* __restrict__ subs,
                                                           const double* __restrict__ V, const double* __restrict__ Z,
                                                           int64_t n0, double* __restrict__ E)
{
    const int p = blockIdx.x;
    const DevSub dj = subs[pair_j[p]], di = subs[pair_i[p]];
    const int mj = dj.m, mi = di.m;
    const int64_t q0 = pair_ptr[p], q1 = pair_ptr[p + 1];
    for (int o = threadIdx.x; o < mj * mi; o += blockDim.x) {
        const int b = o / mi, a = o % mi;
        double acc = 0.0;
        for (int64_t q = q0; q < q1; ++q) acc += V[dj.v_off + (int64_t)pair_rl[q] * mj + b] * Z[pair_zoff[q] + a];
        E[(dj.c_off + b) * n0 + di.c_off + a] = acc;
    }
}

int grid_for(int64_t work, int bs)
{
    const int64_t g = (work + bs - 1) / bs;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace

namespace s2l {

void launch_refactor_fill(cudaStream_t st, int64_t count, const int64_t* src, const int64_t* dst, const double* val,
                          double* F)
{
    if (count > 0) fill_kernel<<<grid_for(count, 256), 256, 0, st>>>(count, src, dst, val, F);
}

size_t refactor_map_bytes(int smax, int warps)
{
    return (size_t)std::max(smax, 1) * sizeof(uint16_t) * warps;
}

// warps of a sparse-columns CTA: as many as 32 whose row maps fit the shared memory
static int sparse_warps(int smax)
{
    const size_t cap = 220 * 1024;
    int w = 32;
    while (w > 1 && refactor_map_bytes(smax, w) > cap) --w;
    return w;
}

int refactor_sparse_warps(int smax)
{
    return sparse_warps(smax);
}

void launch_refactor_sparse(cudaStream_t st, const RefactorArgs& a, int nsub, int cs)
{
    const int w = sparse_warps(a.smax);
    // the per-warp tail maps, or (cooperative columns) one map of every row of a subdomain
    const size_t smem = std::max(refactor_map_bytes(a.smax, w), (size_t)a.nlmax * sizeof(uint16_t));
    cudaFuncSetAttribute(sparse_columns_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // a cluster of cs CTAs (cs SMs) per subdomain
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nsub * cs));
    cfg.blockDim = dim3((unsigned)(32 * w));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, sparse_columns_kernel, a);
}

void launch_refactor_tail_columns(cudaStream_t st, const RefactorArgs& a)
{
    if (a.ntc <= 0) return;
    const int w = std::min(8, sparse_warps(a.smax));
    const size_t smem = refactor_map_bytes(a.smax, w);
    cudaFuncSetAttribute(tail_columns_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    tail_columns_kernel<<<(int)((a.ntc + w - 1) / w), 32 * w, smem, st>>>(a);
}

void launch_refactor_gather_tails(cudaStream_t st, const RefactorArgs& a)
{
    if (a.ntc > 0) gather_tails_kernel<<<(int)((a.ntc * 32 + 255) / 256), 256, 0, st>>>(a);
}

template <typename Real>
void launch_tail_inverses(cudaStream_t st, const double* S, const double* B, int s, int llt, Real* linv, Real* uinv)
{
    tail_inverses_kernel<Real><<<grid_for((int64_t)s * s, 256), 256, 0, st>>>(S, B, s, llt, linv, uinv);
}

void launch_tail_growth(cudaStream_t st, const double* S, int s, double tol, int* err)
{
    if (s > 1 && tol > 0.0) tail_growth_kernel<<<grid_for((int64_t)s * s, 256), 256, 0, st>>>(S, s, tol, err);
}

void launch_identity(cudaStream_t st, double* M, int s)
{
    identity_kernel<<<grid_for((int64_t)s * s, 256), 256, 0, st>>>(M, s);
}

template <typename Real>
void launch_refactor_sweep_values(cudaStream_t st, int nsub, const int64_t* fbase, const double* F,
                                  const int64_t* wtask, const int64_t* wslot, const int64_t* went,
                                  const uint32_t* thdr, const int32_t* tslot, const int32_t* src, const DevSub* subs,
                                  const int32_t* dsrc, Real* val)
{
    const int64_t warps = (int64_t)nsub * S2L_SWEEP_WARPS;
    sweep_values_kernel<Real><<<(int)((warps * 32 + 255) / 256), 256, 0, st>>>(nsub, fbase, F, wtask, wslot, went, thdr,
                                                                             tslot, src, subs, dsrc, val);
}

template <typename Real>
void launch_refactor_dinv(cudaStream_t st, int nsub, const DevSub* subs, const int64_t* fbase, const double* F,
                          const int32_t* dsrc, Real* dinv)
{
    dinv_kernel<Real><<<dim3(16, nsub), 256, 0, st>>>(nsub, subs, fbase, F, dsrc, dinv);
}

template <typename Real>
void launch_refactor_blocks(cudaStream_t st, int64_t nblocks, const int64_t* boff, const int64_t* bioff,
                            const int64_t* wsrc, const int64_t* be_off, const int64_t* be_pos, const uint8_t* be_row,
                            const int64_t* be_cp, const uint8_t* bc_b, const int64_t* bc_pos, const double* F,
                            Real* binv, Real* val)
{
    if (nblocks > 0)
        blocks_kernel<Real><<<(int)((nblocks * 32 + 255) / 256), 256, 0, st>>>(nblocks, boff, bioff, wsrc, be_off,
                                                                               be_pos, be_row, be_cp, bc_b, bc_pos,
                                                                               F, binv, val);
}

template <typename Real>
void launch_gather_values(cudaStream_t st, int64_t count, const int64_t* src, const double* F, Real* out)
{
    if (count > 0) gather_values_kernel<Real><<<grid_for(count, 256), 256, 0, st>>>(count, src, F, out);
}

void launch_row_sums(cudaStream_t st, int64_t n, const int32_t* rp, const double* v, double* out)
{
    row_sums_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, rp, v, out);
}

void launch_coarse_direct(cudaStream_t st, int64_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          const int32_t* owner, const int64_t* rs_ptr, const int32_t* rs_sub, const int64_t* rs_zoff,
                          int npairs, const int32_t* pair_j, const int32_t* pair_i, const int64_t* pair_ptr,
                          const int32_t* pair_rl, const int64_t* pair_zoff, const DevSub* subs, const double* V,
                          double* Z, int64_t n0, double* E)
{
    coarse_z_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, rp, ci, v, owner, rs_ptr, rs_sub, rs_zoff, subs, V, Z);
    cudaMemsetAsync(E, 0, (size_t)n0 * n0 * sizeof(double), st);
    if (npairs > 0)
        coarse_pairs_kernel<<<npairs, 256, 0, st>>>(pair_j, pair_i, pair_ptr, pair_rl, pair_zoff, subs, V, Z, n0, E);
}

void launch_unit_block(cudaStream_t st, int64_t n0, int c0, double* Y)
{
    unit_block_kernel<<<grid_for(n0 * 16, 256), 256, 0, st>>>(n0, c0, Y);
}

void launch_scatter_columns(cudaStream_t st, int64_t n0, int c0, const double* C, double* E)
{
    scatter_columns_kernel<<<grid_for(n0 * 16, 256), 256, 0, st>>>(n0, c0, C, E);
}

template void launch_refactor_sweep_values<double>(cudaStream_t, int, const int64_t*, const double*, const int64_t*,
                                                   const int64_t*, const int64_t*, const uint32_t*, const int32_t*,
                                                   const int32_t*, const DevSub*, const int32_t*, double*);
template void launch_refactor_sweep_values<float>(cudaStream_t, int, const int64_t*, const double*, const int64_t*,
                                                  const int64_t*, const int64_t*, const uint32_t*, const int32_t*,
                                                  const int32_t*, const DevSub*, const int32_t*, float*);
template void launch_refactor_dinv<double>(cudaStream_t, int, const DevSub*, const int64_t*, const double*,
                                           const int32_t*, double*);
template void launch_refactor_dinv<float>(cudaStream_t, int, const DevSub*, const int64_t*, const double*,
                                          const int32_t*, float*);
template void launch_refactor_blocks<double>(cudaStream_t, int64_t, const int64_t*, const int64_t*, const int64_t*,
                                             const int64_t*, const int64_t*, const uint8_t*, const int64_t*,
                                             const uint8_t*, const int64_t*, const double*, double*, double*);
template void launch_refactor_blocks<float>(cudaStream_t, int64_t, const int64_t*, const int64_t*, const int64_t*,
                                            const int64_t*, const int64_t*, const uint8_t*, const int64_t*,
                                            const uint8_t*, const int64_t*, const double*, float*, float*);
template void launch_tail_inverses<double>(cudaStream_t, const double*, const double*, int, int, double*, double*);
template void launch_tail_inverses<float>(cudaStream_t, const double*, const double*, int, int, float*, float*);
template void launch_gather_values<double>(cudaStream_t, int64_t, const int64_t*, const double*, double*);
template void launch_gather_values<float>(cudaStream_t, int64_t, const int64_t*, const double*, float*);

}  // namespace s2l
