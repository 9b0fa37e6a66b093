// sm_100a kernels of the solve phase.
//
// All reductions are deterministic: every reduction-producing kernel runs on a fixed grid of
// S2L_NB_RED blocks, writes one partial per block and column, and reduce_kernel sums them in a
// fixed order.  The same input therefore gives bitwise-identical results, alone or in a batch.
#include "s2l_internal.cuh"

namespace s2l {

namespace {

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the warp, valid in every lane (butterfly)
template <typename Real>
__device__ __forceinline__ Real warp_allsum(Real v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA; the result is valid in thread 0.  sh holds one value per warp.
template <int BS>
__device__ __forceinline__ double block_sum(double v, double* sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < BS / 32) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// ------------------------------------------------------------------------------ SpMV (K1, K10)
// y = A x, or y = b - A x when b != nullptr; with partials, also sum(y^2) per block.
// TPR threads per row (sub-warp groups), grid-stride over rows; the loop is warp-uniform so
// the group shuffles always see the full warp.
template <int TPR>
__global__ void __launch_bounds__(S2L_BS_VEC) spmv_kernel(int64_t n, const int32_t* __restrict__ rp,
                                                          const int32_t* __restrict__ ci,
                                                          const double* __restrict__ v,
                                                          const double* __restrict__ x, double* __restrict__ y,
                                                          const double* __restrict__ b, double* __restrict__ partials)
{
    __shared__ double sh[S2L_BS_VEC / 32];
    const int lane = threadIdx.x % TPR;
    const int64_t g0 = ((int64_t)blockIdx.x * S2L_BS_VEC + threadIdx.x) / TPR;
    const int64_t stride = (int64_t)gridDim.x * (S2L_BS_VEC / TPR);
    double acc = 0.0;
    for (int64_t row = g0; __any_sync(0xffffffffu, row < n); row += stride) {
        double s = 0.0;
        if (row < n) {
            const int e1 = rp[row + 1];
            int e = rp[row] + lane;
            // four entries of the lane at once (loads, then gathers), added in entry order
            for (; e + 3 * TPR < e1; e += 4 * TPR) {
                const int c0 = ci[e], c1 = ci[e + TPR], c2 = ci[e + 2 * TPR], c3 = ci[e + 3 * TPR];
                const double a0 = v[e], a1 = v[e + TPR], a2 = v[e + 2 * TPR], a3 = v[e + 3 * TPR];
                const double x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
                s += a0 * x0;
                s += a1 * x1;
                s += a2 * x2;
                s += a3 * x3;
            }
            for (; e < e1; e += TPR) s += v[e] * __ldg(x + ci[e]);
        }
#pragma unroll
        for (int o = TPR / 2; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && row < n) {
            const double yv = b ? b[row] - s : s;
            y[row] = yv;
            acc += yv * yv;
        }
    }
    if (partials) {
        const double t = block_sum<S2L_BS_VEC>(acc, sh);
        if (threadIdx.x == 0) partials[blockIdx.x] = t;
    }
}

// out[c] = sum over blocks of partials[b * ncols + c]; one warp per column, fixed order.
__global__ void __launch_bounds__(256) reduce_kernel(const double* __restrict__ partials, int nblocks, int ncols,
                                                     double* __restrict__ out)
{
    const int col = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (col >= ncols) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[(int64_t)b * ncols + col];
    s = warp_sum(s);
    if (lane == 0) out[col] = s;
}

// ------------------------------------------------------------------------------ CGS2 (K7)
// h = V(:, 0:k)^T w.  A CTA takes 1024-row tiles (w staged in shared memory), each warp owns the
// columns warp + 8q; partials[b * k + c].
__global__ void __launch_bounds__(256) mdot_kernel(int64_t n, const double* __restrict__ V, int64_t ldv, int k,
                                                   const double* __restrict__ w, double* __restrict__ partials)
{
    __shared__ double ws[1024];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.0;
    for (int64_t t0 = (int64_t)blockIdx.x * 1024; t0 < n; t0 += (int64_t)gridDim.x * 1024) {
        const int cnt = (int)((n - t0) < 1024 ? (n - t0) : 1024);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += 256) ws[i] = w[t0 + i];
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = warp + 8 * q;
            if (c < k) {
                const double* vc = V + (int64_t)c * ldv + t0;
                double s0 = 0.0, s1 = 0.0;
                int i = lane;
                for (; i + 32 < cnt; i += 64) {
                    s0 += vc[i] * ws[i];
                    s1 += vc[i + 32] * ws[i + 32];
                }
                if (i < cnt) s0 += vc[i] * ws[i];
                acc[q] += s0 + s1;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int c = warp + 8 * q;
        if (c < k) {
            const double s = warp_sum(acc[q]);
            if (lane == 0) partials[(int64_t)blockIdx.x * k + c] = s;
        }
    }
}

// w += alpha * V(:, 0:k) h (h on the device); with partials, also sum(w^2) of the new w.
__global__ void __launch_bounds__(256) gemv_update_kernel(int64_t n, const double* __restrict__ V, int64_t ldv, int k,
                                                          const double* __restrict__ h, double alpha,
                                                          double* __restrict__ w, double* __restrict__ partials)
{
    __shared__ double hs[S2L_MAX_RED_COLS];
    __shared__ double sh[8];
    for (int c = threadIdx.x; c < k; c += 256) hs[c] = h[c];
    __syncthreads();
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += V[i + (int64_t)c * ldv] * hs[c];
        const double wn = w[i] + alpha * s;
        w[i] = wn;
        acc += wn * wn;
    }
    if (partials) {
        const double t = block_sum<256>(acc, sh);
        if (threadIdx.x == 0) partials[blockIdx.x] = t;
    }
}

// u = V(:, 0:k) y (y on the device)
__global__ void __launch_bounds__(256) gemv_kernel(int64_t n, const double* __restrict__ V, int64_t ldv, int k,
                                                   const double* __restrict__ y, double* __restrict__ u)
{
    __shared__ double ys[S2L_MAX_RED_COLS];
    for (int c = threadIdx.x; c < k; c += 256) ys[c] = y[c];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += V[i + (int64_t)c * ldv] * ys[c];
        u[i] = s;
    }
}

__global__ void axpby_kernel(int64_t n, double a, const double* __restrict__ x, double b, double* __restrict__ y)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (b == 0.0) ? a * x[i] : a * x[i] + b * y[i];
}

// partials of x.y and (z != nullptr) x.z
__global__ void __launch_bounds__(256) dot2_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                                   const double* __restrict__ z, double* __restrict__ partials)
{
    __shared__ double sh[8];
    double a = 0.0, b = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        a += x[i] * y[i];
        if (z) b += x[i] * z[i];
    }
    const double ta = block_sum<256>(a, sh);
    const double tb = block_sum<256>(b, sh);
    if (threadIdx.x == 0) {
        partials[(int64_t)blockIdx.x * 2] = ta;
        partials[(int64_t)blockIdx.x * 2 + 1] = tb;
    }
}

// ------------------------------------------------------------------------------ OpenFOAM stopping norm
// partials[b * 2 + 0] = sum |a_i - alpha c_i| (c may be nullptr), partials[b * 2 + 1] = sum a_i
__global__ void __launch_bounds__(256) l1_kernel(int64_t n, const double* __restrict__ a, double alpha,
                                                 const double* __restrict__ c, double* __restrict__ partials)
{
    __shared__ double sh[8];
    double s1 = 0.0, s0 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        const double ai = a[i];
        s1 += fabs(c ? ai - alpha * c[i] : ai);
        s0 += ai;
    }
    const double t1 = block_sum<256>(s1, sh);
    const double t0 = block_sum<256>(s0, sh);
    if (threadIdx.x == 0) {
        partials[(int64_t)blockIdx.x * 2] = t1;
        partials[(int64_t)blockIdx.x * 2 + 1] = t0;
    }
}

// partials[b] = sum_i |(V(:, 0:k) q)_i| (q on the device): the 1-norm of a combination of the
// Krylov basis without writing it
__global__ void __launch_bounds__(256) gemv_l1_kernel(int64_t n, const double* __restrict__ V, int64_t ldv, int k,
                                                      const double* __restrict__ q, double* __restrict__ partials)
{
    __shared__ double qs[S2L_MAX_RED_COLS];
    __shared__ double sh[8];
    for (int c = threadIdx.x; c < k; c += 256) qs[c] = q[c];
    __syncthreads();
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += V[i + (int64_t)c * ldv] * qs[c];
        acc += fabs(s);
    }
    const double t = block_sum<256>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// ------------------------------------------------------------------------------ BiCGStab (K9)
__global__ void bicg_p_kernel(int64_t n, const double* __restrict__ r, const double* __restrict__ v, double beta,
                              double omega, double* __restrict__ p, int first)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = first ? r[i] : r[i] + beta * (p[i] - omega * v[i]);
}

// s = r - alpha v; partials: s.s
__global__ void __launch_bounds__(256) bicg_s_kernel(int64_t n, const double* __restrict__ r,
                                                     const double* __restrict__ v, double alpha,
                                                     double* __restrict__ s, double* __restrict__ partials)
{
    __shared__ double sh[8];
    double a = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        const double si = r[i] - alpha * v[i];
        s[i] = si;
        a += si * si;
    }
    const double t = block_sum<256>(a, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// x += alpha y + omega z; r = s - omega t; partials: r.r, rh.r
__global__ void __launch_bounds__(256) bicg_x_kernel(int64_t n, double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ z, double alpha, double omega,
                                                     double* __restrict__ r, const double* __restrict__ s,
                                                     const double* __restrict__ t, const double* __restrict__ rh,
                                                     double* __restrict__ partials)
{
    __shared__ double sh[8];
    double a = 0.0, b = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        x[i] += alpha * y[i] + omega * z[i];
        const double ri = s[i] - omega * t[i];
        r[i] = ri;
        a += ri * ri;
        b += rh[i] * ri;
    }
    const double ta = block_sum<256>(a, sh);
    const double tb = block_sum<256>(b, sh);
    if (threadIdx.x == 0) {
        partials[(int64_t)blockIdx.x * 2] = ta;
        partials[(int64_t)blockIdx.x * 2 + 1] = tb;
    }
}

// ------------------------------------------------------------------------------ local solves (K2, K3)
// Sparse sweep of one factor, one CTA per subdomain, x in shared memory (or, when it does not
// fit, in the local-space buffers with global ready flags).
//
// Rows are slots in solve order (every dependency of slot p is a slot of a lower level).  The rows
// of each level are packed into tasks: a task is R rows of one level with G = 32 / R lanes each
// (G follows the row length), and each warp runs its own list of tasks in level order.  Rows of
// one task never depend on each other, a warp only waits for rows of lower levels, and the lowest
// unfinished level always has its inputs ready, so the sweep cannot deadlock.  A task's entries
// are stored lane-interleaved, so every load is coalesced and its address depends on no loaded
// value; the chunks of a task are loaded in batches (all loads of a batch issued before the first
// wait on a ready flag) and the next batch is hinted into L2.  For each entry a lane waits until
// the ready flag of the column is set; 1/diag is folded into the values and the right-hand side,
// so a row ends with x = b - sum, one write and its flag.  Every wait is bounded: after
// a.spin_limit polls (the setup option "spin_limit", S2L_SPIN_LIMIT by default) the CTA raises
// *err and all warps leave.
// One batch of N chunks of a sweep task for one lane: its N entries (column slot, value) loaded
// together, a wait until all N columns are ready (their flags polled together, one round trip
// per poll), then the N products added in entry order.  With x in shared memory a padding entry
// points at the sentinel slot T (ready, x = 0, value 0), so the batch has no branch per entry; in
// the global-flag layout it is skipped (column >= T).  Returns true when the sweep gave up.
template <typename Real, bool SMEM, int KC, int N>
__device__ __forceinline__ bool sweep_batch(const int32_t* __restrict__ colp, const Real* __restrict__ valp,
                                            volatile const uint8_t* flag, volatile const Real* x, int xstride,
                                            int T, Real (&acc)[KC], volatile int& abort_flag, int* err,
                                            int spin_limit, int sleep_ns)
{
    int lc[N];
    Real lv[N];
#pragma unroll
    for (int q = 0; q < N; ++q) {  // read once: streaming loads, so they do not evict the warp's other lines
        lc[q] = __ldcs(colp + q * 32);
        lv[q] = __ldcs(valp + q * 32);
    }
    int spin = 0;
    for (;;) {
        int ready = 1;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            if (SMEM)
                ready &= (int)flag[lc[q]];
            else if (lc[q] < T)
                ready &= (int)flag[lc[q]];
        }
        if (ready) break;
        if ((++spin & 31) == 0) {  // the abort word and the limit, every 32 polls
            if (abort_flag) return true;
            if (spin > spin_limit) {
                abort_flag = 1;
                atomicExch(err, 1);
                return true;
            }
        }
        // a waiting lane pauses, leaving the issue slots to the warps that compute its columns
        if (sleep_ns > 0) __nanosleep((unsigned)sleep_ns);
    }
#pragma unroll
    for (int q = 0; q < N; ++q) {
        if (SMEM || lc[q] < T) {
#pragma unroll
            for (int r = 0; r < KC; ++r) acc[r] += lv[q] * x[lc[q] * xstride + r];
        }
    }
    return false;
}

template <typename Real, bool SMEM, bool FWD, int KC>
__global__ void __launch_bounds__(S2L_BS_SWEEP, 1) sweep_kernel(const LocalSolveArgs<Real> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int abort_word;
    volatile int& abort_flag = abort_word;
    // chunks per batch: 8 (FP32), 6 (FP64, one column: the registers of 1024 threads), 4 (FP64 blocks)
    constexpr int Q = sizeof(Real) == 4 ? S2L_BATCH_CHUNKS : (KC > 1 ? S2L_BATCH_CHUNKS / 2 : S2L_BATCH_CHUNKS * 3 / 4);
    // KC right-hand sides per CTA: CTA b takes subdomain b / ngrp and columns grp * KC .. + KC of
    // the K interleaved columns (the CTAs of one subdomain are neighbours, so they share the
    // factor stream in L2)
    const int K = a.K;
    const int ngrp = K / KC;
    const int grp = (int)blockIdx.x % ngrp;
    const int g0 = grp * KC;
    const int sidx = (int)blockIdx.x / ngrp;
    const int sid = a.sub_list ? a.sub_list[sidx] : sidx;
    const DevSub sd = a.subs[sid];
    const int64_t lo = sd.loc_off;
    const int T = sd.T;
    const SweepFactor<Real> F = a.f[FWD ? 0 : 1];
    Real* xs;
    volatile uint8_t* flag;
    int xstride;  // x of slot k, column r: xs[k * xstride + r]
    if (SMEM) {
        const size_t off1 = (((size_t)(T + 1) * KC * sizeof(Real)) + 15) & ~(size_t)15;  // T slots + the sentinel
        xs = reinterpret_cast<Real*>(smem_raw);
        flag = reinterpret_cast<volatile uint8_t*>(smem_raw + off1);
        xstride = KC;
    } else {
        xs = (FWD ? a.ybuf : a.xbuf) + lo * K + g0;
        flag = a.gflags + (int64_t)grp * a.nloc + lo;
        xstride = K;
    }
    volatile Real* x = xs;
    if (threadIdx.x == 0) abort_flag = 0;
    // the right-hand side of every slot (scaled by 1/diag): iterations are independent, so four are
    // unrolled to keep their gathers in flight together
#pragma unroll 4
    for (int k = threadIdx.x; k < T; k += S2L_BS_SWEEP) {
        const Real d = F.dinv[lo + k];
        const int64_t src = FWD ? (int64_t)a.gather[lo + k] * K : (lo + a.u2l[lo + k]) * K;
#pragma unroll
        for (int r = 0; r < KC; ++r) {
            const Real b = FWD ? (Real)a.in[src + g0 + r] : a.ybuf[src + g0 + r];
            xs[k * xstride + r] = b * d;
        }
        flag[k] = 0;
    }
    if (SMEM && threadIdx.x == 0) {  // the sentinel slot T of the padding entries: ready, x = 0
#pragma unroll
        for (int r = 0; r < KC; ++r) xs[T * xstride + r] = Real(0);
        flag[T] = 1;
    }
    __syncthreads();
    // chain blocks: right-hand side of block B becomes W^-1 b(B) (W^-1 packed lower, solve order);
    // row i of the block only needs b(0..i), so the rows are overwritten from the last one down
    {
        const int b1 = F.blk_first[sid + 1];
        for (int b = F.blk_first[sid] + threadIdx.x; b < b1; b += S2L_BS_SWEEP) {
            const int64_t o = F.blk_off[b];
            const int k = (int)(F.blk_off[b + 1] - o);
            const Real* W = F.blk_inv + F.blk_ioff[b];
            for (int i = k - 1; i >= 0; --i) {
                const Real* Wi = W + i * (i + 1) / 2;
                Real v[KC];
#pragma unroll
                for (int r = 0; r < KC; ++r) v[r] = Real(0);
                // four entries' loads (slot, W) in flight together, added in entry order
#pragma unroll 4
                for (int j = 0; j <= i; ++j) {
                    const int sj = F.blk_slot[o + j];
#pragma unroll
                    for (int r = 0; r < KC; ++r) v[r] += Wi[j] * xs[sj * xstride + r];
                }
                const int si = F.blk_slot[o + i];
#pragma unroll
                for (int r = 0; r < KC; ++r) xs[si * xstride + r] = v[r];
            }
        }
        __syncthreads();
    }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wi = (int64_t)sid * S2L_SWEEP_WARPS + wid;
    const int64_t t1 = F.wtask[wi + 1];
    int64_t so = F.wslot[wi], eo = F.went[wi];
    const int64_t e_end = F.went[wi + 1];  // the warp's entries are [went[wi], went[wi + 1])
    bool dead = false;
    // task headers 32 at a time: lane j holds the header of task hbase + j (one coalesced load),
    // each task takes its own by a shuffle instead of a load of its own
    int64_t hbase = F.wtask[wi];
    uint32_t hwin = hbase + lane < t1 ? F.thdr[hbase + lane] : 0u;
    for (int64_t t = F.wtask[wi]; t < t1; ++t) {
        if (t - hbase == 32) {  // the same for the whole warp
            hbase = t;
            hwin = hbase + lane < t1 ? F.thdr[hbase + lane] : 0u;
        }
        const uint32_t h = __shfl_sync(0xffffffffu, hwin, (int)(t - hbase));
        const int C = (int)(h & 0xFFFFu), gl2 = (int)((h >> 16) & 7u), R = (int)((h >> 19) & 31u) + 1;
        // the warp's entries are one contiguous stream: hint the first a.sweep_pf chunks after this
        // task (the next tasks' loads) into L2 while this task waits on its ready flags
        if (lane < a.sweep_pf) {
            const int64_t e = eo + (int64_t)(C + lane) * 32;
            if (e < e_end) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.col + e));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e));
                if (sizeof(Real) == 8) asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e + 16));
            }
        }
        const int k = lane >> gl2;
        const int slot = k < R ? F.tslot[so + k] : -1;
        so += R;
        Real acc[KC];
#pragma unroll
        for (int r = 0; r < KC; ++r) acc[r] = Real(0);
        for (int c0 = 0; c0 < C && !dead; c0 += Q) {  // C is the same for the whole warp
            // hint the next batch into L2: lane q < Q takes chunk q of it (lines of 128 bytes)
            if (lane < Q && c0 + Q + lane < C) {
                const int64_t e = eo + (int64_t)(c0 + Q + lane) * 32;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.col + e));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e));
                if (sizeof(Real) == 8) asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e + 16));
            }
            const int64_t e = eo + (int64_t)c0 * 32 + lane;
            const int32_t* cp = F.col + e;
            const Real* vp = F.val + e;
            // a batch of exactly the chunks left (at most Q): no work for absent chunks
            switch (min(C - c0, Q)) {
#define S2L_SWEEP_BATCH(n_)                                                                                        \
    case n_:                                                                                                   \
        if constexpr (n_ <= Q)                                                                                 \
            dead = sweep_batch<Real, SMEM, KC, n_>(cp, vp, flag, x, xstride, T, acc, abort_flag, a.err,         \
                                                   a.spin_limit, a.spin_sleep_ns);                             \
        break;
                S2L_SWEEP_BATCH(1)
                S2L_SWEEP_BATCH(2)
                S2L_SWEEP_BATCH(3)
                S2L_SWEEP_BATCH(4)
                S2L_SWEEP_BATCH(5)
                S2L_SWEEP_BATCH(6)
                S2L_SWEEP_BATCH(7)
                S2L_SWEEP_BATCH(8)
#undef S2L_SWEEP_BATCH
            default: break;
            }
        }
        eo += (int64_t)C * 32;
        dead = __any_sync(0xffffffffu, dead);  // one decision per warp before its shuffles
        if (dead) break;
#pragma unroll
        for (int r = 0; r < KC; ++r)
            for (int o = (1 << gl2) >> 1; o; o >>= 1) acc[r] += __shfl_down_sync(0xffffffffu, acc[r], o, 1 << gl2);
        if ((lane & ((1 << gl2) - 1)) == 0 && slot >= 0) {
#pragma unroll
            for (int r = 0; r < KC; ++r) x[slot * xstride + r] = x[slot * xstride + r] - acc[r];
            __threadfence_block();
            flag[slot] = 1;
        }
    }
    __syncthreads();
    if (FWD) {
        if (SMEM)
            for (int k = threadIdx.x; k < T; k += S2L_BS_SWEEP)
#pragma unroll
                for (int r = 0; r < KC; ++r) a.ybuf[(lo + k) * K + g0 + r] = xs[k * KC + r];
        return;
    }
    // epilogue of the backward sweep: x_local[j] from its backward slot (< T) or tail row (>= T)
    const int n = sd.n_local;
    auto val_at = [&](int q, int r) -> double {
        return q < T ? (double)xs[q * xstride + r] : (double)a.ybuf[(lo + q) * K + g0 + r];
    };
    if (a.mode == 0) {
        for (int j = threadIdx.x; j < sd.n_owned; j += S2L_BS_SWEEP) {
            const int q = a.gout[lo + j];
            const int64_t o = (sd.begin + j) * K + g0;
#pragma unroll
            for (int r = 0; r < KC; ++r) {
                double v = val_at(q, r);
                if (a.base) v += a.base[o + r];
                a.out[o + r] = v;
            }
        }
    } else if (a.mode == 1) {
        for (int j = threadIdx.x; j < n; j += S2L_BS_SWEEP) {
            const int q = a.gout[lo + j];
#pragma unroll
            for (int r = 0; r < KC; ++r) a.ylocal[(lo + j) * K + g0 + r] = val_at(q, r);
        }
    } else {
        for (int j = threadIdx.x; j < n; j += S2L_BS_SWEEP) a.out[j] = val_at(a.gout[lo + j], 0);
    }
}

// v[0..K) = p[0..K) with 16-byte (or 8-byte) loads; p is K-aligned in a block vector, so its byte
// offset is a multiple of K * sizeof(Real)
template <typename Real, int K>
__device__ __forceinline__ void load_k(const Real* __restrict__ p, Real (&v)[K])
{
    if constexpr (sizeof(Real) * K % 16 == 0) {
#pragma unroll
        for (int i = 0; i < (int)(sizeof(Real) * K / 16); ++i) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(p) + i);
            __builtin_memcpy(&v[i * 16 / sizeof(Real)], &t, 16);
        }
    } else if constexpr (sizeof(Real) * K == 8) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        __builtin_memcpy(&v[0], &t, 8);
    } else {
#pragma unroll
        for (int r = 0; r < K; ++r) v[r] = p[r];
    }
}

// acc[r] = sum_e val[e] * x[col[e] * K + r] over e in [e0, e1), one warp; for K = 1 four
// independent gathers are in flight per lane, for K > 1 the K columns give the independence
template <typename Real, int K>
__device__ __forceinline__ void warp_gather_dot(const Real* __restrict__ val, const int32_t* __restrict__ col,
                                                int64_t e0, int64_t e1, const Real* __restrict__ x, int lane,
                                                Real (&acc)[K])
{
    if (K == 1) {
        Real a0 = Real(0), a1 = Real(0), a2 = Real(0), a3 = Real(0);
        int64_t e = e0 + lane;
        for (; e + 96 < e1; e += 128) {
            const int c0 = col[e], c1 = col[e + 32], c2 = col[e + 64], c3 = col[e + 96];
            const Real v0 = val[e], v1 = val[e + 32], v2 = val[e + 64], v3 = val[e + 96];
            a0 += v0 * x[c0];
            a1 += v1 * x[c1];
            a2 += v2 * x[c2];
            a3 += v3 * x[c3];
        }
        for (; e < e1; e += 32) a0 += val[e] * x[col[e]];
        acc[0] = warp_sum((a0 + a1) + (a2 + a3));
    } else {
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] = Real(0);
        int64_t e = e0 + lane;
        for (; e + 96 < e1; e += 128) {  // four entries in flight per lane
            const int c0 = col[e], c1 = col[e + 32], c2 = col[e + 64], c3 = col[e + 96];
            const Real v0 = val[e], v1 = val[e + 32], v2 = val[e + 64], v3 = val[e + 96];
            Real x0[K], x1[K], x2[K], x3[K];
            load_k<Real, K>(x + (int64_t)c0 * K, x0);
            load_k<Real, K>(x + (int64_t)c1 * K, x1);
            load_k<Real, K>(x + (int64_t)c2 * K, x2);
            load_k<Real, K>(x + (int64_t)c3 * K, x3);
#pragma unroll
            for (int r = 0; r < K; ++r) acc[r] += (v0 * x0[r] + v1 * x1[r]) + (v2 * x2[r] + v3 * x3[r]);
        }
        for (; e + 32 < e1; e += 64) {
            const int c0 = col[e], c1 = col[e + 32];
            const Real v0 = val[e], v1 = val[e + 32];
            Real x0[K], x1[K];
            load_k<Real, K>(x + (int64_t)c0 * K, x0);
            load_k<Real, K>(x + (int64_t)c1 * K, x1);
#pragma unroll
            for (int r = 0; r < K; ++r) acc[r] += v0 * x0[r] + v1 * x1[r];
        }
        if (e < e1) {
            const Real v0 = val[e];
            Real x0[K];
            load_k<Real, K>(x + (int64_t)col[e] * K, x0);
#pragma unroll
            for (int r = 0; r < K; ++r) acc[r] += v0 * x0[r];
        }
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] = warp_allsum(acc[r]);  // lane r writes column r
    }
}

// lane r < K gets acc[r] (a register array indexed by a runtime lane)
template <typename Real, int K>
__device__ __forceinline__ Real pick(const Real (&acc)[K], int lane)
{
    Real mine = acc[0];
#pragma unroll
    for (int r = 1; r < K; ++r)
        if (lane == r) mine = acc[r];
    return mine;
}

// Tail right-hand side: t(T+i) = b(T+i) - L(T+i, 0:T) y(0:T), one warp per tail row, K columns.
template <typename Real, int K>
__global__ void __launch_bounds__(256) tail_rhs_kernel(const LocalSolveArgs<Real> a, int q0, int count)
{
    const int q = q0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= q0 + count) return;
    const DevSub sd = a.subs[a.tr_sub[q]];
    const int64_t lo = sd.loc_off;
    const int k = sd.T + a.tr_i[q];
    Real acc[K];
    warp_gather_dot<Real, K>(a.lts_val, a.lts_col, a.lts_ptr[q], a.lts_ptr[q + 1], a.ybuf + lo * K, lane, acc);
    if (lane < K)
        a.ybuf[(lo + k) * K + lane] = (Real)a.in[(int64_t)a.gather[lo + k] * K + lane] - pick<Real, K>(acc, lane);
}

// Dense tail: out(T+i) = sum_j Minv(i, j) in(T+j), j <= i (lower) or j >= i (upper); warp per row,
// K columns (Minv is read once for all of them).  The row is streamed with 16-byte loads (VEC
// entries per lane, two in flight per lane: 1 KB per warp), the few entries before the first
// 16-byte boundary and after the last full vector one per lane.  Every column's sum runs in the same
// order whatever K is.
template <typename Real, bool LOWER, int K>
__global__ void __launch_bounds__(256) tail_gemv_kernel(const LocalSolveArgs<Real> a, const Real* __restrict__ Minv,
                                                        const Real* __restrict__ vin, Real* __restrict__ vout,
                                                        int q0, int count)
{
    constexpr int VEC = 16 / (int)sizeof(Real);
    const int q = q0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= q0 + count) return;
    const DevSub sd = a.subs[a.tr_sub[q]];
    const int s = sd.n_local - sd.T;
    const int i = a.tr_i[q];
    const int64_t base = sd.loc_off + sd.T;
    const Real* row = Minv + sd.d_off + (int64_t)i * s;
    const int j0 = LOWER ? 0 : i, j1 = LOWER ? i + 1 : s;
    const Real* v = vin + base * K;
    Real acc[K];
#pragma unroll
    for (int r = 0; r < K; ++r) acc[r] = Real(0);
    auto fma_entry = [&](Real m, int j) {
        Real x[K];
        load_k<Real, K>(v + (int64_t)j * K, x);
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] += m * x[r];
    };
    // first 16-byte boundary at or after j0 (the allocation is 256-byte aligned)
    const int mis = (int)((reinterpret_cast<uintptr_t>(row + j0) & 15) / sizeof(Real));
    const int ja = mis ? min(j1, j0 + (VEC - mis)) : j0;
    if (j0 + lane < ja) fma_entry(row[j0 + lane], j0 + lane);
    const int nvec = (j1 - ja) / VEC;  // full 16-byte vectors
    const uint4* rv = reinterpret_cast<const uint4*>(row + ja);
    int t = lane;
    for (; t + 32 < nvec; t += 64) {
        const uint4 w0 = __ldg(rv + t), w1 = __ldg(rv + t + 32);
        Real m0[VEC], m1[VEC];
        __builtin_memcpy(m0, &w0, 16);
        __builtin_memcpy(m1, &w1, 16);
#pragma unroll
        for (int u = 0; u < VEC; ++u) fma_entry(m0[u], ja + t * VEC + u);
#pragma unroll
        for (int u = 0; u < VEC; ++u) fma_entry(m1[u], ja + (t + 32) * VEC + u);
    }
    if (t < nvec) {
        const uint4 w0 = __ldg(rv + t);
        Real m0[VEC];
        __builtin_memcpy(m0, &w0, 16);
#pragma unroll
        for (int u = 0; u < VEC; ++u) fma_entry(m0[u], ja + t * VEC + u);
    }
    const int jt = ja + nvec * VEC;  // fewer than VEC entries left
    if (jt + lane < j1) fma_entry(row[jt + lane], jt + lane);
    if (K == 1) {
        const Real sum = warp_sum(acc[0]);
        if (lane == 0) vout[base + i] = sum;
    } else {
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] = warp_allsum(acc[r]);  // lane r writes column r
        if (lane < K) vout[(base + i) * K + lane] = pick<Real, K>(acc, lane);
    }
}

// Backward coupling: y(r) -= U(r, T:n) x(T:n) for the sparse rows that have tail columns, K columns.
// One warp per unit of rows of about the same length (stored longest first): with n rows in the
// unit, G = 32 / n lanes (a power of two) take each row, each lane with four entries in flight,
// and the G partial sums of a row are added by a butterfly within its lane group.
template <typename Real, int K>
__global__ void __launch_bounds__(256) sparse_coupling_kernel(const LocalSolveArgs<Real> a, int u0, int ucount)
{
    const int u = u0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (u >= u0 + ucount) return;
    const int qa = a.uu[u], n = a.uu[u + 1] - qa;  // 1 <= n <= 32
    int lg = 5;
    while ((n << lg) > 32) --lg;  // G = 2^lg lanes per row, the largest with G n <= 32
    const int G = 1 << lg, ri = lane >> lg, sl = lane & (G - 1);
    const bool valid = ri < n;
    const int q = qa + (valid ? ri : 0);
    int64_t e = a.ust_ptr[q] + sl;
    const int64_t e1 = valid ? a.ust_ptr[q + 1] : e;
    Real acc[K];
#pragma unroll
    for (int r = 0; r < K; ++r) acc[r] = Real(0);
    for (; e + 3 * G < e1; e += 4 * G) {
        const int c0 = a.ust_col[e], c1 = a.ust_col[e + G], c2 = a.ust_col[e + 2 * G], c3 = a.ust_col[e + 3 * G];
        const Real v0 = a.ust_val[e], v1 = a.ust_val[e + G], v2 = a.ust_val[e + 2 * G], v3 = a.ust_val[e + 3 * G];
        Real x0[K], x1[K], x2[K], x3[K];
        load_k<Real, K>(a.ybuf + (int64_t)c0 * K, x0);
        load_k<Real, K>(a.ybuf + (int64_t)c1 * K, x1);
        load_k<Real, K>(a.ybuf + (int64_t)c2 * K, x2);
        load_k<Real, K>(a.ybuf + (int64_t)c3 * K, x3);
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] += (v0 * x0[r] + v1 * x1[r]) + (v2 * x2[r] + v3 * x3[r]);
    }
    for (; e < e1; e += G) {
        const Real v0 = a.ust_val[e];
        Real x0[K];
        load_k<Real, K>(a.ybuf + (int64_t)a.ust_col[e] * K, x0);
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] += v0 * x0[r];
    }
#pragma unroll
    for (int r = 0; r < K; ++r)
        for (int o = G >> 1; o; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if (valid && sl == 0) {
        const int64_t o = (a.subs[a.us_sub[q]].loc_off + a.us_r[q]) * K;
#pragma unroll
        for (int r = 0; r < K; ++r) a.ybuf[o + r] -= acc[r];
    }
}

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// out[g] = base[g] + sum over the copies c of g of w_c * ylocal[pos_c] (w = 1 when cp_w is null)
__global__ void combine_kernel(int64_t n, const int64_t* __restrict__ cp_ptr, const int32_t* __restrict__ cp_pos,
                               const double* __restrict__ cp_w, const double* __restrict__ ylocal,
                               const double* __restrict__ base, double* __restrict__ out)
{
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t e = cp_ptr[g]; e < cp_ptr[g + 1]; ++e) s += (cp_w ? cp_w[e] : 1.0) * ylocal[cp_pos[e]];
        out[g] = base ? base[g] + s : s;
    }
}

// ------------------------------------------------------------------------------ coarse space (K4-K6)
__global__ void coarse_reduce_kernel(const DevSub* __restrict__ subs, const int32_t* __restrict__ t_first, int mmax,
                                     const double* __restrict__ partials, double* __restrict__ cvec)
{
    const int i = blockIdx.x;
    const DevSub sd = subs[i];
    for (int c = threadIdx.x; c < sd.m; c += blockDim.x) {
        double s = 0.0;
        for (int t = t_first[i]; t < t_first[i + 1]; ++t) s += partials[(int64_t)t * mmax + c];
        cvec[sd.c_off + c] = s;
    }
}

// y = M x, M dense row-major n0 x n0, one warp per row
__global__ void __launch_bounds__(256) dense_gemv_kernel(int n0, const double* __restrict__ M,
                                                         const double* __restrict__ x, double* __restrict__ y)
{
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n0) return;
    const double* mr = M + (int64_t)row * n0;
    double s = 0.0;
    for (int c = lane; c < n0; c += 32) s += mr[c] * x[c];
    s = warp_sum(s);
    if (lane == 0) y[row] = s;
}

// ------------------------------------------------------------------------------ K right-hand sides
// Block vectors hold K interleaved columns: entry i of column r at i * K + r.

// Y = A X (or B - A X), K columns; with partials, also sum(Y(:, r)^2) per block and column.
template <int TPR, int K>
__global__ void __launch_bounds__(S2L_BS_VEC) spmv_block_kernel(int64_t n, const int32_t* __restrict__ rp,
                                                                const int32_t* __restrict__ ci,
                                                                const double* __restrict__ v,
                                                                const double* __restrict__ X, double* __restrict__ Y,
                                                                const double* __restrict__ B,
                                                                double* __restrict__ partials)
{
    __shared__ double sh[S2L_BS_VEC / 32][K];
    const int lane = threadIdx.x % TPR;
    const int64_t g0 = ((int64_t)blockIdx.x * S2L_BS_VEC + threadIdx.x) / TPR;
    const int64_t stride = (int64_t)gridDim.x * (S2L_BS_VEC / TPR);
    double nrm[K];
#pragma unroll
    for (int r = 0; r < K; ++r) nrm[r] = 0.0;
    for (int64_t row = g0; __any_sync(0xffffffffu, row < n); row += stride) {
        double acc[K];
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] = 0.0;
        if (row < n) {
            const int e1 = rp[row + 1];
            int e = rp[row] + lane;
            // two entries of the lane at once (loads, then gathers), added in entry order
            for (; e + TPR < e1; e += 2 * TPR) {
                const int c0 = ci[e], c1 = ci[e + TPR];
                const double a0 = v[e], a1 = v[e + TPR];
                double x0[K], x1[K];
                load_k<double, K>(X + (int64_t)c0 * K, x0);
                load_k<double, K>(X + (int64_t)c1 * K, x1);
#pragma unroll
                for (int r = 0; r < K; ++r) acc[r] += a0 * x0[r];
#pragma unroll
                for (int r = 0; r < K; ++r) acc[r] += a1 * x1[r];
            }
            if (e < e1) {
                const double a0 = v[e];
                double x0[K];
                load_k<double, K>(X + (int64_t)ci[e] * K, x0);
#pragma unroll
                for (int r = 0; r < K; ++r) acc[r] += a0 * x0[r];
            }
        }
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int o = TPR / 2; o; o >>= 1) acc[r] += __shfl_down_sync(0xffffffffu, acc[r], o, TPR);
        if (lane == 0 && row < n) {
#pragma unroll
            for (int r = 0; r < K; ++r) {
                const double y = B ? B[row * K + r] - acc[r] : acc[r];
                Y[row * K + r] = y;
                nrm[r] += y * y;
            }
        }
    }
    if (partials) {
        const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const double t = warp_sum(nrm[r]);
            if (wl == 0) sh[warp][r] = t;
        }
        __syncthreads();
        if (threadIdx.x < K) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < S2L_BS_VEC / 32; ++w) t += sh[w][threadIdx.x];
            partials[(int64_t)blockIdx.x * K + threadIdx.x] = t;
        }
    }
}

// Y = A X (or B - A X) for short rows, K columns (chunk mode, spmv_tpr 1).  A warp takes 32
// consecutive rows; their entries are contiguous in the CSR arrays, so the warp loads them with
// coalesced loads, multiplies each by the gathered row of X and leaves the products in shared
// memory (pieces of `cap` entries); lane j then adds row j's products in entry order.  With
// partials, also sum(Y(:, r)^2) per block and column.
template <int K>
__global__ void __launch_bounds__(S2L_BS_VEC) spmv_chunk_kernel(int64_t n, const int32_t* __restrict__ rp,
                                                                const int32_t* __restrict__ ci,
                                                                const double* __restrict__ v,
                                                                const double* __restrict__ X, double* __restrict__ Y,
                                                                const double* __restrict__ B,
                                                                double* __restrict__ partials)
{
    constexpr int CAP = 512 / K;  // entries of a piece: 4 KB of products per warp
    __shared__ double prod[S2L_BS_VEC / 32][CAP * K];
    __shared__ double sh[S2L_BS_VEC / 32][K];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* wp = prod[warp];
    double nrm[K];
#pragma unroll
    for (int r = 0; r < K; ++r) nrm[r] = 0.0;
    const int64_t nchunks = (n + 31) / 32;
    for (int64_t ch = (int64_t)blockIdx.x * (S2L_BS_VEC / 32) + warp; ch < nchunks;
         ch += (int64_t)gridDim.x * (S2L_BS_VEC / 32)) {
        const int64_t r0 = ch * 32, row = r0 + lane;
        const int64_t rend = r0 + 32 < n ? r0 + 32 : n;
        const int e_lo = rp[r0], e_hi = rp[rend];
        const int my0 = row < n ? rp[row] : e_hi, my1 = row < n ? rp[row + 1] : e_hi;
        double acc[K];
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] = 0.0;
        for (int base = e_lo; base < e_hi; base += CAP) {
            const int cnt = e_hi - base < CAP ? e_hi - base : CAP;
            // U entries per lane at once: all their loads, then all their gathers, are in flight together
            constexpr int U = K == 1 ? 8 : 4;
            for (int e0 = lane; e0 < cnt; e0 += 32 * U) {
                int c[U];
                double a[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = e0 + 32 * u;
                    c[u] = e < cnt ? ci[base + e] : 0;
                    a[u] = e < cnt ? v[base + e] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = e0 + 32 * u;
                    if (e < cnt) {
                        double x[K];
                        load_k<double, K>(X + (int64_t)c[u] * K, x);
#pragma unroll
                        for (int r = 0; r < K; ++r) wp[e * K + r] = a[u] * x[r];
                    }
                }
            }
            __syncwarp();
            const int s0 = (my0 > base ? my0 : base) - base, s1 = (my1 < base + cnt ? my1 : base + cnt) - base;
            for (int e = s0; e < s1; ++e)
#pragma unroll
                for (int r = 0; r < K; ++r) acc[r] += wp[e * K + r];
            __syncwarp();
        }
        if (row < n) {
#pragma unroll
            for (int r = 0; r < K; ++r) {
                const double y = B ? B[row * K + r] - acc[r] : acc[r];
                Y[row * K + r] = y;
                nrm[r] += y * y;
            }
        }
    }
    if (partials) {
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const double t = warp_sum(nrm[r]);
            if (lane == 0) sh[warp][r] = t;
        }
        __syncthreads();
        if (threadIdx.x < K) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < S2L_BS_VEC / 32; ++w) t += sh[w][threadIdx.x];
            partials[(int64_t)blockIdx.x * K + threadIdx.x] = t;
        }
    }
}

// Sum over the lanes of a warp that hold the same column (lane % K): afterwards lanes 0..K-1 hold
// the column sums (K a power of two, at most 32).
template <int K>
__device__ __forceinline__ double col_sum(double v)
{
#pragma unroll
    for (int o = 16; o >= K; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// h(j, r) = V_j(:, r) . w(:, r) for j < J (V_j at V + ring_block(j) * ldv, n x K interleaved); tiles
// of 1024 entries (w staged in shared memory, entry e of a tile is column e % K), warp owns the
// columns j = warp + 8q; partials[(b * J + j) * K + r].  Each (j, r) is summed in the same order
// whatever J, the ring position and the other columns hold.
__device__ __forceinline__ int64_t ring_block(int j, int j0, int ring)
{
    return ring ? (j0 + j) % ring : j0 + j;
}

template <int K>
__global__ void __launch_bounds__(256) mdot_block_kernel(int64_t nk, const double* __restrict__ V, int64_t ldv, int J,
                                                         const double* __restrict__ w, double* __restrict__ partials,
                                                         int j0, int ring)
{
    __shared__ double ws[1024];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.0;
    for (int64_t t0 = (int64_t)blockIdx.x * 1024; t0 < nk; t0 += (int64_t)gridDim.x * 1024) {
        const int cnt = (int)((nk - t0) < 1024 ? (nk - t0) : 1024);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += 256) ws[i] = w[t0 + i];
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int j = warp + 8 * q;
            if (j < J) {
                const double* vj = V + ring_block(j, j0, ring) * ldv + t0;
                double s0 = 0.0;
                for (int i = lane; i < cnt; i += 32) s0 += vj[i] * ws[i];
                acc[q] += s0;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int j = warp + 8 * q;
        if (j < J) {
            const double t = col_sum<K>(acc[q]);
            if (lane < K) partials[((int64_t)blockIdx.x * J + j) * K + lane] = t;
        }
    }
}

// w(:, r) += alpha * sum_j V_j(:, r) h(j, r); with partials, also sum(w(:, r)^2) per block.  With
// `first`, h(j, r) counts as zero for j < first.f[r] (a column whose own basis starts later in the
// window): the terms before it add exact zeros, so the sum is the same as over its own basis.
template <int K>
__global__ void __launch_bounds__(256) gemv_update_block_kernel(int64_t nk, const double* __restrict__ V, int64_t ldv,
                                                                int J, const double* __restrict__ h, double alpha,
                                                                double* __restrict__ w, double* __restrict__ partials,
                                                                int j0, int ring, ColFirst first, int masked)
{
    __shared__ double hs[S2L_MAX_BLOCK_COLS];
    __shared__ double sh[8][K];
    for (int c = threadIdx.x; c < J * K; c += 256) hs[c] = (masked && c / K < first.f[c % K]) ? 0.0 : h[c];
    __syncthreads();
    const int r = (int)(threadIdx.x % K);  // every stride below is a multiple of K
    double nrm = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < nk; e += (int64_t)gridDim.x * 256) {
        double s = 0.0;
        for (int j = 0; j < J; ++j) s += V[e + ring_block(j, j0, ring) * ldv] * hs[j * K + r];
        const double wn = w[e] + alpha * s;
        w[e] = wn;
        nrm += wn * wn;
    }
    if (partials) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const double t = col_sum<K>(nrm);
        if (lane < K) sh[warp][lane] = t;
        __syncthreads();
        if (threadIdx.x < K) {
            double u = 0.0;
#pragma unroll
            for (int q = 0; q < 8; ++q) u += sh[q][threadIdx.x];
            partials[(int64_t)blockIdx.x * K + threadIdx.x] = u;
        }
    }
}

// u(:, r) = sum_j V_j(:, r) y(j, r)
template <int K>
__global__ void __launch_bounds__(256) gemv_block_kernel(int64_t nk, const double* __restrict__ V, int64_t ldv, int J,
                                                         const double* __restrict__ y, double* __restrict__ u, int j0,
                                                         int ring)
{
    __shared__ double ys[S2L_MAX_BLOCK_COLS];
    for (int c = threadIdx.x; c < J * K; c += 256) ys[c] = y[c];
    __syncthreads();
    const int r = (int)(threadIdx.x % K);
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < nk; e += (int64_t)gridDim.x * 256) {
        double s = 0.0;
        for (int j = 0; j < J; ++j) s += V[e + ring_block(j, j0, ring) * ldv] * ys[j * K + r];
        u[e] = s;
    }
}

// y(:, r) = a(r) x(:, r) + b(r) y(:, r) (b null: y is not read); a, b on the device, K each
template <int K>
__global__ void __launch_bounds__(256) axpby_block_kernel(int64_t nk, const double* __restrict__ a,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          double* __restrict__ y)
{
    const int r = (int)(threadIdx.x % K);
    const double ar = a[r], br = b ? b[r] : 0.0;
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < nk; e += (int64_t)gridDim.x * 256)
        y[e] = b ? ar * x[e] + br * y[e] : ar * x[e];
}

// y(:, r) = a(r) x(:, r) + c(r) z(:, r), a source with a zero coefficient not read (so a stale
// value there never reaches y); a, c by value
template <int K>
__global__ void __launch_bounds__(256) combine2_block_kernel(int64_t nk, ColScale a, const double* __restrict__ x,
                                                             ColScale c, const double* __restrict__ z,
                                                             double* __restrict__ y)
{
    const int r = (int)(threadIdx.x % K);
    const double ar = a.v[r], cr = c.v[r];
    for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < nk; e += (int64_t)gridDim.x * 256) {
        const double p = ar != 0.0 ? ar * x[e] : 0.0;
        const double q = cr != 0.0 ? cr * z[e] : 0.0;
        y[e] = p + q;
    }
}

// column r of dst (n x K interleaved) from src (n), or (out) src column r to dst
__global__ void column_in_kernel(int64_t n, int K, int r, const double* __restrict__ src, double* __restrict__ dst)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i * K + r] = src[i];
}

__global__ void column_out_kernel(int64_t n, int K, int r, const double* __restrict__ src, double* __restrict__ dst)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i * K + r];
}

// column r of every block of a ring (count blocks of n x K) set to v
__global__ void column_fill_kernel(int64_t n, int K, int r, int count, int64_t ld, double v, double* __restrict__ dst)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * count; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = e / n, i = e - b * n;
        dst[b * ld + i * K + r] = v;
    }
}

// dst (n x K interleaved) from k columns src + r * n (r < k); columns k..K-1 are zero
__global__ void interleave_kernel(int64_t n, int K, int k, const double* __restrict__ src, double* __restrict__ dst)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / K;
        const int r = (int)(e % K);
        dst[e] = r < k ? src[(int64_t)r * n + i] : 0.0;
    }
}

// k columns dst + r * n from src (n x K interleaved)
__global__ void deinterleave_kernel(int64_t n, int K, int k, const double* __restrict__ src, double* __restrict__ dst)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * k; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / n);
        const int64_t i = e % n;
        dst[e] = src[i * K + r];
    }
}

// out(g, r) = base(g, r) + sum over the copies of g of w_e ylocal(pos, r) (K columns)
template <int K>
__global__ void combine_block_kernel(int64_t n, const int64_t* __restrict__ cp_ptr, const int32_t* __restrict__ cp_pos,
                                     const double* __restrict__ cp_w, const double* __restrict__ ylocal,
                                     const double* __restrict__ base, double* __restrict__ out)
{
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        double s[K];
#pragma unroll
        for (int r = 0; r < K; ++r) s[r] = 0.0;
        for (int64_t e = cp_ptr[g]; e < cp_ptr[g + 1]; ++e) {
            const double* y = ylocal + (int64_t)cp_pos[e] * K;
            const double wgt = cp_w ? cp_w[e] : 1.0;
#pragma unroll
            for (int r = 0; r < K; ++r) s[r] += wgt * y[r];
        }
#pragma unroll
        for (int r = 0; r < K; ++r) out[g * K + r] = base ? base[g * K + r] + s[r] : s[r];
    }
}

// Coarse restriction of one tile (up to S2L_TILE_ROWS rows of one subdomain), K columns:
// partials(tile, c, r) = sum_i V(row0 + i, c) R(g(row0 + i), r).  The tile's rows of R are staged
// in shared memory first; the tile's block of V (nr x m, contiguous row-major) is then streamed by
// all threads, with 16-byte loads when m is even: thread (g, p) takes the column pair p of rows
// g, g + G, ... (G = threads / pairs, so all lanes load), and the G partial sums of each (c, r)
// are added in order of g.  Every (c, r) sums in the same order whatever K is.
template <int K>
__global__ void __launch_bounds__(S2L_TILE_ROWS) coarse_restrict_block_kernel(
    const int32_t* __restrict__ t_sub, const int32_t* __restrict__ t_row0, const int32_t* __restrict__ t_nrow,
    const DevSub* __restrict__ subs, const double* __restrict__ V, const int32_t* __restrict__ l2g, int boolean_pou,
    const double* __restrict__ R, int mmax, double* __restrict__ partials)
{
    extern __shared__ double sm[];  // Rs[S2L_TILE_ROWS * K], then red[G * m * K] (G m <= 2 S2L_TILE_ROWS)
    const int tile = blockIdx.x;
    const DevSub sd = subs[t_sub[tile]];
    const int m = sd.m, nr = t_nrow[tile], row0 = t_row0[tile];
    if (m == 0) return;  // the prolongation's zero tiles of subdomains without a coarse basis
    double* Rs = sm;
    double* red = sm + S2L_TILE_ROWS * K;
    for (int e = threadIdx.x; e < nr * K; e += S2L_TILE_ROWS) {
        const int i = e / K, r = e % K;
        const int l = row0 + i;
        const int64_t g = boolean_pou ? sd.begin + l : (int64_t)l2g[sd.loc_off + l];
        Rs[e] = R[g * K + r];
    }
    __syncthreads();
    const double* Vt = V + sd.v_off + (int64_t)row0 * m;
    const bool vec = (m & 1) == 0 && (reinterpret_cast<uintptr_t>(Vt) & 15) == 0;
    const int W = vec ? 2 : 1;  // columns per thread
    const int P = (m + W - 1) / W, G = S2L_TILE_ROWS / P;
    const int p = threadIdx.x % P, g = threadIdx.x / P;
    if (g < G) {
        double a0[K], a1[K];
#pragma unroll
        for (int r = 0; r < K; ++r) a0[r] = a1[r] = 0.0;
        if (vec) {
#pragma unroll 4
            for (int i = g; i < nr; i += G) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(Vt + (int64_t)i * m) + p);
#pragma unroll
                for (int r = 0; r < K; ++r) {
                    const double x = Rs[i * K + r];
                    a0[r] += v.x * x;
                    a1[r] += v.y * x;
                }
            }
        } else {
#pragma unroll 4
            for (int i = g; i < nr; i += G) {
                const double v = __ldg(Vt + (int64_t)i * m + p);
#pragma unroll
                for (int r = 0; r < K; ++r) a0[r] += v * Rs[i * K + r];
            }
        }
        const int c = p * W;
#pragma unroll
        for (int r = 0; r < K; ++r) red[((size_t)g * m + c) * K + r] = a0[r];
        if (vec)
#pragma unroll
            for (int r = 0; r < K; ++r) red[((size_t)g * m + c + 1) * K + r] = a1[r];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < m * K; e += S2L_TILE_ROWS) {
        double t = 0.0;
        for (int q = 0; q < G; ++q) t += red[(size_t)q * m * K + e];
        partials[(int64_t)tile * mmax * K + e] = t;
    }
}

template <int K>
__global__ void coarse_reduce_block_kernel(const DevSub* __restrict__ subs, const int32_t* __restrict__ t_first,
                                           int mmax, const double* __restrict__ partials, double* __restrict__ cvec)
{
    const int i = blockIdx.x;
    const DevSub sd = subs[i];
    for (int e = threadIdx.x; e < sd.m * K; e += blockDim.x) {
        double s = 0.0;
        for (int t = t_first[i]; t < t_first[i + 1]; ++t) s += partials[(int64_t)t * mmax * K + e];
        cvec[sd.c_off * K + e] = s;
    }
}

// Y = M X, M dense row-major n0 x n0, K columns; one warp per row (M is read once for all columns)
template <int K>
__global__ void __launch_bounds__(256) dense_gemm_kernel(int n0, const double* __restrict__ M,
                                                         const double* __restrict__ X, double* __restrict__ Y)
{
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n0) return;
    const double* mr = M + (int64_t)row * n0;
    double s[K];
#pragma unroll
    for (int r = 0; r < K; ++r) s[r] = 0.0;
    for (int c = lane; c < n0; c += 32) {
        const double m = mr[c];
#pragma unroll
        for (int r = 0; r < K; ++r) s[r] += m * X[(int64_t)c * K + r];
    }
#pragma unroll
    for (int r = 0; r < K; ++r) {
        const double t = warp_sum(s[r]);
        if (lane == 0) Y[(int64_t)row * K + r] = t;
    }
}

// X0 = V_i Y_i on the owned rows (boolean PoU) or on Omega_i (plocal), K columns.  With `staged`,
// the tile's rows of V (nr x m contiguous doubles) are first copied to shared memory with coalesced
// loads (rows padded to m + 1 doubles) and Y_i next to them; a thread then sums its row there.
template <int K>
__global__ void __launch_bounds__(S2L_TILE_ROWS) coarse_prolong_block_kernel(
    const int32_t* __restrict__ t_sub, const int32_t* __restrict__ t_row0, const int32_t* __restrict__ t_nrow,
    const DevSub* __restrict__ subs, const double* __restrict__ V, int boolean_pou, const double* __restrict__ Y,
    double* __restrict__ out, double* __restrict__ plocal, int staged)
{
    extern __shared__ double sm[];
    const int tile = blockIdx.x;
    const DevSub sd = subs[t_sub[tile]];
    const int m = sd.m, nr = t_nrow[tile], row0 = t_row0[tile];
    const double* vr;
    const double* yc;
    if (staged) {
        const int ld = m + 1;
        double* vs = sm;
        double* ys = sm + (size_t)S2L_TILE_ROWS * ld;
        const double* src = V + sd.v_off + (int64_t)row0 * m;
        for (int e = threadIdx.x; e < nr * m; e += S2L_TILE_ROWS) {
            const int l = e / m;
            vs[l * ld + (e - l * m)] = src[e];
        }
        for (int e = threadIdx.x; e < m * K; e += S2L_TILE_ROWS) ys[e] = Y[sd.c_off * K + e];
        __syncthreads();
        vr = vs + (size_t)threadIdx.x * ld;
        yc = ys;
    } else {
        vr = V + sd.v_off + (int64_t)(row0 + (int)threadIdx.x) * m;
        yc = Y + sd.c_off * K;
    }
    if ((int)threadIdx.x >= nr) return;
    const int l = row0 + threadIdx.x;
    double s[K];
#pragma unroll
    for (int r = 0; r < K; ++r) s[r] = 0.0;
    for (int c = 0; c < m; ++c) {
        const double v = vr[c];
#pragma unroll
        for (int r = 0; r < K; ++r) s[r] += v * yc[c * K + r];
    }
    double* o = boolean_pou ? out + (sd.begin + l) * K : plocal + (sd.loc_off + l) * K;
#pragma unroll
    for (int r = 0; r < K; ++r) o[r] = s[r];
}

inline int grid_for(int64_t n, int bs, int cap)
{
    const int64_t g = (n + bs - 1) / bs;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

// ------------------------------------------------------------------------------ launch wrappers
void launch_spmv(cudaStream_t st, int64_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* x,
                 double* y, const double* b, double* partials, double* red_out, int tpr)
{
    // the norm partials need the fixed grid (deterministic reduction); a plain product takes one
    // lane group per row
    const int grid = partials ? S2L_NB_RED : grid_for(n * tpr, S2L_BS_VEC, 1 << 20);
    switch (tpr) {
    case 1: spmv_chunk_kernel<1><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    case 2: spmv_kernel<2><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    case 4: spmv_kernel<4><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    case 16: spmv_kernel<16><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    case 32: spmv_kernel<32><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    default: spmv_kernel<8><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, x, y, b, partials); break;
    }
    if (partials) reduce_kernel<<<1, 256, 0, st>>>(partials, grid, 1, red_out);
}

void launch_reduce(cudaStream_t st, const double* partials, int nblocks, int ncols, double* out)
{
    reduce_kernel<<<(ncols + 7) / 8, 256, 0, st>>>(partials, nblocks, ncols, out);
}

void launch_mdot(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* w, double* partials,
                 double* out)
{
    mdot_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, V, ldv, k, w, partials);
    reduce_kernel<<<(k + 7) / 8, 256, 0, st>>>(partials, S2L_NB_RED, k, out);
}

void launch_gemv_update(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* h, double alpha,
                        double* w, double* partials)
{
    gemv_update_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, V, ldv, k, h, alpha, w, partials);
}

void launch_gemv(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* y, double* u)
{
    gemv_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, V, ldv, k, y, u);
}

void launch_axpby(cudaStream_t st, int64_t n, double a, const double* x, double b, double* y)
{
    axpby_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, a, x, b, y);
}

void launch_dot2(cudaStream_t st, int64_t n, const double* x, const double* y, const double* z, double* partials,
                 double* out)
{
    dot2_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, x, y, z, partials);
    reduce_kernel<<<1, 256, 0, st>>>(partials, S2L_NB_RED, 2, out);
}

// ---- K right-hand sides (K = 1, 2, 4, 8 or 16)
#define S2L_KSWITCH(K, CALL)                             \
    switch (K) {                                         \
    case 1: { constexpr int KK = 1; CALL; break; }       \
    case 2: { constexpr int KK = 2; CALL; break; }       \
    case 4: { constexpr int KK = 4; CALL; break; }       \
    case 8: { constexpr int KK = 8; CALL; break; }       \
    default: { constexpr int KK = 16; CALL; break; }     \
    }

void launch_spmv_block(cudaStream_t st, int64_t n, int K, const int32_t* rp, const int32_t* ci, const double* v,
                       const double* X, double* Y, const double* B, double* partials, double* red_out, int tpr)
{
    const int grid = partials ? S2L_NB_RED : grid_for(n * tpr, S2L_BS_VEC, 1 << 20);
    if (tpr == 1) {
        S2L_KSWITCH(K, (spmv_chunk_kernel<KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    } else if (tpr == 2) {
        S2L_KSWITCH(K, (spmv_block_kernel<2, KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    } else if (tpr == 4) {
        S2L_KSWITCH(K, (spmv_block_kernel<4, KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    } else if (tpr == 16) {
        S2L_KSWITCH(K, (spmv_block_kernel<16, KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    } else if (tpr == 32) {
        S2L_KSWITCH(K, (spmv_block_kernel<32, KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    } else {
        S2L_KSWITCH(K, (spmv_block_kernel<8, KK><<<grid, S2L_BS_VEC, 0, st>>>(n, rp, ci, v, X, Y, B, partials)));
    }
    if (partials) reduce_kernel<<<(K + 7) / 8, 256, 0, st>>>(partials, grid, K, red_out);
}

void launch_mdot_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* w,
                       double* partials, double* out, int j0, int ring)
{
    S2L_KSWITCH(K, (mdot_block_kernel<KK><<<S2L_NB_RED, 256, 0, st>>>(n * K, V, ldv, J, w, partials, j0, ring)));
    reduce_kernel<<<(J * K + 7) / 8, 256, 0, st>>>(partials, S2L_NB_RED, J * K, out);
}

void launch_gemv_update_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* h,
                              double alpha, double* w, double* partials, double* red_out, int j0, int ring,
                              const ColFirst* first)
{
    const ColFirst f = first ? *first : ColFirst{};
    const int masked = first ? 1 : 0;
    S2L_KSWITCH(K, (gemv_update_block_kernel<KK><<<S2L_NB_RED, 256, 0, st>>>(n * K, V, ldv, J, h, alpha, w, partials,
                                                                             j0, ring, f, masked)));
    if (partials) reduce_kernel<<<(K + 7) / 8, 256, 0, st>>>(partials, S2L_NB_RED, K, red_out);
}

void launch_gemv_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* y,
                       double* u, int j0, int ring)
{
    S2L_KSWITCH(K, (gemv_block_kernel<KK><<<grid_for(n * K, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n * K, V, ldv, J, y, u,
                                                                                                 j0, ring)));
}

void launch_combine2_block(cudaStream_t st, int64_t n, int K, const ColScale& a, const double* x, const ColScale& c,
                           const double* z, double* y)
{
    S2L_KSWITCH(K, (combine2_block_kernel<KK><<<grid_for(n * K, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n * K, a, x, c, z,
                                                                                                     y)));
}

void launch_column_in(cudaStream_t st, int64_t n, int K, int r, const double* src, double* dst)
{
    column_in_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, K, r, src, dst);
}

void launch_column_out(cudaStream_t st, int64_t n, int K, int r, const double* src, double* dst)
{
    column_out_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, K, r, src, dst);
}

void launch_column_fill(cudaStream_t st, int64_t n, int K, int r, int count, int64_t ld, double v, double* dst)
{
    if (count > 0) column_fill_kernel<<<grid_for(n * count, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, K, r, count, ld, v, dst);
}

void launch_axpby_block(cudaStream_t st, int64_t n, int K, const double* a, const double* x, const double* b,
                        double* y)
{
    S2L_KSWITCH(K, (axpby_block_kernel<KK><<<grid_for(n * K, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n * K, a, x, b, y)));
}

void launch_interleave(cudaStream_t st, int64_t n, int K, int k, const double* src, double* dst)
{
    interleave_kernel<<<grid_for(n * K, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, K, k, src, dst);
}

void launch_deinterleave(cudaStream_t st, int64_t n, int K, int k, const double* src, double* dst)
{
    deinterleave_kernel<<<grid_for(n * k, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, K, k, src, dst);
}

void launch_combine_block(cudaStream_t st, int64_t n, int K, const int64_t* cp_ptr, const int32_t* cp_pos,
                          const double* cp_w, const double* ylocal, const double* base, double* out)
{
    S2L_KSWITCH(K, (combine_block_kernel<KK><<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, cp_ptr, cp_pos, cp_w,
                                                                                                ylocal, base, out)));
}

static void restrict_tiles(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                           const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                           int boolean_pou, const double* R, int mmax, double* partials)
{
    if (ntiles <= 0) return;
    // staged R rows + the row groups' partial sums (G m <= 2 S2L_TILE_ROWS): <= 96 KB for K = 16
    const size_t smem = (size_t)3 * S2L_TILE_ROWS * K * sizeof(double);
    S2L_KSWITCH(K, (cudaFuncSetAttribute(coarse_restrict_block_kernel<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)((size_t)3 * S2L_TILE_ROWS * KK * sizeof(double))),
                    coarse_restrict_block_kernel<KK><<<ntiles, S2L_TILE_ROWS, smem, st>>>(
                        t_sub, t_row0, t_nrow, subs, V, l2g, boolean_pou, R, mmax, partials)));
}

void launch_coarse_restrict_block(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                                  const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                                  int boolean_pou, const double* R, int mmax, double* partials)
{
    restrict_tiles(st, K, ntiles, t_sub, t_row0, t_nrow, subs, V, l2g, boolean_pou, R, mmax, partials);
}

void launch_coarse_reduce_block(cudaStream_t st, int K, int nsub, const DevSub* subs, const int32_t* t_first, int mmax,
                                const double* partials, double* cvec)
{
    S2L_KSWITCH(K, (coarse_reduce_block_kernel<KK><<<nsub, 128, 0, st>>>(subs, t_first, mmax, partials, cvec)));
}

void launch_dense_gemm(cudaStream_t st, int K, int n0, const double* M, const double* X, double* Y)
{
    if (n0 <= 0) return;
    S2L_KSWITCH(K, (dense_gemm_kernel<KK><<<(n0 + 7) / 8, 256, 0, st>>>(n0, M, X, Y)));
}

static void prolong_tiles(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                          const int32_t* t_nrow, const DevSub* subs, const double* V, int mmax, int boolean_pou,
                          const double* Y, double* out, double* plocal)
{
    if (ntiles <= 0) return;
    // staged through shared memory when a tile's padded rows and Y_i fit (mmax up to about 100)
    const size_t smem = ((size_t)S2L_TILE_ROWS * (mmax + 1) + (size_t)mmax * K) * sizeof(double);
    const int staged = smem <= 200 * 1024 ? 1 : 0;
    S2L_KSWITCH(K, (cudaFuncSetAttribute(coarse_prolong_block_kernel<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024),
                    coarse_prolong_block_kernel<KK><<<ntiles, S2L_TILE_ROWS, staged ? smem : 0, st>>>(
                        t_sub, t_row0, t_nrow, subs, V, boolean_pou, Y, out, plocal, staged)));
}

void launch_coarse_prolong_block(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                                 const int32_t* t_nrow, const DevSub* subs, const double* V, int mmax, int boolean_pou,
                                 const double* Y, double* out, double* plocal)
{
    prolong_tiles(st, K, ntiles, t_sub, t_row0, t_nrow, subs, V, mmax, boolean_pou, Y, out, plocal);
}

void launch_coarse_restrict(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                            const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                            int boolean_pou, const double* r, int mmax, double* partials)
{
    restrict_tiles(st, 1, ntiles, t_sub, t_row0, t_nrow, subs, V, l2g, boolean_pou, r, mmax, partials);
}

void launch_coarse_prolong(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                           const int32_t* t_nrow, const DevSub* subs, const double* V, int mmax, int boolean_pou,
                           const double* y, double* out, double* plocal)
{
    prolong_tiles(st, 1, ntiles, t_sub, t_row0, t_nrow, subs, V, mmax, boolean_pou, y, out, plocal);
}

#undef S2L_KSWITCH

void launch_l1(cudaStream_t st, int64_t n, const double* a, double alpha, const double* c, double* partials,
               double* out)
{
    l1_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, a, alpha, c, partials);
    reduce_kernel<<<1, 256, 0, st>>>(partials, S2L_NB_RED, 2, out);
}

void launch_gemv_l1(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* q, double* partials,
                    double* out)
{
    gemv_l1_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, V, ldv, k, q, partials);
    reduce_kernel<<<1, 256, 0, st>>>(partials, S2L_NB_RED, 1, out);
}

void launch_bicg_p(cudaStream_t st, int64_t n, const double* r, const double* v, double beta, double omega, double* p,
                   int first)
{
    bicg_p_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, r, v, beta, omega, p, first);
}

void launch_bicg_s(cudaStream_t st, int64_t n, const double* r, const double* v, double alpha, double* s,
                   double* partials, double* out)
{
    bicg_s_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, r, v, alpha, s, partials);
    reduce_kernel<<<1, 256, 0, st>>>(partials, S2L_NB_RED, 1, out);
}

void launch_bicg_x(cudaStream_t st, int64_t n, double* x, const double* y, const double* z, double alpha,
                   double omega, double* r, const double* s, const double* t, const double* rh, double* partials,
                   double* out)
{
    bicg_x_kernel<<<S2L_NB_RED, 256, 0, st>>>(n, x, y, z, alpha, omega, r, s, t, rh, partials);
    reduce_kernel<<<1, 256, 0, st>>>(partials, S2L_NB_RED, 2, out);
}

template <typename Real, int KC, int K>
cudaError_t launch_local_solve_k(cudaStream_t st, const LocalSolveArgs<Real>& a, int nblocks, size_t smem, int tr_first,
                                 int tr_count, int uu_first, int uu_count, int* launches)
{
    cudaError_t e;
    const int grid = nblocks * (K / KC);
    if (smem > 0) {
        // the limit is a process-wide attribute of the kernel: always the same cap, so launches of
        // setups with different shared-memory sizes from several threads cannot undercut each other
        if (smem > S2L_SWEEP_SMEM_CAP) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(sweep_kernel<Real, true, true, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 S2L_SWEEP_SMEM_CAP);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(sweep_kernel<Real, true, false, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 S2L_SWEEP_SMEM_CAP);
        if (e != cudaSuccess) return e;
        sweep_kernel<Real, true, true, KC><<<grid, S2L_BS_SWEEP, smem, st>>>(a);
    } else {
        sweep_kernel<Real, false, true, KC><<<grid, S2L_BS_SWEEP, 0, st>>>(a);
    }
    int nl = 1;
    if (tr_count > 0) {
        const int g = (tr_count + 7) / 8;
        tail_rhs_kernel<Real, K><<<g, 256, 0, st>>>(a, tr_first, tr_count);
        tail_gemv_kernel<Real, true, K><<<g, 256, 0, st>>>(a, a.linv, a.ybuf, a.xbuf, tr_first, tr_count);
        tail_gemv_kernel<Real, false, K><<<g, 256, 0, st>>>(a, a.uinv, a.xbuf, a.ybuf, tr_first, tr_count);
        nl += 3;
    }
    if (uu_count > 0) {
        sparse_coupling_kernel<Real, K><<<(uu_count + 7) / 8, 256, 0, st>>>(a, uu_first, uu_count);
        nl += 1;
    }
    if (smem > 0)
        sweep_kernel<Real, true, false, KC><<<grid, S2L_BS_SWEEP, smem, st>>>(a);
    else
        sweep_kernel<Real, false, false, KC><<<grid, S2L_BS_SWEEP, 0, st>>>(a);
    *launches = nl + 1;
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_local_solve(cudaStream_t st, const LocalSolveArgs<Real>& a, int nblocks, size_t smem, int tr_first,
                               int tr_count, int uu_first, int uu_count, int* launches)
{
    // (KC, K): right-hand sides per sweep CTA and in all; the setup's shared memory fixes KC
    const int K = a.K, KC = smem > 0 ? a.KC : 1;
#define S2L_LS(KC_, K_)                                                                                         \
    if (KC == KC_ && K == K_)                                                                                  \
    return launch_local_solve_k<Real, KC_, K_>(st, a, nblocks, smem, tr_first, tr_count, uu_first, uu_count, \
                                               launches)
    S2L_LS(1, 1);
    S2L_LS(1, 2);
    S2L_LS(2, 2);
    S2L_LS(1, 4);
    S2L_LS(2, 4);
    S2L_LS(4, 4);
    S2L_LS(1, 8);
    S2L_LS(2, 8);
    S2L_LS(4, 8);
    S2L_LS(1, 16);
    S2L_LS(2, 16);
    S2L_LS(4, 16);
#undef S2L_LS
    return cudaErrorInvalidValue;
}

template cudaError_t launch_local_solve<double>(cudaStream_t, const LocalSolveArgs<double>&, int, size_t, int, int, int,
                                                int, int*);
template cudaError_t launch_local_solve<float>(cudaStream_t, const LocalSolveArgs<float>&, int, size_t, int, int, int,
                                                int, int*);

void launch_to_float(cudaStream_t st, const double* in, float* out, int64_t n)
{
    to_float_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(in, out, n);
}

void launch_combine(cudaStream_t st, int64_t n, const int64_t* cp_ptr, const int32_t* cp_pos, const double* cp_w,
                    const double* ylocal, const double* base, double* out)
{
    combine_kernel<<<grid_for(n, 256, 4 * S2L_NB_RED), 256, 0, st>>>(n, cp_ptr, cp_pos, cp_w, ylocal, base, out);
}

void launch_coarse_reduce(cudaStream_t st, int nsub, const DevSub* subs, const int32_t* t_first, int mmax,
                          const double* partials, double* c)
{
    coarse_reduce_kernel<<<nsub, 64, 0, st>>>(subs, t_first, mmax, partials, c);
}

void launch_dense_gemv(cudaStream_t st, int n0, const double* M, const double* x, double* y)
{
    dense_gemv_kernel<<<(n0 + 7) / 8, 256, 0, st>>>(n0, M, x, y);
}

}  // namespace s2l
