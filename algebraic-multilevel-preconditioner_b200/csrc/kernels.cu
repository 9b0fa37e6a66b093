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
            for (int e = rp[row] + lane; e < e1; e += TPR) s += v[e] * __ldg(x + ci[e]);
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
// S2L_SPIN_LIMIT polls the CTA raises *err and all warps leave.
template <typename Real, bool SMEM, bool FWD>
__global__ void __launch_bounds__(S2L_BS_SWEEP, 1) sweep_kernel(const LocalSolveArgs<Real> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int abort_word;
    volatile int& abort_flag = abort_word;
    constexpr int Q = S2L_BATCH_CHUNKS;
    const int sid = a.sub_list ? a.sub_list[blockIdx.x] : (int)blockIdx.x;
    const DevSub sd = a.subs[sid];
    const int64_t lo = sd.loc_off;
    const int T = sd.T;
    const SweepFactor<Real> F = a.f[FWD ? 0 : 1];
    Real* xs;
    volatile uint8_t* flag;
    if (SMEM) {
        const size_t off1 = (((size_t)T * sizeof(Real)) + 15) & ~(size_t)15;
        xs = reinterpret_cast<Real*>(smem_raw);
        flag = reinterpret_cast<volatile uint8_t*>(smem_raw + off1);
    } else {
        xs = (FWD ? a.ybuf : a.xbuf) + lo;
        flag = a.gflags + lo;
    }
    volatile Real* x = xs;
    if (threadIdx.x == 0) abort_flag = 0;
    for (int k = threadIdx.x; k < T; k += S2L_BS_SWEEP) {
        const Real b = FWD ? (Real)a.in[a.gather[lo + k]] : a.ybuf[lo + a.u2l[lo + k]];
        xs[k] = b * F.dinv[lo + k];
        flag[k] = 0;
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
                Real v = Real(0);
                for (int j = 0; j <= i; ++j) v += Wi[j] * xs[F.blk_slot[o + j]];
                xs[F.blk_slot[o + i]] = v;
            }
        }
        __syncthreads();
    }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t wi = (int64_t)sid * S2L_SWEEP_WARPS + wid;
    const int64_t t1 = F.wtask[wi + 1];
    int64_t so = F.wslot[wi], eo = F.went[wi];
    bool dead = false;
    for (int64_t t = F.wtask[wi]; t < t1; ++t) {
        const uint32_t h = F.thdr[t];
        const int C = (int)(h & 0xFFFFu), gl2 = (int)((h >> 16) & 7u), R = (int)((h >> 19) & 31u) + 1;
        const int k = lane >> gl2;
        const int slot = k < R ? F.tslot[so + k] : -1;
        so += R;
        Real acc = Real(0);
        for (int c0 = 0; c0 < C; c0 += Q) {  // C is the same for the whole warp
            int lc[Q];
            Real lv[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                lc[q] = -1;
                lv[q] = Real(0);
                if (c0 + q < C) {
                    const int64_t e = eo + (int64_t)(c0 + q) * 32 + lane;
                    lc[q] = F.col[e];
                    lv[q] = F.val[e];
                }
            }
            // hint the next batch into L2: lane q < Q takes chunk q of it (lines of 128 bytes)
            if (lane < Q && c0 + Q + lane < C) {
                const int64_t e = eo + (int64_t)(c0 + Q + lane) * 32;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.col + e));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e));
                if (sizeof(Real) == 8) asm volatile("prefetch.global.L2 [%0];" ::"l"(F.val + e + 16));
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int c = lc[q];
                if (c >= 0 && !dead) {
                    int spin = 0;
                    while (flag[c] == 0) {
                        if (abort_flag) { dead = true; break; }
                        if (++spin > S2L_SPIN_LIMIT) {
                            abort_flag = 1;
                            atomicExch(a.err, 1);
                            dead = true;
                            break;
                        }
                    }
                    acc += lv[q] * x[c];
                }
            }
        }
        eo += (int64_t)C * 32;
        dead = __any_sync(0xffffffffu, dead);  // one decision per warp before its shuffles
        if (dead) break;
        for (int o = (1 << gl2) >> 1; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, 1 << gl2);
        if ((lane & ((1 << gl2) - 1)) == 0 && slot >= 0) {
            x[slot] = x[slot] - acc;
            __threadfence_block();
            flag[slot] = 1;
        }
    }
    __syncthreads();
    if (FWD) {
        if (SMEM)
            for (int k = threadIdx.x; k < T; k += S2L_BS_SWEEP) a.ybuf[lo + k] = xs[k];
        return;
    }
    // epilogue of the backward sweep: x_local[j] from its backward slot (< T) or tail row (>= T)
    const int n = sd.n_local;
    auto val_at = [&](int q) -> double { return q < T ? (double)xs[q] : (double)a.ybuf[lo + q]; };
    if (a.mode == 0) {
        for (int j = threadIdx.x; j < sd.n_owned; j += S2L_BS_SWEEP) {
            double v = val_at(a.gout[lo + j]);
            if (a.base) v += a.base[sd.begin + j];
            a.out[sd.begin + j] = v;
        }
    } else if (a.mode == 1) {
        for (int j = threadIdx.x; j < n; j += S2L_BS_SWEEP) a.ylocal[lo + j] = val_at(a.gout[lo + j]);
    } else {
        for (int j = threadIdx.x; j < n; j += S2L_BS_SWEEP) a.out[j] = val_at(a.gout[lo + j]);
    }
}

// Tail right-hand side: t(T+i) = b(T+i) - L(T+i, 0:T) y(0:T), one warp per tail row.
template <typename Real>
__global__ void __launch_bounds__(256) tail_rhs_kernel(const LocalSolveArgs<Real> a, int q0, int count)
{
    const int q = q0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= q0 + count) return;
    const DevSub sd = a.subs[a.tr_sub[q]];
    const int64_t lo = sd.loc_off;
    const int k = sd.T + a.tr_i[q];
    Real acc = Real(0);
    for (int64_t e = a.lts_ptr[q] + lane; e < a.lts_ptr[q + 1]; e += 32) acc += a.lts_val[e] * a.ybuf[lo + a.lts_col[e]];
    acc = warp_sum(acc);
    if (lane == 0) a.ybuf[lo + k] = (Real)a.in[a.gather[lo + k]] - acc;
}

// Dense tail: out(T+i) = sum_j Minv(i, j) in(T+j), j <= i (lower) or j >= i (upper); warp per row.
template <typename Real, bool LOWER>
__global__ void __launch_bounds__(256) tail_gemv_kernel(const LocalSolveArgs<Real> a, const Real* __restrict__ Minv,
                                                        const Real* __restrict__ vin, Real* __restrict__ vout,
                                                        int q0, int count)
{
    const int q = q0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= q0 + count) return;
    const DevSub sd = a.subs[a.tr_sub[q]];
    const int s = sd.n_local - sd.T;
    const int i = a.tr_i[q];
    const int64_t base = sd.loc_off + sd.T;
    const Real* row = Minv + sd.d_off + (int64_t)i * s;
    const int j0 = LOWER ? 0 : i, j1 = LOWER ? i + 1 : s;
    Real acc0 = Real(0), acc1 = Real(0);
    int j = j0 + lane;
    for (; j + 32 < j1; j += 64) {
        acc0 += row[j] * vin[base + j];
        acc1 += row[j + 32] * vin[base + j + 32];
    }
    if (j < j1) acc0 += row[j] * vin[base + j];
    const Real acc = warp_sum(acc0 + acc1);
    if (lane == 0) vout[base + i] = acc;
}

// Backward coupling: y(r) -= U(r, T:n) x(T:n) for the sparse rows that have tail columns.
template <typename Real>
__global__ void __launch_bounds__(256) sparse_coupling_kernel(const LocalSolveArgs<Real> a, int q0, int count)
{
    const int q = q0 + blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= q0 + count) return;
    const DevSub sd = a.subs[a.us_sub[q]];
    const int64_t lo = sd.loc_off;
    Real acc = Real(0);
    for (int64_t e = a.ust_ptr[q] + lane; e < a.ust_ptr[q + 1]; e += 32) acc += a.ust_val[e] * a.ybuf[lo + a.ust_col[e]];
    acc = warp_sum(acc);
    if (lane == 0) a.ybuf[lo + a.us_r[q]] -= acc;
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
// c_i = V_i^T r per 256-row tile of one subdomain: partials[tile * mmax + c].
__global__ void __launch_bounds__(S2L_TILE_ROWS) coarse_restrict_kernel(const int32_t* __restrict__ t_sub,
                                                                        const int32_t* __restrict__ t_row0,
                                                                        const int32_t* __restrict__ t_nrow,
                                                                        const DevSub* __restrict__ subs,
                                                                        const double* __restrict__ V,
                                                                        const int32_t* __restrict__ l2g,
                                                                        int boolean_pou, const double* __restrict__ r,
                                                                        int mmax, double* __restrict__ partials)
{
    __shared__ double red[S2L_TILE_ROWS / 32][S2L_MAX_RED_COLS];
    const int tile = blockIdx.x;
    const DevSub sd = subs[t_sub[tile]];
    const int m = sd.m, nr = t_nrow[tile];
    const int l = t_row0[tile] + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool act = threadIdx.x < nr;
    double rv = 0.0;
    const double* vr = V;
    if (act) {
        rv = boolean_pou ? r[sd.begin + l] : r[l2g[sd.loc_off + l]];
        vr = V + sd.v_off + (int64_t)l * m;
    }
    for (int c = 0; c < m; ++c) {
        const double p = warp_sum(act ? rv * vr[c] : 0.0);
        if (lane == 0) red[warp][c] = p;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < m; c += S2L_TILE_ROWS) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < S2L_TILE_ROWS / 32; ++w) s += red[w][c];
        partials[(int64_t)tile * mmax + c] = s;
    }
}

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

// x0 = V_i y_i on the owned rows (boolean PoU: direct global write) or on Omega_i (plocal, summed
// over the copies afterwards).
__global__ void __launch_bounds__(S2L_TILE_ROWS) coarse_prolong_kernel(const int32_t* __restrict__ t_sub,
                                                                       const int32_t* __restrict__ t_row0,
                                                                       const int32_t* __restrict__ t_nrow,
                                                                       const DevSub* __restrict__ subs,
                                                                       const double* __restrict__ V, int boolean_pou,
                                                                       const double* __restrict__ y,
                                                                       double* __restrict__ out,
                                                                       double* __restrict__ plocal)
{
    const int tile = blockIdx.x;
    if ((int)threadIdx.x >= t_nrow[tile]) return;
    const DevSub sd = subs[t_sub[tile]];
    const int l = t_row0[tile] + threadIdx.x;
    const double* vr = V + sd.v_off + (int64_t)l * sd.m;
    const double* yc = y + sd.c_off;
    double s = 0.0;
    for (int c = 0; c < sd.m; ++c) s += vr[c] * yc[c];
    if (boolean_pou)
        out[sd.begin + l] = s;
    else
        plocal[sd.loc_off + l] = s;
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
    const int grid = S2L_NB_RED;
    switch (tpr) {
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

template <typename Real>
cudaError_t launch_local_solve(cudaStream_t st, const LocalSolveArgs<Real>& a, int nblocks, size_t smem, int tr_first,
                               int tr_count, int us_first, int us_count, int* launches)
{
    cudaError_t e;
    if (smem > 0) {
        // the limit is a process-wide attribute of the kernel: always the same cap, so launches of
        // setups with different shared-memory sizes from several threads cannot undercut each other
        if (smem > S2L_SWEEP_SMEM_CAP) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(sweep_kernel<Real, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 S2L_SWEEP_SMEM_CAP);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(sweep_kernel<Real, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 S2L_SWEEP_SMEM_CAP);
        if (e != cudaSuccess) return e;
        sweep_kernel<Real, true, true><<<nblocks, S2L_BS_SWEEP, smem, st>>>(a);
    } else {
        sweep_kernel<Real, false, true><<<nblocks, S2L_BS_SWEEP, 0, st>>>(a);
    }
    int nl = 1;
    if (tr_count > 0) {
        const int grid = (tr_count + 7) / 8;
        tail_rhs_kernel<Real><<<grid, 256, 0, st>>>(a, tr_first, tr_count);
        tail_gemv_kernel<Real, true><<<grid, 256, 0, st>>>(a, a.linv, a.ybuf, a.xbuf, tr_first, tr_count);
        tail_gemv_kernel<Real, false><<<grid, 256, 0, st>>>(a, a.uinv, a.xbuf, a.ybuf, tr_first, tr_count);
        nl += 3;
    }
    if (us_count > 0) {
        sparse_coupling_kernel<Real><<<(us_count + 7) / 8, 256, 0, st>>>(a, us_first, us_count);
        nl += 1;
    }
    if (smem > 0)
        sweep_kernel<Real, true, false><<<nblocks, S2L_BS_SWEEP, smem, st>>>(a);
    else
        sweep_kernel<Real, false, false><<<nblocks, S2L_BS_SWEEP, 0, st>>>(a);
    *launches = nl + 1;
    return cudaGetLastError();
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

void launch_coarse_restrict(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                            const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                            int boolean_pou, const double* r, int mmax, double* partials)
{
    coarse_restrict_kernel<<<ntiles, S2L_TILE_ROWS, 0, st>>>(t_sub, t_row0, t_nrow, subs, V, l2g, boolean_pou, r,
                                                             mmax, partials);
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

void launch_coarse_prolong(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                           const int32_t* t_nrow, const DevSub* subs, const double* V, int boolean_pou,
                           const double* y, double* out, double* plocal)
{
    coarse_prolong_kernel<<<ntiles, S2L_TILE_ROWS, 0, st>>>(t_sub, t_row0, t_nrow, subs, V, boolean_pou, y, out,
                                                            plocal);
}

}  // namespace s2l
