// AMG local solves (the reference's --local-approx amg, src/linalg/inexact_solver.cpp:45-178): one
// V-cycle from x = 0 per subdomain, every subdomain at once.
//
// Layout: level l of every subdomain that has it is concatenated into the level space l (subdomain
// i at lvl_off[l][i]); A_l, R_l (rows in level l + 1) and P_l (rows in level l) are block-diagonal
// CSR matrices over these spaces, so a residual, a restriction or a prolongation is one launch for
// all subdomains.  Gauss-Seidel sweeps run one CTA per subdomain over wavefronts of its rows (rows
// of one wavefront read no row updated in the same wavefront, and no row of a later wavefront has
// been updated yet), a group of lanes per row.
// The coarsest level of a subdomain is solved with its dense inverse.
#include "s2l_internal.cuh"

#include <algorithm>

namespace {

int amg_grid(int64_t work, int bs)
{
    const int64_t g = (work + bs - 1) / bs;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// x(i) = (f(i) - sum_{j != i} A(i, j) x(j)) / A(i, i) over the rows of each wavefront in turn, a
// group of G lanes per row (the lanes split the row's entries, then add their parts by shuffles;
// the sum is reassociated, the serial sweep's rounding is not kept).  With SMEM the subdomain's x
// (rows [o, o + n) of the level space) lives in shared memory for the whole sweep (the operator is
// block-diagonal, so a row reads no other subdomain's x).
template <bool SMEM, int G, typename Real>
__global__ void __launch_bounds__(1024) gs_sweep_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                        const Real* __restrict__ v, const Real* __restrict__ f,
                                                        Real* x, const int32_t* __restrict__ sched,
                                                        const int64_t* __restrict__ wf_ptr,
                                                        const int32_t* __restrict__ sub_wf,
                                                        const int64_t* __restrict__ sub_off,
                                                        const int32_t* __restrict__ sub_n)
{
    extern __shared__ __align__(16) unsigned char gs_smem[];
    Real* xs = reinterpret_cast<Real*>(gs_smem);
    const int b = blockIdx.x;
    const int64_t o = sub_off[b];
    const int n = sub_n[b];
    const int lg = threadIdx.x & (G - 1), grp = threadIdx.x / G, ngrp = blockDim.x / G;
    if (SMEM) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) xs[k] = x[o + k];
        __syncthreads();
    }
    for (int w = sub_wf[b]; w < sub_wf[b + 1]; ++w) {
        const int64_t end = wf_ptr[w + 1];
        for (int64_t kb = wf_ptr[w]; kb < end; kb += ngrp) {  // the same trip count for every lane
            const int64_t k = kb + grp;
            const bool valid = k < end;
            const int i = valid ? sched[k] : 0;
            Real part = Real(0), dpart = Real(0);
            int has = 0;
            if (valid)
                for (int64_t e = rp[i] + lg; e < rp[i + 1]; e += G) {
                    const int c = ci[e];
                    const Real a = v[e];
                    if (c == i) {
                        dpart = a;
                        has = 1;
                    } else {
                        part += a * (SMEM ? xs[c - o] : x[c]);
                    }
                }
#pragma unroll
            for (int m = G / 2; m; m >>= 1) {
                part += __shfl_xor_sync(0xffffffffu, part, m, G);
                dpart += __shfl_xor_sync(0xffffffffu, dpart, m, G);
                has += __shfl_xor_sync(0xffffffffu, has, m, G);
            }
            if (valid && lg == 0) {
                const Real D = has ? dpart : Real(1);
                const Real val = (Real(1) / D) * (f[i] - part);
                if (SMEM) xs[i - o] = val;
                else x[i] = val;
            }
        }
        __syncthreads();
    }
    if (SMEM)
        for (int k = threadIdx.x; k < n; k += blockDim.x) x[o + k] = xs[k];
}

// mode 0: y = M x, 1: y += M x, 2: y = f - M x.  A warp takes 32 consecutive rows: their entries
// are contiguous, so the warp loads them with coalesced loads and leaves the products in shared
// memory (pieces of 512 entries); lane j then adds row j's products in entry order.
template <typename Real>
__global__ void __launch_bounds__(256) csr_chunk_kernel(int64_t n, const int64_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const Real* __restrict__ v,
                                                        const Real* __restrict__ x, const Real* __restrict__ f,
                                                        Real* __restrict__ y, int mode)
{
    constexpr int CAP = 512;
    __shared__ Real prod[8][CAP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Real* wp = prod[warp];
    const int64_t nchunks = (n + 31) / 32;
    for (int64_t ch = (int64_t)blockIdx.x * 8 + warp; ch < nchunks; ch += (int64_t)gridDim.x * 8) {
        const int64_t r0 = ch * 32, row = r0 + lane;
        const int64_t rend = r0 + 32 < n ? r0 + 32 : n;
        const int64_t e_lo = rp[r0], e_hi = rp[rend];
        const int64_t my0 = row < n ? rp[row] : e_hi, my1 = row < n ? rp[row + 1] : e_hi;
        Real s = Real(0);
        for (int64_t base = e_lo; base < e_hi; base += CAP) {
            const int cnt = (int)(e_hi - base < CAP ? e_hi - base : CAP);
            for (int e = lane; e < cnt; e += 32) wp[e] = v[base + e] * x[ci[base + e]];
            __syncwarp();
            const int64_t s0 = (my0 > base ? my0 : base) - base;
            const int64_t s1 = (my1 < base + cnt ? my1 : base + cnt) - base;
            for (int64_t e = s0; e < s1; ++e) s += wp[e];
            __syncwarp();
        }
        if (row < n) y[row] = mode == 2 ? f[row] - s : (mode == 1 ? y[row] + s : s);
    }
}

// x_c = C^-1 f_c for every subdomain whose coarsest level is this one (one CTA each; C^-1 stored
// column by column, so the threads of a row block read consecutive entries)
template <typename Real>
__global__ void coarse_inverse_kernel(const int32_t* __restrict__ c_sub_off, const int32_t* __restrict__ c_n,
                                      const int64_t* __restrict__ c_inv_off, const Real* __restrict__ Cinv,
                                      const Real* __restrict__ f, Real* __restrict__ x)
{
    const int b = blockIdx.x;
    const int n = c_n[b];
    const int64_t o = c_sub_off[b];
    const Real* M = Cinv + c_inv_off[b];
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        Real s = Real(0);
        for (int c = 0; c < n; ++c) s += M[(int64_t)c * n + r] * f[o + c];  // M stored transposed
        x[o + r] = s;
    }
}

// level-0 right-hand side: f(p) = in(l2g(p)) (global input) or local_in(p - off) (one subdomain)
template <typename Real>
__global__ void amg_gather_kernel(int64_t n, const int32_t* __restrict__ l2g, const double* __restrict__ in,
                                  const double* __restrict__ local_in, int64_t lo, int64_t hi,
                                  Real* __restrict__ f)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        if (local_in) f[p] = (Real)((p >= lo && p < hi) ? local_in[p - lo] : 0.0);
        else f[p] = (Real)in[l2g[p]];
    }
}

// outputs of the level-0 solution: owned rows to out (+ base), the local space, or one subdomain
template <typename Real>
__global__ void amg_scatter_kernel(int64_t n, const int32_t* __restrict__ out_idx, const Real* __restrict__ x,
                                   const double* __restrict__ base, double* __restrict__ out, int mode, int64_t lo,
                                   int64_t hi)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const double xp = (double)x[p];
        if (mode == 0) {
            const int32_t g = out_idx[p];
            if (g >= 0) out[g] = base ? xp + base[g] : xp;
        } else if (mode == 1) {
            out[p] = xp;
        } else if (p >= lo && p < hi) {
            out[p - lo] = xp;
        }
    }
}

}  // namespace

namespace s2l {

template <int G, typename Real>
void gs_launch(cudaStream_t st, int nsub_lvl, bool sm, size_t smem, const int64_t* rp, const int32_t* ci,
               const Real* v, const Real* f, Real* x, const int32_t* sched, const int64_t* wf_ptr,
               const int32_t* sub_wf, const int64_t* sub_off, const int32_t* sub_n)
{
    if (sm) {
        cudaFuncSetAttribute(gs_sweep_kernel<true, G, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)S2L_GS_SMEM_CAP);
        gs_sweep_kernel<true, G, Real><<<nsub_lvl, 1024, smem, st>>>(rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off,
                                                                   sub_n);
    } else {
        gs_sweep_kernel<false, G, Real><<<nsub_lvl, 1024, 0, st>>>(rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off,
                                                                 sub_n);
    }
}

template <typename Real>
void launch_gs_sweep(cudaStream_t st, int nsub_lvl, const int64_t* rp, const int32_t* ci, const Real* v, const Real* f,
                     Real* x, const int32_t* sched, const int64_t* wf_ptr, const int32_t* sub_wf,
                     const int64_t* sub_off, const int32_t* sub_n, int max_n, int lanes)
{
    if (nsub_lvl <= 0) return;
    const size_t smem = (size_t)max_n * sizeof(Real);
    const bool sm = smem <= S2L_GS_SMEM_CAP;
    switch (lanes) {
    case 4: gs_launch<4>(st, nsub_lvl, sm, smem, rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off, sub_n); break;
    case 8: gs_launch<8>(st, nsub_lvl, sm, smem, rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off, sub_n); break;
    case 16: gs_launch<16>(st, nsub_lvl, sm, smem, rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off, sub_n); break;
    default: gs_launch<32>(st, nsub_lvl, sm, smem, rp, ci, v, f, x, sched, wf_ptr, sub_wf, sub_off, sub_n); break;
    }
}

template <typename Real>
void launch_csr_mv(cudaStream_t st, int64_t n, const int64_t* rp, const int32_t* ci, const Real* v, const Real* x,
                   Real* y, int accumulate)
{
    if (n > 0)
        csr_chunk_kernel<Real><<<amg_grid(n, 256), 256, 0, st>>>(n, rp, ci, v, x, nullptr, y, accumulate ? 1 : 0);
}

template <typename Real>
void launch_csr_residual(cudaStream_t st, int64_t n, const int64_t* rp, const int32_t* ci, const Real* v,
                         const Real* f, const Real* x, Real* t)
{
    if (n > 0) csr_chunk_kernel<Real><<<amg_grid(n, 256), 256, 0, st>>>(n, rp, ci, v, x, f, t, 2);
}

template <typename Real>
void launch_coarse_inverse(cudaStream_t st, int ncoarse, const int32_t* c_sub_off, const int32_t* c_n,
                           const int64_t* c_inv_off, const Real* Cinv, const Real* f, Real* x)
{
    if (ncoarse > 0) coarse_inverse_kernel<Real><<<ncoarse, 256, 0, st>>>(c_sub_off, c_n, c_inv_off, Cinv, f, x);
}

template <typename Real>
void launch_amg_gather(cudaStream_t st, int64_t n, const int32_t* l2g, const double* in, const double* local_in,
                       int64_t lo, int64_t hi, Real* f)
{
    if (n > 0) amg_gather_kernel<Real><<<amg_grid(n, 256), 256, 0, st>>>(n, l2g, in, local_in, lo, hi, f);
}

template <typename Real>
void launch_amg_scatter(cudaStream_t st, int64_t n, const int32_t* out_idx, const Real* x, const double* base,
                        double* out, int mode, int64_t lo, int64_t hi)
{
    if (n > 0) amg_scatter_kernel<Real><<<amg_grid(n, 256), 256, 0, st>>>(n, out_idx, x, base, out, mode, lo, hi);
}

#define S2L_AMG_INSTANTIATE(Real)                                                                                      \
    template void launch_gs_sweep<Real>(cudaStream_t, int, const int64_t*, const int32_t*, const Real*, const Real*,   \
                                        Real*, const int32_t*, const int64_t*, const int32_t*, const int64_t*,         \
                                        const int32_t*, int, int);                                                     \
    template void launch_csr_mv<Real>(cudaStream_t, int64_t, const int64_t*, const int32_t*, const Real*, const Real*, \
                                      Real*, int);                                                                     \
    template void launch_csr_residual<Real>(cudaStream_t, int64_t, const int64_t*, const int32_t*, const Real*,       \
                                            const Real*, const Real*, Real*);                                          \
    template void launch_coarse_inverse<Real>(cudaStream_t, int, const int32_t*, const int32_t*, const int64_t*,      \
                                              const Real*, const Real*, Real*);                                        \
    template void launch_amg_gather<Real>(cudaStream_t, int64_t, const int32_t*, const double*, const double*, int64_t, \
                                          int64_t, Real*);                                                             \
    template void launch_amg_scatter<Real>(cudaStream_t, int64_t, const int32_t*, const Real*, const double*, double*,  \
                                           int, int64_t, int64_t);
S2L_AMG_INSTANTIATE(double)
S2L_AMG_INSTANTIATE(float)
#undef S2L_AMG_INSTANTIATE

}  // namespace s2l
