// Internal device data layout of the B200 solve phase.
//
// Everything of one matrix lives in HBM for the whole solve phase:
//  * the renumbered global CSR (int32 indices, FP64 values);
//  * the "local space": the concatenation of every subdomain's local vector
//    [owned | ghosts], subdomain i at [loc_off_i, loc_off_i + n_i);
//  * per subdomain, the two triangular factors stored row-wise IN SOLVE ORDER (level by level),
//    diagonal split off as its inverse, columns in the factor's permuted numbering;
//  * the coarse basis row-major (n_rows_i x m_i), the dense inverse of E (n0 x n0, row-major);
//  * a "copies" CSR mapping each global row to its copies in the local space (used when the
//    one-level result or the prolongation must be summed over subdomains).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define S2L_BS_SOLVE 512      // threads of the local-solve CTA (one CTA per subdomain)
#define S2L_BS_VEC 256        // threads of the vector / SpMV kernels
#define S2L_NB_RED 592        // blocks of every kernel that produces reduction partials (4 x 148 SMs)
#define S2L_MAX_RED_COLS 128  // columns of the reduction buffer
#define S2L_TILE_ROWS 256     // rows of one coarse restrict/prolong tile
#define S2L_MODE_CTA 0        // level mode: the whole CTA works on each row of the level

struct DevSub {
    int64_t begin;      // first owned global row
    int64_t loc_off;    // offset of the subdomain in the local space
    int n_owned;
    int n_local;
    // forward (L) and backward (U) schedules
    int64_t lvl_off[2];  // offset into lvl_pos / lvl_mode (nlev+1 entries of lvl_pos per factor)
    int nlev[2];
    // coarse basis
    int m;
    int v_rows;         // rows stored: n_owned (boolean PoU) or n_local
    int64_t v_off;      // offset into coarse_v
    int64_t c_off;      // coarse offset of the subdomain (first coarse unknown)
};

// One triangular factor of every subdomain, in solve order.  Row slot p of subdomain i is
// global slot loc_off_i + p; its row id (permuted numbering) is rows[slot], entries
// ptr[slot]..ptr[slot+1] (off-diagonal only), inverse diagonal dinv[slot].
template <typename Real>
struct DevFactor {
    const int32_t* rows;
    const int64_t* ptr;
    const int32_t* col;
    const Real* val;
    const Real* dinv;
};

template <typename Real>
struct SolveArgs {
    const DevSub* subs;
    const int32_t* sub_list;   // CTA b solves subdomain sub_list[b] (nullptr: b itself)
    DevFactor<Real> f[2];      // 0 = L (forward), 1 = U (backward)
    const int32_t* lvl_pos;    // level boundaries (slot offsets relative to the subdomain)
    const int8_t* lvl_mode;    // group width of each level (1..32) or S2L_MODE_CTA
    const int32_t* gin;        // gather index of slot k: global row of local perm_in[k]
    const int32_t* pin;        // perm_in itself (local-input mode)
    const int32_t* gout;       // perm_out: local j -> slot
    const double* in;          // input vector (global, or local in local-input mode)
    const double* base;        // added to the owned output (x0 of the coarse correction), may be null
    double* out;               // global output (direct mode) or local output
    double* ylocal;            // local space output (sum mode)
    Real* xscratch;            // local space scratch when the vector does not fit shared memory
    int mode;                  // 0 direct owned write, 1 local-space write, 2 local input/output
};

// launch wrappers (kernels.cu)
namespace s2l {

void launch_spmv(cudaStream_t st, int64_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* x,
                 double* y, const double* b, double* partials, double* red_out, int tpr);
void launch_reduce(cudaStream_t st, const double* partials, int nblocks, int ncols, double* out);
void launch_mdot(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* w, double* partials,
                 double* out);
void launch_gemv_update(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* h, double alpha,
                        double* w, double* partials);
void launch_gemv(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* y, double* u);
void launch_axpby(cudaStream_t st, int64_t n, double a, const double* x, double b, double* y);
void launch_scale_copy(cudaStream_t st, int64_t n, const double* x, const double* s_dev, double* y);
void launch_dot2(cudaStream_t st, int64_t n, const double* x, const double* y, const double* z, double* partials,
                 double* out);
void launch_bicg_p(cudaStream_t st, int64_t n, const double* r, const double* v, double beta, double omega, double* p,
                   int first);
void launch_bicg_s(cudaStream_t st, int64_t n, const double* r, const double* v, double alpha, double* s,
                   const double* rh, double* partials, double* out);
void launch_bicg_x(cudaStream_t st, int64_t n, double* x, const double* y, const double* z, double alpha,
                   double omega, double* r, const double* s, const double* t, const double* rh, double* partials,
                   double* out);

template <typename Real>
cudaError_t launch_local_solve(cudaStream_t st, const SolveArgs<Real>& a, int nblocks, size_t smem_bytes);

void launch_combine(cudaStream_t st, int64_t n, const int64_t* cp_ptr, const int32_t* cp_pos, const double* cp_w,
                    const double* ylocal, const double* base, double* out);
void launch_coarse_restrict(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                            const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                            int boolean_pou, const double* r, int mmax, double* partials);
void launch_coarse_reduce(cudaStream_t st, int nsub, const DevSub* subs, const int32_t* t_first, int mmax,
                          const double* partials, double* c);
void launch_dense_gemv(cudaStream_t st, int n0, const double* M, const double* x, double* y);
void launch_coarse_prolong(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                           const int32_t* t_nrow, const DevSub* subs, const double* V, int boolean_pou,
                           const double* y, double* out, double* plocal);

}  // namespace s2l
