// Internal device data layout of the B200 solve phase.
//
// Everything of one matrix lives in HBM for the whole solve phase:
//  * the renumbered global CSR (int32 indices, FP64 values);
//  * the "local space": the concatenation of every subdomain's local vector, subdomain i at
//    [loc_off_i, loc_off_i + n_i), in the factor's permuted numbering;
//  * per subdomain, each triangular factor split at a tail index T_i:
//      sparse part  rows [0, T) : stored row-wise IN SOLVE ORDER (a topological order of the rows),
//                                 off-diagonal entries only, inverse diagonal apart;
//      coupling     L(T:n, 0:T) rows of the tail / U(0:T, T:n) rows of the sparse part: CSR;
//      dense tail   the inverse of the trailing triangle L(T:n, T:n) / U(T:n, T:n), row-major s x s
//                   (s = n - T), computed once at setup, so the tail solve is a dense GEMV;
//  * the coarse basis row-major (n_rows_i x m_i), the dense inverse of E (n0 x n0, row-major);
//  * a "copies" CSR mapping each global row to its copies in the local space (used when the
//    one-level result or the prolongation must be summed over subdomains).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define S2L_BS_SWEEP 1024    // threads of a sweep CTA (one CTA per subdomain)
#define S2L_BS_VEC 256        // threads of the vector / SpMV kernels
#define S2L_NB_RED 592        // blocks of every kernel that produces reduction partials (4 x 148 SMs)
#define S2L_MAX_RED_COLS 128  // columns of the reduction buffer
#define S2L_MAX_RHS 16        // right-hand sides of one block solve
#define S2L_MAX_BLOCK_COLS 1024  // Krylov coefficients of a block step: (restart + 1) x K at most
#define S2L_TILE_ROWS 256     // rows of one coarse restrict/prolong tile
#define S2L_SWEEP_WARPS (S2L_BS_SWEEP / 32)
#define S2L_BATCH_CHUNKS 8    // chunks of a task loaded together (all loads issued before the first wait)
#define S2L_CHAIN_DEFAULT 8   // rows of a chain block (setup option "chain_block")
#define S2L_CHAIN_MAX 16
#define S2L_SWEEP_SMEM_CAP (227 * 1024 - 64)  // dynamic shared memory of a sweep CTA, at most
#define S2L_ADMIT_WAIT_S 600   // longest wait of a call for a free workspace when the HBM budget is full
#ifndef S2L_SPIN_SLEEP_NS
#define S2L_SPIN_SLEEP_NS 0   // pause of a sweep warp after a poll that found a column not ready (ns; 0 = none)
#endif
#define S2L_SPIN_LIMIT (1 << 24)  // polls of one ready flag before a sweep gives up (error 1)
#define S2L_GS_SMEM_CAP (224 * 1024)  // shared memory of a Gauss-Seidel sweep CTA (its subdomain's x)

struct DevSub {
    int64_t begin;      // first owned global row
    int64_t loc_off;    // offset of the subdomain in the local space
    int n_owned;
    int n_local;
    int T;              // rows [0, T) sparse, [T, n_local) dense tail
    int tr_first;       // first entry of the subdomain in the tail-row list
    int us_first;       // first entry of the subdomain in the sparse-row coupling list
    int pad;
    int64_t d_off;      // offset of the subdomain's s x s inverse tails
    // coarse basis
    int m;
    int v_rows;         // rows stored: n_owned (boolean PoU) or n_local
    int64_t v_off;      // offset into coarse_v
    int64_t c_off;      // coarse offset of the subdomain (first coarse unknown)
};

// Sparse part of one factor of every subdomain.  Its rows are renumbered in solve order (slot =
// row: a topological order, rows of one dependency level next to each other), and so are the
// columns, so a sweep needs no row-index array.  Slot p belongs to group p % NG; the entries of a
// group's rows are stored one row after the other, so a group finds the start of its next row by
// adding the lengths of its previous rows, without a load from memory.
template <typename Real>
struct SweepFactor {
    const int32_t* col;        // column slots (-1: padding), per warp, each task lane-interleaved
    const Real* val;           // values times 1/diag of their row
    const Real* dinv;          // per slot (local space layout); the right-hand side is scaled by it
    const uint32_t* thdr;      // per task: chunks C (bits 0-15), log2 G (16-18), rows R - 1 (19-23)
    const int32_t* tslot;      // per task: its R slots
    const int64_t* wtask;      // per (subdomain, warp), plus one: first task
    const int64_t* wslot;      //   first entry of the slot lists
    const int64_t* went;       //   first entry of col / val
    // chain blocks: blocks blk_first[i] .. blk_first[i + 1] of subdomain i; block b has the slots
    // blk_slot[blk_off[b] .. blk_off[b + 1]) (solve order) and W^-1 packed at blk_inv + blk_ioff[b]
    const int32_t* blk_first;
    const int64_t* blk_off;
    const int64_t* blk_ioff;
    const int32_t* blk_slot;
    const Real* blk_inv;
};

template <typename Real>
struct LocalSolveArgs {
    const DevSub* subs;
    const int32_t* sub_list;   // CTA b of a sweep works on subdomain sub_list[b] (nullptr: b)
    SweepFactor<Real> f[2];    // 0 = L (forward), 1 = U (backward)
    // tail rows of every subdomain: (sub, i) pairs, L(T+i, 0:T) coupling CSR
    const int32_t* tr_sub;
    const int32_t* tr_i;
    const int64_t* lts_ptr;
    const int32_t* lts_col;
    const Real* lts_val;
    // sparse rows with U(r, T:n) coupling: (sub, r) pairs and CSR (columns as local-space indices,
    // loc_off + tail row), longest rows first within a subdomain; unit u (one warp) holds the rows
    // uu[u] .. uu[u + 1] - 1, 32 / (its row count) lanes per row
    const int32_t* us_sub;
    const int32_t* us_r;
    const int64_t* ust_ptr;
    const int32_t* ust_col;
    const Real* ust_val;
    const int32_t* uu;
    const Real* linv;          // inverse tails, row-major per subdomain
    const Real* uinv;
    const int32_t* gather;     // slot k -> index into `in` (global gather, or perm_in for a local input)
    const int32_t* gout;       // local j -> x position: backward slot (< T) or tail row (>= T)
    const int32_t* u2l;        // backward slot -> forward slot (the hand-off between the two sweeps)
    const double* in;
    const double* base;        // added to the owned output (x0 of the coarse correction), may be null
    double* out;               // global output (direct mode) or local output (mode 2)
    double* ylocal;            // local-space output (mode 1)
    Real* ybuf;                // local-space work vectors
    Real* xbuf;
    uint8_t* gflags;           // ready flags when a sweep does not fit shared memory
    int* err;                  // device error word (1: a sweep wait gave up)
    int mode;                  // 0 direct owned write, 1 local-space write, 2 local input/output
    // right-hand sides: every vector above holds K interleaved columns (entry i of column r at
    // i * K + r); a sweep CTA takes KC of them (K / KC CTAs per subdomain); single solves: 1, 1
    int K;
    int KC;
    int64_t nloc;              // local-space size (stride of the per-column-group ready flags)
    int spin_limit;            // polls of one ready flag before a sweep gives up (S2L_SPIN_LIMIT by default)
    int spin_sleep_ns;         // pause of a warp after a poll that found a column not ready (0: none)
    int sweep_pf;              // chunks after a task that a sweep warp hints into L2 (0 .. 32)
};

// Numeric refactorization of every subdomain's factors on their kept patterns (s2l_gpu_refactor).
// The factor values live in F, subdomain i's pattern column by column ("combined" CSC: for LU the
// strict upper rows, the diagonal, then the strict lower rows of each column; for LL^T the lower
// rows, diagonal first).  Columns are numbered in the local space (loc_off + j).
struct RefactorArgs {
    const DevSub* subs;
    double* F;
    const int64_t* fbase;      // per subdomain: its first position in F
    const int64_t* fcp;        // per column (nloc + 1): first position (absolute)
    const int32_t* fri;        // per position: row (subdomain-local), increasing within a column
    const int32_t* fdg;        // per column: index of the diagonal within the column
    const uint8_t* fllt;       // per column: 1 if its subdomain's factor is L L^T
    const int64_t* frp;        // L L^T: per column j (nloc + 1), range of its row entries L(j, k), k < j
    const int32_t* frpos;      //   position of L(j, k) (relative to the subdomain's fbase)
    const int32_t* frk;        //   k (subdomain-local), increasing
    const int32_t* lv_first;   // per subdomain (nsub + 1): first dependency level of its sparse columns
    const int64_t* lv_off;     // per level (+1): range in lv_col
    const int32_t* lv_col;     // sparse columns (j < T, subdomain-local) level by level
    const int32_t* tc_sub;     // tail columns (j >= T): subdomain and local column
    const int32_t* tc_col;
    int64_t ntc;
    double* S;                 // dense tails (s x s row-major at subs[i].d_off)
    int smax;                  // largest tail: the per-warp row maps hold smax uint16 positions
    int maxcol;                // longest column of F
    int nlmax;                 // largest subdomain (rows): the cooperative column map
    double* part;              // partial columns of the cooperative column updates: per subdomain
                               // and warp, maxcol doubles
    int* err;                  // first failure: 1 zero / non-positive pivot of a sparse column, 4 an LU
                               // pivot below pivot_tol relative to its column (0: none)
    double pivot_tol;          // LU: largest allowed multiplier is 1 / pivot_tol (0: no check)
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
void launch_dot2(cudaStream_t st, int64_t n, const double* x, const double* y, const double* z, double* partials,
                 double* out);
// K right-hand sides (block vectors n x K interleaved; K = 1, 2, 4, 8 or 16)
void launch_spmv_block(cudaStream_t st, int64_t n, int K, const int32_t* rp, const int32_t* ci, const double* v,
                       const double* X, double* Y, const double* B, double* partials, double* red_out, int tpr);
// Block Krylov bases may sit in a ring of `ring` blocks: basis vector j is block (j0 + j) % ring
// (ring 0: block j0 + j).  A ColFirst mask makes the update coefficients h(j, r) with j < f[r]
// zero (column r's own basis starts there).
struct ColFirst {
    int f[S2L_MAX_RHS];
};
struct ColScale {
    double v[S2L_MAX_RHS];
};
void launch_mdot_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* w,
                       double* partials, double* out, int j0 = 0, int ring = 0);
void launch_gemv_update_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* h,
                              double alpha, double* w, double* partials, double* red_out, int j0 = 0, int ring = 0,
                              const ColFirst* first = nullptr);
void launch_gemv_block(cudaStream_t st, int64_t n, int K, const double* V, int64_t ldv, int J, const double* y,
                       double* u, int j0 = 0, int ring = 0);
// y(:, r) = a(r) x(:, r) + c(r) z(:, r) (a source with a zero coefficient is not read)
void launch_combine2_block(cudaStream_t st, int64_t n, int K, const ColScale& a, const double* x, const ColScale& c,
                           const double* z, double* y);
// column r of an n x K interleaved block from / to a plain vector; column r of count blocks set to v
void launch_column_in(cudaStream_t st, int64_t n, int K, int r, const double* src, double* dst);
void launch_column_out(cudaStream_t st, int64_t n, int K, int r, const double* src, double* dst);
void launch_column_fill(cudaStream_t st, int64_t n, int K, int r, int count, int64_t ld, double v, double* dst);
void launch_axpby_block(cudaStream_t st, int64_t n, int K, const double* a, const double* x, const double* b,
                        double* y);
void launch_interleave(cudaStream_t st, int64_t n, int K, int k, const double* src, double* dst);
void launch_deinterleave(cudaStream_t st, int64_t n, int K, int k, const double* src, double* dst);
void launch_combine_block(cudaStream_t st, int64_t n, int K, const int64_t* cp_ptr, const int32_t* cp_pos,
                          const double* cp_w, const double* ylocal, const double* base, double* out);
void launch_coarse_restrict_block(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                                  const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                                  int boolean_pou, const double* R, int mmax, double* partials);
void launch_coarse_reduce_block(cudaStream_t st, int K, int nsub, const DevSub* subs, const int32_t* t_first, int mmax,
                                const double* partials, double* cvec);
void launch_dense_gemm(cudaStream_t st, int K, int n0, const double* M, const double* X, double* Y);
void launch_coarse_prolong_block(cudaStream_t st, int K, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                                 const int32_t* t_nrow, const DevSub* subs, const double* V, int mmax, int boolean_pou,
                                 const double* Y, double* out, double* plocal);
// out[0] = sum |a - alpha c| (c may be nullptr), out[1] = sum a
void launch_l1(cudaStream_t st, int64_t n, const double* a, double alpha, const double* c, double* partials,
               double* out);
// out[0] = sum |V(:, 0:k) q|
void launch_gemv_l1(cudaStream_t st, int64_t n, const double* V, int64_t ldv, int k, const double* q, double* partials,
                    double* out);
void launch_bicg_p(cudaStream_t st, int64_t n, const double* r, const double* v, double beta, double omega, double* p,
                   int first);
void launch_bicg_s(cudaStream_t st, int64_t n, const double* r, const double* v, double alpha, double* s,
                   double* partials, double* out);
void launch_bicg_x(cudaStream_t st, int64_t n, double* x, const double* y, const double* z, double alpha,
                   double omega, double* r, const double* s, const double* t, const double* rh, double* partials,
                   double* out);

// The local solve of every subdomain (or one): forward sweep, tail coupling, two dense tail GEMVs,
// backward coupling, backward sweep + epilogue.  `tr_range`/`us_range` restrict the row-list
// kernels (first, count); `launches` receives the number of kernels issued.
template <typename Real>
cudaError_t launch_local_solve(cudaStream_t st, const LocalSolveArgs<Real>& a, int nblocks, size_t smem_bytes,
                               int tr_first, int tr_count, int uu_first, int uu_count, int* launches);

void launch_combine(cudaStream_t st, int64_t n, const int64_t* cp_ptr, const int32_t* cp_pos, const double* cp_w,
                    const double* ylocal, const double* base, double* out);
void launch_coarse_restrict(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                            const int32_t* t_nrow, const DevSub* subs, const double* V, const int32_t* l2g,
                            int boolean_pou, const double* r, int mmax, double* partials);
void launch_coarse_reduce(cudaStream_t st, int nsub, const DevSub* subs, const int32_t* t_first, int mmax,
                          const double* partials, double* c);
void launch_dense_gemv(cudaStream_t st, int n0, const double* M, const double* x, double* y);
void launch_coarse_prolong(cudaStream_t st, int ntiles, const int32_t* t_sub, const int32_t* t_row0,
                           const int32_t* t_nrow, const DevSub* subs, const double* V, int mmax, int boolean_pou,
                           const double* y, double* out, double* plocal);
void launch_to_float(cudaStream_t st, const double* in, float* out, int64_t n);

// AMG local solves (amg.cu), in the precision Real of the hierarchy (double, or float for the
// reference's --local-precision single)
// a Gauss-Seidel sweep of every smoothed subdomain of a level (CTA b: rows [sub_off[b], + sub_n[b])
// of the level space, kept in shared memory when max_n values fit S2L_GS_SMEM_CAP), `lanes`
// (4, 8, 16 or 32) lanes per row
template <typename Real>
void launch_gs_sweep(cudaStream_t st, int nsub_lvl, const int64_t* rp, const int32_t* ci, const Real* v, const Real* f,
                     Real* x, const int32_t* sched, const int64_t* wf_ptr, const int32_t* sub_wf,
                     const int64_t* sub_off, const int32_t* sub_n, int max_n, int lanes);
template <typename Real>
void launch_csr_mv(cudaStream_t st, int64_t n, const int64_t* rp, const int32_t* ci, const Real* v, const Real* x,
                   Real* y, int accumulate);
template <typename Real>
void launch_csr_residual(cudaStream_t st, int64_t n, const int64_t* rp, const int32_t* ci, const Real* v,
                         const Real* f, const Real* x, Real* t);
template <typename Real>
void launch_coarse_inverse(cudaStream_t st, int ncoarse, const int32_t* c_sub_off, const int32_t* c_n,
                           const int64_t* c_inv_off, const Real* Cinv, const Real* f, Real* x);
template <typename Real>
void launch_amg_gather(cudaStream_t st, int64_t n, const int32_t* l2g, const double* in, const double* local_in,
                       int64_t lo, int64_t hi, Real* f);
template <typename Real>
void launch_amg_scatter(cudaStream_t st, int64_t n, const int32_t* out_idx, const Real* x, const double* base,
                        double* out, int mode, int64_t lo, int64_t hi);

// refactorization (refactor.cu)
void launch_refactor_fill(cudaStream_t st, int64_t count, const int64_t* src, const int64_t* dst, const double* val,
                          double* F);
// cs CTAs (a thread-block cluster) per subdomain; the partial columns hold nsub x cs x
// refactor_sparse_warps(smax) x maxcol doubles
void launch_refactor_sparse(cudaStream_t st, const RefactorArgs& a, int nsub, int cs);
int refactor_sparse_warps(int smax);
size_t refactor_map_bytes(int smax, int warps);
void launch_refactor_tail_columns(cudaStream_t st, const RefactorArgs& a);
void launch_refactor_gather_tails(cudaStream_t st, const RefactorArgs& a);
void launch_tail_growth(cudaStream_t st, const double* S, int s, double tol, int* err);
void launch_identity(cudaStream_t st, double* M, int s);
template <typename Real>
void launch_tail_inverses(cudaStream_t st, const double* S, const double* B, int s, int llt, Real* linv, Real* uinv);
template <typename Real>
void launch_refactor_sweep_values(cudaStream_t st, int nsub, const int64_t* fbase, const double* F,
                                  const int64_t* wtask, const int64_t* wslot, const int64_t* went,
                                  const uint32_t* thdr, const int32_t* tslot, const int32_t* src, const DevSub* subs,
                                  const int32_t* dsrc, Real* val);
template <typename Real>
void launch_refactor_dinv(cudaStream_t st, int nsub, const DevSub* subs, const int64_t* fbase, const double* F,
                          const int32_t* dsrc, Real* dinv);
template <typename Real>
void launch_refactor_blocks(cudaStream_t st, int64_t nblocks, const int64_t* boff, const int64_t* bioff,
                            const int64_t* wsrc, const int64_t* be_off, const int64_t* be_pos, const uint8_t* be_row,
                            const int64_t* be_cp, const uint8_t* bc_b, const int64_t* bc_pos, const double* F,
                            Real* binv, Real* val);
template <typename Real>
void launch_gather_values(cudaStream_t st, int64_t count, const int64_t* src, const double* F, Real* out);
void launch_row_sums(cudaStream_t st, int64_t n, const int32_t* rp, const double* v, double* out);
// coarse matrix for a boolean partition of unity, directly: per row the products with the bases of
// the subdomains owning its columns (Z), then one block of E per pair of subdomains meeting in a row
void launch_coarse_direct(cudaStream_t st, int64_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          const int32_t* owner, const int64_t* rs_ptr, const int32_t* rs_sub, const int64_t* rs_zoff,
                          int npairs, const int32_t* pair_j, const int32_t* pair_i, const int64_t* pair_ptr,
                          const int32_t* pair_rl, const int64_t* pair_zoff, const DevSub* subs, const double* V,
                          double* Z, int64_t n0, double* E);
// coarse matrix refresh, general partition of unity: unit block, E columns
void launch_unit_block(cudaStream_t st, int64_t n0, int c0, double* Y);
void launch_scatter_columns(cudaStream_t st, int64_t n0, int c0, const double* C, double* E);

}  // namespace s2l
