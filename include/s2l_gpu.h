/*
 * s2l_gpu.h - C ABI of the B200 solve phase of the two-level Schwarz preconditioner.
 *
 * One GPU holds every subdomain of a matrix.  The host (the reference's setup, or any caller)
 * uploads once per matrix: the renumbered global CSR, and per subdomain its ghost list, partition
 * of unity, local triangular factors and coarse basis, then the coarse matrix.  After that the
 * solve phase runs on the device: preconditioner applications and whole Krylov solves.
 *
 * Conventions (kept from the reference's interfaces):
 *  - vectors are in the renumbered ordering, subdomain i owning rows [begin_i, begin_i + n_I,i);
 *  - local numbering of subdomain i is [owned rows | ghosts in increasing global id];
 *  - every call returns S2L_OK (0) or an S2L_ERR_* code; s2l_gpu_last_error() gives the message.
 *    The reference reports the same failures with exceptions (std::invalid_argument for bad
 *    arguments, std::runtime_error for numerical failures, std::logic_error for misuse);
 *  - calls on different setups are independent; solve-phase calls on one setup may overlap from
 *    several host threads, each on a workspace of its own (the reference's apply() is not
 *    re-entrant, include/preconditioner/two_level_schwarz.hpp:220; this one is);
 *  - pointer arguments of the solve-phase calls are host or device memory, as `ptr_kind` says.
 *    Host pointers are copied in and out on the setup's stream inside the call.
 *
 * Entry points and the reference interface each one replaces:
 *  s2l_gpu_create/destroy           no reference counterpart (device context)
 *  s2l_gpu_setup_begin .. _end      the state built by TwoLevelSchwarz's constructor
 *                                   (src/preconditioner/two_level_schwarz.cpp:20-28), uploaded
 *  s2l_gpu_spmv                     DistributedMatrix::apply (include/linalg/distributed_matrix.hpp:33-38)
 *  s2l_gpu_local_solve              LocalSolver::solve (include/linalg/local_solver.hpp:95)
 *  s2l_gpu_coarse_apply             CoarseSpace::apply (src/preconditioner/coarse_space.cpp:234-246)
 *  s2l_gpu_one_level_apply          OneLevelSchwarz::apply (src/preconditioner/one_level_schwarz.cpp:80-99)
 *  s2l_gpu_apply                    Preconditioner::apply / TwoLevelSchwarz::apply
 *                                   (include/preconditioner/preconditioner.hpp:73,
 *                                    src/preconditioner/two_level_schwarz.cpp:134-163)
 *  s2l_gpu_gmres                    Gmres::solve (include/solver/gmres.hpp:53-54, src/solver/gmres.cpp:18-161)
 *  s2l_gpu_bicgstab                 BiCgStab::solve (src/solver/bicgstab.cpp:15-154)
 */
#ifndef S2L_GPU_H
#define S2L_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct s2l_ctx s2l_ctx;
typedef struct s2l_setup s2l_setup;

/* status codes */
enum {
    S2L_OK = 0,
    S2L_ERR_BADARG = 1,    /* invalid argument (reference: std::invalid_argument) */
    S2L_ERR_OOM = 2,       /* device memory or the HBM budget exhausted */
    S2L_ERR_CUDA = 3,      /* a CUDA call failed */
    S2L_ERR_NUMERIC = 4,   /* singular coarse matrix, non-finite values (reference: std::runtime_error) */
    S2L_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
    S2L_ERR_BREAKDOWN = 6, /* Krylov breakdown */
    S2L_ERR_STATE = 7,     /* call out of order (reference: std::logic_error) */
    S2L_ERR_CANCELED = 8   /* an asynchronous solve was canceled (s2l_gpu_cancel) */
};

/* preconditioner variants (include/core/config.hpp:61-64) */
enum { S2L_ONE_LEVEL_RAS = 0, S2L_ONE_LEVEL_ASM = 1 };
enum { S2L_COARSE_NONE = 0, S2L_COARSE_ADDITIVE = 1, S2L_COARSE_DEFLATED = 2 };
enum { S2L_POU_BOOLEAN = 0, S2L_POU_MULTIPLICITY = 1 };

/* local factor kinds (include/linalg/local_solver.hpp:51-52) and storage precision */
enum { S2L_FACTOR_LU = 0, S2L_FACTOR_LLT = 1, S2L_FACTOR_LDLT = 2 };
enum { S2L_REAL_F64 = 0, S2L_REAL_F32 = 1 };

/* where a vector argument lives */
enum { S2L_PTR_HOST = 0, S2L_PTR_DEVICE = 1 };

/* Krylov methods and options (include/core/config.hpp:94-103) */
enum { S2L_KRYLOV_GMRES = 0, S2L_KRYLOV_BICGSTAB = 1 };
/* stopping norms (include/solver/krylov.hpp:21-35):
 *  S2L_STOP_L2:       ||b - A x||_2 <= rtol ||b||_2;
 *  S2L_STOP_OPENFOAM: sum|b - A x| <= max(rtol sum|b - A x0|, atol F), F the OpenFOAM normalisation
 *                     factor of x0 (sum|A x0 - xm A 1| + sum|b - xm A 1| + 1e-20, xm = mean of x0);
 *                     no iteration when x0 already satisfies it. */
enum { S2L_STOP_L2 = 0, S2L_STOP_OPENFOAM = 1 };

typedef struct {
    int restart;        /* GMRES restart length m */
    double rtol;        /* ||b - A x||_2 <= rtol ||b||_2 */
    int maxit;          /* maximum applications of the preconditioner */
    int flexible;       /* 1: flexible GMRES (stores Z_j = M^-1 v_j); 0: the reference's GMRES */
    int strict_true_residual; /* 1: converged only if the recomputed true residual is <= rtol;
                                 0: the reference's 10% slack (src/solver/gmres.cpp:148-156) */
    int history_cap;    /* capacity of result->history (0: no history) */
    int stop_norm;      /* S2L_STOP_L2 (0) or S2L_STOP_OPENFOAM */
    double atol;        /* absolute tolerance of the OpenFOAM test (0: none; needs S2L_STOP_OPENFOAM) */
} s2l_krylov_opts;

typedef struct {
    int converged;
    int breakdown;
    int iterations;           /* applications of M^-1 inside the iteration (include/solver/krylov.hpp:46) */
    int restarts;
    double rel_residual;      /* last Krylov residual estimate / ||b|| */
    double true_rel_residual; /* ||b - A x|| / ||b|| recomputed in FP64 at the end */
    int history_len;
    double* history;          /* caller-owned, history_cap entries: ||r||/||b|| after every M^-1 */
    double initial_residual_of; /* OpenFOAM normalised residual of x0 (S2L_STOP_OPENFOAM only) */
    double final_residual_of;   /* OpenFOAM normalised residual of x, recomputed (S2L_STOP_OPENFOAM only) */
} s2l_result;

/* ---- context ---------------------------------------------------------------------------- */
int s2l_gpu_create(int device, size_t hbm_budget_bytes, s2l_ctx** ctx);
int s2l_gpu_destroy(s2l_ctx* ctx);
const char* s2l_gpu_last_error(const s2l_ctx* ctx);

/* ---- setup upload (once per matrix) ---------------------------------------------------- */
int s2l_gpu_setup_begin(s2l_ctx* ctx, int64_t n, int nsub, int one_level, int coarse, int pou, s2l_setup** setup);

/* Renumbered global matrix, CSR with sorted columns (rowptr has n+1 entries). */
int s2l_gpu_set_matrix(s2l_setup* s, const int64_t* rowptr, const int64_t* col, const double* val);

/*
 * Subdomain i.  ghosts: n_ghost sorted global ids.  D: partition of unity (n_local = n_owned + n_ghost).
 * The local factor solves A_ii x = b as: t[k] = b[perm_in[k]]; L u = t; U v = u; x[j] = v[perm_out[j]].
 *   S2L_FACTOR_LU  : L unit lower (diagonal entries may be present; they are ignored), U upper with diagonal.
 *   S2L_FACTOR_LLT : L lower with diagonal, U = L^T (U_* arguments ignored).
 *   S2L_FACTOR_LDLT: L unit lower, U = diag(ldlt_d) L^T (U_* ignored).
 * L/U are CSR over the n_local rows with sorted columns; values are double or float (real_type).
 * V: coarse basis, n_local x m, column-major (m may be 0).
 */
int s2l_gpu_add_subdomain(s2l_setup* s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t* ghosts,
                          const double* D, int factor_kind, int real_type, const int32_t* perm_in,
                          const int32_t* perm_out, const int64_t* L_rowptr, const int32_t* L_col, const void* L_val,
                          const int64_t* U_rowptr, const int32_t* U_col, const void* U_val, const void* ldlt_d,
                          int m, const double* V);

/* Subdomain i with the reference's inexact local solver instead of exact factors: one AMG V-cycle
 * from x = 0 approximates A_ii^-1 (--local-approx amg, src/linalg/inexact_solver.cpp:45-178;
 * AMGCL smoothed aggregation with Gauss-Seidel smoothing).  The hierarchy is built on the host and
 * given level by level: nlev smoothed levels, level l with nrow[l] rows (nrow[0] = n_local) and
 * its operator A_l (CSR, sorted columns), and unless it is a last level without a coarser one, P_l
 * (nrow[l] x next) and R_l (next x nrow[l]) to the next level, whose size is nrow[l + 1] or, after
 * the last smoothed level, n_coarse.  The coarsest level (n_coarse rows, row-major operator; 0 for
 * none) is solved exactly.  A level is smoothed by `sweeps` forward Gauss-Seidel sweeps before the
 * coarse correction and `sweeps` backward sweeps after it.  FP64; every subdomain of a setup uses
 * the same kind of local solver and the same sweeps; block calls (s2l_gpu_apply_block,
 * s2l_gpu_gmres_block) need factors.  Owned range, ghosts, D, m and V as for s2l_gpu_add_subdomain. */
int s2l_gpu_add_subdomain_amg(s2l_setup* s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t* ghosts,
                              const double* D, int nlev, int sweeps, const int32_t* nrow,
                              const int64_t* const* A_rowptr, const int32_t* const* A_col, const double* const* A_val,
                              const int64_t* const* P_rowptr, const int32_t* const* P_col, const double* const* P_val,
                              const int64_t* const* R_rowptr, const int32_t* const* R_col, const double* const* R_val,
                              int n_coarse, const double* coarse, int m, const double* V);

/* ---- AMG hierarchies on the host (no device needed) ---------------------------------------
 * The hierarchy of one local matrix A_ii (n rows, CSR with sorted unique columns) as the
 * reference's AMGCL setup builds it for --local-approx amg (src/linalg/inexact_solver.cpp:45-178,
 * default parameters): S2L_AMG_SA smoothed aggregation or S2L_AMG_RS Ruge-Stuben
 * (--amg-coarsening), levels while a level has more than coarse_enough rows, the last one dense.
 * s2l_amg_rebuild keeps the transfer operators of `old` and recomputes the coarser operators
 * R (A P) for new values of the same pattern (--amg-reuse, AMGCL's amg::rebuild).  The levels are
 * read with s2l_amg_shape / s2l_amg_matrix (which: 0 A_l, 1 P_l, 2 R_l; rows = 0 for a last level
 * without a coarser one) / s2l_amg_coarse (row-major, n_coarse^2) in the layout
 * s2l_gpu_add_subdomain_amg takes; the pointers stay valid until s2l_amg_free. */
typedef struct s2l_amg s2l_amg;
/* coarsening, optionally | S2L_AMG_SINGLE: the whole setup in single precision, as the reference's
 * --local-precision single builds it (AMGCL's builtin<float> backend); every value returned is then a
 * float widened to double.  s2l_amg_rebuild keeps the precision of `old`. */
enum { S2L_AMG_SA = 0, S2L_AMG_RS = 1, S2L_AMG_SINGLE = 16 };
int s2l_amg_build(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, int coarse_enough,
                  int coarsening, s2l_amg** out);
int s2l_amg_rebuild(const s2l_amg* old, const int64_t* rowptr, const int32_t* col, const double* val, s2l_amg** out);
int s2l_amg_shape(const s2l_amg* h, int* nlev, int64_t* n_coarse);
int s2l_amg_matrix(const s2l_amg* h, int level, int which, int64_t* rows, int64_t* cols, const int64_t** rowptr,
                   const int32_t** col, const double** val);
int s2l_amg_coarse(const s2l_amg* h, const double** dense);
int s2l_amg_free(s2l_amg* h);

/* Coarse matrix E = R0 A R0^T (n0 x n0, row-major) and coarse offsets (nsub+1 entries). */
int s2l_gpu_set_coarse(s2l_setup* s, int64_t n0, const int64_t* offsets, const double* E);

/*
 * Layout options, before s2l_gpu_setup_end (no reference counterpart: they only choose how the
 * same factors are laid out on the device).  Each factor is split at a tail index T: rows [0, T)
 * are solved by the sparse sweeps, the trailing triangle [T, n) through its dense inverse.  T is
 * chosen per subdomain to minimise 2 * hop_us * (sparse dependency levels) + bytes * nsub / bw_gbs.
 *   "tail_min" (rows, default 64), "tail_max" (default 4096): bounds of a non-empty tail;
 *   "tail_rows" (default 0 = cost model): force every subdomain's tail to this many rows;
 *   "hop_us" (default 0.25), "bw_gbs" (default 6000): the cost model's parameters;
 *   "sweep_group" (0 = 16, 8, 16 or 32): most lanes a sparse-sweep row gets (rows of up to
 *   sweep_epl G entries get G lanes, 32 / G rows of one dependency level share a warp);
 *   "sweep_epl" (2, 4, 8 or 16, default 4): entries per lane a sparse-sweep row is sized for (a
 *   row of len entries gets the fewest lanes G, a power of two up to sweep_group, with
 *   G sweep_epl >= len): larger values pack more rows into one task, so a warp has fewer tasks,
 *   each with more entries per lane;
 *   "spmv_tpr" (0 = automatic, 1, 2, 4, 8, 16 or 32): lanes per row of the products with A; 1 is
 *   chunk mode (a warp per 32 consecutive rows, their entries loaded together); automatic: about
 *   four entries per lane from the mean row length, at least 2;
 *   "block_width" (0 = automatic, 1, 2, 4, 8 or 16): the most right-hand sides s2l_gpu_gmres_block
 *   puts in one block; larger k run as several blocks at once (automatic: the widest block whose
 *   sparse-sweep CTAs fit the SMs in one wave);
 *   "chain_block" (1..16, default 8; 1 = off): rows of a chain block.  Runs of sparse rows where
 *   each row depends on the one solved just before it (the rows of a supernode) are cut into
 *   blocks of up to this many rows; a block's rows are stored multiplied by the inverse of its
 *   diagonal block, so the block is one dependency level of the sweep instead of one per row;
 *   "refactor" (0 or 1, default 0): keep the factor patterns and their maps to the solve layout
 *   on the device so s2l_gpu_refactor can refactorize for new matrix values;
 *   "pivot_tol" (default 1e-6, 0 = no check): s2l_gpu_refactor of LU (and LDL^T) factors keeps
 *   the setup's pivot order, and reports S2L_ERR_NUMERIC when a pivot has become small against the
 *   entries it divides (a multiplier larger than 1 / pivot_tol);
 *   "spin_limit" (default 2^24): polls of one ready flag after which a sparse sweep gives up and
 *   the call returns S2L_ERR_TIMEOUT (every wait of the sweeps is bounded).  Unlike the options
 *   above it may also be set after s2l_gpu_setup_end; it applies to the launches that follow and
 *   must not be changed while a solve-phase call runs on the setup;
 *   "spin_sleep_ns" (default 0, at most 1e6): a sparse-sweep warp whose poll found a column not
 *   ready pauses this long (__nanosleep) before the next poll, leaving the issue slots to the warps
 *   that compute the rows it waits for.  Like "spin_limit" it may be set after s2l_gpu_setup_end;
 *   "sweep_prefetch" (default 8, 0 to 32): chunks of 32 entries after its current task that a
 *   sparse-sweep warp hints into L2; may be set after s2l_gpu_setup_end.
 */
int s2l_gpu_setup_option(s2l_setup* s, const char* name, double value);

int s2l_gpu_setup_end(s2l_setup* s);
int s2l_gpu_setup_destroy(s2l_setup* s);

/* New values of A with the pattern given to s2l_gpu_set_matrix (nnz doubles, host or device as
 * ptr_kind says); the preconditioner (factors, coarse basis, E) is kept.  This is the reference's
 * UpdateLevel::Reuse along a sequence of matrices (include/preconditioner/preconditioner.hpp:20-30):
 * the Krylov solves then use the new operator with the lagged preconditioner.  Refused
 * (S2L_ERR_STATE) while a solve-phase call runs or solves are queued on the setup. */
int s2l_gpu_update_matrix(s2l_setup* s, const double* val, int ptr_kind);

/* New values of A with the pattern given to s2l_gpu_set_matrix, and a new preconditioner for them
 * on the device: the reference's UpdateLevel::Refactorize (include/preconditioner/preconditioner.hpp:
 * 15-30, src/preconditioner/two_level_schwarz.cpp:30-41).  Every local factor is refactorized
 * numerically on its kept pattern and permutations (LocalSolver::refactorize,
 * src/linalg/local_solver.cpp:111-118; LU keeps the setup's row order, it does not pivot again),
 * and E = W^T A W is recomputed with the kept coarse basis and inverted (CoarseSpace::refresh,
 * src/preconditioner/coarse_space.cpp:95-105).  Needs the setup option "refactor" = 1, which keeps
 * the factor patterns and their maps to the solve layout on the device (setup stat
 * "refactor_bytes"); LU, LL^T and LDL^T factors.  S2L_ERR_NUMERIC for a non-finite value, a zero
 * (LU) or non-positive (LL^T) pivot, an LU pivot small against its column (option "pivot_tol": the
 * reference's refactorization would pivot again, this one keeps the order, so the caller rebuilds)
 * or a singular E, and then the setup is unchanged.  Refused
 * (S2L_ERR_STATE) while a solve-phase call runs or solves are queued on the setup. */
int s2l_gpu_refactor(s2l_setup* s, const double* val, int ptr_kind);

/* Device bytes held by the setup (matrix, factors, basis, schedules) and its workspaces. */
int s2l_gpu_setup_bytes(const s2l_setup* s, size_t* bytes);
/* Layout statistics after setup_end: "sparse_nnz", "coupling_nnz", "dense_entries", "tail_rows",
   "sweep_group", "smem_bytes", "levels_max" / "levels_mean" (dependency levels of a sparse sweep,
   largest and mean over subdomains and both factors), "chain_blocks", "sweep_tasks" and
   "sweep_padding" (padding entries of the lane-interleaved task layout), both factors;
   "local_solve_column_bytes": the part of s2l_gpu_local_solve_bytes that each further right-hand
   side of a block adds (a block of k reads the factors once: bytes + (k - 1) x this);
   "kc_max": right-hand sides a sparse-sweep CTA holds in shared memory; "spmv_tpr": lanes per row
   of the products with A; "block_width": the block
   width s2l_gpu_gmres_block uses; "refactor_bytes": device bytes of the refactorization plan
   (option "refactor"); "refactor_ms": host time of the last s2l_gpu_refactor. */
int s2l_gpu_setup_stat(const s2l_setup* s, const char* name, double* value);

/* ---- solve phase ----------------------------------------------------------------------
 * Every call below returns when its results are complete (host or device pointers alike).
 * Calls on one setup may come from several host threads at once.  Each call holds a workspace
 * (stream, work vectors, Krylov basis, error word) for its duration.  Workspace 0 runs on the
 * stream of s2l_gpu_set_stream and is taken when free.  A call that finds every workspace busy
 * creates one more, with its own stream ordered after the work already queued on the
 * s2l_gpu_set_stream stream, and the setup keeps it until s2l_gpu_setup_destroy.  The factors,
 * matrix and coarse data are shared and only read.  s2l_gpu_set_stream, s2l_gpu_profile_* and
 * s2l_gpu_setup_destroy must not overlap solve-phase calls. */
int s2l_gpu_spmv(s2l_setup* s, const double* x, double* y, int ptr_kind);
int s2l_gpu_local_solve(s2l_setup* s, int i, const double* b_local, double* x_local, int ptr_kind);
int s2l_gpu_coarse_apply(s2l_setup* s, const double* r, double* x0, int ptr_kind);
int s2l_gpu_one_level_apply(s2l_setup* s, const double* r, double* z, int ptr_kind);
int s2l_gpu_apply(s2l_setup* s, const double* r, double* z, int ptr_kind);

/*
 * The coarse correction x0 = R0^T E^-1 R0 r of s2l_gpu_coarse_apply, for callers that cannot
 * allocate device memory when they call it: code that hands all device memory to its own pool
 * or allocator (a framework's caching allocator, a memory-capped serving process), or that must
 * not allocate once its solve loop runs.  No counterpart in the reference (it has no device).
 *
 * It allocates nothing and uses none of the setup's scratch buffers: the restriction partials and
 * the two coarse vectors live in one static device array of S2L_NOALLOC_SCRATCH_DOUBLES doubles
 * (2 MiB), which every GPU that loads this library holds until the process exits.  A setup needs
 * (coarse tiles x largest m) + 2 n0 doubles of it, plus the local-space size for the multiplicity
 * partition of unity; a setup that needs more is rejected with S2L_ERR_BADARG before any launch.
 * r and x0 are device pointers (n doubles each).  The call makes the setup's device current (as
 * every solve-phase call does), enqueues the kernels on the setup's stream (s2l_gpu_set_stream) and
 * returns; x0 is ready once that stream is synchronized.  Synchronize that stream before calling
 * s2l_gpu_update_matrix, s2l_gpu_refactor, s2l_gpu_set_stream or s2l_gpu_setup_destroy on the same
 * setup: they change what the enqueued kernels read.
 *
 * The first call on a context looks up the device address of the static array (with the
 * context's device current) and the context keeps it: make that first call before any stream
 * capture on the device.  A context created after a reset of the device (cudaDeviceReset) looks it
 * up anew.  Every call shares the one array and leaves its contents behind; every scratch element
 * a call reads is written earlier in the same call, so nothing needs clearing, but calls that
 * overlap on the GPU (other streams, other setups on the same device) race on it.
 */
#define S2L_NOALLOC_SCRATCH_DOUBLES 262144
int s2l_gpu_coarse_apply_noalloc(s2l_setup* s, const double* r, double* x0);

int s2l_gpu_gmres(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* opts,
                  s2l_result* result);
int s2l_gpu_bicgstab(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* opts,
                     s2l_result* result);

/* ---- batched and asynchronous solves ------------------------------------------------------
 * No counterpart in the reference (it solves one right-hand side at a time per process); these
 * serve several right-hand sides of one matrix, or requests over several matrices, from one GPU.
 */
/* k solves of A x_j = b_j on one setup at once, each on its own workspace and stream (k - 1 extra
 * host threads); returns when all are done.  method: S2L_KRYLOV_GMRES or S2L_KRYLOV_BICGSTAB.
 * b[j], x[j]: host or device vectors as ptr_kind says; results[j], status[j] per solve; the
 * return value is the first failing status (or S2L_OK). */
int s2l_gpu_solve_batch(s2l_setup* s, int method, int k, const double* const* b, double* const* x, int ptr_kind,
                        const s2l_krylov_opts* opts, s2l_result* results, int* status);

/* k right-hand sides of one matrix in one block (1 <= k <= 16): every preconditioner application,
 * product with A and orthogonalization runs once for all k columns (the factors, the matrix and
 * the coarse basis are read once for all of them), while each column keeps its own GMRES
 * recurrence, restarts and convergence test (L2 test only).  b and x hold k vectors of n doubles
 * one after another (column r at b + r * n), on the host or the device as ptr_kind says;
 * results[r] per column.  s2l_gpu_apply_block is the preconditioner alone, z = M^-1 r per column. */
int s2l_gpu_apply_block(s2l_setup* s, int k, const double* r, double* z, int ptr_kind);
int s2l_gpu_gmres_block(s2l_setup* s, int k, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* opts,
                        s2l_result* results);

/* Asynchronous solves: s2l_gpu_serve_start starts `workers` native threads on the context; each
 * s2l_gpu_submit queues one solve (first in, first out) and returns a ticket at once.  b, x,
 * result (and result->history) stay owned by the caller and must stay valid until the ticket is
 * finished; opts is copied.  Solves on different setups of the context, and on one setup, run
 * concurrently up to the number of workers (each holds a workspace of its setup).
 * s2l_gpu_cancel drops a queued solve, or stops a running one before its next iteration (status
 * S2L_ERR_CANCELED; x is then unspecified).  s2l_gpu_setup_destroy refuses (S2L_ERR_STATE) while
 * solves are queued or running on the setup; s2l_gpu_destroy cancels queued solves, waits for
 * running ones and joins the workers.  A finished ticket is released with s2l_gpu_ticket_free. */
typedef struct s2l_ticket s2l_ticket;
enum { S2L_JOB_QUEUED = 0, S2L_JOB_RUNNING = 1, S2L_JOB_DONE = 2, S2L_JOB_CANCELED = 3 };
int s2l_gpu_serve_start(s2l_ctx* ctx, int workers);
/* Continuous batching of the asynchronous GMRES solves (on by default, slots < 0: automatic).
 * A worker that takes a GMRES request (L2 stopping test, restart <= 63, exact local factors) runs
 * a block runner for its setup, restart length and variant: up to `slots` requests at once (the
 * automatic width is the setup's block width, s2l_gpu_setup_stat "block_width", at most 4), each in a column
 * of one block, so the preconditioner, the product with A and the orthogonalization of every
 * Arnoldi step run once for all of them.  Each request keeps its own GMRES recurrence, restart
 * cycle and convergence test; a request that arrives while the runner works takes a free slot at
 * the next Arnoldi step and a request that converges returns at once, giving its slot to the next.
 * A request's result does not depend on which others share the block (it is bitwise the same as
 * alone in a runner of the same width).  More requests than slots start more runners on more
 * workers; when a runner's block buffers do not fit the HBM budget it uses half the slots.
 * slots = 0 turns batching off: every request then runs alone on its worker (first in, first
 * out), as BiCGStab requests, the OpenFOAM stopping test and AMG local solvers always do. */
int s2l_gpu_serve_batching(s2l_ctx* ctx, int slots);
int s2l_gpu_submit(s2l_setup* s, int method, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* opts,
                   s2l_result* result, s2l_ticket** ticket);
/* state: S2L_JOB_* */
int s2l_gpu_poll(s2l_ticket* t, int* state);
/* Waits until the ticket is finished (timeout_s < 0: no limit); returns S2L_ERR_TIMEOUT if it is
 * not finished in time, else S2L_OK with the solve's status in *status. */
int s2l_gpu_wait(s2l_ticket* t, double timeout_s, int* status);
int s2l_gpu_cancel(s2l_ticket* t);
/* Time in the queue and running [ms] (host clock, submit to start to finish) and the message of a
 * failed solve (valid until the ticket is freed). */
int s2l_gpu_ticket_info(s2l_ticket* t, double* queue_ms, double* run_ms, const char** error);
int s2l_gpu_ticket_free(s2l_ticket* t);

/* ---- streams and measurement -------------------------------------------------------------- */
/* Launch on this CUDA stream (cudaStream_t passed as a pointer; NULL = the setup's own stream). */
int s2l_gpu_set_stream(s2l_setup* s, void* stream);
/* Kernel classes timed with CUDA events on the launching stream (bit mask; 0 = off). */
enum { S2L_PROF_SPMV = 1, S2L_PROF_LOCAL_SOLVE = 2, S2L_PROF_COARSE = 4, S2L_PROF_COMBINE = 8,
       S2L_PROF_KRYLOV_VEC = 16, S2L_PROF_ALL = 31 };
/* Enables the classes of `mask` and resets the accumulators and the launch counter. */
int s2l_gpu_profile_enable(s2l_setup* s, int mask);
/* Accumulated event time [ms] and launch count of one kernel class, summed over the workspaces;
   names: "spmv", "local_solve", "coarse", "combine", "krylov_vec", "all"; "launches" gives every
   kernel launch of the setup since the last s2l_gpu_profile_enable (timed or not) in *launches. */
int s2l_gpu_profile_get(s2l_setup* s, const char* name, double* ms, long* launches);
/* Algorithmic bytes read+written by one local_solve launch (the roofline numerator). */
int s2l_gpu_local_solve_bytes(const s2l_setup* s, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* S2L_GPU_H */
