// C ABI of the B200 solve phase (include/s2l_gpu.h): setup upload, schedules, apply, Krylov.
//
// Host code.  Setup converts the caller's arrays once into the device layout of
// s2l_internal.cuh (factors in level order, index maps, tiles of the coarse basis, E^-1); the
// solve phase is a sequence of kernel launches on the setup's stream.  Krylov scalars
// (Givens rotations, the small least-squares solve, BiCGStab coefficients) run on the host in
// FP64 from device reductions read back once per orthogonalization step.
#include "s2l_internal.cuh"
#include "../../include/s2l_gpu.h"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <numeric>
#include <string>
#include <vector>

using namespace s2l;

struct s2l_ticket;
namespace {
struct Runner;
}

// Worker threads of the asynchronous solves (s2l_gpu_serve_start / s2l_gpu_submit)
struct s2l_serve {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<s2l_ticket*> queue;
    std::vector<std::thread> workers;
    bool stop = false;
    // continuous batching (s2l_gpu_serve_batching): slots per block runner (< 0 automatic, 0 off)
    // and the runners at work
    int slots = -1;
    std::vector<Runner*> runners;
};

struct s2l_ctx {
    int device = 0;
    size_t budget = 0;
    size_t used = 0;
    std::string err;
    std::mutex mu;
    s2l_serve* serve = nullptr;
    // device address of the static scratch of s2l_gpu_coarse_apply_noalloc, looked up by the first
    // such call on this context (with its device current); a context created after a reset of the
    // device looks it up anew
    double* noalloc_scratch = nullptr;
};

namespace {
thread_local std::string t_last_error;  // message of this thread's last failure (tickets read it)
void serve_stop(s2l_ctx* ctx);
}

namespace {

enum { PC_SPMV = 0, PC_SOLVE, PC_COARSE, PC_COMBINE, PC_VEC, PC_N };

struct s2l_tail_model {
    int force_rows = 0;      // > 0: every subdomain gets a tail of this many rows
    int tail_min = 64;       // smallest tail considered (0 rows is always allowed)
    int tail_max = 4096;
    double hop_s = 0.25e-6;  // time of one dependency level of a sweep
    double bw = 6.0e12;      // bytes/s shared by all subdomains
    double nsub = 1.0;
    double real_bytes = 8.0;
    double smem_cap = (double)S2L_SWEEP_SMEM_CAP;
    int chain = S2L_CHAIN_DEFAULT;  // chain block rows (1 = no blocking)
};
const char* kProfNames[PC_N] = {"spmv", "local_solve", "coarse", "combine", "krylov_vec"};

struct HostCsr {
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v;  // values widened to double on the host
};

struct HostSub {
    bool set = false;
    int64_t begin = 0;
    int n_owned = 0, n_ghost = 0;
    std::vector<int64_t> ghosts;
    std::vector<double> D;
    int kind = S2L_FACTOR_LU;
    std::vector<int32_t> pin, pout;
    HostCsr L, U;
    std::vector<double> d;
    int m = 0;
    std::vector<double> V;  // column-major n_local x m
    // AMG local solver instead of factors (s2l_gpu_add_subdomain_amg): smoothed levels and the
    // coarsest operator (row-major, amg_nc x amg_nc; none when amg_nc is 0)
    bool amg = false;
    int amg_sweeps = 1;
    std::vector<HostCsr> amgA, amgP, amgR;
    int amg_nc = 0;
    std::vector<double> amgC;
    int n_local() const { return n_owned + n_ghost; }
};

// sparse part of one triangular factor of one subdomain, renumbered in solve order
struct Sweep {
    std::vector<int32_t> order;   // slot -> row
    std::vector<int32_t> pos;     // row -> slot
    std::vector<uint16_t> len;    // entries per slot
    std::vector<double> dinv;     // per slot
    std::vector<int32_t> col;     // column slots (T, the sentinel slot: padding), per warp, per task lane-interleaved
    std::vector<double> val;      // values times 1/diag of their row
    std::vector<uint32_t> thdr;   // per task: chunks C (bits 0-15), log2 G (16-18), rows R - 1 (19-23)
    std::vector<int32_t> tslot;   // per task: its R slots
    std::vector<int64_t> wtask, wslot, went;  // per warp (nw + 1): first task, slot and entry
    int64_t pad = 0, ntask = 0;
    int nlev = 0;
    // chain blocks (>= 2 rows): block b holds the slots blk_slot[blk_off[b] .. blk_off[b + 1]) in
    // solve order and the packed lower triangle of W^-1 at blk_inv[blk_ioff[b] ...]
    std::vector<int64_t> blk_off{0}, blk_ioff{0};
    std::vector<int32_t> blk_slot;
    std::vector<double> blk_inv;
    // refactorization maps (built when build_sweep is given the factor position of every entry of
    // its matrix): per entry of `col` the position of its value (-1 padding, -2 a row of a chain
    // block), per slot the position of the row's diagonal (-1: 1 / diagonal = 1), per block the
    // positions of W packed like blk_inv (-1: 0 off the diagonal, 1 on it), and the entries of the
    // blocks' rewritten rows: entry index in `col`, row within the block, and its contributions
    // (block row b, position of M(B[b], c)) of  sum_b W^-1(row, b) M(B[b], c)
    std::vector<int32_t> src, dsrc, blk_wsrc;
    std::vector<int64_t> be_off{0}, be_pos, be_cp{0};
    std::vector<uint8_t> be_row, bc_b;
    std::vector<int32_t> bc_pos;
};

}  // namespace

struct s2l_work;

struct s2l_setup {
    s2l_ctx* ctx = nullptr;
    int64_t n = 0;
    int nsub = 0;
    int one_level = 0, coarse = 0, pou = 0;
    int real = -1;
    int local_kind = -1;  // 0: exact factors (s2l_gpu_add_subdomain), 1: AMG (s2l_gpu_add_subdomain_amg)
    bool ended = false;
    cudaStream_t setup_stream = nullptr;  // uploads and the tail inversion

    // host staging
    HostCsr A;
    bool have_A = false;
    std::vector<HostSub> hs;
    int64_t n0 = 0;
    std::vector<int64_t> coff;
    std::vector<double> E;
    bool have_coarse = false;

    // device memory (read-only after setup_end)
    std::vector<void*> allocs;
    size_t bytes = 0;
    int32_t *d_rp = nullptr, *d_ci = nullptr;
    double* d_av = nullptr;
    double* d_rowsum = nullptr;  // A 1 (OpenFOAM normalisation factor)
    int64_t nnz = 0;
    int tpr = 8;
    std::vector<DevSub> h_subs;
    DevSub* d_subs = nullptr;
    int64_t nloc = 0;
    int max_nl = 0;
    int64_t *d_wtask[2] = {nullptr, nullptr}, *d_wslot[2] = {nullptr, nullptr}, *d_went[2] = {nullptr, nullptr};
    uint32_t* d_thdr[2] = {nullptr, nullptr};
    int32_t* d_tslot[2] = {nullptr, nullptr};
    int32_t* d_bfirst[2] = {nullptr, nullptr};
    int64_t *d_boff[2] = {nullptr, nullptr}, *d_bioff[2] = {nullptr, nullptr};
    int32_t* d_bslot[2] = {nullptr, nullptr};
    void* d_binv[2] = {nullptr, nullptr};
    int32_t* d_col[2] = {nullptr, nullptr};
    int32_t* d_u2l = nullptr;
    void* d_val[2] = {nullptr, nullptr};
    void* d_dinv[2] = {nullptr, nullptr};
    int32_t *d_tr_sub = nullptr, *d_tr_i = nullptr, *d_lts_col = nullptr;
    int64_t* d_lts_ptr = nullptr;
    void* d_lts_val = nullptr;
    int32_t *d_us_sub = nullptr, *d_us_r = nullptr, *d_ust_col = nullptr, *d_uu = nullptr;
    int64_t* d_ust_ptr = nullptr;
    void* d_ust_val = nullptr;
    void *d_linv = nullptr, *d_uinv = nullptr;
    bool need_gflags = false;
    std::vector<int> tr_first_h, us_first_h, uu_first_h;  // per subdomain, nsub+1 entries
    int sweep_group = 32;
    // options (s2l_gpu_setup_option)
    int opt_tail_min = 64, opt_tail_max = 4096, opt_group = 0, opt_tail_rows = 0, opt_chain = S2L_CHAIN_DEFAULT, opt_block_width = 0,
        opt_tpr = 0, opt_epl = 4;
    double opt_hop_us = 0.25, opt_bw_gbs = 6000.0;
    std::atomic<int> opt_spin_limit{S2L_SPIN_LIMIT};  // polls of a sweep wait before it gives up
    std::atomic<int> opt_spin_sleep{S2L_SPIN_SLEEP_NS};  // back-off of a sweep poll that found a column not ready
    std::atomic<int> opt_sweep_pf{S2L_BATCH_CHUNKS};     // chunks a sweep warp hints into L2 ahead of its task
    double opt_pivot_tol = 1e-6;  // refactorization of LU factors: largest multiplier 1 / pivot_tol
    int opt_amg_single = 0;       // AMG local solvers in single precision (--local-precision single)
    // statistics
    int64_t st_sparse_nnz = 0, st_coupling_nnz = 0, st_dense_entries = 0, st_tail_rows = 0;
    int64_t st_levels_max = 0, st_levels_sum = 0;  // sweep dependency levels (both factors)
    int64_t st_blocks = 0;                         // chain blocks (both factors)
    int64_t st_tasks = 0, st_pad = 0;              // sweep tasks and padding entries (both factors)
    int32_t *d_gin = nullptr, *d_pin = nullptr, *d_gout = nullptr, *d_l2g = nullptr;
    double* d_D = nullptr;
    int64_t* d_cp_ptr = nullptr;
    int32_t* d_cp_pos = nullptr;
    double* d_cp_w = nullptr;
    bool need_copies = false;
    // coarse
    double* d_V = nullptr;
    int32_t *d_t_sub = nullptr, *d_t_row0 = nullptr, *d_t_nrow = nullptr, *d_t_first = nullptr;
    int ntiles = 0, mmax = 0;
    double* d_Einv = nullptr;
    size_t smem_bytes = 0;
    double solve_bytes = 0.0;
    double solve_vec_bytes = 0.0;  // the part of solve_bytes that every further right-hand side adds
    int max_T = 0;   // largest sparse part of a subdomain (rows)
    int kc_max = 1;  // right-hand sides a sweep CTA can hold in shared memory (1, 2 or 4)
    // workspaces: one per concurrent solve-phase call (workspace 0 is the caller's default)
    mutable std::mutex wmu;
    std::condition_variable wcv;  // a workspace came free
    std::vector<s2l_work*> works;
    std::vector<char> busy;
    cudaStream_t user_stream = nullptr;  // s2l_gpu_set_stream: used by workspace 0
    unsigned prof_mask = 0;              // s2l_gpu_profile_enable: inherited by new workspaces

    std::atomic<int> pending{0};  // asynchronous solves queued or running on this setup
    std::atomic<int> runners{0};  // block runners of the serving workers holding a workspace of it

    // AMG local solvers (s2l_gpu_add_subdomain_amg): level spaces and block-diagonal operators
    struct AmgDev {
        bool on = false;
        int nlev = 0;                       // level spaces (smoothed levels and coarsest ones)
        int sweeps = 1;
        std::vector<int64_t> nspace;        // per level space: rows
        std::vector<int64_t> voff;          // per level space: offset of its vectors in a workspace block
        int64_t vtotal = 0;                 // doubles of one of the three work vectors (f, x, t)
        std::vector<int64_t*> Arp, Rrp, Prp;
        std::vector<int32_t*> Aci, Rci, Pci;
        std::vector<double*> Av, Rv, Pv;    // values (float arrays when `single`, cast at use)
        bool single = false;                // setup option "amg_single": hierarchy and V-cycle in float
        std::vector<int> nsmooth;           // per level: subdomains smoothed on it (CTAs of a sweep)
        std::vector<int32_t*> fsched, bsched, fsub, bsub;
        std::vector<int64_t*> fwf, bwf;
        std::vector<int64_t*> soff;         // per level: level-space offset of each smoothed subdomain
        std::vector<int32_t*> sn;           //   and its rows
        std::vector<int> smax;              //   the most rows
        std::vector<int> lanes;             // per level: lanes per row of a sweep (from the mean row length)
        std::vector<int> ncoarse;           // per level: subdomains whose coarsest level it is
        std::vector<int32_t*> c_off, c_n;
        std::vector<int64_t*> c_inv;
        double* Cinv = nullptr;
        int32_t* out_idx = nullptr;         // local-space row -> owned global row, or -1
        double cycle_bytes = 0.0;           // algorithmic bytes of one V-cycle of every subdomain
    } amgd;

    // numeric refactorization (setup option "refactor"): factor patterns and the maps from them to
    // the solve layout, kept on the device (RefactorArgs)
    int opt_refactor = 0;
    struct Refac {
        bool on = false;
        int64_t nF = 0, nfill = 0, ntc = 0, nlts = 0, nust = 0, nblk[2] = {0, 0};
        double* F = nullptr;
        double* S = nullptr;      // dense tails (FP64)
        double* stage = nullptr;  // the new matrix values until they are committed
        double* part = nullptr;   // partial columns of the cooperative column updates
        int maxcol = 1;
        int cs = 1;               // CTAs (a cluster) per subdomain in the sparse-column walk
        int* err = nullptr;
        int64_t *fbase = nullptr, *fcp = nullptr, *frp = nullptr, *lv_off = nullptr;
        int32_t *fri = nullptr, *fdg = nullptr, *frpos = nullptr, *frk = nullptr, *lv_first = nullptr,
                *lv_col = nullptr, *tc_sub = nullptr, *tc_col = nullptr;
        uint8_t* fllt = nullptr;
        int64_t *fill_src = nullptr, *fill_dst = nullptr, *lts_src = nullptr, *ust_src = nullptr;
        int32_t *sw_src[2] = {nullptr, nullptr}, *sw_dsrc[2] = {nullptr, nullptr};
        int64_t *wsrc[2] = {nullptr, nullptr}, *be_off[2] = {nullptr, nullptr}, *be_pos[2] = {nullptr, nullptr},
                *be_cp[2] = {nullptr, nullptr}, *bc_pos[2] = {nullptr, nullptr};
        uint8_t *be_row[2] = {nullptr, nullptr}, *bc_b[2] = {nullptr, nullptr};
        std::vector<int> sz;     // tail size per subdomain
        std::vector<char> llt;   // per subdomain
        std::vector<int64_t> d_off;
        size_t bytes = 0;        // device bytes of the plan
        // dense tails factorized and inverted on RF_STREAMS streams at once, each with its cuSOLVER
        // handle and its factorization and inversion workspaces
        static constexpr int RF_STREAMS = 8;
        cudaStream_t tstream[RF_STREAMS] = {};
        cudaEvent_t tev[RF_STREAMS + 1] = {};
        cusolverDnHandle_t tsolver[RF_STREAMS] = {};
        double* swork[RF_STREAMS] = {};
        int lwork = 0;
        void* iwork[RF_STREAMS] = {};         // triangular inversion workspace (device) per stream
        double* B[RF_STREAMS] = {};           // copy of an LU tail whose unit lower triangle is inverted
        size_t iwork_bytes = 0;
        std::vector<char> ihost[RF_STREAMS];  // and its host part
        int* info = nullptr;  // per subdomain: the dense tail factorization's status
        // coarse matrix refresh: E and its inversion, 16 unit vectors through prolong / A / restrict
        double *E = nullptr, *Einv = nullptr, *Y = nullptr, *X = nullptr, *AX = nullptr, *cpart = nullptr,
               *C = nullptr, *plocal = nullptr, *rowsum = nullptr, *ework = nullptr;
        // direct coarse assembly (boolean partition of unity): row slots and subdomain pairs
        bool direct = false;
        int npairs = 0;
        int32_t *owner = nullptr, *rs_sub = nullptr, *pair_j = nullptr, *pair_i = nullptr, *pair_rl = nullptr;
        int64_t *rs_ptr = nullptr, *rs_zoff = nullptr, *pair_ptr = nullptr, *pair_zoff = nullptr;
        double* Z = nullptr;
        int* piv = nullptr;
        int elwork = 0;
        double last_ms = 0.0;
        double phase_ms[6] = {0, 0, 0, 0, 0, 0};  // coarse matrix, its inverse, sparse columns, tail columns,
                                                  // dense tails, commit
    } rf;

    int fail(int code, const std::string& msg)
    {
        t_last_error = msg;
        if (ctx) {
            std::lock_guard<std::mutex> g(ctx->mu);
            ctx->err = msg;
        }
        return code;
    }
};

// Work state of one solve-phase call: its stream, work vectors, Krylov basis, reduction buffers,
// error word and kernel timers.  The setup's data is only read.
struct s2l_work {
    s2l_setup* s = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;  // orders this workspace's stream after the caller's stream
    std::vector<void*> allocs;
    std::vector<size_t> alloc_bytes;  // size of each of allocs
    size_t bytes = 0;
    void *d_ybuf = nullptr, *d_xbuf = nullptr;
    uint8_t* d_gflags = nullptr;
    int* d_err = nullptr;
    double* d_cpart = nullptr;
    double *d_c = nullptr, *d_y = nullptr;
    double *d_ylocal = nullptr, *d_x0 = nullptr, *d_w = nullptr, *d_in = nullptr, *d_out = nullptr;
    double* d_plocal = nullptr;
    double* d_part = nullptr;
    double* d_red = nullptr;
    double* h_red = nullptr;
    // Krylov work (lazy)
    int kr_m = -1;
    bool kr_flex = false;
    double *d_V_kr = nullptr, *d_Z_kr = nullptr, *d_r = nullptr, *d_z = nullptr, *d_kw = nullptr, *d_b = nullptr,
           *d_xk = nullptr, *d_u = nullptr;
    double *d_rh = nullptr, *d_p = nullptr, *d_v = nullptr, *d_s = nullptr, *d_t = nullptr, *d_yb = nullptr;
    double* d_coef = nullptr;
    double* d_amg = nullptr;  // AMG local solves: f, x, t of every level space
    // block solves (K interleaved right-hand sides), allocated on first use
    struct Block {
        int K = 0, m = -1;
        bool flex = false;
        void *ybuf = nullptr, *xbuf = nullptr;
        uint8_t* gflags = nullptr;
        double *ylocal = nullptr, *plocal = nullptr, *x0 = nullptr, *wv = nullptr, *cpart = nullptr, *c = nullptr,
               *y = nullptr;
        double *V = nullptr, *Z = nullptr, *r = nullptr, *z = nullptr, *kw = nullptr, *b = nullptr, *xk = nullptr,
               *u = nullptr, *coef = nullptr, *scal = nullptr, *part = nullptr, *red = nullptr, *h_red = nullptr;
        std::vector<void*> allocs;
    } blk;
    // profiling
    unsigned prof = 0;  // bit c: time kernel class c
    long launches = 0;  // kernel launches issued through this workspace
    struct Ev {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Ev> evs;
    std::vector<cudaEvent_t> pool;
    double acc_ms[PC_N] = {0, 0, 0, 0, 0};
    long acc_n[PC_N] = {0, 0, 0, 0, 0};

    int fail(int code, const std::string& msg) { return s->fail(code, msg); }
};

#define CUDA_OK(s, call)                                                                                             \
    do {                                                                                                             \
        cudaError_t _e = (call);                                                                                     \
        if (_e != cudaSuccess) return (s)->fail(S2L_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));  \
    } while (0)

#define RET_IF(x)         \
    do {                  \
        int _r = (x);     \
        if (_r) return _r; \
    } while (0)

namespace {

int check_err(s2l_work* w);

int dev_alloc(s2l_setup* s, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    {
        std::lock_guard<std::mutex> g(s->ctx->mu);
        if (s->ctx->budget && s->ctx->used + bytes > s->ctx->budget) {
            s->ctx->err = "HBM budget exceeded: need " + std::to_string(s->ctx->used + bytes) + " of " +
                          std::to_string(s->ctx->budget) + " bytes";
            return S2L_ERR_OOM;
        }
        s->ctx->used += bytes;
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(s->ctx->mu);
        s->ctx->used -= bytes;
        s->ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return S2L_ERR_OOM;
    }
    s->allocs.push_back(*p);
    s->bytes += bytes;
    return S2L_OK;
}

template <typename T>
int upload(s2l_setup* s, T** dst, const T* src, size_t count)
{
    RET_IF(dev_alloc(s, reinterpret_cast<void**>(dst), count * sizeof(T)));
    if (count) CUDA_OK(s, cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s->setup_stream));
    return S2L_OK;
}

template <typename T>
int upload(s2l_setup* s, T** dst, const std::vector<T>& v)
{
    return upload(s, dst, v.data(), v.size());
}

// Chain blocks of the sparse part, in solve order (lower: rows 0, 1, ..; upper: T-1, T-2, ..): a
// block grows while its next row depends on the row solved just before it, up to `chain` rows.
// Returns, per block, the rows in solve order.
std::vector<std::vector<int32_t>> chain_blocks(const HostCsr& M, int T, bool lower, int chain)
{
    std::vector<std::vector<int32_t>> blocks;
    auto seq = [&](int t) { return lower ? t : T - 1 - t; };
    auto has = [&](int r, int c) {  // entry (r, c) present (sorted columns)
        const int32_t* b = M.ci.data() + M.rp[r];
        const int32_t* e = M.ci.data() + M.rp[r + 1];
        const int32_t* it = std::lower_bound(b, e, c);
        return it != e && *it == c;
    };
    for (int t = 0; t < T;) {
        std::vector<int32_t> blk{(int32_t)seq(t)};
        while (t + (int)blk.size() < T && (int)blk.size() < chain && has(seq(t + (int)blk.size()), blk.back()))
            blk.push_back((int32_t)seq(t + (int)blk.size()));
        t += (int)blk.size();
        blocks.push_back(std::move(blk));
    }
    return blocks;
}

// Sweep layout of the sparse part (rows [0, T)): slots in level order, columns as slots, the rows
// of each level packed into tasks of the nw warps of a sweep CTA (below).
//
// Chain blocks: for a block B of k rows solved one after another (row a depends on row a - 1),
// W = M(B, B) (k x k, lower in solve order).  The block's rows are replaced by W^-1 M(B, outside),
// which depend only on rows solved before the block, and the right-hand side of the block by
// W^-1 b(B) (the sweep's prologue): the k-step chain becomes one level.  The replaced rows hold
// the union of the block rows' patterns; a block stops before a row that would reach 65535 entries.
// f(i) for i in [0, n) on up to hardware_concurrency host threads (each i independent)
void parallel_for(int n, const std::function<void(int)>& f)
{
    const int nt = std::max(1, std::min(n, (int)std::thread::hardware_concurrency()));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&] {
            for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
        });
    for (auto& x : th) x.join();
}

void build_sweep(const HostCsr& M, int T, bool lower, bool unit_diag, int nw, int gmax, int epl, int chain, Sweep& out,
                 std::string& err, const std::vector<int32_t>* mpos = nullptr)
{
    const bool track = mpos != nullptr;
    // rows of the sparse part, original numbering: (column, value) outside the diagonal, and diagonal
    std::vector<std::vector<std::pair<int32_t, double>>> rows(T);
    std::vector<double> diag(T, 1.0);
    std::vector<std::vector<int32_t>> rpos(track ? T : 0);  // factor position of each entry of rows[r]
    std::vector<int32_t> dpos(track ? T : 0, -1);
    for (int r = 0; r < T; ++r) {
        double dg = 1.0;
        for (int64_t e = M.rp[r]; e < M.rp[r + 1]; ++e) {
            const int c = M.ci[e];
            if (c == r) {
                dg = M.v[e];
                if (track) dpos[r] = (*mpos)[e];
                continue;
            }
            if (lower ? (c > r) : (c < r || c >= T)) continue;
            rows[r].emplace_back(c, M.v[e]);
            if (track) rpos[r].push_back((*mpos)[e]);
        }
        if (unit_diag) {
            dg = 1.0;
            if (track) dpos[r] = -1;
        }
        if (dg == 0.0 || !std::isfinite(dg)) {
            err = "zero or non-finite diagonal in a triangular factor";
            return;
        }
        diag[r] = dg;
    }
    // chain blocks: rewrite their rows
    std::vector<std::vector<int32_t>> blocks = chain_blocks(M, T, lower, std::max(chain, 1));
    std::vector<char> inblk(T, 0);
    std::vector<double> acc(T, 0.0);
    std::vector<int32_t> mark(T, -1), touched;
    std::vector<std::vector<double>> winv_of;  // per block, packed lower W^-1
    std::vector<int> blk_ids;                  // blocks of >= 2 rows, in solve order
    // tracking: per rewritten row its block (order in blk_ids) and row, and per entry its
    // contributions; per kept block the positions of W
    std::vector<std::pair<int32_t, int32_t>> rblk(track ? T : 0, {-1, -1});
    std::vector<std::vector<std::vector<std::pair<uint8_t, int32_t>>>> rcons(track ? T : 0);
    std::vector<std::vector<int32_t>> wsrc_of;
    std::vector<int32_t> tix(track ? T : 0, -1);
    for (int bi = 0; bi < (int)blocks.size(); ++bi) {
        std::vector<int32_t>& B = blocks[bi];
        int k = (int)B.size();
        if (k < 2) continue;
        for (int32_t r : B) inblk[r] = 1;
        // W (k x k, lower in solve order) and its inverse by forward substitution, column by column
        std::vector<double> W((size_t)k * k, 0.0);
        std::vector<int32_t> Wp(track ? (size_t)k * k : 0, -1);
        for (int a2 = 0; a2 < k; ++a2) {
            W[(size_t)a2 * k + a2] = diag[B[a2]];
            if (track) Wp[(size_t)a2 * k + a2] = dpos[B[a2]];
            for (size_t q = 0; q < rows[B[a2]].size(); ++q) {
                const auto& cv = rows[B[a2]][q];
                for (int b2 = 0; b2 < a2; ++b2)
                    if (cv.first == B[b2]) {
                        W[(size_t)a2 * k + b2] = cv.second;
                        if (track) Wp[(size_t)a2 * k + b2] = rpos[B[a2]][q];
                    }
            }
        }
        std::vector<double> Wi((size_t)k * k, 0.0);
        for (int j = 0; j < k; ++j)
            for (int i = j; i < k; ++i) {
                double v = i == j ? 1.0 : 0.0;
                for (int q = j; q < i; ++q) v -= W[(size_t)i * k + q] * Wi[(size_t)q * k + j];
                Wi[(size_t)i * k + j] = v / W[(size_t)i * k + i];
            }
        // new row a = sum_{b <= a} W^-1(a, b) M(B[b], outside the block)
        std::vector<std::vector<std::pair<int32_t, double>>> nrows(k);
        std::vector<std::vector<std::vector<std::pair<uint8_t, int32_t>>>> ncons(track ? k : 0);
        std::vector<std::vector<std::pair<uint8_t, int32_t>>> tcons;
        int kept = k;
        for (int a2 = 0; a2 < k; ++a2) {
            touched.clear();
            tcons.clear();
            for (int b2 = 0; b2 <= a2; ++b2) {
                const double w = Wi[(size_t)a2 * k + b2];
                for (size_t q = 0; q < rows[B[b2]].size(); ++q) {
                    const auto& cv = rows[B[b2]][q];
                    if (inblk[cv.first]) continue;
                    if (mark[cv.first] != a2 + 1 + bi * 64) {
                        mark[cv.first] = a2 + 1 + bi * 64;
                        acc[cv.first] = 0.0;
                        if (track) {
                            tix[cv.first] = (int32_t)touched.size();
                            tcons.emplace_back();
                        }
                        touched.push_back(cv.first);
                    }
                    acc[cv.first] += w * cv.second;
                    if (track) tcons[tix[cv.first]].emplace_back((uint8_t)b2, rpos[B[b2]][q]);
                }
            }
            if (touched.size() >= 65535) {
                kept = a2;
                break;
            }
            std::sort(touched.begin(), touched.end());
            for (int32_t c : touched) nrows[a2].emplace_back(c, acc[c]);
            if (track)
                for (int32_t c : touched) ncons[a2].push_back(std::move(tcons[tix[c]]));
        }
        if (kept < 2) {  // too long to block: leave the rows as they are
            for (int32_t r : B) inblk[r] = 0;
            continue;
        }
        if (kept < k) {
            // shorten the block: W^-1 of the leading rows is the leading part of W^-1, and the rows
            // already rewritten never reference the dropped rows (those are solved after them)
            for (int a2 = kept; a2 < k; ++a2) inblk[B[a2]] = 0;
            B.resize(kept);
            std::vector<double> Wk((size_t)kept * kept);
            for (int i = 0; i < kept; ++i)
                for (int j = 0; j < kept; ++j) Wk[(size_t)i * kept + j] = Wi[(size_t)i * k + j];
            Wi.swap(Wk);
            if (track) {
                std::vector<int32_t> Wpk((size_t)kept * kept);
                for (int i = 0; i < kept; ++i)
                    for (int j = 0; j < kept; ++j) Wpk[(size_t)i * kept + j] = Wp[(size_t)i * k + j];
                Wp.swap(Wpk);
            }
            k = kept;
        }
        for (int a2 = 0; a2 < k; ++a2) {
            rows[B[a2]].swap(nrows[a2]);
            diag[B[a2]] = 1.0;
            inblk[B[a2]] = 0;  // the marker covers the block being rewritten only
            if (track) {
                rblk[B[a2]] = {(int32_t)blk_ids.size(), a2};
                rcons[B[a2]] = std::move(ncons[a2]);
            }
        }
        std::vector<double> packed;
        std::vector<int32_t> wpacked;
        for (int i = 0; i < k; ++i)
            for (int j = 0; j <= i; ++j) {
                packed.push_back(Wi[(size_t)i * k + j]);
                if (track) wpacked.push_back(Wp[(size_t)i * k + j]);
            }
        winv_of.push_back(std::move(packed));
        if (track) wsrc_of.push_back(std::move(wpacked));
        blk_ids.push_back(bi);
    }
    // dependency levels of the rewritten rows, in solve order
    std::vector<int32_t> level(T, 0);
    out.nlev = 0;
    for (int t = 0; t < T; ++t) {
        const int r = lower ? t : T - 1 - t;
        int lv = 0;
        for (const auto& cv : rows[r]) lv = std::max(lv, level[cv.first] + 1);
        level[r] = lv;
        out.nlev = std::max(out.nlev, lv + 1);
    }
    std::vector<int32_t> cnt(out.nlev + 1, 0);
    for (int r = 0; r < T; ++r) ++cnt[level[r] + 1];
    for (int l = 0; l < out.nlev; ++l) cnt[l + 1] += cnt[l];
    out.order.assign(T, 0);
    out.pos.assign(T, 0);
    {
        std::vector<int32_t> next(cnt.begin(), cnt.end() - 1);
        if (lower)
            for (int r = 0; r < T; ++r) out.order[next[level[r]]++] = r;
        else
            for (int r = T - 1; r >= 0; --r) out.order[next[level[r]]++] = r;
    }
    for (int p = 0; p < T; ++p) out.pos[out.order[p]] = p;
    out.len.assign(T, 0);
    out.dinv.assign(T, 1.0);
    for (int p = 0; p < T; ++p) {
        const int r = out.order[p];
        if (rows[r].size() >= 65535) {
            err = "a sparse row has 65535 or more entries";
            return;
        }
        out.len[p] = (uint16_t)rows[r].size();
        out.dinv[p] = 1.0 / diag[r];
    }
    // Tasks: the rows of one level, R = 32 / G of them with G lanes each (G from the row length,
    // about epl entries per lane, at most gmax), sorted by width and length so a task's rows
    // are alike.  Each task goes to the warp with the least work so far; a warp's tasks stay in
    // level order.  Entries are stored lane-interleaved: chunk c of a task holds, for lane
    // k * G + j, entry c * G + j of its row k (column T, the sentinel slot, and value 0 past the
    // row's end), with
    // 1/diag folded into the values (the sweep scales the right-hand side by 1/diag too).
    auto width = [&](int len) {
        int g = 1;
        while (g < gmax && g * epl < len) g <<= 1;
        return g;
    };
    struct WarpOut {
        std::vector<uint32_t> hdr;
        std::vector<int32_t> slot, col, src;
        std::vector<double> val;
        double cost = 0.0;
    };
    // tracking: entries of rewritten rows as (block, row in block, entry index within its warp,
    // warp, row, entry of the row)
    struct BlkEnt {
        int32_t blk, arow, w, r, e;
        int64_t idx;
    };
    std::vector<BlkEnt> bents;
    std::vector<WarpOut> wo(nw);
    out.pad = 0;
    out.ntask = 0;
    std::vector<std::pair<int, int>> items;  // (width, slot)
    for (int l = 0; l < out.nlev; ++l) {
        items.clear();
        for (int p = cnt[l]; p < cnt[l + 1]; ++p) items.emplace_back(width(out.len[p]), p);
        std::sort(items.begin(), items.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
            if (a.first != b.first) return a.first < b.first;
            if (out.len[a.second] != out.len[b.second]) return out.len[a.second] < out.len[b.second];
            return a.second < b.second;
        });
        for (size_t i0 = 0; i0 < items.size();) {
            const int G = items[i0].first;
            size_t i1 = i0;
            while (i1 < items.size() && items[i1].first == G && (int)(i1 - i0) < 32 / G) ++i1;
            const int R = (int)(i1 - i0);
            int C = 0;
            for (size_t i = i0; i < i1; ++i) C = std::max(C, (out.len[items[i].second] + G - 1) / G);
            int wbest = 0;
            for (int w = 1; w < nw; ++w)
                if (wo[w].cost < wo[wbest].cost) wbest = w;
            WarpOut& W = wo[wbest];
            W.cost += C + 3.0;
            int gl2 = 0;
            while ((1 << gl2) < G) ++gl2;
            W.hdr.push_back((uint32_t)C | ((uint32_t)gl2 << 16) | ((uint32_t)(R - 1) << 19));
            for (size_t i = i0; i < i1; ++i) W.slot.push_back(items[i].second);
            for (int c = 0; c < C; ++c)
                for (int lane = 0; lane < 32; ++lane) {
                    const int k = lane / G, j = lane % G, e = c * G + j;
                    int32_t colv = T, sv = -1;
                    double v = 0.0;
                    if (k < R) {
                        const int p = items[i0 + k].second;
                        const int r = out.order[p];
                        const auto& row = rows[r];
                        if (e < (int)row.size()) {
                            colv = out.pos[row[e].first];
                            v = row[e].second * out.dinv[p];
                            if (track) {
                                if (rblk[r].first >= 0) {
                                    sv = -2;
                                    bents.push_back({rblk[r].first, rblk[r].second, wbest, r, e, (int64_t)W.col.size()});
                                } else {
                                    sv = rpos[r][e];
                                }
                            }
                        }
                    }
                    if (colv == T) ++out.pad;
                    W.col.push_back(colv);
                    W.val.push_back(v);
                    if (track) W.src.push_back(sv);
                }
            ++out.ntask;
            i0 = i1;
        }
    }
    out.wtask.assign(nw + 1, 0);
    out.wslot.assign(nw + 1, 0);
    out.went.assign(nw + 1, 0);
    out.thdr.clear();
    out.tslot.clear();
    out.col.clear();
    out.val.clear();
    for (int w = 0; w < nw; ++w) {
        out.wtask[w] = (int64_t)out.thdr.size();
        out.wslot[w] = (int64_t)out.tslot.size();
        out.went[w] = (int64_t)out.col.size();
        out.thdr.insert(out.thdr.end(), wo[w].hdr.begin(), wo[w].hdr.end());
        out.tslot.insert(out.tslot.end(), wo[w].slot.begin(), wo[w].slot.end());
        out.col.insert(out.col.end(), wo[w].col.begin(), wo[w].col.end());
        out.val.insert(out.val.end(), wo[w].val.begin(), wo[w].val.end());
        if (track) out.src.insert(out.src.end(), wo[w].src.begin(), wo[w].src.end());
    }
    out.wtask[nw] = (int64_t)out.thdr.size();
    out.wslot[nw] = (int64_t)out.tslot.size();
    out.went[nw] = (int64_t)out.col.size();
    out.blk_off.assign(1, 0);
    out.blk_ioff.assign(1, 0);
    out.blk_slot.clear();
    out.blk_inv.clear();
    for (size_t q = 0; q < blk_ids.size(); ++q) {
        for (int32_t r : blocks[blk_ids[q]]) out.blk_slot.push_back(out.pos[r]);
        out.blk_off.push_back((int64_t)out.blk_slot.size());
        out.blk_inv.insert(out.blk_inv.end(), winv_of[q].begin(), winv_of[q].end());
        out.blk_ioff.push_back((int64_t)out.blk_inv.size());
    }
    if (!track) return;
    out.dsrc.assign(T, -1);
    for (int p = 0; p < T; ++p) {
        const int r = out.order[p];
        out.dsrc[p] = rblk[r].first >= 0 ? -1 : dpos[r];
    }
    for (const auto& w : wsrc_of) out.blk_wsrc.insert(out.blk_wsrc.end(), w.begin(), w.end());
    std::sort(bents.begin(), bents.end(), [&](const BlkEnt& a, const BlkEnt& b) {
        if (a.blk != b.blk) return a.blk < b.blk;
        return out.went[a.w] + a.idx < out.went[b.w] + b.idx;
    });
    size_t q = 0;
    for (size_t b = 0; b < blk_ids.size(); ++b) {
        for (; q < bents.size() && bents[q].blk == (int32_t)b; ++q) {
            const BlkEnt& be = bents[q];
            out.be_pos.push_back(out.went[be.w] + be.idx);
            out.be_row.push_back((uint8_t)be.arow);
            for (const auto& cb : rcons[be.r][be.e]) {
                out.bc_b.push_back(cb.first);
                out.bc_pos.push_back(cb.second);
            }
            out.be_cp.push_back((int64_t)out.bc_b.size());
        }
        out.be_off.push_back((int64_t)out.be_pos.size());
    }
}

// Tail split of one subdomain: T minimising  2 hop levels(T) + bytes(T) nsub / bw, where levels is
// the dependency depth of the sparse rows < T (forward levels of L, a row's level depends on
// smaller rows only) and bytes what one local solve reads for this split: sparse entries of L and
// U, coupling entries L(T:n, 0:T) and U(0:T, T:n), and the two dense triangles of the tail.  The
// tail is at most tail_max rows; the sweep's shared memory must hold T rows.
// Lanes of the U-coupling kernel for a row of `len` entries: about four entries per lane, a power
// of two, 1 to 32 (a warp takes 32 / lanes rows of about that length)
int coupling_lanes(int len)
{
    int g = 1;
    while (g < 32 && 4 * g < len) g <<= 1;
    return g;
}

int choose_tail(const HostCsr& L, const HostCsr& U, int n, const s2l_tail_model& tm)
{
    if (tm.force_rows > 0) return std::max(1, n - std::min(tm.force_rows, n - 1));
    // forward levels of L after chain blocking, and the entries blocking adds to each row
    std::vector<int32_t> level(n, 0), extra(n, 0);
    {
        std::vector<int32_t> mark(n, -1);
        int stamp = 0;
        for (const auto& B : chain_blocks(L, n, true, std::max(tm.chain, 1))) {
            const int r0 = B.front();
            int lv = 0, uni = 0;
            ++stamp;
            for (int32_t r : B) {
                int raw = 0;
                for (int64_t e = L.rp[r]; e < L.rp[r + 1]; ++e) {
                    const int c = L.ci[e];
                    if (c >= r) continue;
                    ++raw;
                    if (c >= r0) continue;  // inside the block
                    lv = std::max(lv, level[c] + 1);
                    if (mark[c] != stamp) {
                        mark[c] = stamp;
                        ++uni;
                    }
                }
                level[r] = lv;
                if (B.size() > 1) extra[r] = uni - raw;
            }
        }
    }
    std::vector<int32_t> maxlev(n + 1, 0);  // levels of rows [0, T)
    for (int r = 0; r < n; ++r) maxlev[r + 1] = std::max(maxlev[r], level[r] + 1);
    // entry counts as functions of T (difference arrays)
    std::vector<double> sp(n + 2, 0.0), cp(n + 2, 0.0);
    auto account = [&](const HostCsr& M, bool lower) {
        for (int r = 0; r < n; ++r)
            for (int64_t e = M.rp[r]; e < M.rp[r + 1]; ++e) {
                const int c = M.ci[e];
                if (c == r || (lower ? c > r : c < r)) continue;
                const int lo = std::min(r, c), hi = std::max(r, c);
                // sparse-part entry iff hi < T  ->  T in [hi + 1, n]
                sp[hi + 1] += 1.0;
                // coupling entry iff lo < T <= hi  ->  T in [lo + 1, hi]
                cp[lo + 1] += 1.0;
                cp[hi + 1] -= 1.0;
            }
    };
    account(L, true);
    account(U, false);
    for (int r = 0; r < n; ++r) sp[r + 1] += 2.0 * extra[r];  // fill of the blocked rows (L and U alike)
    const double rs = tm.real_bytes, idx = 4.0;
    double best = 1e300;
    int bestT = n;
    double spc = 0.0, cpc = 0.0;
    std::vector<double> spT(n + 1, 0.0), cpT(n + 1, 0.0);
    for (int T = 0; T <= n; ++T) {
        spc += sp[T];
        cpc += cp[T];
        spT[T] = spc;
        cpT[T] = cpc;
    }
    for (int T = n; T >= std::max(1, n - tm.tail_max); --T) {
        const double sz = n - T;
        if (sz > 0 && sz < tm.tail_min) continue;
        if ((double)T * (rs + 1.0) + 64.0 > tm.smem_cap) continue;
        const double bytes = (spT[T] + cpT[T]) * (rs + idx) + sz * (sz + 1.0) * rs + 2.0 * T * (rs + 2.0);
        const double cost = 2.0 * tm.hop_s * maxlev[T] + bytes * tm.nsub / tm.bw;
        if (cost < best) {
            best = cost;
            bestT = T;
        }
    }
    return bestT;
}

// Combined column pattern of one subdomain's factors (RefactorArgs): L L^T the columns of L, LU and
// LDL^T the strict upper rows (from U), the diagonal (U's), then the strict lower rows (from L).
// Rows increase within a column.
struct FPat {
    std::vector<int64_t> cp;
    std::vector<int32_t> ri;
    std::vector<int32_t> dg;
    int32_t find(int r, int c) const
    {
        const auto b = ri.begin() + cp[c], e = ri.begin() + cp[c + 1];
        const auto it = std::lower_bound(b, e, r);
        return (it != e && *it == r) ? (int32_t)(it - ri.begin()) : -1;
    }
};

bool make_fpattern(const HostCsr& L, const HostCsr& U, int n, bool llt, FPat& P)
{
    P.cp.assign(n + 1, 0);
    auto visit = [&](const std::function<void(int, int)>& f) {
        for (int r = 0; r < n; ++r) {
            for (int64_t e = L.rp[r]; e < L.rp[r + 1]; ++e) {
                const int c = L.ci[e];
                if (llt ? c <= r : c < r) f(r, c);
            }
            if (!llt)
                for (int64_t e = U.rp[r]; e < U.rp[r + 1]; ++e) {
                    const int c = U.ci[e];
                    if (c >= r) f(r, c);
                }
        }
    };
    visit([&](int, int c) { ++P.cp[c + 1]; });
    for (int c = 0; c < n; ++c) P.cp[c + 1] += P.cp[c];
    P.ri.resize(P.cp[n]);
    std::vector<int64_t> nx(P.cp.begin(), P.cp.end() - 1);
    visit([&](int r, int c) { P.ri[nx[c]++] = r; });  // rows visited in increasing order
    P.dg.assign(n, 0);
    for (int c = 0; c < n; ++c) {
        int64_t q = P.cp[c];
        while (q < P.cp[c + 1] && P.ri[q] < c) ++q;
        if (q == P.cp[c + 1] || P.ri[q] != c) return false;
        P.dg[c] = (int32_t)(q - P.cp[c]);
    }
    return true;
}

// transpose of a lower CSR (values scaled by rowscale[c] of the result rows if given)
HostCsr transpose_lower(const HostCsr& L, int n, const std::vector<double>* rowscale)
{
    HostCsr U;
    U.rp.assign(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int64_t e = L.rp[r]; e < L.rp[r + 1]; ++e) ++U.rp[L.ci[e] + 1];
    for (int i = 0; i < n; ++i) U.rp[i + 1] += U.rp[i];
    U.ci.resize(U.rp[n]);
    U.v.resize(U.rp[n]);
    std::vector<int64_t> nx(U.rp.begin(), U.rp.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int64_t e = L.rp[r]; e < L.rp[r + 1]; ++e) {
            const int c = L.ci[e];
            const int64_t q = nx[c]++;
            U.ci[q] = r;
            U.v[q] = L.v[e] * (rowscale ? (*rowscale)[c] : 1.0);
        }
    return U;
}

// dense inverse by LU with partial pivoting (FP64); false if singular
bool dense_inverse(std::vector<double>& A, int n, std::vector<double>& Ainv)
{
    std::vector<int> piv(n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            const double v = std::fabs(A[(size_t)i * n + k]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (best == 0.0 || !std::isfinite(best)) return false;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
        const double inv = 1.0 / A[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) {
            double& lik = A[(size_t)i * n + k];
            lik *= inv;
            if (lik != 0.0) {
                const double* rk = &A[(size_t)k * n];
                double* ri = &A[(size_t)i * n];
                for (int j = k + 1; j < n; ++j) ri[j] -= lik * rk[j];
            }
        }
    }
    Ainv.assign((size_t)n * n, 0.0);
    std::vector<double> col(n);
    for (int j = 0; j < n; ++j) {
        std::fill(col.begin(), col.end(), 0.0);
        col[j] = 1.0;
        // apply the row interchanges
        for (int k = 0; k < n; ++k) std::swap(col[k], col[piv[k]]);
        for (int i = 0; i < n; ++i) {
            double s = col[i];
            for (int k = 0; k < i; ++k) s -= A[(size_t)i * n + k] * col[k];
            col[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = col[i];
            for (int k = i + 1; k < n; ++k) s -= A[(size_t)i * n + k] * col[k];
            col[i] = s / A[(size_t)i * n + i];
        }
        for (int i = 0; i < n; ++i) Ainv[(size_t)i * n + j] = col[i];
    }
    return true;
}

template <typename Real>
int upload_real(s2l_setup* s, void** dst, const std::vector<double>& v)
{
    std::vector<Real> t(v.begin(), v.end());
    Real* p = nullptr;
    RET_IF(upload(s, &p, t));
    *dst = p;
    return S2L_OK;
}

// ------------------------------------------------------------------------------ profiling
int check_ready(s2l_setup* s)
{
    if (!s) return S2L_ERR_BADARG;
    if (!s->ended) return s->fail(S2L_ERR_STATE, "setup_end() was not called");
    return S2L_OK;
}

int work_alloc(s2l_work* w, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    s2l_ctx* c = w->s->ctx;
    {
        std::lock_guard<std::mutex> g(c->mu);
        if (c->budget && c->used + bytes > c->budget) {
            c->err = "HBM budget exceeded: need " + std::to_string(c->used + bytes) + " of " + std::to_string(c->budget) +
                     " bytes";
            return S2L_ERR_OOM;
        }
        c->used += bytes;
    }
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(c->mu);
        c->used -= bytes;
        c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return S2L_ERR_OOM;
    }
    w->allocs.push_back(*p);
    w->alloc_bytes.push_back(bytes);
    w->bytes += bytes;
    return S2L_OK;
}

int work_doubles(s2l_work* w, double** p, size_t count)
{
    return work_alloc(w, reinterpret_cast<void**>(p), count * sizeof(double));
}

void work_free(s2l_work* w, void* p)
{
    for (size_t i = 0; i < w->allocs.size(); ++i)
        if (w->allocs[i] == p) {
            const size_t bytes = w->alloc_bytes[i];
            cudaFree(p);
            w->allocs.erase(w->allocs.begin() + (long)i);
            w->alloc_bytes.erase(w->alloc_bytes.begin() + (long)i);
            w->bytes -= bytes;
            std::lock_guard<std::mutex> g(w->s->ctx->mu);
            w->s->ctx->used -= std::min(w->s->ctx->used, bytes);
            return;
        }
}

void prof_begin(s2l_work* w, int cls, cudaEvent_t* a)
{
    if (!(w->prof & (1u << cls))) return;
    if (w->pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        w->pool.push_back(e);
    }
    *a = w->pool.back();
    w->pool.pop_back();
    cudaEventRecord(*a, w->stream);
    (void)cls;
}

void prof_end(s2l_work* w, int cls, cudaEvent_t a)
{
    if (!(w->prof & (1u << cls))) return;
    if (w->pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        w->pool.push_back(e);
    }
    cudaEvent_t b = w->pool.back();
    w->pool.pop_back();
    cudaEventRecord(b, w->stream);
    w->evs.push_back({cls, a, b});
}

void prof_drain(s2l_work* w)
{
    if (w->evs.empty()) return;
    cudaStreamSynchronize(w->stream);
    for (auto& e : w->evs) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
            w->acc_ms[e.cls] += ms;
            w->acc_n[e.cls] += 1;
        }
        w->pool.push_back(e.a);
        w->pool.push_back(e.b);
    }
    w->evs.clear();
}

struct Prof {
    s2l_work* w;
    int cls;
    cudaEvent_t a{};
    Prof(s2l_work* w_, int c) : w(w_), cls(c) { prof_begin(w, cls, &a); }
    ~Prof() { prof_end(w, cls, a); }
};

// ------------------------------------------------------------------------------ solve-phase pieces
template <typename Real>
LocalSolveArgs<Real> solve_args(s2l_work* w)
{
    s2l_setup* s = w->s;
    LocalSolveArgs<Real> a{};
    a.subs = s->d_subs;
    for (int f = 0; f < 2; ++f)
        a.f[f] = {s->d_col[f],   (const Real*)s->d_val[f], (const Real*)s->d_dinv[f], s->d_thdr[f],
                  s->d_tslot[f], s->d_wtask[f],            s->d_wslot[f],             s->d_went[f],
                  s->d_bfirst[f], s->d_boff[f],            s->d_bioff[f],             s->d_bslot[f],
                  (const Real*)s->d_binv[f]};
    a.u2l = s->d_u2l;
    a.tr_sub = s->d_tr_sub;
    a.tr_i = s->d_tr_i;
    a.lts_ptr = s->d_lts_ptr;
    a.lts_col = s->d_lts_col;
    a.lts_val = (const Real*)s->d_lts_val;
    a.us_sub = s->d_us_sub;
    a.us_r = s->d_us_r;
    a.ust_ptr = s->d_ust_ptr;
    a.ust_col = s->d_ust_col;
    a.ust_val = (const Real*)s->d_ust_val;
    a.uu = s->d_uu;
    a.linv = (const Real*)s->d_linv;
    a.uinv = (const Real*)s->d_uinv;
    a.gout = s->d_gout;
    a.ylocal = w->d_ylocal;
    a.ybuf = (Real*)w->d_ybuf;
    a.xbuf = (Real*)w->d_xbuf;
    a.gflags = w->d_gflags;
    a.err = w->d_err;
    a.K = 1;
    a.KC = 1;
    a.nloc = s->nloc;
    a.spin_limit = s->opt_spin_limit.load();
    a.spin_sleep_ns = s->opt_spin_sleep.load();
    a.sweep_pf = s->opt_sweep_pf.load();
    return a;
}

// Local solves of every subdomain (only_sub < 0) or of one: in -> (mode 0) out[owned] (+ base),
// (mode 1) ylocal, (mode 2: local input/output of subdomain only_sub) out.
// The AMG local solves of every subdomain: one V-cycle from x = 0 (the reference's
// --local-approx amg), with the outputs of run_local_solve's modes.
template <typename Real>
int amg_local_solve_t(s2l_work* w, const double* in, const double* base, double* out, int mode, int only_sub,
                      const double* local_in)
{
    s2l_setup* s = w->s;
    const auto& G = s->amgd;
    cudaStream_t st = w->stream;
    const int L = G.nlev;
    Real* f = reinterpret_cast<Real*>(w->d_amg);
    Real* x = f + G.vtotal;
    Real* t = f + 2 * G.vtotal;
    auto V = [](double* p) { return reinterpret_cast<const Real*>(p); };
    int64_t lo = 0, hi = 0;
    if (only_sub >= 0) {
        lo = s->h_subs[only_sub].loc_off;
        hi = lo + s->h_subs[only_sub].n_local;
    }
    launch_amg_gather<Real>(st, G.nspace[0], s->d_l2g, in, mode == 2 ? local_in : nullptr, lo, hi, f);
    CUDA_OK(w, cudaMemsetAsync(x, 0, (size_t)G.vtotal * sizeof(Real), st));
    int launched = 2;
    for (int l = 0; l < L; ++l) {
        Real *fl = f + G.voff[l], *xl = x + G.voff[l], *tl = t + G.voff[l];
        for (int k = 0; k < G.sweeps; ++k)
            launch_gs_sweep(st, G.nsmooth[l], G.Arp[l], G.Aci[l], V(G.Av[l]), fl, xl, G.fsched[l], G.fwf[l], G.fsub[l],
                            G.soff[l], G.sn[l], G.smax[l], G.lanes[l]);
        launch_coarse_inverse(st, G.ncoarse[l], G.c_off[l], G.c_n[l], G.c_inv[l], V(G.Cinv), f + G.voff[l], xl);
        launched += G.sweeps + 1;
        if (l + 1 < L) {
            launch_csr_residual(st, G.nspace[l], G.Arp[l], G.Aci[l], V(G.Av[l]), fl, xl, tl);
            launch_csr_mv(st, G.nspace[l + 1], G.Rrp[l], G.Rci[l], V(G.Rv[l]), tl, f + G.voff[l + 1], 0);
            launched += 2;
        }
    }
    // the deepest level space: its smoothed subdomains have no coarser level (backward sweeps now)
    for (int k = 0; k < G.sweeps; ++k)
        launch_gs_sweep(st, G.nsmooth[L - 1], G.Arp[L - 1], G.Aci[L - 1], V(G.Av[L - 1]), f + G.voff[L - 1],
                        x + G.voff[L - 1], G.bsched[L - 1], G.bwf[L - 1], G.bsub[L - 1], G.soff[L - 1], G.sn[L - 1],
                        G.smax[L - 1], G.lanes[L - 1]);
    for (int l = L - 2; l >= 0; --l) {
        Real *fl = f + G.voff[l], *xl = x + G.voff[l];
        launch_csr_mv(st, G.nspace[l], G.Prp[l], G.Pci[l], V(G.Pv[l]), x + G.voff[l + 1], xl, 1);
        for (int k = 0; k < G.sweeps; ++k)
            launch_gs_sweep(st, G.nsmooth[l], G.Arp[l], G.Aci[l], V(G.Av[l]), fl, xl, G.bsched[l], G.bwf[l], G.bsub[l],
                            G.soff[l], G.sn[l], G.smax[l], G.lanes[l]);
        launched += G.sweeps + 1;
    }
    launch_amg_scatter<Real>(st, G.nspace[0], G.out_idx, x, base, mode == 1 ? w->d_ylocal : out, mode, lo, hi);
    w->launches += launched + 1;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return w->fail(S2L_ERR_CUDA, std::string("AMG local solve launch: ") + cudaGetErrorString(e));
    return S2L_OK;
}

int amg_local_solve(s2l_work* w, const double* in, const double* base, double* out, int mode, int only_sub,
                    const double* local_in)
{
    return w->s->amgd.single ? amg_local_solve_t<float>(w, in, base, out, mode, only_sub, local_in)
                             : amg_local_solve_t<double>(w, in, base, out, mode, only_sub, local_in);
}

int run_local_solve(s2l_work* w, const double* in, const double* base, double* out, int mode, int only_sub,
                    const double* local_in)
{
    s2l_setup* s = w->s;
    Prof pr(w, PC_SOLVE);
    if (s->amgd.on) return amg_local_solve(w, in, base, out, mode, only_sub, local_in);
    const int nb = only_sub >= 0 ? 1 : s->nsub;
    int32_t* sub_list = nullptr;
    int tr0 = 0, trn = s->tr_first_h[s->nsub], us0 = 0, usn = s->uu_first_h[s->nsub];
    if (only_sub >= 0) {
        sub_list = reinterpret_cast<int32_t*>(w->d_red + 500);  // scratch slot for one index
        int32_t v = only_sub;
        CUDA_OK(w, cudaMemcpyAsync(sub_list, &v, sizeof(v), cudaMemcpyHostToDevice, w->stream));
        tr0 = s->tr_first_h[only_sub];
        trn = s->tr_first_h[only_sub + 1] - tr0;
        us0 = s->uu_first_h[only_sub];
        usn = s->uu_first_h[only_sub + 1] - us0;
    }
    cudaError_t e;
    int launched = 0;
    const size_t smem = w->d_gflags ? 0 : s->smem_bytes;
    if (s->real == S2L_REAL_F32) {
        LocalSolveArgs<float> a = solve_args<float>(w);
        a.sub_list = sub_list;
        a.gather = mode == 2 ? s->d_pin : s->d_gin;
        a.in = mode == 2 ? local_in : in;
        a.base = base;
        a.out = out;
        a.mode = mode;
        e = launch_local_solve<float>(w->stream, a, nb, smem, tr0, trn, us0, usn, &launched);
    } else {
        LocalSolveArgs<double> a = solve_args<double>(w);
        a.sub_list = sub_list;
        a.gather = mode == 2 ? s->d_pin : s->d_gin;
        a.in = mode == 2 ? local_in : in;
        a.base = base;
        a.out = out;
        a.mode = mode;
        e = launch_local_solve<double>(w->stream, a, nb, smem, tr0, trn, us0, usn, &launched);
    }
    w->launches += launched;
    if (e != cudaSuccess) return w->fail(S2L_ERR_CUDA, std::string("local_solve launch: ") + cudaGetErrorString(e));
    return S2L_OK;
}

// z = M1^-1 in (+ base), M1 = RAS or ASM
int one_level(s2l_work* w, const double* in, const double* base, double* out)
{
    s2l_setup* s = w->s;
    if (s->pou == S2L_POU_BOOLEAN && s->one_level == S2L_ONE_LEVEL_RAS) return run_local_solve(w, in, base, out, 0, -1, nullptr);
    RET_IF(run_local_solve(w, in, nullptr, nullptr, 1, -1, nullptr));
    Prof pr(w, PC_COMBINE);
    launch_combine(w->stream, s->n, s->d_cp_ptr, s->d_cp_pos, s->one_level == S2L_ONE_LEVEL_RAS ? s->d_cp_w : nullptr,
                   w->d_ylocal, base, out);
    w->launches += 1;
    return S2L_OK;
}

// x0 = R0^T E^-1 R0 r
int coarse_apply(s2l_work* w, const double* r, double* x0)
{
    s2l_setup* s = w->s;
    Prof pr(w, PC_COARSE);
    const int boolean = s->pou == S2L_POU_BOOLEAN;
    launch_coarse_restrict(w->stream, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->d_l2g,
                           boolean, r, s->mmax, w->d_cpart);
    launch_coarse_reduce(w->stream, s->nsub, s->d_subs, s->d_t_first, s->mmax, w->d_cpart, w->d_c);
    launch_dense_gemv(w->stream, (int)s->n0, s->d_Einv, w->d_c, w->d_y);
    launch_coarse_prolong(w->stream, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->mmax,
                          boolean, w->d_y, x0, w->d_plocal);
    if (!boolean) launch_combine(w->stream, s->n, s->d_cp_ptr, s->d_cp_pos, nullptr, w->d_plocal, nullptr, x0);
    w->launches += boolean ? 4 : 5;
    return S2L_OK;
}

int spmv_dev(s2l_work* w, const double* x, double* y, const double* b, bool with_norm)
{
    s2l_setup* s = w->s;
    Prof pr(w, PC_SPMV);
    launch_spmv(w->stream, s->n, s->d_rp, s->d_ci, s->d_av, x, y, b, with_norm ? w->d_part : nullptr,
                w->d_red + 256, s->tpr);
    w->launches += with_norm ? 2 : 1;
    return S2L_OK;
}

// z = M^-1 r (two-level Schwarz, src/preconditioner/two_level_schwarz.cpp:134-163); r and z distinct
int apply_dev(s2l_work* w, const double* r, double* z)
{
    s2l_setup* s = w->s;
    if (s->coarse == S2L_COARSE_NONE || s->n0 == 0) return one_level(w, r, nullptr, z);
    RET_IF(coarse_apply(w, r, w->d_x0));
    if (s->coarse == S2L_COARSE_ADDITIVE) return one_level(w, r, w->d_x0, z);
    RET_IF(spmv_dev(w, w->d_x0, w->d_w, r, false));  // w = r - A x0
    return one_level(w, w->d_w, w->d_x0, z);
}


// ------------------------------------------------------------------------------ block solve pieces
// Block vectors: n x K, entry i of column r at i * K + r.

// Buffers of a block solve with K columns and restart m (reallocated when a call needs others).
int ensure_block(s2l_work* w, int K, int m, bool flex)
{
    s2l_setup* s = w->s;
    s2l_work::Block& B = w->blk;
    if (B.K == K && B.m >= m && (!flex || B.flex)) return S2L_OK;
    CUDA_OK(w, cudaStreamSynchronize(w->stream));
    for (void* p : B.allocs) work_free(w, p);
    if (B.h_red) cudaFreeHost(B.h_red);
    B = s2l_work::Block{};
    const size_t rs = s->real == S2L_REAL_F32 ? 4 : 8;
    const int64_t loc = std::max<int64_t>(s->nloc, 1), n = s->n;
    int rc = S2L_OK;
    auto A = [&](void** p, size_t bytes) {
        if (rc == S2L_OK) {
            rc = work_alloc(w, p, bytes);
            if (rc == S2L_OK) B.allocs.push_back(*p);
        }
    };
    auto D = [&](double** p, size_t count) { A(reinterpret_cast<void**>(p), count * sizeof(double)); };
    A(&B.ybuf, (size_t)loc * K * rs);
    A(&B.xbuf, (size_t)loc * K * rs);
    if (s->need_gflags) A(reinterpret_cast<void**>(&B.gflags), (size_t)loc * K);
    D(&B.ylocal, (size_t)loc * K);
    D(&B.plocal, (size_t)loc * K);
    D(&B.x0, (size_t)n * K);
    D(&B.wv, (size_t)n * K);
    if (s->ntiles > 0) {
        D(&B.cpart, (size_t)s->ntiles * s->mmax * K);
        D(&B.c, (size_t)std::max<int64_t>(s->n0, 1) * K);
        D(&B.y, (size_t)std::max<int64_t>(s->n0, 1) * K);
    }
    D(&B.V, (size_t)n * K * (m + 1));
    if (flex) D(&B.Z, (size_t)n * K * (m + 1));  // m + 1: the serving runners keep Z in a ring like V
    D(&B.r, (size_t)n * K);
    D(&B.z, (size_t)n * K);
    D(&B.kw, (size_t)n * K);
    D(&B.b, (size_t)n * K);
    D(&B.xk, (size_t)n * K);
    D(&B.u, (size_t)n * K);
    D(&B.coef, S2L_MAX_BLOCK_COLS);
    D(&B.scal, 4 * S2L_MAX_RHS);
    D(&B.part, (size_t)S2L_NB_RED * S2L_MAX_BLOCK_COLS);
    D(&B.red, 3 * S2L_MAX_BLOCK_COLS);
    if (rc == S2L_OK && cudaMallocHost(&B.h_red, 3 * S2L_MAX_BLOCK_COLS * sizeof(double)) != cudaSuccess)
        rc = w->fail(S2L_ERR_OOM, "cannot allocate pinned host memory");
    if (rc != S2L_OK) {
        for (void* p : B.allocs) work_free(w, p);
        B = s2l_work::Block{};
        return rc;
    }
    B.K = K;
    B.m = m;
    B.flex = flex;
    return S2L_OK;
}

// Widest block that keeps one wave of sparse-sweep CTAs: K/KC CTAs per subdomain on the SMs.
int block_width_best(s2l_setup* s)
{
    if (s->opt_block_width > 0) return s->opt_block_width;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->ctx->device) != cudaSuccess || sms <= 0) sms = 148;
    const int kc = s->need_gflags ? 1 : s->kc_max;
    int w = kc * std::max(1, sms / std::max(s->nsub, 1));
    int p = 1;
    while (p * 2 <= w && p * 2 <= S2L_MAX_RHS) p *= 2;
    return p;
}

size_t sweep_smem(const s2l_setup* s, int kc)
{
    const size_t rs = s->real == S2L_REAL_F32 ? 4 : 8;
    const size_t slots = (size_t)s->max_T + 1;  // the sparse rows and the sentinel slot of the padding
    return (((slots * kc * rs) + 15) & ~(size_t)15) + ((slots + 15) & ~(size_t)15);
}

// local solves of every subdomain for K columns: (mode 0) out[owned] (+ base), (mode 1) ylocal
template <typename Real>
int local_solve_block_t(s2l_work* w, int K, const double* in, const double* base, double* out, int mode)
{
    s2l_setup* s = w->s;
    s2l_work::Block& B = w->blk;
    LocalSolveArgs<Real> a = solve_args<Real>(w);
    a.gather = s->d_gin;
    a.in = in;
    a.base = base;
    a.out = out;
    a.mode = mode;
    a.ylocal = B.ylocal;
    a.ybuf = (Real*)B.ybuf;
    a.xbuf = (Real*)B.xbuf;
    a.gflags = B.gflags;
    a.K = K;
    a.KC = B.gflags ? 1 : std::min(K, s->kc_max);
    const size_t smem = B.gflags ? 0 : sweep_smem(s, a.KC);
    int launched = 0;
    const cudaError_t e = launch_local_solve<Real>(w->stream, a, s->nsub, smem, 0, s->tr_first_h[s->nsub], 0,
                                                   s->uu_first_h[s->nsub], &launched);
    w->launches += launched;
    if (e != cudaSuccess) return w->fail(S2L_ERR_CUDA, std::string("block local_solve launch: ") + cudaGetErrorString(e));
    return S2L_OK;
}

int one_level_block(s2l_work* w, int K, const double* in, const double* base, double* out)
{
    s2l_setup* s = w->s;
    const bool direct = s->pou == S2L_POU_BOOLEAN && s->one_level == S2L_ONE_LEVEL_RAS;
    {
        Prof pr(w, PC_SOLVE);
        if (s->real == S2L_REAL_F32) RET_IF(local_solve_block_t<float>(w, K, in, base, out, direct ? 0 : 1));
        else RET_IF(local_solve_block_t<double>(w, K, in, base, out, direct ? 0 : 1));
    }
    if (direct) return S2L_OK;
    Prof pr(w, PC_COMBINE);
    launch_combine_block(w->stream, s->n, K, s->d_cp_ptr, s->d_cp_pos,
                         s->one_level == S2L_ONE_LEVEL_RAS ? s->d_cp_w : nullptr, w->blk.ylocal, base, out);
    w->launches += 1;
    return S2L_OK;
}

int coarse_block(s2l_work* w, int K, const double* r, double* x0)
{
    s2l_setup* s = w->s;
    s2l_work::Block& B = w->blk;
    Prof pr(w, PC_COARSE);
    const int boolean = s->pou == S2L_POU_BOOLEAN;
    launch_coarse_restrict_block(w->stream, K, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V,
                                 s->d_l2g, boolean, r, s->mmax, B.cpart);
    launch_coarse_reduce_block(w->stream, K, s->nsub, s->d_subs, s->d_t_first, s->mmax, B.cpart, B.c);
    launch_dense_gemm(w->stream, K, (int)s->n0, s->d_Einv, B.c, B.y);
    launch_coarse_prolong_block(w->stream, K, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V,
                                s->mmax, boolean, B.y, x0, B.plocal);
    if (!boolean) launch_combine_block(w->stream, s->n, K, s->d_cp_ptr, s->d_cp_pos, nullptr, B.plocal, nullptr, x0);
    w->launches += boolean ? 4 : 5;
    return S2L_OK;
}

int spmv_block(s2l_work* w, int K, const double* X, double* Y, const double* Bv, bool with_norm)
{
    s2l_setup* s = w->s;
    Prof pr(w, PC_SPMV);
    launch_spmv_block(w->stream, s->n, K, s->d_rp, s->d_ci, s->d_av, X, Y, Bv, with_norm ? w->blk.part : nullptr,
                      w->blk.red + 2 * S2L_MAX_BLOCK_COLS, s->tpr);
    w->launches += with_norm ? 2 : 1;
    return S2L_OK;
}

// Z = M^-1 R for K columns (two-level Schwarz); R and Z distinct
int apply_block(s2l_work* w, int K, const double* R, double* Z)
{
    s2l_setup* s = w->s;
    s2l_work::Block& B = w->blk;
    if (s->coarse == S2L_COARSE_NONE || s->n0 == 0) return one_level_block(w, K, R, nullptr, Z);
    RET_IF(coarse_block(w, K, R, B.x0));
    if (s->coarse == S2L_COARSE_ADDITIVE) return one_level_block(w, K, R, B.x0, Z);
    RET_IF(spmv_block(w, K, B.x0, B.wv, R, false));  // W = R - A X0
    return one_level_block(w, K, B.wv, B.x0, Z);
}

// host/device staging of a global vector argument
int stage_in(s2l_work* w, const double* p, int kind, int64_t count, double* tmp, const double** dev)
{
    if (kind == S2L_PTR_DEVICE) {
        *dev = p;
        return S2L_OK;
    }
    if (kind != S2L_PTR_HOST) return w->fail(S2L_ERR_BADARG, "ptr_kind must be S2L_PTR_HOST or S2L_PTR_DEVICE");
    CUDA_OK(w, cudaMemcpyAsync(tmp, p, count * sizeof(double), cudaMemcpyHostToDevice, w->stream));
    *dev = tmp;
    return S2L_OK;
}

int finish_out(s2l_work* w, double* dst, const double* dev, int kind, int64_t count)
{
    if (kind == S2L_PTR_HOST)
        CUDA_OK(w, cudaMemcpyAsync(dst, dev, count * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
    else if (dst != dev)
        CUDA_OK(w, cudaMemcpyAsync(dst, dev, count * sizeof(double), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_OK(w, cudaStreamSynchronize(w->stream));
    CUDA_OK(w, cudaGetLastError());
    return check_err(w);
}

int ensure_krylov(s2l_work* w, int m, bool flexible)
{
    s2l_setup* s = w->s;
    if (w->kr_m >= m && (!flexible || w->kr_flex)) return S2L_OK;
    if (m + 1 > S2L_MAX_RED_COLS - 1) return w->fail(S2L_ERR_BADARG, "restart too large (max 120)");
    const size_t n = (size_t)s->n;
    std::vector<double*> fresh;  // undone if a later allocation fails (admission retries it)
    int rc = S2L_OK;
    auto D = [&](double** p, size_t count) {
        double* q = nullptr;
        if (rc == S2L_OK) rc = work_doubles(w, &q, count);
        if (rc == S2L_OK) fresh.push_back(q);
        return q;
    };
    double* V = D(nullptr, n * (m + 1));
    double* Z = flexible ? D(nullptr, n * m) : nullptr;
    double *r = nullptr, *z = nullptr, *kw = nullptr, *b = nullptr, *xk = nullptr, *u = nullptr, *coef = nullptr;
    if (w->kr_m < 0) {
        r = D(nullptr, n);
        z = D(nullptr, n);
        kw = D(nullptr, n);
        b = D(nullptr, n);
        xk = D(nullptr, n);
        u = D(nullptr, n);
        coef = D(nullptr, 2 * S2L_MAX_RED_COLS);
    }
    if (rc != S2L_OK) {
        for (double* q : fresh) work_free(w, q);
        return rc;
    }
    if (w->d_V_kr) work_free(w, w->d_V_kr);
    w->d_V_kr = V;
    if (flexible) {
        if (w->d_Z_kr) work_free(w, w->d_Z_kr);
        w->d_Z_kr = Z;
    }
    if (w->kr_m < 0) {
        w->d_r = r;
        w->d_z = z;
        w->d_kw = kw;
        w->d_b = b;
        w->d_xk = xk;
        w->d_u = u;
        w->d_coef = coef;
    }
    w->kr_m = m;
    w->kr_flex = w->kr_flex || flexible;
    return S2L_OK;
}

int read_red(s2l_work* w, int off, int count)
{
    CUDA_OK(w, cudaMemcpyAsync(w->h_red + off, w->d_red + off, count * sizeof(double), cudaMemcpyDeviceToHost,
                               w->stream));
    return check_err(w);
}

int norm2_dev(s2l_work* w, const double* x, double* out_host)
{
    s2l_setup* s = w->s;
    {
        Prof pr(w, PC_VEC);
        launch_dot2(w->stream, s->n, x, x, nullptr, w->d_part, w->d_red + 256);
        w->launches += 2;
    }
    RET_IF(read_red(w, 256, 1));
    *out_host = std::sqrt(w->h_red[256]);
    return S2L_OK;
}

// sum|a - alpha c| (c may be nullptr) and sum a
int l1_dev(s2l_work* w, const double* a, double alpha, const double* c, double* l1, double* sum)
{
    s2l_setup* s = w->s;
    {
        Prof pr(w, PC_VEC);
        launch_l1(w->stream, s->n, a, alpha, c, w->d_part, w->d_red + 300);
        w->launches += 2;
    }
    RET_IF(read_red(w, 300, 2));
    *l1 = w->h_red[300];
    if (sum) *sum = w->h_red[301];
    return S2L_OK;
}

// OpenFOAM normalisation factor of x0 (src/solver/krylov.cpp:48-58), Ax0 = A x0:
// F = sum|A x0 - xm A 1| + sum|b - xm A 1| + 1e-20, xm the mean of x0 (A 1 not needed when xm = 0)
int of_norm_factor(s2l_work* w, const double* b, const double* x0, const double* Ax0, double* F)
{
    s2l_setup* s = w->s;
    double unused = 0.0, sx = 0.0, a1 = 0.0, a2 = 0.0;
    RET_IF(l1_dev(w, x0, 0.0, nullptr, &unused, &sx));
    const double xm = s->n > 0 ? sx / (double)s->n : 0.0;
    RET_IF(l1_dev(w, Ax0, xm, xm == 0.0 ? nullptr : s->d_rowsum, &a1, nullptr));
    RET_IF(l1_dev(w, b, xm, xm == 0.0 ? nullptr : s->d_rowsum, &a2, nullptr));
    *F = a1 + a2 + 1e-20;
    return S2L_OK;
}

// checks of the stopping-norm options (src/solver/krylov.cpp:14-33)
int check_stop(s2l_setup* s, const s2l_krylov_opts* o)
{
    if (o->stop_norm != S2L_STOP_L2 && o->stop_norm != S2L_STOP_OPENFOAM)
        return s->fail(S2L_ERR_BADARG, "unknown stopping norm (S2L_STOP_L2 | S2L_STOP_OPENFOAM)");
    if (!(o->atol >= 0.0)) return s->fail(S2L_ERR_BADARG, "atol must be >= 0");
    if (o->atol > 0.0 && o->stop_norm != S2L_STOP_OPENFOAM)
        return s->fail(S2L_ERR_BADARG, "an absolute tolerance needs the OpenFOAM stopping norm");
    return S2L_OK;
}

// Inverses of the dense tails: X = L_tt^-1 and Y = U_tt^-1, row-major, through cuBLAS DTRSM on
// the identity.  A row-major triangle is the column-major transpose, so solving with the
// transposed triangle leaves the row-major inverse in place.
int invert_tails(s2l_setup* s, const std::vector<std::vector<double>>& Ltt, const std::vector<std::vector<double>>& Utt,
                 const std::vector<int64_t>& d_off)
{
    int max_sz = 0;
    for (size_t i = 0; i < Ltt.size(); ++i)
        if (!Ltt[i].empty()) max_sz = std::max(max_sz, (int)std::lround(std::sqrt((double)Ltt[i].size())));
    if (max_sz == 0) return S2L_OK;
    double *dA = nullptr, *dB = nullptr;
    const size_t mb = (size_t)max_sz * max_sz * sizeof(double);
    if (cudaMalloc(&dA, mb) != cudaSuccess || cudaMalloc(&dB, mb) != cudaSuccess) {
        cudaFree(dA);
        return s->fail(S2L_ERR_OOM, "no device memory for the tail inversion");
    }
    cublasHandle_t hb = nullptr;
    int rc = S2L_OK;
    if (cublasCreate(&hb) != CUBLAS_STATUS_SUCCESS) rc = s->fail(S2L_ERR_CUDA, "cublasCreate failed");
    if (rc == S2L_OK) cublasSetStream(hb, s->setup_stream);
    std::vector<double> eye;
    for (size_t i = 0; i < Ltt.size() && rc == S2L_OK; ++i) {
        if (Ltt[i].empty()) continue;
        const int sz = (int)std::lround(std::sqrt((double)Ltt[i].size()));
        eye.assign((size_t)sz * sz, 0.0);
        for (int k = 0; k < sz; ++k) eye[(size_t)k * sz + k] = 1.0;
        const double one = 1.0;
        for (int f = 0; f < 2 && rc == S2L_OK; ++f) {
            const std::vector<double>& M = f == 0 ? Ltt[i] : Utt[i];
            if (cudaMemcpyAsync(dA, M.data(), (size_t)sz * sz * sizeof(double), cudaMemcpyHostToDevice, s->setup_stream) != cudaSuccess ||
                cudaMemcpyAsync(dB, eye.data(), (size_t)sz * sz * sizeof(double), cudaMemcpyHostToDevice, s->setup_stream) != cudaSuccess) {
                rc = s->fail(S2L_ERR_CUDA, "tail upload failed");
                break;
            }
            // row-major lower L = column-major upper L^T (and row-major upper U = column-major lower U^T)
            const cublasFillMode_t fill = f == 0 ? CUBLAS_FILL_MODE_UPPER : CUBLAS_FILL_MODE_LOWER;
            if (cublasDtrsm(hb, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, sz, sz, &one, dA, sz, dB, sz) !=
                CUBLAS_STATUS_SUCCESS) {
                rc = s->fail(S2L_ERR_CUDA, "cublasDtrsm failed");
                break;
            }
            void* dst = f == 0 ? s->d_linv : s->d_uinv;
            if (s->real == S2L_REAL_F32) {
                launch_to_float(s->setup_stream, dB, (float*)dst + d_off[i], (int64_t)sz * sz);
            } else if (cudaMemcpyAsync((double*)dst + d_off[i], dB, (size_t)sz * sz * sizeof(double),
                                       cudaMemcpyDeviceToDevice, s->setup_stream) != cudaSuccess) {
                rc = s->fail(S2L_ERR_CUDA, "tail copy failed");
            }
            // the host copies of M and eye are reused: finish before the next upload
            if (cudaStreamSynchronize(s->setup_stream) != cudaSuccess) rc = s->fail(S2L_ERR_CUDA, "tail inversion failed");
        }
    }
    if (hb) cublasDestroy(hb);
    cudaFree(dA);
    cudaFree(dB);
    return rc;
}

// error word of the sweeps: a bounded wait gave up
int check_err(s2l_work* w)
{
    int e = 0;
    CUDA_OK(w, cudaMemcpyAsync(&e, w->d_err, sizeof(int), cudaMemcpyDeviceToHost, w->stream));
    CUDA_OK(w, cudaStreamSynchronize(w->stream));
    if (e) {
        CUDA_OK(w, cudaMemsetAsync(w->d_err, 0, sizeof(int), w->stream));
        return w->fail(S2L_ERR_TIMEOUT, "a sparse sweep gave up waiting for a row (bounded wait exceeded)");
    }
    return S2L_OK;
}

// ------------------------------------------------------------------------------ workspaces
int work_create(s2l_setup* s, s2l_work** out)
{
    *out = nullptr;
    auto* w = new s2l_work;
    w->s = s;
    if (cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete w;
        return s->fail(S2L_ERR_CUDA, "cannot create a stream");
    }
    w->stream = w->own_stream;
    w->prof = s->prof_mask;
    if (cudaEventCreateWithFlags(&w->join, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(w->own_stream);
        delete w;
        return s->fail(S2L_ERR_CUDA, "cannot create an event");
    }
    const size_t rs = s->real == S2L_REAL_F32 ? 4 : 8;
    const int64_t loc = std::max<int64_t>(s->nloc, 1);
    int rc = S2L_OK;
    auto A = [&](void** p, size_t b) {
        if (rc == S2L_OK) rc = work_alloc(w, p, b);
    };
    A(&w->d_ybuf, (size_t)loc * rs);
    A(&w->d_xbuf, (size_t)loc * rs);
    A(reinterpret_cast<void**>(&w->d_err), 16);
    if (s->need_gflags) A(reinterpret_cast<void**>(&w->d_gflags), (size_t)loc);
    if (s->ntiles > 0) {
        A(reinterpret_cast<void**>(&w->d_cpart), (size_t)s->ntiles * s->mmax * sizeof(double));
        A(reinterpret_cast<void**>(&w->d_c), (size_t)std::max<int64_t>(s->n0, 1) * sizeof(double));
        A(reinterpret_cast<void**>(&w->d_y), (size_t)std::max<int64_t>(s->n0, 1) * sizeof(double));
    }
    A(reinterpret_cast<void**>(&w->d_ylocal), (size_t)loc * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_plocal), (size_t)loc * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_x0), (size_t)s->n * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_w), (size_t)s->n * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_in), (size_t)std::max<int64_t>(s->n, s->max_nl) * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_out), (size_t)std::max<int64_t>(s->n, s->max_nl) * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_part), (size_t)S2L_NB_RED * S2L_MAX_RED_COLS * sizeof(double));
    A(reinterpret_cast<void**>(&w->d_red), 512 * sizeof(double));
    if (s->amgd.on) A(reinterpret_cast<void**>(&w->d_amg), (size_t)std::max<int64_t>(3 * s->amgd.vtotal, 1) * sizeof(double));
    if (rc == S2L_OK && cudaMallocHost(&w->h_red, 512 * sizeof(double)) != cudaSuccess)
        rc = s->fail(S2L_ERR_OOM, "cannot allocate pinned host memory");
    if (rc == S2L_OK && cudaMemsetAsync(w->d_err, 0, 16, w->stream) != cudaSuccess) rc = S2L_ERR_CUDA;
    if (rc == S2L_OK && cudaStreamSynchronize(w->stream) != cudaSuccess) rc = S2L_ERR_CUDA;
    if (rc != S2L_OK) {
        for (void* p : w->allocs) cudaFree(p);
        {
            std::lock_guard<std::mutex> g(s->ctx->mu);
            s->ctx->used -= std::min(s->ctx->used, w->bytes);
        }
        if (w->h_red) cudaFreeHost(w->h_red);
        cudaEventDestroy(w->join);
        cudaStreamDestroy(w->own_stream);
        delete w;
        return rc;
    }
    *out = w;
    return S2L_OK;
}

void work_destroy(s2l_work* w)
{
    if (!w) return;
    cudaStreamSynchronize(w->stream);
    cudaStreamSynchronize(w->own_stream);
    prof_drain(w);
    for (void* p : w->allocs) cudaFree(p);
    {
        std::lock_guard<std::mutex> g(w->s->ctx->mu);
        w->s->ctx->used -= std::min(w->s->ctx->used, w->bytes);
    }
    if (w->h_red) cudaFreeHost(w->h_red);
    if (w->blk.h_red) cudaFreeHost(w->blk.h_red);
    for (auto e : w->pool) cudaEventDestroy(e);
    cudaEventDestroy(w->join);
    cudaStreamDestroy(w->own_stream);
    delete w;
}

// A free workspace for one solve-phase call: workspace 0 when it is free (it carries the caller's
// stream and timers), another free one, or a new one when every workspace is busy (concurrent
// calls on one setup from several threads).
// A workspace for one solve-phase call: workspace 0 when it is free (it carries the caller's
// stream and timers), another free one, or a new one when every workspace is busy (concurrent
// calls on one setup from several threads).  `prepare` allocates what the call needs on the
// workspace (Krylov basis, block buffers).
//
// Admission by HBM footprint: when those allocations do not fit the context's budget, the call
// waits for a busy workspace of this setup to come free (it usually has them already) and tries
// again; it fails with S2L_ERR_OOM only when no workspace is busy or after S2L_ADMIT_WAIT_S seconds.
struct Lease {
    s2l_setup* s;
    s2l_work* w = nullptr;
    int idx = -1;
    int rc = S2L_OK;
    explicit Lease(s2l_setup* s_, const std::function<int(s2l_work*)>& prepare = {}) : s(s_)
    {
        if (cudaSetDevice(s->ctx->device) != cudaSuccess) {
            rc = s->fail(S2L_ERR_CUDA, "cudaSetDevice failed");
            return;
        }
        std::unique_lock<std::mutex> g(s->wmu);
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::seconds(S2L_ADMIT_WAIT_S);
        auto take = [&](size_t i) -> int {  // reserve workspace i and prepare it (lock released meanwhile)
            s->busy[i] = 1;
            s2l_work* cand = s->works[i];
            g.unlock();
            const int r = prepare ? prepare(cand) : S2L_OK;
            g.lock();
            if (r != S2L_OK) s->busy[i] = 0;
            return r;
        };
        for (;;) {
            for (size_t i = 0; i < s->works.size() && idx < 0; ++i) {
                if (s->busy[i]) continue;
                const int r = take(i);
                if (r == S2L_OK) idx = (int)i;
                else if (r != S2L_ERR_OOM) {
                    rc = r;
                    return;
                }
            }
            if (idx >= 0) break;
            s2l_work* nw = nullptr;
            int r = work_create(s, &nw);
            if (r == S2L_OK) {
                s->works.push_back(nw);
                s->busy.push_back(0);
                const size_t i = s->works.size() - 1;
                r = take(i);
                if (r == S2L_OK) {
                    idx = (int)i;
                    break;
                }
            }
            if (r != S2L_ERR_OOM) {
                rc = r;
                return;
            }
            bool anybusy = false;
            for (char b : s->busy) anybusy = anybusy || b;
            if (!anybusy || s->wcv.wait_until(g, deadline) == std::cv_status::timeout) {
                rc = S2L_ERR_OOM;  // the message of the failed allocation stays in last_error
                return;
            }
        }
        w = s->works[idx];
        // another workspace's stream starts after the work already queued on the caller's stream
        if (idx != 0 && s->user_stream) {
            if (cudaEventRecord(w->join, s->user_stream) != cudaSuccess ||
                cudaStreamWaitEvent(w->stream, w->join, 0) != cudaSuccess)
                rc = s->fail(S2L_ERR_CUDA, "cannot order a workspace after the caller's stream");
        }
    }
    ~Lease()
    {
        if (idx < 0) return;
        {
            std::lock_guard<std::mutex> g(s->wmu);
            s->busy[idx] = 0;
        }
        s->wcv.notify_all();
    }
};

}  // namespace

// ================================================================================= C ABI
extern "C" {

int s2l_gpu_create(int device, size_t hbm_budget_bytes, s2l_ctx** ctx)
{
    if (!ctx) return S2L_ERR_BADARG;
    *ctx = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return S2L_ERR_CUDA;
    if (device < 0 || device >= count) return S2L_ERR_BADARG;
    if (cudaSetDevice(device) != cudaSuccess) return S2L_ERR_CUDA;
    auto* c = new s2l_ctx;
    c->device = device;
    c->budget = hbm_budget_bytes;
    *ctx = c;
    return S2L_OK;
}

int s2l_gpu_destroy(s2l_ctx* ctx)
{
    if (!ctx) return S2L_OK;
    serve_stop(ctx);
    delete ctx;
    return S2L_OK;
}

const char* s2l_gpu_last_error(const s2l_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int s2l_gpu_setup_begin(s2l_ctx* ctx, int64_t n, int nsub, int one_level, int coarse, int pou, s2l_setup** out)
{
    if (!ctx || !out) return S2L_ERR_BADARG;
    *out = nullptr;
    auto bad = [&](const char* m) {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->err = m;
        return S2L_ERR_BADARG;
    };
    if (n <= 0 || n >= (int64_t)INT32_MAX) return bad("n must be in [1, 2^31)");
    if (nsub <= 0) return bad("nsub must be positive");
    if (one_level != S2L_ONE_LEVEL_RAS && one_level != S2L_ONE_LEVEL_ASM) return bad("unknown one-level variant");
    if (coarse < S2L_COARSE_NONE || coarse > S2L_COARSE_DEFLATED) return bad("unknown coarse correction");
    if (pou != S2L_POU_BOOLEAN && pou != S2L_POU_MULTIPLICITY) return bad("unknown partition of unity");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return S2L_ERR_CUDA;
    auto* s = new s2l_setup;
    s->ctx = ctx;
    s->n = n;
    s->nsub = nsub;
    s->one_level = one_level;
    s->coarse = coarse;
    s->pou = pou;
    s->hs.resize(nsub);
    if (cudaStreamCreateWithFlags(&s->setup_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return S2L_ERR_CUDA;
    }
    *out = s;
    return S2L_OK;
}

int s2l_gpu_set_matrix(s2l_setup* s, const int64_t* rowptr, const int64_t* col, const double* val)
{
    if (!s || !rowptr || !col || !val) return S2L_ERR_BADARG;
    if (s->ended) return s->fail(S2L_ERR_STATE, "set_matrix after setup_end");
    const int64_t n = s->n;
    if (rowptr[0] != 0) return s->fail(S2L_ERR_BADARG, "rowptr[0] must be 0");
    const int64_t nnz = rowptr[n];
    if (nnz < 0 || nnz >= (int64_t)INT32_MAX) return s->fail(S2L_ERR_BADARG, "nnz must be in [0, 2^31)");
    for (int64_t r = 0; r < n; ++r)  // monotone: every row ends within [0, nnz]
        if (rowptr[r + 1] < rowptr[r]) return s->fail(S2L_ERR_BADARG, "rowptr not monotone");
    s->A.rp.assign(rowptr, rowptr + n + 1);
    s->A.ci.resize(nnz);
    for (int64_t r = 0; r < n; ++r) {
        for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            if (col[e] < 0 || col[e] >= n) return s->fail(S2L_ERR_BADARG, "column index out of range");
            s->A.ci[e] = (int32_t)col[e];
        }
    }
    s->A.v.assign(val, val + nnz);
    s->have_A = true;
    return S2L_OK;
}

int s2l_gpu_add_subdomain(s2l_setup* s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t* ghosts,
                          const double* D, int factor_kind, int real_type, const int32_t* perm_in,
                          const int32_t* perm_out, const int64_t* L_rowptr, const int32_t* L_col, const void* L_val,
                          const int64_t* U_rowptr, const int32_t* U_col, const void* U_val, const void* ldlt_d,
                          int m, const double* V)
{
    if (!s) return S2L_ERR_BADARG;
    if (s->ended) return s->fail(S2L_ERR_STATE, "add_subdomain after setup_end");
    if (i < 0 || i >= s->nsub) return s->fail(S2L_ERR_BADARG, "subdomain index out of range");
    if (n_owned <= 0 || n_ghost < 0) return s->fail(S2L_ERR_BADARG, "n_owned must be > 0 and n_ghost >= 0");
    if (begin < 0 || begin + n_owned > s->n) return s->fail(S2L_ERR_BADARG, "owned range outside [0, n)");
    if (real_type != S2L_REAL_F64 && real_type != S2L_REAL_F32) return s->fail(S2L_ERR_BADARG, "unknown real type");
    if (s->real >= 0 && s->real != real_type)
        return s->fail(S2L_ERR_BADARG, "all subdomains must store their factors in the same precision");
    if (s->local_kind == 1) return s->fail(S2L_ERR_BADARG, "a setup's subdomains all use factors or all AMG");
    s->local_kind = 0;
    if (factor_kind < S2L_FACTOR_LU || factor_kind > S2L_FACTOR_LDLT) return s->fail(S2L_ERR_BADARG, "unknown factor kind");
    if (!D || !perm_in || !perm_out || !L_rowptr || !L_col || !L_val || (n_ghost && !ghosts))
        return s->fail(S2L_ERR_BADARG, "null array");
    if (factor_kind == S2L_FACTOR_LU && (!U_rowptr || !U_col || !U_val)) return s->fail(S2L_ERR_BADARG, "LU needs U");
    if (factor_kind == S2L_FACTOR_LDLT && !ldlt_d) return s->fail(S2L_ERR_BADARG, "LDLT needs d");
    if (m < 0 || m > S2L_MAX_RED_COLS || (m > 0 && !V)) return s->fail(S2L_ERR_BADARG, "bad coarse basis (m <= 128)");
    s->real = real_type;
    HostSub& h = s->hs[i];
    h = HostSub();
    const int nl = n_owned + n_ghost;
    h.begin = begin;
    h.n_owned = n_owned;
    h.n_ghost = n_ghost;
    h.ghosts.assign(ghosts, ghosts + n_ghost);
    for (int k = 0; k < n_ghost; ++k) {
        if (ghosts[k] < 0 || ghosts[k] >= s->n) return s->fail(S2L_ERR_BADARG, "ghost id out of range");
        if (ghosts[k] >= begin && ghosts[k] < begin + n_owned) return s->fail(S2L_ERR_BADARG, "ghost is an owned row");
        if (k && ghosts[k] <= ghosts[k - 1]) return s->fail(S2L_ERR_BADARG, "ghosts must be sorted and unique");
    }
    h.D.assign(D, D + nl);
    h.kind = factor_kind;
    h.pin.assign(perm_in, perm_in + nl);
    h.pout.assign(perm_out, perm_out + nl);
    {
        std::vector<char> seen(nl, 0), seen2(nl, 0);
        for (int k = 0; k < nl; ++k) {
            if (perm_in[k] < 0 || perm_in[k] >= nl || seen[perm_in[k]]) return s->fail(S2L_ERR_BADARG, "perm_in is not a permutation");
            if (perm_out[k] < 0 || perm_out[k] >= nl || seen2[perm_out[k]]) return s->fail(S2L_ERR_BADARG, "perm_out is not a permutation");
            seen[perm_in[k]] = seen2[perm_out[k]] = 1;
        }
    }
    auto copy_csr = [&](HostCsr& dst, const int64_t* rp, const int32_t* ci, const void* v, bool lower) -> int {
        if (rp[0] != 0) return s->fail(S2L_ERR_BADARG, "factor rowptr[0] must be 0");
        for (int r = 0; r < nl; ++r)
            if (rp[r + 1] < rp[r]) return s->fail(S2L_ERR_BADARG, "factor rowptr not monotone");
        dst.rp.assign(rp, rp + nl + 1);
        const int64_t nz = rp[nl];
        dst.ci.assign(ci, ci + nz);
        dst.v.resize(nz);
        if (real_type == S2L_REAL_F64)
            std::copy((const double*)v, (const double*)v + nz, dst.v.begin());
        else
            std::copy((const float*)v, (const float*)v + nz, dst.v.begin());
        for (int r = 0; r < nl; ++r) {
            for (int64_t e = rp[r]; e < rp[r + 1]; ++e) {
                const int c = ci[e];
                if (c < 0 || c >= nl) return s->fail(S2L_ERR_BADARG, "factor column out of range");
                if (lower ? c > r : c < r) return s->fail(S2L_ERR_BADARG, lower ? "L has an entry above the diagonal" : "U has an entry below the diagonal");
            }
        }
        return S2L_OK;
    };
    RET_IF(copy_csr(h.L, L_rowptr, L_col, L_val, true));
    if (factor_kind == S2L_FACTOR_LU) RET_IF(copy_csr(h.U, U_rowptr, U_col, U_val, false));
    if (factor_kind == S2L_FACTOR_LDLT) {
        h.d.resize(nl);
        for (int k = 0; k < nl; ++k)
            h.d[k] = real_type == S2L_REAL_F64 ? ((const double*)ldlt_d)[k] : ((const float*)ldlt_d)[k];
    }
    h.m = m;
    if (m) h.V.assign(V, V + (size_t)nl * m);
    h.set = true;
    return S2L_OK;
}

int s2l_gpu_add_subdomain_amg(s2l_setup* s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t* ghosts,
                              const double* D, int nlev, int sweeps, const int32_t* nrow,
                              const int64_t* const* A_rowptr, const int32_t* const* A_col, const double* const* A_val,
                              const int64_t* const* P_rowptr, const int32_t* const* P_col, const double* const* P_val,
                              const int64_t* const* R_rowptr, const int32_t* const* R_col, const double* const* R_val,
                              int n_coarse, const double* coarse, int m, const double* V)
{
    if (!s) return S2L_ERR_BADARG;
    if (s->ended) return s->fail(S2L_ERR_STATE, "add_subdomain_amg after setup_end");
    if (i < 0 || i >= s->nsub) return s->fail(S2L_ERR_BADARG, "subdomain index out of range");
    if (n_owned <= 0 || n_ghost < 0) return s->fail(S2L_ERR_BADARG, "n_owned must be > 0 and n_ghost >= 0");
    if (begin < 0 || begin + n_owned > s->n) return s->fail(S2L_ERR_BADARG, "owned range outside [0, n)");
    if (s->local_kind == 0) return s->fail(S2L_ERR_BADARG, "a setup's subdomains all use factors or all AMG");
    if (s->real == S2L_REAL_F32) return s->fail(S2L_ERR_BADARG, "AMG local solvers run in FP64");
    if (!D || (n_ghost && !ghosts)) return s->fail(S2L_ERR_BADARG, "null array");
    if (nlev < 0 || nlev > 32 || sweeps < 1 || sweeps > 16 || n_coarse < 0)
        return s->fail(S2L_ERR_BADARG, "bad AMG hierarchy: levels in [0, 32], sweeps in [1, 16]");
    if (m < 0 || m > S2L_MAX_RED_COLS || (m > 0 && !V)) return s->fail(S2L_ERR_BADARG, "bad coarse basis (m <= 128)");
    const int nl = n_owned + n_ghost;
    if (nlev == 0 && n_coarse != nl) return s->fail(S2L_ERR_BADARG, "a hierarchy without levels needs a coarse solve of n_local rows");
    if (nlev > 0 && (!nrow || nrow[0] != nl)) return s->fail(S2L_ERR_BADARG, "the first AMG level must have n_local rows");
    if (n_coarse > 0 && !coarse) return s->fail(S2L_ERR_BADARG, "null coarse operator");
    s->local_kind = 1;
    s->real = S2L_REAL_F64;
    HostSub& h = s->hs[i];
    h = HostSub();
    h.begin = begin;
    h.n_owned = n_owned;
    h.n_ghost = n_ghost;
    h.ghosts.assign(ghosts, ghosts + n_ghost);
    for (int k = 0; k < n_ghost; ++k) {
        if (ghosts[k] < 0 || ghosts[k] >= s->n) return s->fail(S2L_ERR_BADARG, "ghost id out of range");
        if (ghosts[k] >= begin && ghosts[k] < begin + n_owned) return s->fail(S2L_ERR_BADARG, "ghost is an owned row");
        if (k && ghosts[k] <= ghosts[k - 1]) return s->fail(S2L_ERR_BADARG, "ghosts must be sorted and unique");
    }
    h.D.assign(D, D + nl);
    h.amg = true;
    h.amg_sweeps = sweeps;
    auto copy = [&](HostCsr& dst, int rows, int cols, const int64_t* rp, const int32_t* ci, const double* v) -> int {
        if (!rp || !ci || !v || rp[0] != 0) return s->fail(S2L_ERR_BADARG, "bad AMG level matrix");
        for (int r = 0; r < rows; ++r)
            if (rp[r + 1] < rp[r]) return s->fail(S2L_ERR_BADARG, "AMG level matrix: rowptr not monotone");
        dst.rp.assign(rp, rp + rows + 1);
        const int64_t nz = rp[rows];
        dst.ci.assign(ci, ci + nz);
        dst.v.assign(v, v + nz);
        for (int r = 0; r < rows; ++r) {
            for (int64_t e = rp[r]; e < rp[r + 1]; ++e)
                if (ci[e] < 0 || ci[e] >= cols || (e > rp[r] && ci[e] <= ci[e - 1]))
                    return s->fail(S2L_ERR_BADARG, "AMG level matrix: columns out of range or not sorted");
        }
        return S2L_OK;
    };
    h.amgA.resize(nlev);
    h.amgP.resize(nlev);
    h.amgR.resize(nlev);
    for (int l = 0; l < nlev; ++l) {
        if (nrow[l] <= 0) return s->fail(S2L_ERR_BADARG, "an AMG level without rows");
        RET_IF(copy(h.amgA[l], nrow[l], nrow[l], A_rowptr[l], A_col[l], A_val[l]));
        const int next = l + 1 < nlev ? nrow[l + 1] : n_coarse;
        if (next > 0) {  // the transfer operators to the next level (none after a last smoothed-only level)
            RET_IF(copy(h.amgP[l], nrow[l], next, P_rowptr[l], P_col[l], P_val[l]));
            RET_IF(copy(h.amgR[l], next, nrow[l], R_rowptr[l], R_col[l], R_val[l]));
        } else if (l + 1 < nlev) {
            return s->fail(S2L_ERR_BADARG, "only the last AMG level may have no coarser level");
        }
    }
    h.amg_nc = n_coarse;
    if (n_coarse > 0) h.amgC.assign(coarse, coarse + (size_t)n_coarse * n_coarse);
    h.m = m;
    if (m) h.V.assign(V, V + (size_t)nl * m);
    h.pin.resize(nl);
    h.pout.resize(nl);
    for (int k = 0; k < nl; ++k) h.pin[k] = h.pout[k] = k;
    h.set = true;
    return S2L_OK;
}

int s2l_gpu_set_coarse(s2l_setup* s, int64_t n0, const int64_t* offsets, const double* E)
{
    if (!s) return S2L_ERR_BADARG;
    if (s->ended) return s->fail(S2L_ERR_STATE, "set_coarse after setup_end");
    if (n0 < 0 || (n0 > 0 && (!offsets || !E))) return s->fail(S2L_ERR_BADARG, "bad coarse arguments");
    if (n0 > 65536) return s->fail(S2L_ERR_BADARG, "coarse dimension too large for the dense inverse (max 65536)");
    s->n0 = n0;
    s->coff.assign(offsets, offsets + s->nsub + 1);
    s->E.assign(E, E + (size_t)n0 * n0);
    s->have_coarse = true;
    return S2L_OK;
}

}  // extern "C"

namespace {

// Gauss-Seidel wavefronts of one matrix (rows in sweep order: increasing when forward): a row
// comes after every earlier row it reads or that reads it, so a wavefront's rows see exactly the
// values a serial sweep would.  Returns per row its wavefront.
std::vector<int32_t> gs_wavefronts(const HostCsr& A, int n, bool forward)
{
    std::vector<int32_t> wf(n, 0);
    for (int q = 0; q < n; ++q) {
        const int r = forward ? q : n - 1 - q;
        auto earlier = [&](int c) { return forward ? c < r : c > r; };
        int w = wf[r];
        for (int64_t e = A.rp[r]; e < A.rp[r + 1]; ++e)
            if (earlier(A.ci[e])) w = std::max(w, wf[A.ci[e]] + 1);
        wf[r] = w;
        for (int64_t e = A.rp[r]; e < A.rp[r + 1]; ++e) {
            const int c = A.ci[e];
            if (c != r && !earlier(c)) wf[c] = std::max(wf[c], w + 1);  // c reads r's new value later
        }
    }
    return wf;
}

// Device data of the AMG local solvers: per level space the block-diagonal A, R, P, the sweeps'
// wavefronts and the coarsest levels' inverses.
int amg_build(s2l_setup* s)
{
    auto& G = s->amgd;
    const int nsub = s->nsub;
    int L = 0;
    for (int i = 0; i < nsub; ++i) {
        const HostSub& h = s->hs[i];
        L = std::max(L, (int)h.amgA.size() + (h.amg_nc > 0 ? 1 : 0));
        G.sweeps = h.amg_sweeps;
    }
    for (int i = 0; i < nsub; ++i)
        if (s->hs[i].amg_sweeps != G.sweeps) return s->fail(S2L_ERR_BADARG, "all AMG hierarchies need the same sweeps");
    G.nlev = L;
    G.single = s->opt_amg_single != 0;
    const double vb = G.single ? 4.0 : 8.0;  // bytes of a value
    // values in the hierarchy's precision (float arrays behind the double pointers when single)
    auto upload_vals = [&](double** dst, const std::vector<double>& src) -> int {
        if (!G.single) return upload(s, dst, src);
        std::vector<float> f(src.begin(), src.end());
        float* p = nullptr;
        RET_IF(upload(s, &p, f));
        *dst = reinterpret_cast<double*>(p);
        return S2L_OK;
    };
    auto rows_at = [&](const HostSub& h, int l) -> int64_t {
        const int nl = (int)h.amgA.size();
        if (l < nl) return (int64_t)h.amgA[l].rp.size() - 1;
        return (l == nl && h.amg_nc > 0) ? h.amg_nc : 0;
    };
    std::vector<std::vector<int64_t>> off(L + 1, std::vector<int64_t>(nsub + 1, 0));
    G.nspace.assign(L, 0);
    G.voff.assign(L + 1, 0);
    for (int l = 0; l < L; ++l) {
        for (int i = 0; i < nsub; ++i) off[l][i + 1] = off[l][i] + rows_at(s->hs[i], l);
        G.nspace[l] = off[l][nsub];
        G.voff[l + 1] = G.voff[l] + G.nspace[l];
    }
    G.vtotal = G.voff[L];
    if (L == 0 || G.nspace[0] != s->nloc) return s->fail(S2L_ERR_BADARG, "the AMG first levels must span the local space");
    G.Arp.assign(L, nullptr), G.Rrp.assign(L, nullptr), G.Prp.assign(L, nullptr);
    G.Aci.assign(L, nullptr), G.Rci.assign(L, nullptr), G.Pci.assign(L, nullptr);
    G.Av.assign(L, nullptr), G.Rv.assign(L, nullptr), G.Pv.assign(L, nullptr);
    G.fsched.assign(L, nullptr), G.bsched.assign(L, nullptr), G.fsub.assign(L, nullptr), G.bsub.assign(L, nullptr);
    G.fwf.assign(L, nullptr), G.bwf.assign(L, nullptr);
    G.soff.assign(L, nullptr), G.sn.assign(L, nullptr), G.smax.assign(L, 0), G.lanes.assign(L, 32);
    G.nsmooth.assign(L, 0), G.ncoarse.assign(L, 0);
    G.c_off.assign(L, nullptr), G.c_n.assign(L, nullptr), G.c_inv.assign(L, nullptr);
    std::vector<double> cinv_all;
    double bytes = 0.0;
    const double sw = (double)G.sweeps;
    for (int l = 0; l < L; ++l) {
        // concatenated A_l (rows of space l), P_l (rows of space l), R_l (rows of space l + 1)
        std::vector<int64_t> arp(1, 0), prp(1, 0), rrp(1, 0);
        std::vector<int32_t> aci, pci, rci;
        std::vector<double> av, pv, rv;
        std::vector<int32_t> fs, bs, fsub(1, 0), bsub(1, 0), coff, cn, sn;
        std::vector<int64_t> soff;
        std::vector<int64_t> fwf(1, 0), bwf(1, 0), cinvoff;
        for (int i = 0; i < nsub; ++i) {
            const HostSub& h = s->hs[i];
            const int nlv = (int)h.amgA.size();
            const int64_t o = off[l][i], on = l + 1 < L ? off[l + 1][i] : 0;
            if (l < nlv) {
                const HostCsr& A = h.amgA[l];
                const int n = (int)A.rp.size() - 1;
                for (int r = 0; r < n; ++r) {
                    for (int64_t e = A.rp[r]; e < A.rp[r + 1]; ++e) {
                        aci.push_back((int32_t)(o + A.ci[e]));
                        av.push_back(A.v[e]);
                    }
                    arp.push_back((int64_t)aci.size());
                }
                const bool transfer = !h.amgP[l].rp.empty();
                for (int r = 0; r < n; ++r) {
                    if (transfer)
                        for (int64_t e = h.amgP[l].rp[r]; e < h.amgP[l].rp[r + 1]; ++e) {
                            pci.push_back((int32_t)(on + h.amgP[l].ci[e]));
                            pv.push_back(h.amgP[l].v[e]);
                        }
                    prp.push_back((int64_t)pci.size());
                }
                if (transfer) {
                    const int nr = (int)h.amgR[l].rp.size() - 1;
                    for (int r = 0; r < nr; ++r) {
                        for (int64_t e = h.amgR[l].rp[r]; e < h.amgR[l].rp[r + 1]; ++e) {
                            rci.push_back((int32_t)(o + h.amgR[l].ci[e]));
                            rv.push_back(h.amgR[l].v[e]);
                        }
                        rrp.push_back((int64_t)rci.size());
                    }
                    bytes += (double)(h.amgP[l].ci.size() + h.amgR[l].ci.size()) * (4.0 + vb);
                }
                // sweeps' wavefronts (rows as level-space indices)
                for (int f = 0; f < 2; ++f) {
                    const std::vector<int32_t> wf = gs_wavefronts(A, n, f == 0);
                    int nw = 0;
                    for (int32_t x : wf) nw = std::max(nw, x + 1);
                    std::vector<int64_t> cnt(nw + 1, 0);
                    for (int32_t x : wf) ++cnt[x + 1];
                    for (int k = 0; k < nw; ++k) cnt[k + 1] += cnt[k];
                    std::vector<int32_t> ord(n);
                    std::vector<int64_t> nx(cnt.begin(), cnt.end() - 1);
                    for (int r = 0; r < n; ++r) ord[nx[wf[r]]++] = (int32_t)(o + r);
                    std::vector<int32_t>& sched = f == 0 ? fs : bs;
                    std::vector<int64_t>& wptr = f == 0 ? fwf : bwf;
                    std::vector<int32_t>& sub = f == 0 ? fsub : bsub;
                    const int64_t base = (int64_t)sched.size();
                    sched.insert(sched.end(), ord.begin(), ord.end());
                    for (int k = 0; k < nw; ++k) wptr.push_back(base + cnt[k + 1]);
                    sub.push_back((int32_t)(wptr.size() - 1));
                }
                G.nsmooth[l] += 1;
                soff.push_back(o);
                sn.push_back(n);
                G.smax[l] = std::max(G.smax[l], n);
                bytes += (double)A.ci.size() * (4.0 + vb) * (2.0 * sw + 1.0) + (double)n * vb * 6.0;
            } else {
                const int64_t n = rows_at(h, l);  // a coarsest level: no rows of A_l, P_l
                for (int64_t r = 0; r < n; ++r) {
                    arp.push_back((int64_t)aci.size());
                    prp.push_back((int64_t)pci.size());
                }
                if (l == nlv && h.amg_nc > 0) {
                    const int nc = h.amg_nc;
                    std::vector<double> Cc = h.amgC, Ci;
                    if (!dense_inverse(Cc, nc, Ci))
                        return s->fail(S2L_ERR_NUMERIC, "subdomain " + std::to_string(i) + ": singular coarsest AMG level");
                    coff.push_back((int32_t)o);
                    cn.push_back(nc);
                    cinvoff.push_back((int64_t)cinv_all.size());
                    for (int c = 0; c < nc; ++c)  // stored transposed (column by column)
                        for (int r = 0; r < nc; ++r) cinv_all.push_back(Ci[(size_t)r * nc + c]);
                    G.ncoarse[l] += 1;
                    bytes += (double)nc * nc * vb;
                }
            }
            // rows of space l + 1 that come from subdomains without a transfer at level l
            if (l + 1 < L && !(l < nlv && !h.amgP[l].rp.empty()))
                for (int64_t r = off[l + 1][i]; r < off[l + 1][i + 1]; ++r) rrp.push_back((int64_t)rci.size());
        }
        RET_IF(upload(s, &G.Arp[l], arp));
        RET_IF(upload(s, &G.Aci[l], aci));
        RET_IF(upload_vals(&G.Av[l], av));
        RET_IF(upload(s, &G.Prp[l], prp));
        RET_IF(upload(s, &G.Pci[l], pci));
        RET_IF(upload_vals(&G.Pv[l], pv));
        RET_IF(upload(s, &G.Rrp[l], rrp));
        RET_IF(upload(s, &G.Rci[l], rci));
        RET_IF(upload_vals(&G.Rv[l], rv));
        RET_IF(upload(s, &G.fsched[l], fs));
        RET_IF(upload(s, &G.bsched[l], bs));
        RET_IF(upload(s, &G.fwf[l], fwf));
        RET_IF(upload(s, &G.bwf[l], bwf));
        RET_IF(upload(s, &G.fsub[l], fsub));
        RET_IF(upload(s, &G.bsub[l], bsub));
        {
            const double mean = arp.size() > 1 && aci.size() ? (double)aci.size() / (double)(arp.size() - 1) : 0.0;
            G.lanes[l] = mean <= 10.0 ? 4 : (mean <= 20.0 ? 8 : (mean <= 40.0 ? 16 : 32));
        }
        RET_IF(upload(s, &G.soff[l], soff));
        RET_IF(upload(s, &G.sn[l], sn));
        RET_IF(upload(s, &G.c_off[l], coff));
        RET_IF(upload(s, &G.c_n[l], cn));
        RET_IF(upload(s, &G.c_inv[l], cinvoff));
    }
    RET_IF(upload_vals(&G.Cinv, cinv_all));
    std::vector<int32_t> out_idx((size_t)s->nloc, -1);
    for (int i = 0; i < nsub; ++i) {
        const DevSub& d = s->h_subs[i];
        for (int j = 0; j < d.n_owned; ++j) out_idx[(size_t)(d.loc_off + j)] = (int32_t)(d.begin + j);
    }
    RET_IF(upload(s, &G.out_idx, out_idx));
    G.cycle_bytes = bytes;
    G.on = true;
    return S2L_OK;
}

// A block runner of the serving workers gives its workspace back right after its last request
// finishes.  Calls that need the setup idle (update, refactor, destroy) wait for that, bounded, when
// no request is queued or running on the setup.
int wait_runners_gone(s2l_setup* s)
{
    if (s->pending.load() > 0) return S2L_OK;  // the caller refuses
    for (int i = 0; s->runners.load() > 0; ++i) {
        if (i > 100000) return s->fail(S2L_ERR_STATE, "a serving block runner still holds a workspace of this setup");
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    return S2L_OK;
}

}  // namespace

extern "C" {

int s2l_gpu_setup_end(s2l_setup* s)
{
    if (!s) return S2L_ERR_BADARG;
    if (s->ended) return s->fail(S2L_ERR_STATE, "setup_end called twice");
    if (!s->have_A) return s->fail(S2L_ERR_STATE, "set_matrix was not called");
    if (cudaSetDevice(s->ctx->device) != cudaSuccess) return S2L_ERR_CUDA;
    const int nsub = s->nsub;
    if (s->local_kind == 1 && s->opt_refactor)
        return s->fail(S2L_ERR_BADARG, "the option refactor needs exact local factors");
    // ---- ownership checks: contiguous ranges covering [0, n)
    {
        int64_t next = 0;
        for (int i = 0; i < nsub; ++i) {
            if (!s->hs[i].set) return s->fail(S2L_ERR_STATE, "subdomain " + std::to_string(i) + " was not added");
            if (s->hs[i].begin != next) return s->fail(S2L_ERR_BADARG, "owned ranges must be contiguous in subdomain order");
            next += s->hs[i].n_owned;
        }
        if (next != s->n) return s->fail(S2L_ERR_BADARG, "owned ranges do not cover [0, n)");
    }
    if (s->coarse != S2L_COARSE_NONE) {
        if (!s->have_coarse) return s->fail(S2L_ERR_STATE, "set_coarse was not called");
        if (s->coff[0] != 0 || s->coff[nsub] != s->n0) return s->fail(S2L_ERR_BADARG, "coarse offsets inconsistent with n0");
        for (int i = 0; i < nsub; ++i)
            if (s->coff[i + 1] - s->coff[i] != s->hs[i].m)
                return s->fail(S2L_ERR_BADARG, "coarse offsets do not match the basis sizes");
    }
    const bool boolean = s->pou == S2L_POU_BOOLEAN;
    s->need_copies = !(boolean && s->one_level == S2L_ONE_LEVEL_RAS);

    // ---- global matrix
    {
        std::vector<int32_t> rp(s->n + 1);
        for (int64_t r = 0; r <= s->n; ++r) rp[r] = (int32_t)s->A.rp[r];
        s->nnz = s->A.rp[s->n];
        RET_IF(upload(s, &s->d_rp, rp));
        RET_IF(upload(s, &s->d_ci, s->A.ci));
        RET_IF(upload(s, &s->d_av, s->A.v));
        std::vector<double> rowsum(s->n, 0.0);  // A 1, summed in row order as a CSR product does
        for (int64_t r = 0; r < s->n; ++r)
            for (int64_t e = s->A.rp[r]; e < s->A.rp[r + 1]; ++e) rowsum[r] += s->A.v[e];
        RET_IF(upload(s, &s->d_rowsum, rowsum));
        const double avg = (double)s->nnz / (double)s->n;
        // lanes per row for about four entries per lane, between 2 and 32 (each lane with four
        // entries in flight: on a 7-point matrix 2 lanes per row beat the chunk mode, a warp per 32
        // rows with coalesced entry loads, spmv_tpr 1, by 1.3x for one column and 1.5x for four)
        int tpr = 2;
        while (tpr < 32 && tpr * 4 < avg) tpr *= 2;
        s->tpr = s->opt_tpr ? s->opt_tpr : tpr;
    }

    // ---- per-subdomain factor split, sweep layouts and index maps
    s->h_subs.resize(nsub);
    const size_t rs = s->real == S2L_REAL_F32 ? 4 : 8;
    // pass 1: full U of every subdomain and its tail split
    std::vector<HostCsr> Us(nsub);
    std::vector<int> Ts(nsub);
    s2l_tail_model tm;
    tm.force_rows = s->opt_tail_rows;
    tm.tail_min = s->opt_tail_min;
    tm.tail_max = s->opt_tail_max;
    tm.hop_s = s->opt_hop_us * 1e-6;
    tm.bw = s->opt_bw_gbs * 1e9;
    tm.nsub = nsub;
    tm.real_bytes = (double)rs;
    tm.chain = s->opt_chain;
    // per subdomain and independent of the others: on several host threads
    std::vector<char> ldlt_bad(nsub, 0);
    parallel_for(nsub, [&](int i) {
        HostSub& h = s->hs[i];
        const int nl = h.n_local();
        if (h.amg) {  // no factors: the whole local space is "sparse part" without a tail
            Ts[i] = nl;
            return;
        }
        if (h.kind == S2L_FACTOR_LU) {
            Us[i] = std::move(h.U);
        } else {
            Us[i] = transpose_lower(h.L, nl, nullptr);
            if (h.kind == S2L_FACTOR_LDLT) {
                bool missing = false;
                for (int r = 0; r < nl; ++r) {
                    bool f = false;
                    for (int64_t e = Us[i].rp[r]; e < Us[i].rp[r + 1]; ++e) {
                        if (Us[i].ci[e] == r) {
                            Us[i].v[e] = h.d[r];
                            f = true;
                        } else {
                            Us[i].v[e] *= h.d[r];
                        }
                    }
                    missing = missing || !f;
                }
                if (missing) {
                    ldlt_bad[i] = 1;
                    return;
                }
            }
        }
        Ts[i] = choose_tail(h.L, Us[i], nl, tm);
    });
    for (int i = 0; i < nsub; ++i)
        if (ldlt_bad[i]) return s->fail(S2L_ERR_BADARG, "LDLT: L must store its unit diagonal");
    s->sweep_group = s->opt_group ? s->opt_group : 16;  // widest lane group of a sweep row
    const int nw = S2L_BS_SWEEP / 32;
    // pass 2: layouts
    int64_t loc = 0;
    std::vector<int32_t> gin, pin, gout, l2g, u2l;
    std::vector<double> Dall;
    std::vector<int32_t> sw_col[2], sw_tslot[2];
    std::vector<double> sw_val[2], sw_dinv[2];
    std::vector<uint32_t> sw_thdr[2];
    std::vector<int64_t> sw_wtask[2], sw_wslot[2], sw_went[2];
    std::vector<int32_t> sw_bfirst[2], sw_bslot[2];
    std::vector<int64_t> sw_boff[2] = {{0}, {0}}, sw_bioff[2] = {{0}, {0}};
    std::vector<double> sw_binv[2];
    std::vector<int32_t> tr_sub, tr_i, lts_col, us_sub, us_r, ust_col, uu;
    std::vector<int64_t> lts_ptr(1, 0), ust_ptr(1, 0);
    std::vector<double> lts_val, ust_val;
    std::vector<std::vector<double>> Ltt(nsub), Utt(nsub);
    std::vector<int64_t> d_off(nsub + 1, 0);
    s->tr_first_h.assign(nsub + 1, 0);
    s->us_first_h.assign(nsub + 1, 0);
    s->uu_first_h.assign(nsub + 1, 0);
    double bytes = 0.0;
    int max_T = 0, max_nl = 0;
    int64_t sparse_nnz = 0;
    // refactorization plan (host side; see RefactorArgs)
    const bool rfon = s->opt_refactor != 0;
    std::vector<int64_t> rf_fbase(1, 0), rf_fcp, rf_frp(1, 0), rf_lvoff(1, 0), rf_fill_src, rf_fill_dst, rf_lts, rf_ust;
    std::vector<int32_t> rf_fri, rf_fdg, rf_frpos, rf_frk, rf_lvfirst, rf_lvcol, rf_tcsub, rf_tccol;
    std::vector<uint8_t> rf_fllt;
    std::vector<int32_t> rf_swsrc[2], rf_swdsrc[2];
    std::vector<int64_t> rf_wsrc[2], rf_beoff[2] = {{0}, {0}}, rf_bepos[2], rf_becp[2] = {{0}, {0}}, rf_bcpos[2];
    std::vector<uint8_t> rf_berow[2], rf_bcb[2];
    if (rfon) {
        s->rf.sz.assign(nsub, 0);
        s->rf.llt.assign(nsub, 0);
    }
    // the sweep layouts of both factors and, with the refactorization plan, the combined pattern and
    // the position of every factor entry in it: per subdomain, on several host threads
    struct PreLayout {
        Sweep sl, su;
        FPat P;
        std::vector<int32_t> mposL, mposU;
        std::string err;
        int code = S2L_OK;
    };
    std::vector<PreLayout> pre(nsub);
    s->sweep_group = s->opt_group ? s->opt_group : 16;
    parallel_for(nsub, [&](int i) {
        HostSub& h = s->hs[i];
        if (h.amg) return;
        PreLayout& q = pre[i];
        const HostCsr& U = Us[i];
        const int nl = h.n_local();
        const int T = Ts[i];
        const bool unitL = h.kind != S2L_FACTOR_LLT;
        const bool llt = h.kind == S2L_FACTOR_LLT;
        if (rfon) {
            if (!make_fpattern(h.L, U, nl, llt, q.P)) {
                q.code = S2L_ERR_BADARG;
                q.err = "a factor has no diagonal entry";
                return;
            }
            q.mposL.assign(h.L.ci.size(), -1);
            for (int r = 0; r < nl; ++r)
                for (int64_t e = h.L.rp[r]; e < h.L.rp[r + 1]; ++e) {
                    const int c = h.L.ci[e];
                    if (llt ? c <= r : c < r) q.mposL[e] = q.P.find(r, c);
                }
            q.mposU.assign(U.ci.size(), -1);
            for (int r = 0; r < nl; ++r)
                for (int64_t e = U.rp[r]; e < U.rp[r + 1]; ++e) {
                    const int c = U.ci[e];
                    q.mposU[e] = llt ? q.P.find(c, r) : q.P.find(r, c);
                }
        }
        build_sweep(h.L, T, true, unitL, nw, s->sweep_group, s->opt_epl, s->opt_chain, q.sl, q.err, rfon ? &q.mposL : nullptr);
        if (q.err.empty())
            build_sweep(U, T, false, false, nw, s->sweep_group, s->opt_epl, s->opt_chain, q.su, q.err, rfon ? &q.mposU : nullptr);
        if (!q.err.empty()) q.code = S2L_ERR_NUMERIC;
    });
    for (int i = 0; i < nsub; ++i) {
        HostSub& h = s->hs[i];
        const HostCsr& U = Us[i];
        const int nl = h.n_local();
        max_nl = std::max(max_nl, nl);
        if (pre[i].code != S2L_OK) return s->fail(pre[i].code, "subdomain " + std::to_string(i) + ": " + pre[i].err);
        if (h.amg) {  // AMG local solver: the local space in natural order, no sweeps or tails
            s->tr_first_h[i] = (int)tr_sub.size();
            s->us_first_h[i] = (int)us_sub.size();
            s->uu_first_h[i] = (int)uu.size();
            d_off[i + 1] = d_off[i];
            DevSub d{};
            d.begin = h.begin;
            d.loc_off = loc;
            d.n_owned = h.n_owned;
            d.n_local = nl;
            d.T = nl;
            d.tr_first = s->tr_first_h[i];
            d.us_first = s->us_first_h[i];
            d.d_off = d_off[i];
            d.m = h.m;
            d.v_rows = boolean ? h.n_owned : nl;
            d.c_off = s->coarse != S2L_COARSE_NONE ? s->coff[i] : 0;
            s->h_subs[i] = d;
            for (int j = 0; j < nl; ++j) {
                const int64_t g = j < h.n_owned ? h.begin + j : h.ghosts[j - h.n_owned];
                l2g.push_back((int32_t)g);
            }
            for (int k = 0; k < nl; ++k) {
                gin.push_back(l2g[loc + k]);
                pin.push_back(k);
                gout.push_back(k);
            }
            Dall.insert(Dall.end(), h.D.begin(), h.D.end());
            loc += nl;
            continue;
        }
        const bool unitL = h.kind != S2L_FACTOR_LLT;
        const int T = Ts[i];
        const int sz = nl - T;
        max_T = std::max(max_T, T);
        Sweep& sl = pre[i].sl;
        Sweep& su = pre[i].su;
        const FPat& P = pre[i].P;
        const std::vector<int32_t>& mposL = pre[i].mposL;
        const std::vector<int32_t>& mposU = pre[i].mposU;
        const bool llt = h.kind == S2L_FACTOR_LLT;
        const int64_t fb = rf_fbase.back();
        if (rfon) {
            // the column kernels address a column's tail rows through 16-bit offsets and keep one
            // row map of the tail per warp in shared memory
            for (int c = 0; c < nl; ++c) {
                if (P.cp[c + 1] - P.cp[c] >= 65535)
                    return s->fail(S2L_ERR_BADARG, "refactor: a factor column has 65535 or more entries");
                s->rf.maxcol = std::max(s->rf.maxcol, (int)(P.cp[c + 1] - P.cp[c]));
            }
            if (nl > 100000) return s->fail(S2L_ERR_BADARG, "refactor: a subdomain of more than 100000 rows");
            bool found = true;
            for (int r = 0; r < nl; ++r) {
                for (int64_t e = U.rp[r]; e < U.rp[r + 1]; ++e) found = found && mposU[e] >= 0;
                for (int64_t e = h.L.rp[r]; e < h.L.rp[r + 1]; ++e)
                    if (llt ? h.L.ci[e] <= r : h.L.ci[e] < r) found = found && mposL[e] >= 0;
            }
            if (!found)  // every factor entry must have its place in the combined pattern
                return s->fail(S2L_ERR_BADARG, "subdomain " + std::to_string(i) + ": inconsistent factor patterns");
            s->rf.sz[i] = sz;
            s->rf.llt[i] = llt;
        }
        if (rfon) {
            // pattern, per-column data, L L^T row lists
            for (int c = 0; c < nl; ++c) {
                rf_fcp.push_back(fb + P.cp[c]);
                rf_fllt.push_back(llt);
                if (llt)
                    for (int64_t e = h.L.rp[c]; e < h.L.rp[c + 1]; ++e) {
                        const int k = h.L.ci[e];
                        if (k >= c) break;
                        rf_frpos.push_back(P.find(c, k));
                        rf_frk.push_back(k);
                    }
                rf_frp.push_back((int64_t)rf_frpos.size());
            }
            rf_fri.insert(rf_fri.end(), P.ri.begin(), P.ri.end());
            rf_fdg.insert(rf_fdg.end(), P.dg.begin(), P.dg.end());
            // fill map: A(l2g(a), l2g(b)) -> F(ipin(a), pout(b)) (lower triangle only for L L^T)
            std::vector<int32_t> ipin(nl);
            for (int p = 0; p < nl; ++p) ipin[h.pin[p]] = p;
            for (int a = 0; a < nl; ++a) {
                const int64_t g = a < h.n_owned ? h.begin + a : h.ghosts[a - h.n_owned];
                const int p = ipin[a];
                for (int64_t e = s->A.rp[g]; e < s->A.rp[g + 1]; ++e) {
                    const int64_t cg = s->A.ci[e];
                    int b = -1;
                    if (cg >= h.begin && cg < h.begin + h.n_owned) {
                        b = (int)(cg - h.begin);
                    } else {
                        const auto it = std::lower_bound(h.ghosts.begin(), h.ghosts.end(), cg);
                        if (it != h.ghosts.end() && *it == cg) b = h.n_owned + (int)(it - h.ghosts.begin());
                    }
                    if (b < 0) continue;
                    const int q = h.pout[b];
                    if (llt && p < q) continue;
                    const int32_t pos = P.find(p, q);
                    if (pos < 0)
                        return s->fail(S2L_ERR_BADARG, "subdomain " + std::to_string(i) +
                                                           ": a matrix entry lies outside the factor pattern (refactor)");
                    rf_fill_src.push_back(e);
                    rf_fill_dst.push_back(fb + pos);
                }
            }
            // dependency levels of the sparse columns
            std::vector<int32_t> lev(T, 0);
            int nlev = 0;
            for (int j = 0; j < T; ++j) {
                int lv = 0;
                if (llt) {
                    for (int64_t e = h.L.rp[j]; e < h.L.rp[j + 1]; ++e)
                        if (h.L.ci[e] < j) lv = std::max(lv, lev[h.L.ci[e]] + 1);
                } else {
                    for (int64_t q = P.cp[j]; q < P.cp[j] + P.dg[j]; ++q) lv = std::max(lv, lev[P.ri[q]] + 1);
                }
                lev[j] = lv;
                nlev = std::max(nlev, lv + 1);
            }
            rf_lvfirst.push_back((int32_t)(rf_lvoff.size() - 1));
            {
                std::vector<int64_t> cnt(nlev + 1, 0);
                for (int j = 0; j < T; ++j) ++cnt[lev[j] + 1];
                for (int l = 0; l < nlev; ++l) cnt[l + 1] += cnt[l];
                std::vector<int32_t> cols(T);
                std::vector<int64_t> nx(cnt.begin(), cnt.end() - 1);
                for (int j = 0; j < T; ++j) cols[nx[lev[j]]++] = j;
                const int64_t base = (int64_t)rf_lvcol.size();
                rf_lvcol.insert(rf_lvcol.end(), cols.begin(), cols.end());
                for (int l = 0; l < nlev; ++l) rf_lvoff.push_back(base + cnt[l + 1]);
            }
            for (int j = T; j < nl; ++j) {
                rf_tcsub.push_back(i);
                rf_tccol.push_back(j);
            }
            rf_fbase.push_back(fb + (int64_t)P.ri.size());
        }
        s->st_levels_max = std::max<int64_t>(s->st_levels_max, std::max(sl.nlev, su.nlev));
        s->st_levels_sum += sl.nlev + su.nlev;
        for (int f = 0; f < 2; ++f) {
            const Sweep& q = f == 0 ? sl : su;
            const int64_t e0 = sw_col[f].size(), t0 = sw_thdr[f].size(), s0 = sw_tslot[f].size();
            for (int w = 0; w < nw; ++w) {
                sw_wtask[f].push_back(t0 + q.wtask[w]);
                sw_wslot[f].push_back(s0 + q.wslot[w]);
                sw_went[f].push_back(e0 + q.went[w]);
            }
            sw_col[f].insert(sw_col[f].end(), q.col.begin(), q.col.end());
            sw_val[f].insert(sw_val[f].end(), q.val.begin(), q.val.end());
            sw_thdr[f].insert(sw_thdr[f].end(), q.thdr.begin(), q.thdr.end());
            sw_tslot[f].insert(sw_tslot[f].end(), q.tslot.begin(), q.tslot.end());
            sw_dinv[f].insert(sw_dinv[f].end(), q.dinv.begin(), q.dinv.end());
            sw_dinv[f].resize(sw_dinv[f].size() + sz, 1.0);
            if (rfon) {
                rf_swsrc[f].insert(rf_swsrc[f].end(), q.src.begin(), q.src.end());
                rf_swdsrc[f].insert(rf_swdsrc[f].end(), q.dsrc.begin(), q.dsrc.end());
                rf_swdsrc[f].resize(rf_swdsrc[f].size() + sz, -1);
                for (int32_t w : q.blk_wsrc) rf_wsrc[f].push_back(w >= 0 ? fb + w : -1);
                const int64_t eb = (int64_t)rf_bepos[f].size(), cb = (int64_t)rf_bcb[f].size();
                for (size_t b = 1; b < q.be_off.size(); ++b) rf_beoff[f].push_back(eb + q.be_off[b]);
                for (int64_t x : q.be_pos) rf_bepos[f].push_back(e0 + x);
                rf_berow[f].insert(rf_berow[f].end(), q.be_row.begin(), q.be_row.end());
                for (size_t x = 1; x < q.be_cp.size(); ++x) rf_becp[f].push_back(cb + q.be_cp[x]);
                rf_bcb[f].insert(rf_bcb[f].end(), q.bc_b.begin(), q.bc_b.end());
                for (int32_t x : q.bc_pos) rf_bcpos[f].push_back(fb + x);
            }
            const int64_t real = (int64_t)q.col.size() - q.pad;
            sparse_nnz += real;
            s->st_pad += q.pad;
            s->st_tasks += q.ntask;
            // algorithmic bytes: the real entries, 1/diag and the task slots and headers
            bytes += (double)real * (rs + 4) + (double)T * (rs + 4) + (double)q.ntask * 4;
            // chain blocks (slots stay subdomain-relative)
            sw_bfirst[f].push_back((int32_t)(sw_boff[f].size() - 1));
            const int64_t so = (int64_t)sw_bslot[f].size(), io = (int64_t)sw_binv[f].size();
            sw_bslot[f].insert(sw_bslot[f].end(), q.blk_slot.begin(), q.blk_slot.end());
            sw_binv[f].insert(sw_binv[f].end(), q.blk_inv.begin(), q.blk_inv.end());
            for (size_t b = 1; b < q.blk_off.size(); ++b) {
                sw_boff[f].push_back(so + q.blk_off[b]);
                sw_bioff[f].push_back(io + q.blk_ioff[b]);
            }
            bytes += (double)q.blk_inv.size() * rs + (double)q.blk_slot.size() * 4 + (double)(q.blk_off.size() - 1) * 16;
        }
        // backward slot -> forward slot
        for (int u = 0; u < T; ++u) u2l.push_back(sl.pos[su.order[u]]);
        u2l.resize(u2l.size() + sz, 0);
        // L coupling of the tail rows (columns as forward slots) and the dense lower tail
        s->tr_first_h[i] = (int)tr_sub.size();
        if (sz > 0) {
            Ltt[i].assign((size_t)sz * sz, 0.0);
            for (int k = T; k < nl; ++k) {
                tr_sub.push_back(i);
                tr_i.push_back(k - T);
                for (int64_t e = h.L.rp[k]; e < h.L.rp[k + 1]; ++e) {
                    const int c = h.L.ci[e];
                    if (c < T) {
                        lts_col.push_back(sl.pos[c]);
                        lts_val.push_back(h.L.v[e]);
                        if (rfon) rf_lts.push_back(fb + P.find(k, c));
                    } else if (c < k) {
                        Ltt[i][(size_t)(k - T) * sz + (c - T)] = h.L.v[e];
                    } else if (c == k) {
                        Ltt[i][(size_t)(k - T) * sz + (c - T)] = unitL ? 1.0 : h.L.v[e];
                    }
                }
                if (unitL) Ltt[i][(size_t)(k - T) * sz + (k - T)] = 1.0;
                lts_ptr.push_back((int64_t)lts_col.size());
            }
            Utt[i].assign((size_t)sz * sz, 0.0);
            for (int k = T; k < nl; ++k)
                for (int64_t e = U.rp[k]; e < U.rp[k + 1]; ++e) {
                    const int c = U.ci[e];
                    if (c >= k) Utt[i][(size_t)(k - T) * sz + (c - T)] = U.v[e];
                }
            for (int k = 0; k < sz; ++k)
                if (Utt[i][(size_t)k * sz + k] == 0.0 || Ltt[i][(size_t)k * sz + k] == 0.0)
                    return s->fail(S2L_ERR_NUMERIC, "subdomain " + std::to_string(i) + ": zero pivot in the dense tail");
        }
        // U coupling of the sparse rows: the target is the row's forward slot (ybuf keeps forward order).
        // The rows are stored longest first and grouped into units of one warp: a unit holds rows of
        // about the same length, each taken by the lanes its length needs (coupling_lanes)
        s->us_first_h[i] = (int)us_sub.size();
        s->uu_first_h[i] = (int)uu.size();
        if (sz > 0) {
            std::vector<std::pair<int, int>> rows;  // (tail entries, row)
            for (int r = 0; r < T; ++r) {
                int cnt = 0;
                for (int64_t e = U.rp[r]; e < U.rp[r + 1]; ++e) cnt += U.ci[e] >= T;
                if (cnt) rows.emplace_back(cnt, r);
            }
            std::stable_sort(rows.begin(), rows.end(), [](const std::pair<int, int>& x, const std::pair<int, int>& y) {
                return x.first > y.first;
            });
            const int q0 = (int)us_sub.size();
            for (const auto& pr : rows) {
                const int r = pr.second;
                for (int64_t e = U.rp[r]; e < U.rp[r + 1]; ++e)
                    if (U.ci[e] >= T) {
                        ust_col.push_back((int32_t)(loc + U.ci[e]));  // local-space index of the tail row
                        ust_val.push_back(U.v[e]);
                        if (rfon) rf_ust.push_back(fb + (llt ? P.find(U.ci[e], r) : P.find(r, U.ci[e])));
                    }
                us_sub.push_back(i);
                us_r.push_back(sl.pos[r]);
                ust_ptr.push_back((int64_t)ust_col.size());
            }
            for (size_t k = 0; k < rows.size();) {
                uu.push_back(q0 + (int)k);
                k += std::min(rows.size() - k, (size_t)(32 / coupling_lanes(rows[k].first)));
            }
        }
        d_off[i + 1] = d_off[i] + (int64_t)sz * sz;
        DevSub d{};
        d.begin = h.begin;
        d.loc_off = loc;
        d.n_owned = h.n_owned;
        d.n_local = nl;
        d.T = T;
        d.tr_first = s->tr_first_h[i];
        d.us_first = s->us_first_h[i];
        d.d_off = d_off[i];
        d.m = h.m;
        d.v_rows = boolean ? h.n_owned : nl;
        d.c_off = s->coarse != S2L_COARSE_NONE ? s->coff[i] : 0;
        s->h_subs[i] = d;
        for (int j = 0; j < nl; ++j) {
            const int64_t g = j < h.n_owned ? h.begin + j : h.ghosts[j - h.n_owned];
            l2g.push_back((int32_t)g);
        }
        // forward gather per slot (< T) or tail row (>= T); backward output position per local j
        for (int k = 0; k < nl; ++k) {
            const int prow = k < T ? sl.order[k] : k;
            gin.push_back(l2g[loc + h.pin[prow]]);
            pin.push_back(h.pin[prow]);
        }
        for (int j = 0; j < nl; ++j) {
            const int q = h.pout[j];
            gout.push_back(q < T ? su.pos[q] : q);
        }
        Dall.insert(Dall.end(), h.D.begin(), h.D.end());
        bytes += (double)sz * (sz + 1) * rs;
        loc += nl;
        h.L = HostCsr();
        Us[i] = HostCsr();
    }
    s->tr_first_h[nsub] = (int)tr_sub.size();
    s->us_first_h[nsub] = (int)us_sub.size();
    s->uu_first_h[nsub] = (int)uu.size();
    uu.push_back((int32_t)us_sub.size());  // the end of the last unit
    s->nloc = loc;
    s->st_sparse_nnz = sparse_nnz;
    s->st_coupling_nnz = (int64_t)lts_col.size() + (int64_t)ust_col.size();
    s->st_dense_entries = d_off[nsub];
    s->st_tail_rows = (int64_t)tr_sub.size();
    bytes += (double)s->st_coupling_nnz * (rs + 4) + (double)(tr_sub.size() + us_sub.size()) * (8 + 8 + rs);
    for (int f = 0; f < 2; ++f) {
        sw_wtask[f].push_back((int64_t)sw_thdr[f].size());
        sw_wslot[f].push_back((int64_t)sw_tslot[f].size());
        sw_went[f].push_back((int64_t)sw_col[f].size());
        RET_IF(upload(s, &s->d_wtask[f], sw_wtask[f]));
        RET_IF(upload(s, &s->d_wslot[f], sw_wslot[f]));
        RET_IF(upload(s, &s->d_went[f], sw_went[f]));
        RET_IF(upload(s, &s->d_thdr[f], sw_thdr[f]));
        RET_IF(upload(s, &s->d_tslot[f], sw_tslot[f]));
        sw_thdr[f] = {};
        sw_tslot[f] = {};
        sw_bfirst[f].push_back((int32_t)(sw_boff[f].size() - 1));
        RET_IF(upload(s, &s->d_bfirst[f], sw_bfirst[f]));
        RET_IF(upload(s, &s->d_boff[f], sw_boff[f]));
        RET_IF(upload(s, &s->d_bioff[f], sw_bioff[f]));
        RET_IF(upload(s, &s->d_bslot[f], sw_bslot[f]));
        if (s->real == S2L_REAL_F32) RET_IF(upload_real<float>(s, &s->d_binv[f], sw_binv[f]));
        else RET_IF(upload_real<double>(s, &s->d_binv[f], sw_binv[f]));
        s->st_blocks += (int64_t)sw_boff[f].size() - 1;
        RET_IF(upload(s, &s->d_col[f], sw_col[f]));
        if (s->real == S2L_REAL_F32) {
            RET_IF(upload_real<float>(s, &s->d_val[f], sw_val[f]));
            RET_IF(upload_real<float>(s, &s->d_dinv[f], sw_dinv[f]));
        } else {
            RET_IF(upload_real<double>(s, &s->d_val[f], sw_val[f]));
            RET_IF(upload_real<double>(s, &s->d_dinv[f], sw_dinv[f]));
        }
        sw_col[f] = {};
        sw_val[f] = {};
    }
    RET_IF(upload(s, &s->d_u2l, u2l));
    RET_IF(upload(s, &s->d_tr_sub, tr_sub));
    RET_IF(upload(s, &s->d_tr_i, tr_i));
    RET_IF(upload(s, &s->d_lts_ptr, lts_ptr));
    RET_IF(upload(s, &s->d_lts_col, lts_col));
    RET_IF(upload(s, &s->d_us_sub, us_sub));
    RET_IF(upload(s, &s->d_us_r, us_r));
    RET_IF(upload(s, &s->d_ust_ptr, ust_ptr));
    RET_IF(upload(s, &s->d_ust_col, ust_col));
    RET_IF(upload(s, &s->d_uu, uu));
    if (s->real == S2L_REAL_F32) {
        RET_IF(upload_real<float>(s, &s->d_lts_val, lts_val));
        RET_IF(upload_real<float>(s, &s->d_ust_val, ust_val));
    } else {
        RET_IF(upload_real<double>(s, &s->d_lts_val, lts_val));
        RET_IF(upload_real<double>(s, &s->d_ust_val, ust_val));
    }
    // ---- dense tail inverses on the device (FP64 triangular solves with the identity)
    RET_IF(dev_alloc(s, &s->d_linv, (size_t)std::max<int64_t>(d_off[nsub], 1) * rs));
    RET_IF(dev_alloc(s, &s->d_uinv, (size_t)std::max<int64_t>(d_off[nsub], 1) * rs));
    RET_IF(invert_tails(s, Ltt, Utt, d_off));
    // input gather and owned output of one local solve (per right-hand side)
    double vec = 0.0;
    for (int i = 0; i < nsub; ++i) {
        const HostSub& h = s->hs[i];
        vec += (double)h.n_local() * (4 + 8) + (double)h.n_owned * (4 + 8 + 8);
    }
    s->solve_bytes = bytes + vec;
    s->solve_vec_bytes = vec;
    RET_IF(upload(s, &s->d_gin, gin));
    RET_IF(upload(s, &s->d_pin, pin));
    RET_IF(upload(s, &s->d_gout, gout));
    RET_IF(upload(s, &s->d_l2g, l2g));
    RET_IF(upload(s, &s->d_D, Dall));

    // ---- copies of every global row in the local space (owner first, then ghosts by subdomain)
    if (s->need_copies) {
        std::vector<int64_t> cnt(s->n + 1, 0);
        for (int64_t p = 0; p < loc; ++p) ++cnt[l2g[p] + 1];
        for (int64_t g = 0; g < s->n; ++g) cnt[g + 1] += cnt[g];
        std::vector<int32_t> pos(loc);
        std::vector<double> w(loc);
        std::vector<int64_t> nx(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < nsub; ++i) {  // owned copies first
            const DevSub& d = s->h_subs[i];
            for (int j = 0; j < d.n_owned; ++j) {
                const int64_t q = nx[d.begin + j]++;
                pos[q] = (int32_t)(d.loc_off + j);
                w[q] = Dall[d.loc_off + j];
            }
        }
        for (int i = 0; i < nsub; ++i) {
            const DevSub& d = s->h_subs[i];
            for (int j = d.n_owned; j < d.n_local; ++j) {
                const int64_t g = l2g[d.loc_off + j];
                const int64_t q = nx[g]++;
                pos[q] = (int32_t)(d.loc_off + j);
                w[q] = Dall[d.loc_off + j];
            }
        }
        RET_IF(upload(s, &s->d_cp_ptr, cnt));
        RET_IF(upload(s, &s->d_cp_pos, pos));
        RET_IF(upload(s, &s->d_cp_w, w));
    }

    // ---- coarse basis (row-major, owned rows for the boolean PoU) and E^-1
    if (s->coarse != S2L_COARSE_NONE && s->n0 > 0) {
        std::vector<double> Vr;
        std::vector<int32_t> tsub, trow0, tnrow, tfirst(nsub + 1, 0);
        int64_t voff = 0;
        int mmax = 0;
        for (int i = 0; i < nsub; ++i) {
            HostSub& h = s->hs[i];
            DevSub& d = s->h_subs[i];
            const int nl = h.n_local();
            d.v_off = voff;
            mmax = std::max(mmax, h.m);
            for (int l = 0; l < d.v_rows; ++l)
                for (int c = 0; c < h.m; ++c) Vr.push_back(h.V[(size_t)c * nl + l]);
            voff += (int64_t)d.v_rows * h.m;
            tfirst[i] = (int32_t)tsub.size();
            if (h.m > 0)
                for (int r0 = 0; r0 < d.v_rows; r0 += S2L_TILE_ROWS) {
                    tsub.push_back(i);
                    trow0.push_back(r0);
                    tnrow.push_back(std::min(S2L_TILE_ROWS, d.v_rows - r0));
                }
        }
        tfirst[nsub] = (int32_t)tsub.size();
        // subdomains with m = 0 contribute no tile; prolong must still zero their rows: add zero tiles
        for (int i = 0; i < nsub; ++i) {
            if (s->hs[i].m > 0) continue;
            for (int r0 = 0; r0 < s->h_subs[i].v_rows; r0 += S2L_TILE_ROWS) {
                tsub.push_back(i);
                trow0.push_back(r0);
                tnrow.push_back(std::min(S2L_TILE_ROWS, s->h_subs[i].v_rows - r0));
            }
        }
        s->ntiles = (int)tsub.size();
        s->mmax = std::max(mmax, 1);
        RET_IF(upload(s, &s->d_V, Vr));
        RET_IF(upload(s, &s->d_t_sub, tsub));
        RET_IF(upload(s, &s->d_t_row0, trow0));
        RET_IF(upload(s, &s->d_t_nrow, tnrow));
        RET_IF(upload(s, &s->d_t_first, tfirst));
        std::vector<double> Ecopy = s->E, Einv;
        if (!dense_inverse(Ecopy, (int)s->n0, Einv)) return s->fail(S2L_ERR_NUMERIC, "coarse matrix E is singular");
        RET_IF(upload(s, &s->d_Einv, Einv));
    }
    RET_IF(upload(s, &s->d_subs, s->h_subs));
    if (s->local_kind == 1) {
        RET_IF(amg_build(s));
        s->solve_bytes = s->amgd.cycle_bytes + s->solve_vec_bytes;
    }
    // refactorization plan and work buffers (after the coarse tiles: the refresh of E uses them)
    if (rfon) {
        auto& R = s->rf;
        const size_t before = s->bytes;
        rf_fcp.push_back(rf_fbase.back());
        rf_lvfirst.push_back((int32_t)(rf_lvoff.size() - 1));
        R.nF = rf_fbase.back();
        R.nfill = (int64_t)rf_fill_src.size();
        R.ntc = (int64_t)rf_tcsub.size();
        R.nlts = (int64_t)rf_lts.size();
        R.nust = (int64_t)rf_ust.size();
        R.d_off = d_off;
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.F), (size_t)std::max<int64_t>(R.nF, 1) * sizeof(double)));
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.S), (size_t)std::max<int64_t>(d_off[nsub], 1) * sizeof(double)));
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.stage), (size_t)std::max<int64_t>(s->nnz, 1) * sizeof(double)));
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.err), sizeof(int)));
        {
            // clusters of 4 or 2 CTAs per subdomain when they fit the SMs at once, else one
            int sms = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->ctx->device) != cudaSuccess || sms <= 0)
                sms = 148;
            R.cs = nsub * 4 <= sms ? 4 : (nsub * 2 <= sms ? 2 : 1);
            int smax = 1;
            for (int sz : R.sz) smax = std::max(smax, sz);
            const size_t warps = (size_t)R.cs * refactor_sparse_warps(smax);
            RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.part), (size_t)nsub * warps * R.maxcol * sizeof(double)));
        }
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.info), (size_t)(nsub + 2) * sizeof(int)));
        RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.rowsum), (size_t)s->n * sizeof(double)));
        {
            auto dbl = [&](double** p, size_t count) {
                return dev_alloc(s, reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(double));
            };
            const int64_t n0 = std::max<int64_t>(s->n0, 1);
            RET_IF(dbl(&R.E, (size_t)n0 * n0));
            RET_IF(dbl(&R.Einv, (size_t)n0 * n0));
            if (s->coarse != S2L_COARSE_NONE && s->n0 > 0 && s->pou == S2L_POU_BOOLEAN) {
                // per row: the subdomains owning its columns (slots of m_i values in Z); per pair
                // (owner of the row, owner of a column): the rows and their slots
                std::vector<int32_t> owner((size_t)s->n), rs_sub, pj, pi, prl;
                std::vector<int64_t> rs_ptr(1, 0), rs_zoff, pptr;
                for (int i = 0; i < nsub; ++i)
                    for (int r = 0; r < s->hs[i].n_owned; ++r) owner[(size_t)(s->hs[i].begin + r)] = i;
                std::vector<std::vector<std::pair<int32_t, int64_t>>> rows_of;  // per pair
                std::vector<std::vector<int32_t>> pair_of(nsub);                // pair id by (j, i)
                std::vector<int32_t> subs_in_row;
                int64_t z = 0;
                for (int64_t r = 0; r < s->n; ++r) {
                    subs_in_row.clear();
                    for (int64_t e = s->A.rp[r]; e < s->A.rp[r + 1]; ++e) {
                        const int32_t i = owner[(size_t)s->A.ci[e]];
                        if (std::find(subs_in_row.begin(), subs_in_row.end(), i) == subs_in_row.end())
                            subs_in_row.push_back(i);
                    }
                    std::sort(subs_in_row.begin(), subs_in_row.end());
                    const int32_t j = owner[(size_t)r];
                    for (int32_t i : subs_in_row) {
                        rs_sub.push_back(i);
                        rs_zoff.push_back(z);
                        if (pair_of[j].empty()) pair_of[j].assign(nsub, -1);
                        if (pair_of[j][i] < 0) {
                            pair_of[j][i] = (int32_t)rows_of.size();
                            rows_of.emplace_back();
                            pj.push_back(j);
                            pi.push_back(i);
                        }
                        rows_of[pair_of[j][i]].emplace_back((int32_t)(r - s->hs[j].begin), z);
                        z += s->hs[i].m;
                    }
                    rs_ptr.push_back((int64_t)rs_sub.size());
                }
                std::vector<int64_t> pzoff;
                pptr.push_back(0);
                for (const auto& v : rows_of) {
                    for (const auto& q : v) {
                        prl.push_back(q.first);
                        pzoff.push_back(q.second);
                    }
                    pptr.push_back((int64_t)prl.size());
                }
                R.npairs = (int)rows_of.size();
                RET_IF(upload(s, &R.owner, owner));
                RET_IF(upload(s, &R.rs_ptr, rs_ptr));
                RET_IF(upload(s, &R.rs_sub, rs_sub));
                RET_IF(upload(s, &R.rs_zoff, rs_zoff));
                RET_IF(upload(s, &R.pair_j, pj));
                RET_IF(upload(s, &R.pair_i, pi));
                RET_IF(upload(s, &R.pair_ptr, pptr));
                RET_IF(upload(s, &R.pair_rl, prl));
                RET_IF(upload(s, &R.pair_zoff, pzoff));
                RET_IF(dbl(&R.Z, (size_t)std::max<int64_t>(z, 1)));
                R.direct = true;
            }
            RET_IF(dev_alloc(s, reinterpret_cast<void**>(&R.piv), (size_t)n0 * sizeof(int)));
            RET_IF(dbl(&R.Y, (size_t)n0 * 16));
            RET_IF(dbl(&R.X, (size_t)s->n * 16));
            RET_IF(dbl(&R.AX, (size_t)s->n * 16));
            RET_IF(dbl(&R.cpart, (size_t)std::max(s->ntiles, 1) * std::max(s->mmax, 1) * 16));
            RET_IF(dbl(&R.C, (size_t)n0 * 16));
            if (s->pou != S2L_POU_BOOLEAN) RET_IF(dbl(&R.plocal, (size_t)s->nloc * 16));
            int smax = 1;
            for (int sz : R.sz) smax = std::max(smax, sz);
            constexpr int NS = s2l_setup::Refac::RF_STREAMS;
            for (int q = 0; q < NS; ++q) {
                CUDA_OK(s, cudaStreamCreateWithFlags(&R.tstream[q], cudaStreamNonBlocking));
                if (cusolverDnCreate(&R.tsolver[q]) != CUSOLVER_STATUS_SUCCESS) {
                    R.tsolver[q] = nullptr;
                    return s->fail(S2L_ERR_CUDA, "cusolverDnCreate failed");
                }
                if (cusolverDnSetStream(R.tsolver[q], R.tstream[q]) != CUSOLVER_STATUS_SUCCESS)
                    return s->fail(S2L_ERR_CUDA, "cannot bind the tail handles to their streams");
            }
            for (auto& e : R.tev) CUDA_OK(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            int l1 = 0, l2 = 0;
            size_t id1 = 0, ih1 = 0, id2 = 0, ih2 = 0;
            if (cusolverDnDpotrf_bufferSize(R.tsolver[0], CUBLAS_FILL_MODE_UPPER, smax, R.S, smax, &l1) !=
                    CUSOLVER_STATUS_SUCCESS ||
                cusolverDnDgetrf_bufferSize(R.tsolver[0], smax, smax, R.S, smax, &l2) != CUSOLVER_STATUS_SUCCESS ||
                cusolverDnXtrtri_bufferSize(R.tsolver[0], CUBLAS_FILL_MODE_UPPER, CUBLAS_DIAG_NON_UNIT, smax,
                                            CUDA_R_64F, R.S, smax, &id1, &ih1) != CUSOLVER_STATUS_SUCCESS ||
                cusolverDnXtrtri_bufferSize(R.tsolver[0], CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_UNIT, smax,
                                            CUDA_R_64F, R.S, smax, &id2, &ih2) != CUSOLVER_STATUS_SUCCESS)
                return s->fail(S2L_ERR_CUDA, "cuSOLVER workspace query failed");
            R.lwork = std::max(std::max(l1, l2), 1);
            R.iwork_bytes = std::max<size_t>(std::max(id1, id2), 16);
            for (int q = 0; q < NS; ++q) {
                RET_IF(dbl(&R.swork[q], (size_t)R.lwork));
                RET_IF(dev_alloc(s, &R.iwork[q], R.iwork_bytes));
                bool any_lu = false;
                for (char l : R.llt) any_lu = any_lu || !l;
                if (any_lu) RET_IF(dbl(&R.B[q], (size_t)smax * smax));
                R.ihost[q].assign(std::max<size_t>(std::max(ih1, ih2), 16), 0);
            }
            int l3 = 0;
            if (cusolverDnDgetrf_bufferSize(R.tsolver[0], (int)n0, (int)n0, R.E, (int)n0, &l3) != CUSOLVER_STATUS_SUCCESS)
                return s->fail(S2L_ERR_CUDA, "cuSOLVER workspace query failed");
            R.elwork = std::max(l3, 1);
            RET_IF(dbl(&R.ework, (size_t)R.elwork));
        }
        RET_IF(upload(s, &R.fbase, rf_fbase));
        RET_IF(upload(s, &R.fcp, rf_fcp));
        RET_IF(upload(s, &R.fri, rf_fri));
        RET_IF(upload(s, &R.fdg, rf_fdg));
        RET_IF(upload(s, &R.fllt, rf_fllt));
        RET_IF(upload(s, &R.frp, rf_frp));
        RET_IF(upload(s, &R.frpos, rf_frpos));
        RET_IF(upload(s, &R.frk, rf_frk));
        RET_IF(upload(s, &R.lv_first, rf_lvfirst));
        RET_IF(upload(s, &R.lv_off, rf_lvoff));
        RET_IF(upload(s, &R.lv_col, rf_lvcol));
        RET_IF(upload(s, &R.tc_sub, rf_tcsub));
        RET_IF(upload(s, &R.tc_col, rf_tccol));
        RET_IF(upload(s, &R.fill_src, rf_fill_src));
        RET_IF(upload(s, &R.fill_dst, rf_fill_dst));
        RET_IF(upload(s, &R.lts_src, rf_lts));
        RET_IF(upload(s, &R.ust_src, rf_ust));
        for (int f = 0; f < 2; ++f) {
            R.nblk[f] = (int64_t)rf_beoff[f].size() - 1;
            RET_IF(upload(s, &R.sw_src[f], rf_swsrc[f]));
            RET_IF(upload(s, &R.sw_dsrc[f], rf_swdsrc[f]));
            RET_IF(upload(s, &R.wsrc[f], rf_wsrc[f]));
            RET_IF(upload(s, &R.be_off[f], rf_beoff[f]));
            RET_IF(upload(s, &R.be_pos[f], rf_bepos[f]));
            RET_IF(upload(s, &R.be_row[f], rf_berow[f]));
            RET_IF(upload(s, &R.be_cp[f], rf_becp[f]));
            RET_IF(upload(s, &R.bc_b[f], rf_bcb[f]));
            RET_IF(upload(s, &R.bc_pos[f], rf_bcpos[f]));
        }
        CUDA_OK(s, cudaStreamSynchronize(s->setup_stream));
        R.bytes = s->bytes - before;
        R.on = true;
    }

    // sweep shared memory: x (T values and the sentinel slot) + one ready byte per slot
    const size_t slots = (size_t)max_T + 1;
    const size_t smem = (((slots * rs) + 15) & ~(size_t)15) + ((slots + 15) & ~(size_t)15);
    const size_t smem_cap = S2L_SWEEP_SMEM_CAP;
    if (smem <= smem_cap) {
        s->smem_bytes = smem;
    } else {
        s->smem_bytes = 0;
        s->need_gflags = true;
    }
    s->max_nl = max_nl;
    s->max_T = max_T;
    s->kc_max = 1;
    if (s->smem_bytes > 0)
        for (int kc = 2; kc <= 4; kc *= 2)
            if ((((slots * kc * rs) + 15) & ~(size_t)15) + ((slots + 15) & ~(size_t)15) <= smem_cap)
                s->kc_max = kc;
    CUDA_OK(s, cudaStreamSynchronize(s->setup_stream));
    // host staging no longer needed
    s->A.ci = {};  // the row pointers stay: s2l_gpu_update_matrix recomputes the row sums with them
    s->A.v = {};
    for (auto& h : s->hs) {
        h.L = HostCsr();
        h.U = HostCsr();
        h.V.clear();
        h.V.shrink_to_fit();
    }
    s2l_work* w0 = nullptr;
    RET_IF(work_create(s, &w0));
    if (s->user_stream) w0->stream = s->user_stream;
    s->works.push_back(w0);
    s->busy.push_back(0);
    s->ended = true;
    return S2L_OK;
}

int s2l_gpu_setup_destroy(s2l_setup* s)
{
    if (!s) return S2L_OK;
    if (s->pending.load() > 0) return s->fail(S2L_ERR_STATE, "asynchronous solves are queued or running on this setup");
    RET_IF(wait_runners_gone(s));
    cudaSetDevice(s->ctx->device);
    for (s2l_work* w : s->works) work_destroy(w);
    if (s->setup_stream) cudaStreamSynchronize(s->setup_stream);
    for (void* p : s->allocs) cudaFree(p);
    {
        std::lock_guard<std::mutex> g(s->ctx->mu);
        s->ctx->used -= std::min(s->ctx->used, s->bytes);
    }
    if (s->setup_stream) cudaStreamDestroy(s->setup_stream);
    for (int q = 0; q < s2l_setup::Refac::RF_STREAMS; ++q) {
        if (s->rf.tsolver[q]) cusolverDnDestroy(s->rf.tsolver[q]);
        if (s->rf.tstream[q]) cudaStreamDestroy(s->rf.tstream[q]);
    }
    for (auto e : s->rf.tev)
        if (e) cudaEventDestroy(e);
    delete s;
    return S2L_OK;
}

// New values of A, same pattern (the reference's UpdateLevel::Reuse,
// include/preconditioner/preconditioner.hpp:20-30): the operator changes, the preconditioner stays.
int s2l_gpu_update_matrix(s2l_setup* s, const double* val, int ptr_kind)
{
    RET_IF(check_ready(s));
    if (!val) return s->fail(S2L_ERR_BADARG, "null values");
    if (ptr_kind != S2L_PTR_HOST && ptr_kind != S2L_PTR_DEVICE)
        return s->fail(S2L_ERR_BADARG, "ptr_kind must be S2L_PTR_HOST or S2L_PTR_DEVICE");
    RET_IF(wait_runners_gone(s));
    std::lock_guard<std::mutex> g(s->wmu);  // no call can take a workspace meanwhile
    for (char b : s->busy)
        if (b) return s->fail(S2L_ERR_STATE, "update_matrix while a solve-phase call runs on the setup");
    if (s->pending.load() > 0) return s->fail(S2L_ERR_STATE, "update_matrix while solves are queued on the setup");
    if (cudaSetDevice(s->ctx->device) != cudaSuccess) return s->fail(S2L_ERR_CUDA, "cudaSetDevice failed");
    const int64_t n = s->n, nnz = s->nnz;
    std::vector<double> v((size_t)nnz);
    if (ptr_kind == S2L_PTR_HOST) {
        std::copy(val, val + nnz, v.begin());
    } else {
        CUDA_OK(s, cudaMemcpyAsync(v.data(), val, nnz * sizeof(double), cudaMemcpyDeviceToHost, s->setup_stream));
        CUDA_OK(s, cudaStreamSynchronize(s->setup_stream));
    }
    for (int64_t e = 0; e < nnz; ++e)
        if (!std::isfinite(v[e])) return s->fail(S2L_ERR_NUMERIC, "non-finite matrix value");
    std::vector<double> rowsum((size_t)n, 0.0);  // A 1, in row order as at setup
    for (int64_t r = 0; r < n; ++r)
        for (int64_t e = s->A.rp[r]; e < s->A.rp[r + 1]; ++e) rowsum[r] += v[e];
    CUDA_OK(s, cudaMemcpyAsync(s->d_av, v.data(), nnz * sizeof(double), cudaMemcpyHostToDevice, s->setup_stream));
    CUDA_OK(s, cudaMemcpyAsync(s->d_rowsum, rowsum.data(), n * sizeof(double), cudaMemcpyHostToDevice, s->setup_stream));
    CUDA_OK(s, cudaStreamSynchronize(s->setup_stream));
    return S2L_OK;
}

}  // extern "C"

namespace {

// E = W^T A W for the matrix values v (device), 16 columns of W at a time: prolongation of unit
// coarse vectors, product with A, restriction (the kernels of the coarse correction)
int coarse_matrix_dev(s2l_setup* s, cudaStream_t st, const double* v, double* E)
{
    auto& R = s->rf;
    const int64_t n = s->n, n0 = s->n0;
    const int K = 16;
    const int boolean = s->pou == S2L_POU_BOOLEAN;
    for (int64_t c0 = 0; c0 < n0; c0 += K) {
        launch_unit_block(st, n0, (int)c0, R.Y);
        launch_coarse_prolong_block(st, K, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->mmax,
                                    boolean, R.Y, R.X, R.plocal);
        if (!boolean) launch_combine_block(st, n, K, s->d_cp_ptr, s->d_cp_pos, nullptr, R.plocal, nullptr, R.X);
        launch_spmv_block(st, n, K, s->d_rp, s->d_ci, v, R.X, R.AX, nullptr, nullptr, nullptr, s->tpr);
        launch_coarse_restrict_block(st, K, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->d_l2g,
                                     boolean, R.AX, s->mmax, R.cpart);
        launch_coarse_reduce_block(st, K, s->nsub, s->d_subs, s->d_t_first, s->mmax, R.cpart, R.C);
        launch_scatter_columns(st, n0, (int)c0, R.C, E);
    }
    CUDA_OK(s, cudaGetLastError());
    return S2L_OK;
}

// fork the tail streams after the work queued on st / join st after them
int tails_fork(s2l_setup* s, cudaStream_t st)
{
    auto& R = s->rf;
    constexpr int NS = s2l_setup::Refac::RF_STREAMS;
    CUDA_OK(s, cudaEventRecord(R.tev[NS], st));
    for (int q = 0; q < NS; ++q) CUDA_OK(s, cudaStreamWaitEvent(R.tstream[q], R.tev[NS], 0));
    return S2L_OK;
}

int tails_join(s2l_setup* s, cudaStream_t st)
{
    auto& R = s->rf;
    constexpr int NS = s2l_setup::Refac::RF_STREAMS;
    for (int q = 0; q < NS; ++q) {
        CUDA_OK(s, cudaEventRecord(R.tev[q], R.tstream[q]));
        CUDA_OK(s, cudaStreamWaitEvent(st, R.tev[q], 0));
    }
    return S2L_OK;
}

// Dense tails in place (S_i, s x s row-major, i.e. S_i^T column-major), the subdomains spread over
// the tail streams: L L^T by Cholesky (potrf, upper in column-major = the lower L row-major); LU by
// an LU without pivoting (getrf with no pivot array) of S^T = L' U', which is S = (U'^T)(L'^T) with
// a lower triangle U'^T and a unit upper L'^T.  A failed pivot leaves info_i > 0.
int refactor_dense_tails(s2l_setup* s, cudaStream_t st)
{
    auto& R = s->rf;
    constexpr int NS = s2l_setup::Refac::RF_STREAMS;
    RET_IF(tails_fork(s, st));
    for (int i = 0; i < s->nsub; ++i) {
        const int sz = R.sz[i];
        if (sz == 0) continue;
        const int q = i % NS;
        double* Si = R.S + R.d_off[i];
        const cusolverStatus_t cs =
            R.llt[i] ? cusolverDnDpotrf(R.tsolver[q], CUBLAS_FILL_MODE_UPPER, sz, Si, sz, R.swork[q], R.lwork, R.info + i)
                     : cusolverDnDgetrf(R.tsolver[q], sz, sz, Si, sz, R.swork[q], nullptr, R.info + i);
        if (cs != CUSOLVER_STATUS_SUCCESS) return s->fail(S2L_ERR_CUDA, "dense tail factorization failed to launch");
        if (!R.llt[i]) launch_tail_growth(R.tstream[q], Si, sz, s->opt_pivot_tol, R.err);
    }
    return tails_join(s, st);
}

template <typename Real>
int refactor_commit_factors(s2l_setup* s, cudaStream_t st)
{
    auto& R = s->rf;
    const int nsub = s->nsub;
    for (int f = 0; f < 2; ++f) {
        launch_refactor_dinv<Real>(st, nsub, s->d_subs, R.fbase, R.F, R.sw_dsrc[f], (Real*)s->d_dinv[f]);
        launch_refactor_sweep_values<Real>(st, nsub, R.fbase, R.F, s->d_wtask[f], s->d_wslot[f], s->d_went[f],
                                           s->d_thdr[f], s->d_tslot[f], R.sw_src[f], s->d_subs, R.sw_dsrc[f],
                                           (Real*)s->d_val[f]);
        launch_refactor_blocks<Real>(st, R.nblk[f], s->d_boff[f], s->d_bioff[f], R.wsrc[f], R.be_off[f], R.be_pos[f],
                                     R.be_row[f], R.be_cp[f], R.bc_b[f], R.bc_pos[f], R.F, (Real*)s->d_binv[f],
                                     (Real*)s->d_val[f]);
    }
    launch_gather_values<Real>(st, R.nlts, R.lts_src, R.F, (Real*)s->d_lts_val);
    launch_gather_values<Real>(st, R.nust, R.ust_src, R.F, (Real*)s->d_ust_val);
    // dense tail inverses: the triangles of each factored tail inverted (cusolverDnXtrtri), the
    // subdomains spread over the tail streams.  Column-major, the tail holds the Cholesky factor
    // U_c (upper; row-major that is the lower L) or U' (upper) and L' (strict lower, unit diagonal);
    // their inverses are row-major Lt^-1 (lower) and Ut^-1 (strict upper, unit diagonal).  U_c / U'
    // is inverted in place, L' in a copy of the tail (the two inversions do not share storage).
    constexpr int NS = s2l_setup::Refac::RF_STREAMS;
    RET_IF(tails_fork(s, st));
    for (int i = 0; i < nsub; ++i) {
        const int sz = R.sz[i];
        if (sz == 0) continue;
        const int q = i % NS;
        cudaStream_t sq = R.tstream[q];
        double* Si = R.S + R.d_off[i];
        double* Bq = R.llt[i] ? nullptr : R.B[q];
        if (Bq) CUDA_OK(s, cudaMemcpyAsync(Bq, Si, (size_t)sz * sz * sizeof(double), cudaMemcpyDeviceToDevice, sq));
        for (int f = 0; f < (Bq ? 2 : 1); ++f) {
            if (cusolverDnXtrtri(R.tsolver[q], f == 0 ? CUBLAS_FILL_MODE_UPPER : CUBLAS_FILL_MODE_LOWER,
                                 f == 0 ? CUBLAS_DIAG_NON_UNIT : CUBLAS_DIAG_UNIT, sz, CUDA_R_64F, f == 0 ? Si : Bq,
                                 sz, R.iwork[q], R.iwork_bytes, R.ihost[q].data(), R.ihost[q].size(), R.info + i) !=
                CUSOLVER_STATUS_SUCCESS)
                return s->fail(S2L_ERR_CUDA, "cusolverDnXtrtri failed");
        }
        launch_tail_inverses<Real>(sq, Si, Bq, sz, R.llt[i], (Real*)s->d_linv + R.d_off[i],
                                   (Real*)s->d_uinv + R.d_off[i]);
    }
    return tails_join(s, st);
}

int refactor_run(s2l_setup* s, const double* val, int ptr_kind)
{
    auto& R = s->rf;
    cudaStream_t st = s->setup_stream;
    const int nsub = s->nsub;
    const int64_t n = s->n, nnz = s->nnz, n0 = s->n0;
    const auto t0 = std::chrono::steady_clock::now();
    // phase timers (events on the setup stream)
    struct Evs {
        cudaEvent_t e[7] = {};
        ~Evs()
        {
            for (auto x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    for (auto& x : ev.e) CUDA_OK(s, cudaEventCreate(&x));
    CUDA_OK(s, cudaMemcpyAsync(R.stage, val, (size_t)nnz * sizeof(double),
                               ptr_kind == S2L_PTR_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
    CUDA_OK(s, cudaMemsetAsync(R.err, 0, sizeof(int), st));
    CUDA_OK(s, cudaMemsetAsync(R.info, 0, (size_t)(nsub + 2) * sizeof(int), st));
    // row sums of the new matrix: the OpenFOAM normalisation, and a finiteness check of every value
    launch_row_sums(st, n, s->d_rp, R.stage, R.rowsum);
    {
        std::vector<double> h((size_t)n);
        CUDA_OK(s, cudaMemcpyAsync(h.data(), R.rowsum, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(s, cudaStreamSynchronize(st));
        for (double v : h)
            if (!std::isfinite(v)) return s->fail(S2L_ERR_NUMERIC, "non-finite matrix value");
    }
    // coarse matrix with the kept basis, and its inverse
    const bool coarse = s->coarse != S2L_COARSE_NONE && n0 > 0;
    CUDA_OK(s, cudaEventRecord(ev.e[0], st));
    if (coarse && R.direct)
        launch_coarse_direct(st, n, s->d_rp, s->d_ci, R.stage, R.owner, R.rs_ptr, R.rs_sub, R.rs_zoff, R.npairs,
                             R.pair_j, R.pair_i, R.pair_ptr, R.pair_rl, R.pair_zoff, s->d_subs, s->d_V, R.Z, n0, R.E);
    else if (coarse)
        RET_IF(coarse_matrix_dev(s, st, R.stage, R.E));
    CUDA_OK(s, cudaEventRecord(ev.e[1], st));
    if (coarse) {
        // E^-1: LU with partial pivoting (E row-major is E^T column-major; the solve against the
        // identity gives (E^T)^-1 column-major = E^-1 row-major); info > 0: singular
        RET_IF(tails_fork(s, st));
        launch_identity(R.tstream[0], R.Einv, (int)n0);
        if (cusolverDnDgetrf(R.tsolver[0], (int)n0, (int)n0, R.E, (int)n0, R.ework, R.piv, R.info + nsub) !=
                CUSOLVER_STATUS_SUCCESS ||
            cusolverDnDgetrs(R.tsolver[0], CUBLAS_OP_N, (int)n0, (int)n0, R.E, (int)n0, R.piv, R.Einv, (int)n0,
                             R.info + nsub + 1) != CUSOLVER_STATUS_SUCCESS)
            return s->fail(S2L_ERR_CUDA, "coarse inversion failed to launch");
        RET_IF(tails_join(s, st));
    }
    // local factors on their kept patterns
    RefactorArgs a{};
    a.subs = s->d_subs;
    a.F = R.F;
    a.fbase = R.fbase;
    a.fcp = R.fcp;
    a.fri = R.fri;
    a.fdg = R.fdg;
    a.fllt = R.fllt;
    a.frp = R.frp;
    a.frpos = R.frpos;
    a.frk = R.frk;
    a.lv_first = R.lv_first;
    a.lv_off = R.lv_off;
    a.lv_col = R.lv_col;
    a.tc_sub = R.tc_sub;
    a.tc_col = R.tc_col;
    a.ntc = R.ntc;
    a.S = R.S;
    a.err = R.err;
    a.pivot_tol = s->opt_pivot_tol;
    a.smax = 1;
    for (int sz : R.sz) a.smax = std::max(a.smax, sz);
    a.maxcol = R.maxcol;
    a.nlmax = s->max_nl;
    a.part = R.part;
    CUDA_OK(s, cudaMemsetAsync(R.F, 0, (size_t)std::max<int64_t>(R.nF, 1) * sizeof(double), st));
    launch_refactor_fill(st, R.nfill, R.fill_src, R.fill_dst, R.stage, R.F);
    CUDA_OK(s, cudaEventRecord(ev.e[2], st));
    launch_refactor_sparse(st, a, nsub, R.cs);
    CUDA_OK(s, cudaEventRecord(ev.e[3], st));
    launch_refactor_tail_columns(st, a);
    CUDA_OK(s, cudaEventRecord(ev.e[4], st));
    CUDA_OK(s, cudaMemsetAsync(R.S, 0, (size_t)std::max<int64_t>(R.d_off[nsub], 1) * sizeof(double), st));
    launch_refactor_gather_tails(st, a);
    RET_IF(refactor_dense_tails(s, st));
    CUDA_OK(s, cudaEventRecord(ev.e[5], st));
    CUDA_OK(s, cudaGetLastError());
    int herr = 0;
    std::vector<int> infos((size_t)nsub + 2);
    CUDA_OK(s, cudaMemcpyAsync(&herr, R.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(s, cudaMemcpyAsync(infos.data(), R.info, (size_t)(nsub + 2) * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(s, cudaStreamSynchronize(st));
    for (int i = 0; i < nsub && herr == 0; ++i)
        if (infos[i] != 0) herr = 2;
    if (herr == 0 && coarse && (infos[nsub] != 0 || infos[nsub + 1] != 0)) herr = 3;
    if (herr == 1) return s->fail(S2L_ERR_NUMERIC, "refactorization: zero or non-positive pivot in a sparse column");
    if (herr == 2) return s->fail(S2L_ERR_NUMERIC, "refactorization: zero or non-positive pivot in a dense tail");
    if (herr == 4)
        return s->fail(S2L_ERR_NUMERIC, "refactorization: an LU pivot is below pivot_tol relative to its column (a "
                                        "multiplier above 1 / pivot_tol); the kept pivot order no longer suits the "
                                        "matrix: rebuild the factorization");
    if (herr == 3) return s->fail(S2L_ERR_NUMERIC, "refactorization: the coarse matrix is singular");
    if (herr) return s->fail(S2L_ERR_NUMERIC, "refactorization failed");
    // commit: the matrix, its row sums, E^-1, then the solve layout of the new factors
    CUDA_OK(s, cudaMemcpyAsync(s->d_av, R.stage, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_OK(s, cudaMemcpyAsync(s->d_rowsum, R.rowsum, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (coarse)
        CUDA_OK(s, cudaMemcpyAsync(s->d_Einv, R.Einv, (size_t)n0 * n0 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (s->real == S2L_REAL_F32) RET_IF(refactor_commit_factors<float>(s, st));
    else RET_IF(refactor_commit_factors<double>(s, st));
    CUDA_OK(s, cudaGetLastError());
    CUDA_OK(s, cudaEventRecord(ev.e[6], st));
    CUDA_OK(s, cudaStreamSynchronize(st));
    R.last_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (int q = 0; q < 6; ++q) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev.e[q], ev.e[q + 1]);
        R.phase_ms[q] = ms;
    }
    return S2L_OK;
}

}  // namespace

extern "C" {

int s2l_gpu_refactor(s2l_setup* s, const double* val, int ptr_kind)
{
    RET_IF(check_ready(s));
    if (!val) return s->fail(S2L_ERR_BADARG, "null values");
    if (ptr_kind != S2L_PTR_HOST && ptr_kind != S2L_PTR_DEVICE)
        return s->fail(S2L_ERR_BADARG, "ptr_kind must be S2L_PTR_HOST or S2L_PTR_DEVICE");
    if (!s->rf.on) return s->fail(S2L_ERR_STATE, "the setup was built without the option refactor = 1");
    RET_IF(wait_runners_gone(s));
    std::lock_guard<std::mutex> g(s->wmu);  // no call can take a workspace meanwhile
    for (char b : s->busy)
        if (b) return s->fail(S2L_ERR_STATE, "refactor while a solve-phase call runs on the setup");
    if (s->pending.load() > 0) return s->fail(S2L_ERR_STATE, "refactor while solves are queued on the setup");
    if (cudaSetDevice(s->ctx->device) != cudaSuccess) return s->fail(S2L_ERR_CUDA, "cudaSetDevice failed");
    return refactor_run(s, val, ptr_kind);
}

int s2l_gpu_setup_bytes(const s2l_setup* s, size_t* bytes)
{
    if (!s || !bytes) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(s->wmu);
    size_t b = s->bytes;
    for (const s2l_work* w : s->works) b += w->bytes;
    *bytes = b;
    return S2L_OK;
}

int s2l_gpu_setup_option(s2l_setup* s, const char* name, double value)
{
    if (!s || !name) return S2L_ERR_BADARG;
    const std::string n(name);
    if (n == "spin_limit") {  // read at every launch: may change after setup_end
        if (!(value >= 1.0 && value <= 2147483647.0)) return s->fail(S2L_ERR_BADARG, "spin_limit must be in [1, 2^31)");
        s->opt_spin_limit.store((int)value);
        return S2L_OK;
    }
    if (n == "sweep_prefetch") {  // read at every launch, like spin_limit
        if (!(value >= 0.0 && value <= 32.0)) return s->fail(S2L_ERR_BADARG, "sweep_prefetch must be in [0, 32]");
        s->opt_sweep_pf.store((int)value);
        return S2L_OK;
    }
    if (n == "spin_sleep_ns") {  // read at every launch, like spin_limit
        if (!(value >= 0.0 && value <= 1000000.0)) return s->fail(S2L_ERR_BADARG, "spin_sleep_ns must be in [0, 1e6]");
        s->opt_spin_sleep.store((int)value);
        return S2L_OK;
    }
    if (s->ended) return s->fail(S2L_ERR_STATE, "setup_option after setup_end");
    if (n == "tail_min") s->opt_tail_min = (int)value;
    else if (n == "tail_max") s->opt_tail_max = (int)value;
    else if (n == "tail_rows") s->opt_tail_rows = (int)value;
    else if (n == "hop_us") s->opt_hop_us = value;
    else if (n == "bw_gbs") s->opt_bw_gbs = value;
    else if (n == "sweep_group") {
        const int g = (int)value;
        if (g != 0 && g != 8 && g != 16 && g != 32) return s->fail(S2L_ERR_BADARG, "sweep_group must be 0, 8, 16 or 32");
        s->opt_group = g;
    } else if (n == "spmv_tpr") {
        const int t = (int)value;
        if (t != 0 && t != 1 && t != 2 && t != 4 && t != 8 && t != 16 && t != 32)
            return s->fail(S2L_ERR_BADARG, "spmv_tpr must be 0, 1, 2, 4, 8, 16 or 32");
        s->opt_tpr = t;
    } else if (n == "block_width") {
        const int bw = (int)value;
        if (bw != 0 && bw != 1 && bw != 2 && bw != 4 && bw != 8 && bw != 16)
            return s->fail(S2L_ERR_BADARG, "block_width must be 0, 1, 2, 4, 8 or 16");
        s->opt_block_width = bw;
    } else if (n == "sweep_epl") {
        const int v = (int)value;
        if (v != 2 && v != 4 && v != 8 && v != 16) return s->fail(S2L_ERR_BADARG, "sweep_epl must be 2, 4, 8 or 16");
        s->opt_epl = v;
    } else if (n == "chain_block") {
        const int c = (int)value;
        if (c < 1 || c > S2L_CHAIN_MAX) return s->fail(S2L_ERR_BADARG, "chain_block must be in [1, 16]");
        s->opt_chain = c;
    } else if (n == "refactor") {
        s->opt_refactor = value != 0.0;
    } else if (n == "amg_single") {
        s->opt_amg_single = value != 0.0;
    } else if (n == "pivot_tol") {
        if (!(value >= 0.0 && value < 1.0)) return s->fail(S2L_ERR_BADARG, "pivot_tol must be in [0, 1)");
        s->opt_pivot_tol = value;
    } else return s->fail(S2L_ERR_BADARG, "unknown setup option " + n);
    return S2L_OK;
}

int s2l_gpu_setup_stat(const s2l_setup* s, const char* name, double* value)
{
    if (!s || !name || !value) return S2L_ERR_BADARG;
    const std::string n(name);
    if (n == "sparse_nnz") *value = (double)s->st_sparse_nnz;
    else if (n == "coupling_nnz") *value = (double)s->st_coupling_nnz;
    else if (n == "dense_entries") *value = (double)s->st_dense_entries;
    else if (n == "tail_rows") *value = (double)s->st_tail_rows;
    else if (n == "sweep_group") *value = (double)s->sweep_group;
    else if (n == "smem_bytes") *value = (double)s->smem_bytes;
    else if (n == "levels_max") *value = (double)s->st_levels_max;
    else if (n == "chain_blocks") *value = (double)s->st_blocks;
    else if (n == "sweep_tasks") *value = (double)s->st_tasks;
    else if (n == "local_solve_column_bytes") *value = s->solve_vec_bytes;
    else if (n == "kc_max") *value = (double)s->kc_max;
    else if (n == "spmv_tpr") *value = (double)s->tpr;
    else if (n == "block_width") *value = (double)block_width_best(const_cast<s2l_setup*>(s));
    else if (n == "sweep_padding") *value = (double)s->st_pad;
    else if (n == "levels_mean") *value = s->nsub ? (double)s->st_levels_sum / (2.0 * s->nsub) : 0.0;
    else if (n == "refactor_bytes") *value = (double)s->rf.bytes;
    else if (n == "refactor_ms") *value = s->rf.last_ms;
    else if (n == "refactor_cluster") *value = (double)s->rf.cs;
    else if (n == "refactor_ms_coarse") *value = s->rf.phase_ms[0];
    else if (n == "refactor_ms_coarse_inverse") *value = s->rf.phase_ms[1];
    else if (n == "refactor_ms_sparse") *value = s->rf.phase_ms[2];
    else if (n == "refactor_ms_tail") *value = s->rf.phase_ms[3];
    else if (n == "refactor_ms_dense") *value = s->rf.phase_ms[4];
    else if (n == "refactor_ms_commit") *value = s->rf.phase_ms[5];
    else return S2L_ERR_BADARG;
    return S2L_OK;
}

int s2l_gpu_set_stream(s2l_setup* s, void* stream)
{
    if (!s) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(s->wmu);
    s->user_stream = (cudaStream_t)stream;
    if (!s->works.empty()) s->works[0]->stream = stream ? (cudaStream_t)stream : s->works[0]->own_stream;
    return S2L_OK;
}

int s2l_gpu_profile_enable(s2l_setup* s, int on)
{
    if (!s) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(s->wmu);
    s->prof_mask = (unsigned)on & 0x1Fu;
    for (s2l_work* w : s->works) {
        prof_drain(w);
        for (int c = 0; c < PC_N; ++c) {
            w->acc_ms[c] = 0.0;
            w->acc_n[c] = 0;
        }
        w->prof = s->prof_mask;
        w->launches = 0;
    }
    return S2L_OK;
}

int s2l_gpu_profile_get(s2l_setup* s, const char* name, double* ms, long* launches)
{
    if (!s || !name || !ms || !launches) return S2L_ERR_BADARG;
    int cls = -2;  // -2 launches, -1 all classes, else one class
    if (std::strcmp(name, "launches") == 0) cls = -2;
    else if (std::strcmp(name, "all") == 0) cls = -1;
    else {
        cls = PC_N;
        for (int c = 0; c < PC_N; ++c)
            if (std::strcmp(name, kProfNames[c]) == 0) cls = c;
        if (cls == PC_N) return s->fail(S2L_ERR_BADARG, std::string("unknown profile class ") + name);
    }
    std::lock_guard<std::mutex> g(s->wmu);
    *ms = 0.0;
    *launches = 0;
    for (s2l_work* w : s->works) {  // summed over the workspaces of concurrent calls
        prof_drain(w);
        if (cls == -2) {
            *launches += w->launches;
            continue;
        }
        for (int c = 0; c < PC_N; ++c)
            if (cls == -1 || cls == c) {
                *ms += w->acc_ms[c];
                *launches += w->acc_n[c];
            }
    }
    return S2L_OK;
}

int s2l_gpu_local_solve_bytes(const s2l_setup* s, double* bytes)
{
    if (!s || !bytes) return S2L_ERR_BADARG;
    *bytes = s->solve_bytes;
    return S2L_OK;
}

// ------------------------------------------------------------------------------ solve-phase calls
int s2l_gpu_spmv(s2l_setup* s, const double* x, double* y, int ptr_kind)
{
    RET_IF(check_ready(s));
    Lease lease(s);
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    if (!x || !y) return s->fail(S2L_ERR_BADARG, "null vector");
    const double* dx;
    RET_IF(stage_in(w, x, ptr_kind, s->n, w->d_in, &dx));
    double* dy = ptr_kind == S2L_PTR_DEVICE ? y : w->d_out;
    RET_IF(spmv_dev(w, dx, dy, nullptr, false));
    return finish_out(w, y, dy, ptr_kind, s->n);
}

int s2l_gpu_local_solve(s2l_setup* s, int i, const double* b_local, double* x_local, int ptr_kind)
{
    RET_IF(check_ready(s));
    Lease lease(s);
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    if (i < 0 || i >= s->nsub) return s->fail(S2L_ERR_BADARG, "subdomain index out of range");
    if (!b_local || !x_local) return s->fail(S2L_ERR_BADARG, "null vector");
    const int nl = s->h_subs[i].n_local;
    const double* db;
    RET_IF(stage_in(w, b_local, ptr_kind, nl, w->d_in, &db));
    double* dx = ptr_kind == S2L_PTR_DEVICE ? x_local : w->d_out;
    RET_IF(run_local_solve(w, nullptr, nullptr, dx, 2, i, db));
    return finish_out(w, x_local, dx, ptr_kind, nl);
}

int s2l_gpu_coarse_apply(s2l_setup* s, const double* r, double* x0, int ptr_kind)
{
    RET_IF(check_ready(s));
    Lease lease(s);
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    if (!r || !x0) return s->fail(S2L_ERR_BADARG, "null vector");
    if (s->coarse == S2L_COARSE_NONE || s->n0 == 0) return s->fail(S2L_ERR_STATE, "no coarse space");
    const double* dr;
    RET_IF(stage_in(w, r, ptr_kind, s->n, w->d_in, &dr));
    double* dx = ptr_kind == S2L_PTR_DEVICE ? x0 : w->d_out;
    RET_IF(coarse_apply(w, dr, dx));
    return finish_out(w, x0, dx, ptr_kind, s->n);
}

}  // extern "C"

// Scratch of s2l_gpu_coarse_apply_noalloc: one static array per device, never allocated.  Host
// code reaches it only through the device address looked up once per device below.
static __device__ __align__(256) double s2l_noalloc_scratch[S2L_NOALLOC_SCRATCH_DOUBLES];

namespace {
// The device address of the static scratch for the context's device.  The device is current when
// this runs (the entry point sets it), so the lookup resolves the array of that device.
int noalloc_scratch(s2l_setup* s, double** out)
{
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (!s->ctx->noalloc_scratch) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, s2l_noalloc_scratch);
        if (e != cudaSuccess) {
            t_last_error = std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e);
            s->ctx->err = t_last_error;
            return S2L_ERR_CUDA;
        }
        s->ctx->noalloc_scratch = static_cast<double*>(p);
    }
    *out = s->ctx->noalloc_scratch;
    return S2L_OK;
}
}  // namespace

extern "C" int s2l_gpu_coarse_apply_noalloc(s2l_setup* s, const double* r, double* x0)
{
    RET_IF(check_ready(s));
    if (!r || !x0) return s->fail(S2L_ERR_BADARG, "null vector");
    if (s->coarse == S2L_COARSE_NONE || s->n0 == 0) return s->fail(S2L_ERR_STATE, "no coarse space");
    const int boolean = s->pou == S2L_POU_BOOLEAN;
    const int64_t need = (int64_t)s->ntiles * s->mmax + 2 * s->n0 + (boolean ? 0 : s->nloc);
    if (need > S2L_NOALLOC_SCRATCH_DOUBLES)
        return s->fail(S2L_ERR_BADARG, "coarse_apply_noalloc: this setup needs " + std::to_string(need) +
                                           " doubles of scratch; the static no-alloc scratch holds " +
                                           std::to_string(S2L_NOALLOC_SCRATCH_DOUBLES));
    // the setup's device is made current, as every other solve-phase call does (its pointers and
    // its stream belong to that device)
    if (cudaSetDevice(s->ctx->device) != cudaSuccess) return s->fail(S2L_ERR_CUDA, "cudaSetDevice failed");
    double* scr = nullptr;
    RET_IF(noalloc_scratch(s, &scr));
    // the stream of workspace 0 (the caller's stream from s2l_gpu_set_stream) is read, and the
    // kernels enqueued, under the workspace lock: s2l_gpu_set_stream, s2l_gpu_update_matrix and
    // s2l_gpu_refactor take the same lock and cannot change the stream or the setup meanwhile
    std::lock_guard<std::mutex> g(s->wmu);
    cudaStream_t st = s->works[0]->stream;
    double* part = scr;
    double* c = part + (int64_t)s->ntiles * s->mmax;
    double* y = c + s->n0;
    double* plocal = y + s->n0;
    launch_coarse_restrict(st, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->d_l2g,
                           boolean, r, s->mmax, part);
    launch_coarse_reduce(st, s->nsub, s->d_subs, s->d_t_first, s->mmax, part, c);
    launch_dense_gemv(st, (int)s->n0, s->d_Einv, c, y);
    launch_coarse_prolong(st, s->ntiles, s->d_t_sub, s->d_t_row0, s->d_t_nrow, s->d_subs, s->d_V, s->mmax, boolean, y,
                          x0, plocal);
    if (!boolean) launch_combine(st, s->n, s->d_cp_ptr, s->d_cp_pos, nullptr, plocal, nullptr, x0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return s->fail(S2L_ERR_CUDA, std::string("coarse_apply_noalloc launch: ") + cudaGetErrorString(e));
    return S2L_OK;
}

extern "C" {

int s2l_gpu_one_level_apply(s2l_setup* s, const double* r, double* z, int ptr_kind)
{
    RET_IF(check_ready(s));
    Lease lease(s);
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    if (!r || !z) return s->fail(S2L_ERR_BADARG, "null vector");
    if (r == z) return s->fail(S2L_ERR_BADARG, "r and z must not alias");
    const double* dr;
    RET_IF(stage_in(w, r, ptr_kind, s->n, w->d_in, &dr));
    double* dz = ptr_kind == S2L_PTR_DEVICE ? z : w->d_out;
    RET_IF(one_level(w, dr, nullptr, dz));
    return finish_out(w, z, dz, ptr_kind, s->n);
}

int s2l_gpu_apply(s2l_setup* s, const double* r, double* z, int ptr_kind)
{
    RET_IF(check_ready(s));
    Lease lease(s);
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    if (!r || !z) return s->fail(S2L_ERR_BADARG, "null vector");
    if (r == z) return s->fail(S2L_ERR_BADARG, "r and z must not alias");
    const double* dr;
    RET_IF(stage_in(w, r, ptr_kind, s->n, w->d_in, &dr));
    double* dz = ptr_kind == S2L_PTR_DEVICE ? z : w->d_out;
    RET_IF(apply_dev(w, dr, dz));
    return finish_out(w, z, dz, ptr_kind, s->n);
}

// Restarted right-preconditioned GMRES(m) with CGS2 (src/solver/gmres.cpp:18-161); flexible variant
// keeps Z_j = M^-1 v_j and updates x += Z y instead of x += M^-1 (V y).
static int gmres_run(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                     s2l_result* res, const std::atomic<int>* cancel)
{
    RET_IF(check_ready(s));
    if (!b || !x || !o || !res) return s->fail(S2L_ERR_BADARG, "null argument");
    if (o->restart < 1 || o->maxit < 0 || !(o->rtol >= 0.0)) return s->fail(S2L_ERR_BADARG, "bad Krylov options");
    RET_IF(check_stop(s, o));
    const bool of = o->stop_norm == S2L_STOP_OPENFOAM;
    const int m = o->restart;
    const bool flex = o->flexible != 0;
    Lease lease(s, [&](s2l_work* lw) { return ensure_krylov(lw, m, flex); });
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    const int64_t n = s->n;
    cudaStream_t st = w->stream;
    double* V = w->d_V_kr;
    double* Z = w->d_Z_kr;
    const double* db;
    if (ptr_kind == S2L_PTR_HOST) {
        CUDA_OK(w, cudaMemcpyAsync(w->d_b, b, n * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(w, cudaMemcpyAsync(w->d_xk, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
        db = w->d_b;
    } else if (ptr_kind == S2L_PTR_DEVICE) {
        db = b;
        CUDA_OK(w, cudaMemcpyAsync(w->d_xk, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
        return s->fail(S2L_ERR_BADARG, "bad ptr_kind");
    }
    double* dx = w->d_xk;
    res->converged = 0;
    res->breakdown = 0;
    res->iterations = 0;
    res->restarts = 0;
    res->history_len = 0;
    res->initial_residual_of = res->final_residual_of = 0.0;
    auto hist = [&](double v) {
        if (res->history && res->history_len < o->history_cap) res->history[res->history_len] = v;
        if (res->history_len < o->history_cap) ++res->history_len;
    };
    double bnorm = 0.0;
    RET_IF(norm2_dev(w, db, &bnorm));
    if (bnorm == 0.0) {
        CUDA_OK(w, cudaMemsetAsync(dx, 0, n * sizeof(double), st));
        res->converged = 1;
        hist(0.0);
        res->rel_residual = res->true_rel_residual = 0.0;
        return finish_out(w, x, dx, ptr_kind, n);
    }
    if (!std::isfinite(bnorm)) return s->fail(S2L_ERR_NUMERIC, "non-finite right-hand side");
    double* r = w->d_r;
    double* z = w->d_z;
    double* wv = w->d_kw;
    // OpenFOAM test: sum|r| <= thr = max(rtol sum|r0|, atol F) (src/solver/gmres.cpp:41-56)
    double normF = 1.0, l1 = 0.0, thr = 0.0;
    if (of) {
        RET_IF(spmv_dev(w, dx, w->d_u, nullptr, false));
        RET_IF(of_norm_factor(w, db, dx, w->d_u, &normF));
    }
    RET_IF(spmv_dev(w, dx, r, db, true));
    RET_IF(read_red(w, 256, 1));
    double beta = std::sqrt(w->h_red[256]);
    hist(beta / bnorm);
    res->rel_residual = beta / bnorm;
    bool converged = false;
    if (of) {
        RET_IF(l1_dev(w, r, 0.0, nullptr, &l1, nullptr));
        res->initial_residual_of = l1 / normF;
        thr = std::max(o->rtol * l1, o->atol * normF);
        converged = l1 <= thr;  // x0 already satisfies the test: no iteration
    } else {
        converged = beta <= o->rtol * bnorm;
    }
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    auto Hc = [&](int i, int j) -> double& { return H[(size_t)j * (m + 1) + i]; };
    while (!converged && res->iterations < o->maxit) {
        if (!std::isfinite(beta)) return s->fail(S2L_ERR_NUMERIC, "non-finite residual");
        {
            Prof pr(w, PC_VEC);
            launch_axpby(st, n, 1.0 / beta, r, 0.0, V);
            w->launches += 1;
        }
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        std::fill(H.begin(), H.end(), 0.0);
        int k = 0;
        bool breakdown = false;
        for (int j = 0; j < m && res->iterations < o->maxit; ++j) {
            if (cancel && cancel->load(std::memory_order_relaxed)) return s->fail(S2L_ERR_CANCELED, "solve canceled");
            double* zj = flex ? Z + (size_t)j * n : z;
            RET_IF(apply_dev(w, V + (size_t)j * n, zj));
            RET_IF(spmv_dev(w, zj, wv, nullptr, false));
            {
                Prof pr(w, PC_VEC);
                launch_mdot(st, n, V, n, j + 1, wv, w->d_part, w->d_red);
                launch_gemv_update(st, n, V, n, j + 1, w->d_red, -1.0, wv, nullptr);
                launch_mdot(st, n, V, n, j + 1, wv, w->d_part, w->d_red + 128);
                launch_gemv_update(st, n, V, n, j + 1, w->d_red + 128, -1.0, wv, w->d_part);
                launch_reduce(st, w->d_part, S2L_NB_RED, 1, w->d_red + 256);
                w->launches += 7;
            }
            CUDA_OK(w, cudaMemcpyAsync(w->h_red, w->d_red, 257 * sizeof(double), cudaMemcpyDeviceToHost, st));
            RET_IF(check_err(w));
            const double hn = std::sqrt(w->h_red[256]);
            for (int i = 0; i <= j; ++i) Hc(i, j) = w->h_red[i] + w->h_red[128 + i];
            Hc(j + 1, j) = hn;
            if (hn > 0.0) {
                Prof pr(w, PC_VEC);
                launch_axpby(st, n, 1.0 / hn, wv, 0.0, V + (size_t)(j + 1) * n);
                w->launches += 1;
            }
            for (int i = 0; i < j; ++i) {
                const double t = cs[i] * Hc(i, j) + sn[i] * Hc(i + 1, j);
                Hc(i + 1, j) = -sn[i] * Hc(i, j) + cs[i] * Hc(i + 1, j);
                Hc(i, j) = t;
            }
            const double den = std::hypot(Hc(j, j), Hc(j + 1, j));
            cs[j] = den > 0.0 ? Hc(j, j) / den : 1.0;
            sn[j] = den > 0.0 ? Hc(j + 1, j) / den : 0.0;
            Hc(j, j) = den;
            Hc(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++k;
            ++res->iterations;
            res->rel_residual = std::fabs(g[j + 1]) / bnorm;
            hist(res->rel_residual);
            if (!std::isfinite(res->rel_residual)) return s->fail(S2L_ERR_NUMERIC, "non-finite GMRES residual");
            bool done = false;
            if (of) {
                // GMRES residual r_j = g_{j+1} V_{j+2} Q^T e_{j+1} (src/solver/gmres.cpp:106-123)
                if (hn == 0.0 || g[j + 1] == 0.0) {
                    l1 = 0.0;
                } else {
                    std::vector<double> q(j + 2, 0.0);
                    q[j + 1] = 1.0;
                    for (int i = j; i >= 0; --i) {
                        const double qa = q[i], qc = q[i + 1];
                        q[i] = cs[i] * qa - sn[i] * qc;
                        q[i + 1] = sn[i] * qa + cs[i] * qc;
                    }
                    double* dq = w->d_coef + S2L_MAX_RED_COLS;
                    CUDA_OK(w, cudaMemcpyAsync(dq, q.data(), (j + 2) * sizeof(double), cudaMemcpyHostToDevice, st));
                    {
                        Prof pr(w, PC_VEC);
                        launch_gemv_l1(st, n, V, n, j + 2, dq, w->d_part, w->d_red + 300);
                        w->launches += 2;
                    }
                    RET_IF(read_red(w, 300, 1));
                    l1 = std::fabs(g[j + 1]) * w->h_red[300];
                }
                done = l1 <= thr;
            } else {
                done = res->rel_residual <= o->rtol;
            }
            if (done) {
                converged = true;
                break;
            }
            if (hn == 0.0) {
                breakdown = true;
                break;
            }
        }
        // y = H_k^-1 g_k (upper triangular), x += M^-1 V_k y (or Z_k y)
        for (int i = k - 1; i >= 0; --i) {
            double t = g[i];
            for (int c = i + 1; c < k; ++c) t -= Hc(i, c) * y[c];
            y[i] = t / Hc(i, i);
        }
        CUDA_OK(w, cudaMemcpyAsync(w->d_coef, y.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
        {
            Prof pr(w, PC_VEC);
            launch_gemv(st, n, flex ? Z : V, n, k, w->d_coef, w->d_u);
            w->launches += 1;
        }
        if (flex) {
            Prof pr(w, PC_VEC);
            launch_axpby(st, n, 1.0, w->d_u, 1.0, dx);
            w->launches += 1;
        } else {
            RET_IF(apply_dev(w, w->d_u, z));
            Prof pr(w, PC_VEC);
            launch_axpby(st, n, 1.0, z, 1.0, dx);
            w->launches += 1;
        }
        RET_IF(spmv_dev(w, dx, r, db, true));
        RET_IF(read_red(w, 256, 1));
        beta = std::sqrt(w->h_red[256]);
        if (of) RET_IF(l1_dev(w, r, 0.0, nullptr, &l1, nullptr));
        const double slack = o->strict_true_residual ? 1.0 : 1.1;
        const bool within = of ? l1 <= thr : beta <= o->rtol * bnorm;
        const bool within_slack = of ? l1 <= slack * thr : beta <= slack * o->rtol * bnorm;
        if (breakdown) converged = within || converged;
        if (converged && !within_slack) converged = false;
        if (beta == 0.0) converged = true;
        if (!converged) ++res->restarts;
    }
    res->converged = converged ? 1 : 0;
    res->true_rel_residual = beta / bnorm;
    if (of) res->final_residual_of = l1 / normF;
    return finish_out(w, x, dx, ptr_kind, n);
}

// Right-preconditioned BiCGStab, L2 or OpenFOAM stopping test (src/solver/bicgstab.cpp:15-154).
static int bicgstab_run(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                        s2l_result* res, const std::atomic<int>* cancel)
{
    RET_IF(check_ready(s));
    if (!b || !x || !o || !res) return s->fail(S2L_ERR_BADARG, "null argument");
    if (o->maxit < 0 || !(o->rtol >= 0.0)) return s->fail(S2L_ERR_BADARG, "bad Krylov options");
    RET_IF(check_stop(s, o));
    const bool of = o->stop_norm == S2L_STOP_OPENFOAM;
    Lease lease(s, [&](s2l_work* lw) -> int {
        RET_IF(ensure_krylov(lw, 1, false));
        if (lw->d_rh) return S2L_OK;
        double* q[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        for (int i = 0; i < 6; ++i) {
            const int r = work_doubles(lw, &q[i], (size_t)s->n);
            if (r != S2L_OK) {
                for (int j = 0; j < i; ++j) work_free(lw, q[j]);
                return r;
            }
        }
        lw->d_rh = q[0];
        lw->d_p = q[1];
        lw->d_v = q[2];
        lw->d_s = q[3];
        lw->d_t = q[4];
        lw->d_yb = q[5];
        return S2L_OK;
    });
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    const int64_t n = s->n;
    cudaStream_t st = w->stream;
    const double* db;
    if (ptr_kind == S2L_PTR_HOST) {
        CUDA_OK(w, cudaMemcpyAsync(w->d_b, b, n * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(w, cudaMemcpyAsync(w->d_xk, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
        db = w->d_b;
    } else if (ptr_kind == S2L_PTR_DEVICE) {
        db = b;
        CUDA_OK(w, cudaMemcpyAsync(w->d_xk, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
        return s->fail(S2L_ERR_BADARG, "bad ptr_kind");
    }
    double* dx = w->d_xk;
    double *r = w->d_r, *rh = w->d_rh, *p = w->d_p, *v = w->d_v, *y = w->d_yb, *sv = w->d_s, *zv = w->d_z,
           *t = w->d_t;
    res->converged = 0;
    res->breakdown = 0;
    res->iterations = 0;
    res->restarts = 0;
    res->history_len = 0;
    res->initial_residual_of = res->final_residual_of = 0.0;
    auto hist = [&](double val) {
        if (res->history && res->history_len < o->history_cap) res->history[res->history_len] = val;
        if (res->history_len < o->history_cap) ++res->history_len;
    };
    double bnorm = 0.0;
    RET_IF(norm2_dev(w, db, &bnorm));
    if (bnorm == 0.0) {
        CUDA_OK(w, cudaMemsetAsync(dx, 0, n * sizeof(double), st));
        res->converged = 1;
        hist(0.0);
        res->rel_residual = res->true_rel_residual = 0.0;
        return finish_out(w, x, dx, ptr_kind, n);
    }
    // OpenFOAM test: sum|r| <= thr = max(rtol sum|r0|, atol F) (src/solver/bicgstab.cpp:33-66)
    double normF = 1.0, l1 = 0.0, thr = 0.0;
    if (of) {
        RET_IF(spmv_dev(w, dx, w->d_u, nullptr, false));
        RET_IF(of_norm_factor(w, db, dx, w->d_u, &normF));
    }
    RET_IF(spmv_dev(w, dx, r, db, true));
    RET_IF(read_red(w, 256, 1));
    double rn = std::sqrt(w->h_red[256]);
    if (of) {
        RET_IF(l1_dev(w, r, 0.0, nullptr, &l1, nullptr));
        res->initial_residual_of = l1 / normF;
        thr = std::max(o->rtol * l1, o->atol * normF);
    }
    hist(rn / bnorm);
    res->rel_residual = rn / bnorm;
    auto satisfied = [&](double slack) { return of ? l1 <= slack * thr : rn <= slack * o->rtol * bnorm; };
    for (;;) {
        if (satisfied(1.0)) {
            res->converged = 1;
            break;
        }
        if (res->iterations >= o->maxit) break;
        CUDA_OK(w, cudaMemcpyAsync(rh, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        const double rhn = rn;
        double rho = rn * rn, rho_old = 1.0, alpha = 1.0, omega = 1.0;
        bool first = true, candidate = false;
        while (res->iterations < o->maxit) {
            if (cancel && cancel->load(std::memory_order_relaxed)) return s->fail(S2L_ERR_CANCELED, "solve canceled");
            {
                Prof pr(w, PC_VEC);
                launch_bicg_p(st, n, r, v, first ? 0.0 : (rho / rho_old) * (alpha / omega), omega, p, first ? 1 : 0);
                w->launches += 1;
            }
            first = false;
            RET_IF(apply_dev(w, p, y));
            RET_IF(spmv_dev(w, y, v, nullptr, false));
            ++res->iterations;
            {
                Prof pr(w, PC_VEC);
                launch_dot2(st, n, rh, v, nullptr, w->d_part, w->d_red + 256);
                w->launches += 2;
            }
            RET_IF(read_red(w, 256, 1));
            const double rhv = w->h_red[256];
            if (rhv == 0.0 || !std::isfinite(rhv)) {
                res->breakdown = 1;
                break;
            }
            alpha = rho / rhv;
            {
                Prof pr(w, PC_VEC);
                launch_bicg_s(st, n, r, v, alpha, sv, w->d_part, w->d_red + 256);
                w->launches += 2;
            }
            RET_IF(read_red(w, 256, 1));
            rn = std::sqrt(w->h_red[256]);
            if (of) RET_IF(l1_dev(w, sv, 0.0, nullptr, &l1, nullptr));
            res->rel_residual = rn / bnorm;
            hist(res->rel_residual);
            if (satisfied(1.0) || res->iterations >= o->maxit) {
                Prof pr(w, PC_VEC);
                launch_axpby(st, n, alpha, y, 1.0, dx);
                w->launches += 1;
                CUDA_OK(w, cudaMemcpyAsync(r, sv, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
                candidate = satisfied(1.0);
                break;
            }
            RET_IF(apply_dev(w, sv, zv));
            RET_IF(spmv_dev(w, zv, t, nullptr, false));
            ++res->iterations;
            {
                Prof pr(w, PC_VEC);
                launch_dot2(st, n, t, t, sv, w->d_part, w->d_red + 256);
                w->launches += 2;
            }
            RET_IF(read_red(w, 256, 2));
            const double tt = w->h_red[256], ts = w->h_red[257];
            omega = tt > 0.0 ? ts / tt : 0.0;
            {
                Prof pr(w, PC_VEC);
                launch_bicg_x(st, n, dx, y, zv, alpha, omega, r, sv, t, rh, w->d_part, w->d_red + 256);
                w->launches += 2;
            }
            RET_IF(read_red(w, 256, 2));
            rho_old = rho;
            rn = std::sqrt(w->h_red[256]);
            rho = w->h_red[257];
            if (of) RET_IF(l1_dev(w, r, 0.0, nullptr, &l1, nullptr));
            res->rel_residual = rn / bnorm;
            hist(res->rel_residual);
            if (satisfied(1.0)) {
                candidate = true;
                break;
            }
            if (omega == 0.0 || std::fabs(rho) < 1e-14 * rhn * rn) break;
        }
        RET_IF(spmv_dev(w, dx, r, db, true));
        RET_IF(read_red(w, 256, 1));
        rn = std::sqrt(w->h_red[256]);
        if (of) RET_IF(l1_dev(w, r, 0.0, nullptr, &l1, nullptr));
        if (res->breakdown) break;
        if (candidate && satisfied(o->strict_true_residual ? 1.0 : 1.1)) {
            res->converged = 1;
            break;
        }
        if (res->iterations >= o->maxit) break;
        ++res->restarts;
    }
    res->true_rel_residual = rn / bnorm;
    if (of) res->final_residual_of = l1 / normF;
    return finish_out(w, x, dx, ptr_kind, n);
}

int s2l_gpu_gmres(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                  s2l_result* res)
{
    return gmres_run(s, b, x, ptr_kind, o, res, nullptr);
}

int s2l_gpu_bicgstab(s2l_setup* s, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                     s2l_result* res)
{
    return bicgstab_run(s, b, x, ptr_kind, o, res, nullptr);
}

// ------------------------------------------------------------------------------ block solves
// Stage k column-major vectors (host or device) into a block vector of K interleaved columns.
static int block_in(s2l_work* w, int K, int k, const double* src, int ptr_kind, double* dst)
{
    s2l_setup* s = w->s;
    const double* d = src;
    if (ptr_kind == S2L_PTR_HOST) {
        CUDA_OK(w, cudaMemcpyAsync(w->blk.u, src, (size_t)s->n * k * sizeof(double), cudaMemcpyHostToDevice, w->stream));
        d = w->blk.u;
    } else if (ptr_kind != S2L_PTR_DEVICE) {
        return w->fail(S2L_ERR_BADARG, "ptr_kind must be S2L_PTR_HOST or S2L_PTR_DEVICE");
    }
    launch_interleave(w->stream, s->n, K, k, d, dst);
    w->launches += 1;
    return S2L_OK;
}

static int block_out(s2l_work* w, int K, int k, const double* src, int ptr_kind, double* dst)
{
    s2l_setup* s = w->s;
    if (ptr_kind == S2L_PTR_HOST) {
        launch_deinterleave(w->stream, s->n, K, k, src, w->blk.u);
        CUDA_OK(w, cudaMemcpyAsync(dst, w->blk.u, (size_t)s->n * k * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
    } else {
        launch_deinterleave(w->stream, s->n, K, k, src, dst);
    }
    w->launches += 1;
    CUDA_OK(w, cudaStreamSynchronize(w->stream));
    CUDA_OK(w, cudaGetLastError());
    return check_err(w);
}

static int block_width(s2l_setup* s, int k, int* K)
{
    if (k < 1 || k > S2L_MAX_RHS) return s->fail(S2L_ERR_BADARG, "a block holds 1 to 16 right-hand sides");
    if (s->amgd.on) return s->fail(S2L_ERR_BADARG, "block solves need exact local factors (AMG: one right-hand side per call)");
    *K = 1;
    while (*K < k) *K <<= 1;
    return S2L_OK;
}

int s2l_gpu_apply_block(s2l_setup* s, int k, const double* r, double* z, int ptr_kind)
{
    RET_IF(check_ready(s));
    if (!r || !z) return s->fail(S2L_ERR_BADARG, "null vector");
    int K = 1;
    RET_IF(block_width(s, k, &K));
    Lease lease(s, [&](s2l_work* lw) { return ensure_block(lw, K, std::max(lw->blk.m, 1), lw->blk.flex); });
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    RET_IF(block_in(w, K, k, r, ptr_kind, w->blk.r));
    RET_IF(apply_block(w, K, w->blk.r, w->blk.z));
    return block_out(w, K, k, w->blk.z, ptr_kind, z);
}

// k right-hand sides solved together: the GMRES of s2l_gpu_gmres (src/solver/gmres.cpp:18-161) run
// in lockstep, each column with its own Hessenberg matrix, rotations, restarts and convergence;
// the preconditioner, the products with A and the orthogonalization act on all columns at once.
// A column that has converged, broken down or used maxit gets a zero basis vector, so the shared
// steps leave it unchanged.  L2 stopping test only.
static int gmres_block_one(s2l_setup* s, int k, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                           s2l_result* res)
{
    RET_IF(check_ready(s));
    if (!b || !x || !o || !res) return s->fail(S2L_ERR_BADARG, "null argument");
    if (o->restart < 1 || o->maxit < 0 || !(o->rtol >= 0.0)) return s->fail(S2L_ERR_BADARG, "bad Krylov options");
    RET_IF(check_stop(s, o));
    if (o->stop_norm != S2L_STOP_L2) return s->fail(S2L_ERR_BADARG, "block solves implement the L2 stopping test");
    int K = 1;
    RET_IF(block_width(s, k, &K));
    const int m = o->restart;
    if ((m + 1) * K > S2L_MAX_BLOCK_COLS) return s->fail(S2L_ERR_BADARG, "restart x right-hand sides too large");
    const bool flex = o->flexible != 0;
    Lease lease(s, [&](s2l_work* lw) { return ensure_block(lw, K, m, flex); });
    RET_IF(lease.rc);
    s2l_work* w = lease.w;
    s2l_work::Block& B = w->blk;
    const int64_t n = s->n, nK = n * K;
    cudaStream_t st = w->stream;
    RET_IF(block_in(w, K, k, b, ptr_kind, B.b));
    RET_IF(block_in(w, K, k, x, ptr_kind, B.xk));
    const int MC = S2L_MAX_BLOCK_COLS;
    auto read = [&](int off, int count) -> int {
        CUDA_OK(w, cudaMemcpyAsync(B.h_red + off, B.red + off, count * sizeof(double), cudaMemcpyDeviceToHost, st));
        return check_err(w);
    };
    auto upload = [&](double* dst, const double* src, int count) -> int {
        CUDA_OK(w, cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, st));
        return S2L_OK;
    };
    for (int r = 0; r < k; ++r) {
        res[r].converged = res[r].breakdown = res[r].iterations = res[r].restarts = 0;
        res[r].history_len = 0;
        res[r].rel_residual = res[r].true_rel_residual = 0.0;
        res[r].initial_residual_of = res[r].final_residual_of = 0.0;
    }
    auto hist = [&](int r, double v) {
        if (res[r].history && res[r].history_len < o->history_cap) res[r].history[res[r].history_len] = v;
        if (res[r].history_len < o->history_cap) ++res[r].history_len;
    };
    // ||b_r||
    {
        Prof pr(w, PC_VEC);
        launch_mdot_block(st, n, K, B.b, nK, 1, B.b, B.part, B.red);
        w->launches += 2;
    }
    RET_IF(read(0, K));
    std::vector<double> bnorm(K, 0.0), beta(K, 0.0);
    for (int r = 0; r < k; ++r) bnorm[r] = std::sqrt(B.h_red[r]);
    for (int r = 0; r < k; ++r)
        if (!std::isfinite(bnorm[r])) return s->fail(S2L_ERR_NUMERIC, "non-finite right-hand side");
    std::vector<char> active(K, 0);
    RET_IF(spmv_block(w, K, B.xk, B.r, B.b, true));
    RET_IF(read(2 * MC, K));
    for (int r = 0; r < k; ++r) {
        if (bnorm[r] == 0.0) {  // x = 0 (src/solver/gmres.cpp:27-32)
            res[r].converged = 1;
            hist(r, 0.0);
            continue;
        }
        beta[r] = std::sqrt(B.h_red[2 * MC + r]);
        hist(r, beta[r] / bnorm[r]);
        res[r].rel_residual = beta[r] / bnorm[r];
        active[r] = beta[r] > o->rtol * bnorm[r];
        res[r].converged = active[r] ? 0 : 1;
    }
    std::vector<double> H((size_t)K * (m + 1) * m), cs((size_t)K * m), sn((size_t)K * m), g((size_t)K * (m + 1));
    std::vector<double> scal(2 * K), coef((size_t)(m + 1) * K), y(m);
    std::vector<int> kr(K, 0);
    std::vector<char> run(K, 0), done(K, 0), brk(K, 0), cand(K, 0);
    auto Hc = [&](int r, int i, int j) -> double& { return H[((size_t)r * m + j) * (m + 1) + i]; };
    for (;;) {
        bool any = false;
        for (int r = 0; r < k; ++r) {
            run[r] = active[r] && res[r].iterations < o->maxit;
            any = any || run[r];
        }
        if (!any) break;
        for (int r = 0; r < K; ++r) {
            if (r < k && !std::isfinite(beta[r]) && run[r]) return s->fail(S2L_ERR_NUMERIC, "non-finite residual");
            scal[r] = r < k && run[r] ? 1.0 / beta[r] : 0.0;
            done[r] = r < k && run[r] ? 0 : 1;
            brk[r] = cand[r] = 0;
            kr[r] = 0;
        }
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        for (int r = 0; r < k; ++r) g[(size_t)r * (m + 1)] = beta[r];
        RET_IF(upload(B.scal, scal.data(), K));
        {
            Prof pr(w, PC_VEC);
            launch_axpby_block(st, n, K, B.scal, B.r, nullptr, B.V);
            w->launches += 1;
        }
        int jmax = 0;
        for (int j = 0; j < m; ++j) {
            bool step = false;
            for (int r = 0; r < k; ++r) step = step || !done[r];
            if (!step) break;
            double* Vj = B.V + (size_t)j * nK;
            double* Zj = flex ? B.Z + (size_t)j * nK : B.z;
            RET_IF(apply_block(w, K, Vj, Zj));
            RET_IF(spmv_block(w, K, Zj, B.kw, nullptr, false));
            {
                Prof pr(w, PC_VEC);
                launch_mdot_block(st, n, K, B.V, nK, j + 1, B.kw, B.part, B.red);
                launch_gemv_update_block(st, n, K, B.V, nK, j + 1, B.red, -1.0, B.kw, nullptr, nullptr);
                launch_mdot_block(st, n, K, B.V, nK, j + 1, B.kw, B.part, B.red + MC);
                launch_gemv_update_block(st, n, K, B.V, nK, j + 1, B.red + MC, -1.0, B.kw, B.part, B.red + 2 * MC);
                w->launches += 7;
            }
            CUDA_OK(w, cudaMemcpyAsync(B.h_red, B.red, 3 * MC * sizeof(double), cudaMemcpyDeviceToHost, st));
            RET_IF(check_err(w));
            for (int r = 0; r < K; ++r) scal[r] = 0.0;
            for (int r = 0; r < k; ++r) {
                if (done[r]) continue;
                const double hn = std::sqrt(B.h_red[2 * MC + r]);
                for (int i = 0; i <= j; ++i) Hc(r, i, j) = B.h_red[i * K + r] + B.h_red[MC + i * K + r];
                Hc(r, j + 1, j) = hn;
                double* c_ = &cs[(size_t)r * m];
                double* s_ = &sn[(size_t)r * m];
                double* g_ = &g[(size_t)r * (m + 1)];
                for (int i = 0; i < j; ++i) {
                    const double t = c_[i] * Hc(r, i, j) + s_[i] * Hc(r, i + 1, j);
                    Hc(r, i + 1, j) = -s_[i] * Hc(r, i, j) + c_[i] * Hc(r, i + 1, j);
                    Hc(r, i, j) = t;
                }
                const double den = std::hypot(Hc(r, j, j), Hc(r, j + 1, j));
                c_[j] = den > 0.0 ? Hc(r, j, j) / den : 1.0;
                s_[j] = den > 0.0 ? Hc(r, j + 1, j) / den : 0.0;
                Hc(r, j, j) = den;
                Hc(r, j + 1, j) = 0.0;
                g_[j + 1] = -s_[j] * g_[j];
                g_[j] = c_[j] * g_[j];
                ++kr[r];
                ++res[r].iterations;
                res[r].rel_residual = std::fabs(g_[j + 1]) / bnorm[r];
                hist(r, res[r].rel_residual);
                if (!std::isfinite(res[r].rel_residual)) return s->fail(S2L_ERR_NUMERIC, "non-finite GMRES residual");
                if (res[r].rel_residual <= o->rtol) {
                    cand[r] = 1;
                    done[r] = 1;
                } else if (hn == 0.0) {
                    brk[r] = 1;
                    done[r] = 1;
                } else if (res[r].iterations >= o->maxit) {
                    done[r] = 1;
                }
                if (!done[r]) scal[r] = 1.0 / hn;
            }
            jmax = j + 1;
            if (j + 1 < m) {  // V_{j+1}: columns still running get w / hn, the others zero
                RET_IF(upload(B.scal, scal.data(), K));
                Prof pr(w, PC_VEC);
                launch_axpby_block(st, n, K, B.scal, B.kw, nullptr, B.V + (size_t)(j + 1) * nK);
                w->launches += 1;
            }
        }
        // y_r = H_r^-1 g_r, x += M^-1 V y (or Z y)
        std::fill(coef.begin(), coef.end(), 0.0);
        for (int r = 0; r < k; ++r) {
            if (!run[r]) continue;
            const double* g_ = &g[(size_t)r * (m + 1)];
            for (int i = kr[r] - 1; i >= 0; --i) {
                double t = g_[i];
                for (int c = i + 1; c < kr[r]; ++c) t -= Hc(r, i, c) * y[c];
                y[i] = t / Hc(r, i, i);
            }
            for (int i = 0; i < kr[r]; ++i) coef[(size_t)i * K + r] = y[i];
        }
        for (int r = 0; r < K; ++r) scal[r] = scal[K + r] = 1.0;
        RET_IF(upload(B.coef, coef.data(), jmax * K));
        RET_IF(upload(B.scal, scal.data(), 2 * K));
        {
            Prof pr(w, PC_VEC);
            launch_gemv_block(st, n, K, flex ? B.Z : B.V, nK, jmax, B.coef, B.u);
            w->launches += 1;
        }
        if (flex) {
            Prof pr(w, PC_VEC);
            launch_axpby_block(st, n, K, B.scal, B.u, B.scal + K, B.xk);
            w->launches += 1;
        } else {
            RET_IF(apply_block(w, K, B.u, B.z));
            Prof pr(w, PC_VEC);
            launch_axpby_block(st, n, K, B.scal, B.z, B.scal + K, B.xk);
            w->launches += 1;
        }
        RET_IF(spmv_block(w, K, B.xk, B.r, B.b, true));
        RET_IF(read(2 * MC, K));
        for (int r = 0; r < k; ++r) {
            if (!run[r]) continue;
            beta[r] = std::sqrt(B.h_red[2 * MC + r]);
            const double slack = o->strict_true_residual ? 1.0 : 1.1;
            const bool within = beta[r] <= o->rtol * bnorm[r];
            const bool within_slack = beta[r] <= slack * o->rtol * bnorm[r];
            bool conv = cand[r] != 0;
            if (brk[r]) conv = within || conv;
            if (conv && !within_slack) conv = false;
            if (beta[r] == 0.0) conv = true;
            res[r].converged = conv ? 1 : 0;
            res[r].true_rel_residual = beta[r] / bnorm[r];
            if (conv) active[r] = 0;
            else ++res[r].restarts;
        }
    }
    RET_IF(block_out(w, K, k, B.xk, ptr_kind, x));
    for (int r = 0; r < k; ++r) {
        if (bnorm[r] != 0.0) continue;
        if (ptr_kind == S2L_PTR_HOST) std::fill(x + (size_t)r * n, x + (size_t)(r + 1) * n, 0.0);
        else CUDA_OK(w, cudaMemsetAsync(x + (size_t)r * n, 0, n * sizeof(double), st));
    }
    CUDA_OK(w, cudaStreamSynchronize(st));
    return S2L_OK;
}

// k right-hand sides: sub-blocks of the best width, run at once on their own workspaces
static int gmres_block_run(s2l_setup* s, int k, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                           s2l_result* res)
{
    RET_IF(check_ready(s));
    if (!b || !x || !o || !res) return s->fail(S2L_ERR_BADARG, "null argument");
    if (k < 1 || k > S2L_MAX_RHS) return s->fail(S2L_ERR_BADARG, "a block holds 1 to 16 right-hand sides");
    if (s->amgd.on) return s->fail(S2L_ERR_BADARG, "block solves need exact local factors (AMG: one right-hand side per call)");
    const int wb = block_width_best(s);
    if (k <= wb) return gmres_block_one(s, k, b, x, ptr_kind, o, res);
    const int64_t n = s->n;
    const int parts = (k + wb - 1) / wb;
    std::vector<int> rc(parts, S2L_OK);
    std::vector<std::thread> th;
    for (int p = 1; p < parts; ++p)
        th.emplace_back([&, p] {
            const int off = p * wb, kk = std::min(wb, k - off);
            rc[p] = gmres_block_one(s, kk, b + off * n, x + off * n, ptr_kind, o, res + off);
        });
    rc[0] = gmres_block_one(s, std::min(wb, k), b, x, ptr_kind, o, res);
    for (auto& t : th) t.join();
    for (int v : rc)
        if (v != S2L_OK) return v;
    return S2L_OK;
}

int s2l_gpu_gmres_block(s2l_setup* s, int k, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* o,
                        s2l_result* results)
{
    return gmres_block_run(s, k, b, x, ptr_kind, o, results);
}

// ------------------------------------------------------------------------------ batched solves
int s2l_gpu_solve_batch(s2l_setup* s, int method, int k, const double* const* b, double* const* x, int ptr_kind,
                        const s2l_krylov_opts* opts, s2l_result* results, int* status)
{
    RET_IF(check_ready(s));
    if (k < 1 || !b || !x || !opts || !results || !status) return s->fail(S2L_ERR_BADARG, "bad batch arguments");
    if (method != S2L_KRYLOV_GMRES && method != S2L_KRYLOV_BICGSTAB)
        return s->fail(S2L_ERR_BADARG, "unknown Krylov method");
    auto one = [&](int j) {
        status[j] = method == S2L_KRYLOV_GMRES ? gmres_run(s, b[j], x[j], ptr_kind, opts, &results[j], nullptr)
                                               : bicgstab_run(s, b[j], x[j], ptr_kind, opts, &results[j], nullptr);
    };
    std::vector<std::thread> th;
    th.reserve(k - 1);
    for (int j = 1; j < k; ++j) th.emplace_back(one, j);
    one(0);
    for (auto& t : th) t.join();
    for (int j = 0; j < k; ++j)
        if (status[j] != S2L_OK) return status[j];
    return S2L_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------ asynchronous solves
struct s2l_ticket {
    s2l_setup* s = nullptr;
    int method = S2L_KRYLOV_GMRES;
    const double* b = nullptr;
    double* x = nullptr;
    int ptr_kind = S2L_PTR_HOST;
    s2l_krylov_opts opts{};
    s2l_result* res = nullptr;
    std::atomic<int> state{S2L_JOB_QUEUED};
    std::atomic<int> cancel{0};
    int status = S2L_OK;
    std::string err;
    std::chrono::steady_clock::time_point t_submit, t_start, t_end;
    std::mutex mu;
    std::condition_variable cv;
};

namespace {

void ticket_finish(s2l_ticket* t, int state, int status)
{
    {
        std::lock_guard<std::mutex> g(t->mu);
        t->status = status;
        t->t_end = std::chrono::steady_clock::now();
        t->state.store(state);
    }
    t->s->pending.fetch_sub(1);
    t->cv.notify_all();
}

// ------------------------------------------------------------------------------ continuous batching
// A block runner serves the GMRES requests of one setup (same restart length and variant) from one
// workspace: up to K requests at once, each in a column slot of a block of K right-hand sides.
// Every Arnoldi step runs the preconditioner, the product with A and both CGS2 passes once for all
// occupied slots; each column keeps its own Hessenberg matrix, rotations, restart cycle and
// convergence test (src/solver/gmres.cpp:18-161).  A request that arrives while the others run
// takes a free slot at the next step boundary and starts its own cycle there; a column that
// converges (or uses maxit) writes its solution out and frees its slot at once.
//
// Columns start their cycles at different steps, so the basis is a ring of restart + 1 blocks:
// the basis vector of every running column at global step T sits in block T % (restart + 1), and a
// column whose cycle started at step t0 owns the blocks of steps t0 .. T.  The orthogonalization
// runs over the union of these windows with the coefficients of blocks outside a column's own
// window set to zero: each column then computes exactly what it computes alone (the extra terms
// add exact zeros), whatever the other slots hold.
struct Runner {
    s2l_setup* s = nullptr;
    int m = 0;
    bool flex = false;
    int K = 1;
    int free_slots = 0;  // slots not holding a request (guarded by the serve mutex)
};

bool batchable(const s2l_serve* sv, const s2l_ticket* t)
{
    const s2l_setup* s = t->s;
    return sv->slots != 0 && t->method == S2L_KRYLOV_GMRES && t->opts.stop_norm == S2L_STOP_L2 &&
           t->opts.atol == 0.0 && !s->amgd.on && t->opts.restart >= 1 && t->opts.restart <= 63 &&
           t->opts.maxit >= 0 && t->opts.rtol >= 0.0;
}

bool runner_takes(const Runner* R, const s2l_ticket* t)
{
    return R->s == t->s && R->m == t->opts.restart && R->flex == (t->opts.flexible != 0);
}

// slots of a runner on setup s with restart m: the setting of s2l_gpu_serve_batching, or
// automatically the setup's best block width but at most 4 (a step costs about the same for 1 to 4
// occupied columns, so a lightly loaded runner stays as fast as a single solve; more load starts
// more runners), and never more than the coefficient buffers hold
int runner_width(const s2l_serve* sv, s2l_setup* s, int m)
{
    int K = sv->slots > 0 ? sv->slots : std::min(block_width_best(s), 4);
    int p = 1;
    while (p * 2 <= K && p * 2 <= S2L_MAX_RHS && (m + 1) * p * 2 <= S2L_MAX_BLOCK_COLS) p *= 2;
    return p;
}

struct Slot {
    s2l_ticket* t = nullptr;
    bool run = false;      // a restart cycle is running
    bool ending = false;   // its cycle ended at the last step: solution update and restart test
    bool cand = false, brk = false;
    int64_t t0 = 0;        // global step of the cycle's first basis vector
    int kr = 0;            // steps of the cycle so far
    double bnorm = 0.0, beta = 0.0, hn = 0.0;
    std::vector<double> H, cs, sn, g;
};

void slot_reset_cycle(Slot& c, int m)
{
    std::fill(c.H.begin(), c.H.end(), 0.0);
    std::fill(c.g.begin(), c.g.end(), 0.0);
    c.kr = 0;
    c.cand = c.brk = false;
    (void)m;
}

void block_runner(s2l_ctx* ctx, Runner* R, s2l_ticket* first)
{
    s2l_serve* sv = ctx->serve;
    s2l_setup* s = R->s;
    const int m = R->m, ring = m + 1;
    const bool flex = R->flex;
    std::vector<s2l_ticket*> incoming{first};
    std::vector<Slot> slots;
    // leaves the runner: every ticket still held fails with rc, the runner is deregistered
    auto leave = [&](int rc, const std::string& msg) {
        std::vector<s2l_ticket*> held;
        for (auto& c : slots)
            if (c.t) held.push_back(c.t);
        for (s2l_ticket* t : incoming) held.push_back(t);
        {
            std::lock_guard<std::mutex> g(sv->mu);
            auto it = std::find(sv->runners.begin(), sv->runners.end(), R);
            if (it != sv->runners.end()) sv->runners.erase(it);
        }
        sv->cv.notify_all();
        for (s2l_ticket* t : held) {
            t->err = msg;
            ticket_finish(t, rc == S2L_ERR_CANCELED ? S2L_JOB_CANCELED : S2L_JOB_DONE, rc);
        }
        delete R;
    };
    // the block buffers of K slots; when they do not fit the HBM budget (and no other workspace of
    // the setup is busy to wait for), half as many slots
    t_last_error.clear();
    std::unique_ptr<Lease> lease;
    for (;;) {
        const int Kt = R->K;
        lease.reset(new Lease(s, [&](s2l_work* lw) { return ensure_block(lw, Kt, m, flex); }));
        if (lease->rc == S2L_ERR_OOM && Kt > 1) {
            lease.reset();
            std::lock_guard<std::mutex> g(sv->mu);
            R->K = Kt / 2;
            R->free_slots = R->K - 1;
            continue;
        }
        break;
    }
    if (lease->rc != S2L_OK) {
        leave(lease->rc, t_last_error);
        return;
    }
    const int K = R->K;
    slots.resize(K);
    for (auto& c : slots) {
        c.H.assign((size_t)(m + 1) * m, 0.0);
        c.cs.assign(m, 0.0);
        c.sn.assign(m, 0.0);
        c.g.assign(m + 1, 0.0);
    }
    s2l_work* w = lease->w;
    s2l_work::Block& B = w->blk;
    const int64_t n = s->n, nK = n * K;
    cudaStream_t st = w->stream;
    const int MC = S2L_MAX_BLOCK_COLS;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        leave(S2L_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    // a clean block: every ring block, the right-hand sides, iterates and work vectors zero
    {
        cudaError_t e = cudaSuccess;
        for (double* p : {B.V, B.Z, B.b, B.xk, B.kw, B.r, B.z, B.u})
            if (p && e == cudaSuccess)
                e = cudaMemsetAsync(p, 0, (size_t)nK * sizeof(double) * (p == B.V || p == B.Z ? ring : 1), st);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    }
    auto read = [&](int off, int count) -> int {
        const cudaError_t e = cudaMemcpyAsync(B.h_red + off, B.red + off, count * sizeof(double),
                                              cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return w->fail(S2L_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
        return check_err(w);
    };
    auto hist = [&](Slot& c, double v) {
        s2l_result* res = c.t->res;
        if (res->history && res->history_len < c.t->opts.history_cap) res->history[res->history_len] = v;
        if (res->history_len < c.t->opts.history_cap) ++res->history_len;
    };
    auto Hc = [&](Slot& c, int i, int j) -> double& { return c.H[(size_t)j * (m + 1) + i]; };
    std::vector<int> done_slots;  // finished at this boundary: tickets to complete after the copies
    std::vector<int> done_state, done_status;
    std::vector<std::string> done_err;
    auto complete = [&](int r, int state, int status, const std::string& err) {
        done_slots.push_back(r);
        done_state.push_back(state);
        done_status.push_back(status);
        done_err.push_back(err);
    };
    // solution column r out to its ticket (host or device), queued on the stream
    auto write_out = [&](int r) -> int {
        s2l_ticket* t = slots[r].t;
        if (t->ptr_kind == S2L_PTR_DEVICE) {
            launch_column_out(st, n, K, r, B.xk, t->x);
            w->launches += 1;
        } else {
            double* stage = B.u;  // n doubles; the outputs of one boundary go one after another
            launch_column_out(st, n, K, r, B.xk, stage);
            w->launches += 1;
            CUDA_OK(w, cudaMemcpyAsync(t->x, stage, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
            CUDA_OK(w, cudaStreamSynchronize(st));
        }
        return S2L_OK;
    };
    int64_t T = 0;  // the next Arnoldi step
    for (;;) {
        // ---------------------------------------------------------------- boundary before step T
        done_slots.clear();
        done_state.clear();
        done_status.clear();
        done_err.clear();
        for (int r = 0; r < K; ++r)
            if (slots[r].t && slots[r].t->cancel.load()) {
                complete(r, S2L_JOB_CANCELED, S2L_ERR_CANCELED, "solve canceled");
                slots[r].run = slots[r].ending = false;
            }
        // requests queued for this runner take the free slots
        {
            std::lock_guard<std::mutex> g(sv->mu);
            int freeable = 0;
            for (int r = 0; r < K; ++r)
                if (!slots[r].t) ++freeable;
            freeable -= (int)incoming.size();
            for (auto it = sv->queue.begin(); it != sv->queue.end() && freeable > 0;) {
                if (runner_takes(R, *it) && batchable(sv, *it) && !(*it)->cancel.load()) {
                    incoming.push_back(*it);
                    it = sv->queue.erase(it);
                    --freeable;
                    --R->free_slots;
                } else {
                    ++it;
                }
            }
        }
        std::vector<int> adm;
        for (s2l_ticket* t : incoming) {
            int r = 0;
            while (slots[r].t) ++r;
            slots[r].t = t;
            slots[r].run = slots[r].ending = false;
            t->t_start = std::chrono::steady_clock::now();
            t->state.store(S2L_JOB_RUNNING);
            s2l_result* res = t->res;
            res->converged = res->breakdown = res->iterations = res->restarts = 0;
            res->history_len = 0;
            res->rel_residual = res->true_rel_residual = 0.0;
            res->initial_residual_of = res->final_residual_of = 0.0;
            adm.push_back(r);
        }
        incoming.clear();
        bool any_end = false;
        for (int r = 0; r < K; ++r) any_end = any_end || slots[r].ending;
        int rc = S2L_OK;
        if (any_end) {
            // x += Z y (flexible) or x += M^-1 (V y) for the columns whose cycle ended at step T - 1
            int64_t tmin = T;
            for (int r = 0; r < K; ++r)
                if (slots[r].ending) tmin = std::min(tmin, slots[r].t0);
            const int Lw = (int)(T - tmin);
            std::vector<double> coef((size_t)Lw * K, 0.0), y(m);
            for (int r = 0; r < K; ++r) {
                Slot& c = slots[r];
                if (!c.ending) continue;
                for (int i = c.kr - 1; i >= 0; --i) {
                    double v = c.g[i];
                    for (int q = i + 1; q < c.kr; ++q) v -= Hc(c, i, q) * y[q];
                    y[i] = v / Hc(c, i, i);
                }
                const int off = (int)(c.t0 - tmin);
                for (int i = 0; i < c.kr; ++i) coef[(size_t)(off + i) * K + r] = y[i];
            }
            cudaError_t e = cudaMemcpyAsync(B.coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
            {
                Prof pr(w, PC_VEC);
                launch_gemv_block(st, n, K, flex ? B.Z : B.V, nK, Lw, B.coef, B.u, (int)(tmin % ring), ring);
                w->launches += 1;
            }
            ColScale one{};
            for (int r = 0; r < K; ++r) one.v[r] = 1.0;
            if (flex) {
                Prof pr(w, PC_VEC);
                launch_combine2_block(st, n, K, one, B.u, one, B.xk, B.xk);
                w->launches += 1;
            } else {
                rc = apply_block(w, K, B.u, B.z);
                if (rc != S2L_OK) return leave(rc, t_last_error);
                Prof pr(w, PC_VEC);
                launch_combine2_block(st, n, K, one, B.z, one, B.xk, B.xk);
                w->launches += 1;
            }
        }
        // the admitted requests' right-hand sides and initial guesses into their columns
        for (int r : adm) {
            s2l_ticket* t = slots[r].t;
            const double* src[2] = {t->b, t->x};
            double* dst[2] = {B.b, B.xk};
            for (int q = 0; q < 2; ++q) {
                if (t->ptr_kind == S2L_PTR_HOST) {
                    cudaError_t e = cudaMemcpyAsync(B.u, src[q], (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
                    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
                    launch_column_in(st, n, K, r, B.u, dst[q]);
                } else {
                    launch_column_in(st, n, K, r, src[q], dst[q]);
                }
                w->launches += 1;
            }
        }
        if (any_end || !adm.empty()) {
            if (!adm.empty()) {
                Prof pr(w, PC_VEC);
                launch_mdot_block(st, n, K, B.b, nK, 1, B.b, B.part, B.red);
                w->launches += 2;
            }
            rc = spmv_block(w, K, B.xk, B.r, B.b, true);
            if (rc == S2L_OK && !adm.empty()) rc = read(0, K);
            if (rc == S2L_OK) rc = read(2 * MC, K);
            if (rc != S2L_OK) return leave(rc, t_last_error);
            for (int r = 0; r < K; ++r) {
                Slot& c = slots[r];
                if (!c.ending) continue;
                c.ending = false;
                s2l_result* res = c.t->res;
                const s2l_krylov_opts& o = c.t->opts;
                c.beta = std::sqrt(B.h_red[2 * MC + r]);
                const double slack = o.strict_true_residual ? 1.0 : 1.1;
                const bool within = c.beta <= o.rtol * c.bnorm;
                const bool within_slack = c.beta <= slack * o.rtol * c.bnorm;
                bool conv = c.cand;
                if (c.brk) conv = within || conv;
                if (conv && !within_slack) conv = false;
                if (c.beta == 0.0) conv = true;
                res->converged = conv ? 1 : 0;
                res->true_rel_residual = c.beta / c.bnorm;
                if (!std::isfinite(c.beta)) {
                    complete(r, S2L_JOB_DONE, S2L_ERR_NUMERIC, "non-finite residual");
                    c.run = false;
                } else if (conv || res->iterations >= o.maxit) {
                    if (write_out(r) != S2L_OK) return leave(S2L_ERR_CUDA, t_last_error);
                    complete(r, S2L_JOB_DONE, S2L_OK, "");
                    c.run = false;
                } else {
                    ++res->restarts;
                    slot_reset_cycle(c, m);
                    c.t0 = T;
                    c.run = true;
                }
            }
            for (int r : adm) {
                Slot& c = slots[r];
                s2l_result* res = c.t->res;
                const s2l_krylov_opts& o = c.t->opts;
                c.bnorm = std::sqrt(B.h_red[r]);
                c.beta = std::sqrt(B.h_red[2 * MC + r]);
                if (!std::isfinite(c.bnorm)) {
                    complete(r, S2L_JOB_DONE, S2L_ERR_NUMERIC, "non-finite right-hand side");
                    continue;
                }
                if (c.bnorm == 0.0) {  // x = 0 (src/solver/gmres.cpp:27-32)
                    hist(c, 0.0);
                    res->converged = 1;
                    launch_column_fill(st, n, K, r, 1, nK, 0.0, B.xk);
                    w->launches += 1;
                    if (write_out(r) != S2L_OK) return leave(S2L_ERR_CUDA, t_last_error);
                    complete(r, S2L_JOB_DONE, S2L_OK, "");
                    continue;
                }
                if (!std::isfinite(c.beta)) {
                    complete(r, S2L_JOB_DONE, S2L_ERR_NUMERIC, "non-finite residual");
                    continue;
                }
                hist(c, c.beta / c.bnorm);
                res->rel_residual = c.beta / c.bnorm;
                res->true_rel_residual = c.beta / c.bnorm;
                if (c.beta <= o.rtol * c.bnorm || o.maxit <= 0) {
                    res->converged = c.beta <= o.rtol * c.bnorm ? 1 : 0;
                    if (write_out(r) != S2L_OK) return leave(S2L_ERR_CUDA, t_last_error);
                    complete(r, S2L_JOB_DONE, S2L_OK, "");
                    continue;
                }
                slot_reset_cycle(c, m);
                c.t0 = T;
                c.run = true;
            }
        }
        // complete the finished tickets (their solutions are on the host or queued before the
        // stream synchronization below); a column that failed is cleared in every ring block so
        // no non-finite value stays behind for the next request of that slot
        if (!done_slots.empty()) {
            for (size_t q = 0; q < done_slots.size(); ++q)
                if (done_status[q] != S2L_OK && done_status[q] != S2L_ERR_CANCELED) {
                    const int r = done_slots[q];
                    launch_column_fill(st, n, K, r, ring, nK, 0.0, B.V);
                    if (flex) launch_column_fill(st, n, K, r, ring, nK, 0.0, B.Z);
                    launch_column_fill(st, n, K, r, 1, nK, 0.0, B.kw);
                    w->launches += flex ? 3 : 2;
                }
            const cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
            {
                std::lock_guard<std::mutex> g(sv->mu);
                R->free_slots += (int)done_slots.size();
            }
            for (size_t q = 0; q < done_slots.size(); ++q) {
                Slot& c = slots[done_slots[q]];
                s2l_ticket* t = c.t;
                c.t = nullptr;
                c.run = c.ending = false;
                if (!done_err[q].empty()) t->err = done_err[q];
                ticket_finish(t, done_state[q], done_status[q]);
            }
            sv->cv.notify_all();
        }
        bool any_run = false;
        for (int r = 0; r < K; ++r) any_run = any_run || slots[r].run;
        if (!any_run) {
            // nothing running: leave unless a request for this runner is queued
            std::lock_guard<std::mutex> g(sv->mu);
            bool more = false;
            for (s2l_ticket* t : sv->queue)
                more = more || (runner_takes(R, t) && batchable(sv, t) && !t->cancel.load());
            if (!more) {
                auto it = std::find(sv->runners.begin(), sv->runners.end(), R);
                if (it != sv->runners.end()) sv->runners.erase(it);
                sv->cv.notify_all();
                delete R;
                return;
            }
            continue;
        }
        // ---------------------------------------------------------------- Arnoldi step T
        const int p = (int)(T % ring);
        ColScale a{}, c0{};
        for (int r = 0; r < K; ++r) {
            const Slot& c = slots[r];
            if (!c.run) continue;
            if (c.t0 == T) c0.v[r] = 1.0 / c.beta;  // first vector of a cycle: r / beta
            else a.v[r] = 1.0 / c.hn;               // next vector: w / h(j + 1, j)
        }
        double* Vp = B.V + (size_t)p * nK;
        {
            Prof pr(w, PC_VEC);
            launch_combine2_block(st, n, K, a, B.kw, c0, B.r, Vp);
            w->launches += 1;
        }
        double* Zp = flex ? B.Z + (size_t)p * nK : B.z;
        rc = apply_block(w, K, Vp, Zp);
        if (rc == S2L_OK) rc = spmv_block(w, K, Zp, B.kw, nullptr, false);
        if (rc != S2L_OK) return leave(rc, t_last_error);
        int64_t tmin = T;
        for (int r = 0; r < K; ++r)
            if (slots[r].run) tmin = std::min(tmin, slots[r].t0);
        const int Lw = (int)(T - tmin + 1), j0 = (int)(tmin % ring);
        ColFirst first{};
        for (int r = 0; r < K; ++r) first.f[r] = slots[r].run ? (int)(slots[r].t0 - tmin) : Lw;
        {
            Prof pr(w, PC_VEC);
            launch_mdot_block(st, n, K, B.V, nK, Lw, B.kw, B.part, B.red, j0, ring);
            launch_gemv_update_block(st, n, K, B.V, nK, Lw, B.red, -1.0, B.kw, nullptr, nullptr, j0, ring, &first);
            launch_mdot_block(st, n, K, B.V, nK, Lw, B.kw, B.part, B.red + MC, j0, ring);
            launch_gemv_update_block(st, n, K, B.V, nK, Lw, B.red + MC, -1.0, B.kw, B.part, B.red + 2 * MC, j0, ring,
                                     &first);
            w->launches += 7;
        }
        {
            const cudaError_t e = cudaMemcpyAsync(B.h_red, B.red, 3 * MC * sizeof(double), cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
            rc = check_err(w);
            if (rc != S2L_OK) return leave(rc, t_last_error);
        }
        for (int r = 0; r < K; ++r) {
            Slot& c = slots[r];
            if (!c.run) continue;
            s2l_result* res = c.t->res;
            const s2l_krylov_opts& o = c.t->opts;
            const int j = (int)(T - c.t0);
            const int f = first.f[r];
            const double hn = std::sqrt(B.h_red[2 * MC + r]);
            for (int i = 0; i <= j; ++i) Hc(c, i, j) = B.h_red[(f + i) * K + r] + B.h_red[MC + (f + i) * K + r];
            Hc(c, j + 1, j) = hn;
            for (int i = 0; i < j; ++i) {
                const double tt = c.cs[i] * Hc(c, i, j) + c.sn[i] * Hc(c, i + 1, j);
                Hc(c, i + 1, j) = -c.sn[i] * Hc(c, i, j) + c.cs[i] * Hc(c, i + 1, j);
                Hc(c, i, j) = tt;
            }
            const double den = std::hypot(Hc(c, j, j), Hc(c, j + 1, j));
            c.cs[j] = den > 0.0 ? Hc(c, j, j) / den : 1.0;
            c.sn[j] = den > 0.0 ? Hc(c, j + 1, j) / den : 0.0;
            Hc(c, j, j) = den;
            Hc(c, j + 1, j) = 0.0;
            if (j == 0) c.g[0] = c.beta;
            c.g[j + 1] = -c.sn[j] * c.g[j];
            c.g[j] = c.cs[j] * c.g[j];
            c.kr = j + 1;
            ++res->iterations;
            res->rel_residual = std::fabs(c.g[j + 1]) / c.bnorm;
            hist(c, res->rel_residual);
            bool end = false;
            if (!std::isfinite(res->rel_residual)) {
                end = true;  // the boundary's residual check reports it
            } else if (res->rel_residual <= o.rtol) {
                c.cand = true;
                end = true;
            } else if (hn == 0.0) {
                c.brk = true;
                res->breakdown = 1;
                end = true;
            } else if (res->iterations >= o.maxit || j + 1 == m) {
                end = true;
            }
            c.hn = hn;
            if (end) {
                c.run = false;
                c.ending = true;
            }
        }
        ++T;
    }
}

// The next ticket this worker runs (serve mutex held): the first queued one that no block runner
// with a free slot is going to take.  A batchable ticket starts a new runner (returned in *nr).
s2l_ticket* pick_ticket(s2l_serve* sv, Runner** nr)
{
    *nr = nullptr;
    std::vector<int> room;  // free slots of each runner not yet promised to a queued ticket
    for (Runner* R : sv->runners) room.push_back(R->free_slots);
    for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
        s2l_ticket* t = *it;
        if (batchable(sv, t) && !t->cancel.load()) {
            bool promised = false;
            for (size_t q = 0; q < sv->runners.size() && !promised; ++q)
                if (room[q] > 0 && runner_takes(sv->runners[q], t)) {
                    --room[q];
                    promised = true;
                }
            if (promised) continue;
            auto* R = new Runner;
            R->s = t->s;
            R->m = t->opts.restart;
            R->flex = t->opts.flexible != 0;
            R->K = runner_width(sv, t->s, R->m);
            R->free_slots = R->K - 1;
            sv->runners.push_back(R);
            t->s->runners.fetch_add(1);
            *nr = R;
        }
        sv->queue.erase(it);
        return t;
    }
    return nullptr;
}

void serve_worker(s2l_ctx* ctx)
{
    s2l_serve* sv = ctx->serve;
    cudaSetDevice(ctx->device);
    for (;;) {
        s2l_ticket* t = nullptr;
        Runner* R = nullptr;
        {
            std::unique_lock<std::mutex> g(sv->mu);
            for (;;) {
                t = pick_ticket(sv, &R);
                if (t) break;
                if (sv->stop && sv->queue.empty()) return;  // stop requested and nothing left
                sv->cv.wait(g);
            }
        }
        if (R) {  // continuous batching: this worker runs the block runner until it has no request left
            s2l_setup* s = R->s;
            block_runner(ctx, R, t);
            s->runners.fetch_sub(1);
            continue;
        }
        if (t->cancel.load()) {
            t->err = "solve canceled before it started";
            ticket_finish(t, S2L_JOB_CANCELED, S2L_ERR_CANCELED);
            continue;
        }
        t->t_start = std::chrono::steady_clock::now();
        t->state.store(S2L_JOB_RUNNING);
        t_last_error.clear();
        const int rc = t->method == S2L_KRYLOV_GMRES
                           ? gmres_run(t->s, t->b, t->x, t->ptr_kind, &t->opts, t->res, &t->cancel)
                           : bicgstab_run(t->s, t->b, t->x, t->ptr_kind, &t->opts, t->res, &t->cancel);
        if (rc != S2L_OK) t->err = t_last_error;
        ticket_finish(t, rc == S2L_ERR_CANCELED ? S2L_JOB_CANCELED : S2L_JOB_DONE, rc);
    }
}

void serve_stop(s2l_ctx* ctx)
{
    s2l_serve* sv = ctx->serve;
    if (!sv) return;
    std::deque<s2l_ticket*> left;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop = true;
        left.swap(sv->queue);
    }
    for (s2l_ticket* t : left) {
        t->err = "context destroyed before the solve started";
        ticket_finish(t, S2L_JOB_CANCELED, S2L_ERR_CANCELED);
    }
    sv->cv.notify_all();
    for (auto& w : sv->workers) w.join();
    delete sv;
    ctx->serve = nullptr;
}

}  // namespace

extern "C" {

int s2l_gpu_serve_start(s2l_ctx* ctx, int workers)
{
    if (!ctx || workers < 1 || workers > 256) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (ctx->serve) {
        ctx->err = "the worker threads are already running";
        return S2L_ERR_STATE;
    }
    ctx->serve = new s2l_serve;
    for (int i = 0; i < workers; ++i) ctx->serve->workers.emplace_back(serve_worker, ctx);
    return S2L_OK;
}

int s2l_gpu_serve_batching(s2l_ctx* ctx, int slots)
{
    if (!ctx || slots > S2L_MAX_RHS) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->serve) {
        ctx->err = "s2l_gpu_serve_start was not called on this context";
        return S2L_ERR_STATE;
    }
    std::lock_guard<std::mutex> q(ctx->serve->mu);
    ctx->serve->slots = slots < 0 ? -1 : slots;
    return S2L_OK;
}

int s2l_gpu_submit(s2l_setup* s, int method, const double* b, double* x, int ptr_kind, const s2l_krylov_opts* opts,
                   s2l_result* result, s2l_ticket** ticket)
{
    RET_IF(check_ready(s));
    if (!ticket) return s->fail(S2L_ERR_BADARG, "null ticket");
    *ticket = nullptr;
    if (!b || !x || !opts || !result) return s->fail(S2L_ERR_BADARG, "null argument");
    if (method != S2L_KRYLOV_GMRES && method != S2L_KRYLOV_BICGSTAB)
        return s->fail(S2L_ERR_BADARG, "unknown Krylov method");
    s2l_serve* sv = s->ctx->serve;
    if (!sv) return s->fail(S2L_ERR_STATE, "s2l_gpu_serve_start was not called on this context");
    auto* t = new s2l_ticket;
    t->s = s;
    t->method = method;
    t->b = b;
    t->x = x;
    t->ptr_kind = ptr_kind;
    t->opts = *opts;
    t->res = result;
    t->t_submit = std::chrono::steady_clock::now();
    s->pending.fetch_add(1);
    {
        std::lock_guard<std::mutex> g(sv->mu);
        if (sv->stop) {
            s->pending.fetch_sub(1);
            delete t;
            return s->fail(S2L_ERR_STATE, "the worker threads are stopping");
        }
        sv->queue.push_back(t);
    }
    sv->cv.notify_all();  // an idle worker, or none when a block runner has a slot for it
    *ticket = t;
    return S2L_OK;
}

int s2l_gpu_poll(s2l_ticket* t, int* state)
{
    if (!t || !state) return S2L_ERR_BADARG;
    *state = t->state.load();
    return S2L_OK;
}

int s2l_gpu_wait(s2l_ticket* t, double timeout_s, int* status)
{
    if (!t) return S2L_ERR_BADARG;
    std::unique_lock<std::mutex> g(t->mu);
    auto finished = [&] { return t->state.load() >= S2L_JOB_DONE; };
    if (timeout_s < 0.0) {
        t->cv.wait(g, finished);
    } else if (!t->cv.wait_for(g, std::chrono::duration<double>(timeout_s), finished)) {
        return S2L_ERR_TIMEOUT;
    }
    if (status) *status = t->status;
    return S2L_OK;
}

int s2l_gpu_cancel(s2l_ticket* t)
{
    if (!t) return S2L_ERR_BADARG;
    t->cancel.store(1);
    return S2L_OK;
}

int s2l_gpu_ticket_info(s2l_ticket* t, double* queue_ms, double* run_ms, const char** error)
{
    if (!t) return S2L_ERR_BADARG;
    std::lock_guard<std::mutex> g(t->mu);
    const int st = t->state.load();
    using ms = std::chrono::duration<double, std::milli>;
    if (queue_ms)
        *queue_ms = st >= S2L_JOB_RUNNING && t->t_start.time_since_epoch().count()
                        ? ms(t->t_start - t->t_submit).count()
                        : (st >= S2L_JOB_DONE ? ms(t->t_end - t->t_submit).count() : 0.0);
    if (run_ms)
        *run_ms = st >= S2L_JOB_DONE && t->t_start.time_since_epoch().count() ? ms(t->t_end - t->t_start).count() : 0.0;
    if (error) *error = t->err.c_str();
    return S2L_OK;
}

int s2l_gpu_ticket_free(s2l_ticket* t)
{
    if (!t) return S2L_OK;
    if (t->state.load() < S2L_JOB_DONE) return S2L_ERR_STATE;
    delete t;
    return S2L_OK;
}

}  // extern "C"
