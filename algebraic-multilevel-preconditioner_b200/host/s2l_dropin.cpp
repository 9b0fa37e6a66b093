/**
 * @file s2l_dropin.cpp
 * @brief Implementation of the drop-in classes (see s2l_dropin.hpp).
 *
 * What crosses the C ABI, per subdomain (include/s2l_gpu.h, s2l_gpu_add_subdomain):
 *  - the owned range and ghost list of part::Subdomain (include/partition/subdomain.hpp:63-88);
 *  - its partition of unity D_i;
 *  - the exact factors of A_ii, in the precision and factorization type the reference's
 *    LocalSolver used (src/linalg/local_solver.cpp:95-153, 400-451).  Eigen's factorizations are
 *    deterministic, so refactorizing sd.Aii() with the same solver class reproduces them; they are
 *    walked into CSR: SparseLU's supernodes (L strictly below the diagonal of each supernode, the
 *    rest plus CoarseSpace's m_mapU to U), SimplicialLLT/LDLT's L with its permutation;
 *  - the coarse basis V_i of CoarseSpace (include/preconditioner/coarse_space.hpp:93).
 * Rank 0 adds E = W^T A W, W = [R_1^T V_1, ..., R_N^T V_N] (what CoarseSpace::assemble sums,
 * src/preconditioner/coarse_space.cpp:107-206), from the gathered bases and rows.
 */
#include "s2l_dropin.hpp"

#include "mpi_utils.hpp"

#include <Eigen/SparseCholesky>
#include <Eigen/SparseLU>

#include <cstring>
#include <stdexcept>
#include <type_traits>

namespace s2l::dropin {

using namespace schwarz2lvl;

namespace {

// ------------------------------------------------------------------------- byte blobs
struct Blob {
    std::vector<char> b;
    template <typename T>
    void put(const T* p, size_t n)
    {
        const uint64_t c = n;
        b.insert(b.end(), (const char*)&c, (const char*)&c + sizeof(c));
        b.insert(b.end(), (const char*)p, (const char*)p + n * sizeof(T));
    }
    template <typename T>
    void put(const std::vector<T>& v) { put(v.data(), v.size()); }
};

struct Reader {
    const char* p;
    template <typename T>
    std::vector<T> get()
    {
        uint64_t c;
        std::memcpy(&c, p, sizeof(c));
        p += sizeof(c);
        std::vector<T> v(c);
        if (c) std::memcpy(v.data(), p, c * sizeof(T));
        p += c * sizeof(T);
        return v;
    }
};

template <typename Real>
using SpMatT = Eigen::SparseMatrix<Real, Eigen::ColMajor, core::LocalIndex>;

template <typename Real>
void triplets_to_csr(int n, std::vector<Eigen::Triplet<Real, int>>& t, std::vector<int64_t>& rp, std::vector<int32_t>& ci,
                     std::vector<Real>& v)
{
    Eigen::SparseMatrix<Real, Eigen::RowMajor, int> M(n, n);
    M.setFromTriplets(t.begin(), t.end());
    M.makeCompressed();
    rp.assign(n + 1, 0);
    ci.clear();
    v.clear();
    for (int r = 0; r < n; ++r) {
        for (typename Eigen::SparseMatrix<Real, Eigen::RowMajor, int>::InnerIterator it(M, r); it; ++it) {
            if (it.value() == Real(0) && it.col() != r) continue;
            ci.push_back(it.col());
            v.push_back(it.value());
        }
        rp[r + 1] = (int64_t)ci.size();
    }
}

template <typename Perm>
std::vector<int32_t> perm_inverse(const Perm& P)
{
    std::vector<int32_t> inv(P.indices().size());
    for (int i = 0; i < (int)inv.size(); ++i) inv[P.indices()[i]] = i;
    return inv;
}

template <typename Perm>
std::vector<int32_t> perm_indices(const Perm& P)
{
    return std::vector<int32_t>(P.indices().data(), P.indices().data() + P.indices().size());
}

// factor of A_ii in the reference's precision and type -> blob: kind, single, pin, pout, L, [U], [d]
template <typename Real>
void export_factor(const core::SpMat& A, linalg::Factorization f, Blob& out)
{
    const int n = (int)A.rows();
    SpMatT<Real> M = A.template cast<Real>();
    using Tr = Eigen::Triplet<Real, int>;
    std::vector<Tr> tl, tu;
    std::vector<int32_t> pin, pout;
    std::vector<Real> d;
    int kind;
    if (f == linalg::Factorization::LU) {
        Eigen::SparseLU<SpMatT<Real>, Eigen::COLAMDOrdering<core::LocalIndex>> s;
        s.analyzePattern(M);
        s.factorize(M);
        if (s.info() != Eigen::Success) throw std::runtime_error("GPU export: SparseLU of A_ii failed");
        auto Lr = s.matrixL();
        const auto& Lm = Lr.m_mapL;
        using SC = typename std::decay<decltype(Lm)>::type;
        for (int c = 0; c < n; ++c) {
            tl.emplace_back(c, c, Real(1));
            for (typename SC::InnerIterator it(Lm, c); it; ++it) {
                if ((int)it.row() > c) tl.emplace_back((int)it.row(), c, it.value());
                else tu.emplace_back((int)it.row(), c, it.value());
            }
        }
        auto Ur = s.matrixU();
        const auto& Um = Ur.m_mapU;
        using MU = typename std::decay<decltype(Um)>::type;
        for (int c = 0; c < n; ++c)
            for (typename MU::InnerIterator it(Um, c); it; ++it) tu.emplace_back((int)it.row(), c, it.value());
        pin = perm_inverse(s.rowsPermutation());
        pout = perm_indices(s.colsPermutation());
        kind = S2L_FACTOR_LU;
    } else if (f == linalg::Factorization::Cholesky) {
        Eigen::SimplicialLLT<SpMatT<Real>> s(M);
        if (s.info() != Eigen::Success) throw std::runtime_error("GPU export: Cholesky of A_ii failed");
        SpMatT<Real> L = s.matrixL();
        for (int c = 0; c < n; ++c)
            for (typename SpMatT<Real>::InnerIterator it(L, c); it; ++it) tl.emplace_back((int)it.row(), c, it.value());
        pin = perm_inverse(s.permutationP());
        pout = perm_indices(s.permutationP());
        kind = S2L_FACTOR_LLT;
    } else {
        Eigen::SimplicialLDLT<SpMatT<Real>> s(M);
        if (s.info() != Eigen::Success) throw std::runtime_error("GPU export: LDLT of A_ii failed");
        SpMatT<Real> L = s.matrixL();
        for (int c = 0; c < n; ++c) {
            tl.emplace_back(c, c, Real(1));
            for (typename SpMatT<Real>::InnerIterator it(L, c); it; ++it)
                if ((int)it.row() > c) tl.emplace_back((int)it.row(), c, it.value());
        }
        auto D = s.vectorD();
        d.assign(D.data(), D.data() + n);
        pin = perm_inverse(s.permutationP());
        pout = perm_indices(s.permutationP());
        kind = S2L_FACTOR_LDLT;
    }
    std::vector<int64_t> meta = {kind, std::is_same_v<Real, float> ? 1 : 0};
    out.put(meta);
    out.put(pin);
    out.put(pout);
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<Real> v;
    triplets_to_csr<Real>(n, tl, rp, ci, v);
    out.put(rp);
    out.put(ci);
    out.put(v);
    if (kind == S2L_FACTOR_LU) {
        triplets_to_csr<Real>(n, tu, rp, ci, v);
        out.put(rp);
        out.put(ci);
        out.put(v);
    }
    if (kind == S2L_FACTOR_LDLT) out.put(d);
}

int one_level_code(const core::SolverConfig& c) { return c.one_level == "asm" ? S2L_ONE_LEVEL_ASM : S2L_ONE_LEVEL_RAS; }
int coarse_code(const core::SolverConfig& c)
{
    return c.coarse == "none" ? S2L_COARSE_NONE : (c.coarse == "additive" ? S2L_COARSE_ADDITIVE : S2L_COARSE_DEFLATED);
}

}  // namespace

// ------------------------------------------------------------------------- GpuSolvePhase
GpuSolvePhase::GpuSolvePhase(const part::Subdomain& sd, const prec::OneLevelSchwarz& one,
                             const prec::TwoLevelSchwarz* two, const core::SolverConfig& cfg, int device,
                             size_t hbm_budget, bool refactorize)
    : comm_(sd.comm()), sd_(&sd), cfg_(cfg), device_(device), hbm_budget_(hbm_budget), refactorize_(refactorize)
{
    op_version_ = prec_version_ = sd.valuesVersion();
    rank_ = core::mpiRank(comm_);
    np_ = core::mpiSize(comm_);
    const core::LocalSystem& sys = sd.system();
    n_ = sys.n_global;
    counts_.resize(np_);
    displs_.resize(np_);
    for (int p = 0; p < np_; ++p) {
        counts_[p] = (int)(sys.ownership[p + 1] - sys.ownership[p]);
        displs_[p] = (int)sys.ownership[p];
    }
    if (cfg.local_approx != "none" && cfg.local_approx != "amg")
        throw std::invalid_argument("unknown local approximation '" + cfg.local_approx + "' (none|amg)");
    amg_on_ = cfg.local_approx == "amg";
    coarse_ = two && two->coarse().dimension() > 0 && cfg.coarse != "none";
    if (two && two->coarse().dimension() > 0) {
        const core::Mat& V = two->coarse().basis();
        m_ = (int)V.cols();
        V_.assign(V.data(), V.data() + V.size());
    }
    if (amg_on_) buildAmg(false);
    else factorization_ = (int)one.localSolver().factorization();
    upload();
}

void GpuSolvePhase::buildAmg(bool keep_transfer)
{
    // A_ii in CSR with sorted columns (what AMGCL receives from the reference, inexact_solver.cpp:62)
    Eigen::SparseMatrix<double, Eigen::RowMajor, int> R = sd_->Aii();
    R.makeCompressed();
    const int64_t n = R.rows();
    std::vector<int64_t> rp(R.outerIndexPtr(), R.outerIndexPtr() + n + 1);
    std::vector<int32_t> ci(R.innerIndexPtr(), R.innerIndexPtr() + R.nonZeros());
    s2l_amg* h = nullptr;
    int st;
    if (keep_transfer && amg_) {
        st = s2l_amg_rebuild(amg_, rp.data(), ci.data(), R.valuePtr(), &h);
    } else {
        // --local-precision single: the hierarchy built in float, as the reference's AMGCL<float>
        st = s2l_amg_build(n, rp.data(), ci.data(), R.valuePtr(), cfg_.amg_coarse_enough,
                           (cfg_.amg_coarsening == "rs" ? S2L_AMG_RS : S2L_AMG_SA) |
                               (cfg_.local_precision == "single" ? S2L_AMG_SINGLE : 0),
                           &h);
    }
    int worst = st;
    MPI_Allreduce(&st, &worst, 1, MPI_INT, MPI_MAX, comm_);
    if (worst != S2L_OK) {
        if (h) s2l_amg_free(h);
        throw std::invalid_argument("GPU setup: the host AMG setup of A_ii failed on a rank (status " +
                                    std::to_string(worst) + ")");
    }
    if (amg_) s2l_amg_free(amg_);
    amg_ = h;
}

void GpuSolvePhase::upload()
{
    const core::LocalSystem& sys = sd_->system();
    const part::Subdomain& sd = *sd_;
    // ---- this rank's part
    Blob blob;
    {
        std::vector<int64_t> meta = {(int64_t)sys.rowBegin(), (int64_t)sd.nOwned(), (int64_t)sd.nGhost()};
        blob.put(meta);
        blob.put(sys.row_ptr);
        blob.put(sys.col);
        blob.put(sys.val);
        blob.put(sd.ghosts());
        blob.put(sd.pou().data(), (size_t)sd.pou().size());
        if (amg_on_) {
            // AMG levels: kind -1, sweeps, levels, coarsest size; per level A, P, R ([rows, cols] and
            // CSR; rows = 0 for none); the coarsest operator, row-major
            int nlev = 0;
            int64_t nc = 0;
            s2l_amg_shape(amg_, &nlev, &nc);
            std::vector<int64_t> fmeta = {-1, (int64_t)cfg_.amg_sweeps, (int64_t)nlev, nc};
            blob.put(fmeta);
            for (int l = 0; l < nlev; ++l)
                for (int which = 0; which < 3; ++which) {
                    int64_t rows = 0, cols = 0;
                    const int64_t* mrp = nullptr;
                    const int32_t* mci = nullptr;
                    const double* mv = nullptr;
                    s2l_amg_matrix(amg_, l, which, &rows, &cols, &mrp, &mci, &mv);
                    std::vector<int64_t> shape = {rows, cols};
                    blob.put(shape);
                    const int64_t nz = rows ? mrp[rows] : 0;
                    blob.put(mrp, rows ? (size_t)rows + 1 : 0);
                    blob.put(mci, (size_t)nz);
                    blob.put(mv, (size_t)nz);
                }
            const double* dense = nullptr;
            s2l_amg_coarse(amg_, &dense);
            blob.put(dense, (size_t)(nc * nc));
        } else {
            const auto f = (linalg::Factorization)factorization_;
            if (cfg_.local_precision == "single")
                export_factor<float>(sd.Aii(), f, blob);
            else
                export_factor<double>(sd.Aii(), f, blob);
        }
        std::vector<int64_t> vm = {(int64_t)m_};
        blob.put(vm);
        blob.put(V_);
    }
    // ---- rank 0 receives every part in rank order and uploads it as a new setup
    int status = S2L_OK;
    std::string msg;
    const int tag = 7311;
    if (rank_ != 0) {
        long long sz = (long long)blob.b.size();
        MPI_Send(&sz, 1, MPI_LONG_LONG, 0, tag, comm_);
        MPI_Send(blob.b.data(), (int)sz, MPI_CHAR, 0, tag + 1, comm_);
    } else {
        const core::SolverConfig& cfg = cfg_;
        const bool coarse = coarse_;
        if (setup_) {
            s2l_gpu_setup_destroy(setup_);
            setup_ = nullptr;
        }
        nnz_counts_.clear();
        nnz_displs_.clear();
        if (!ctx_) status = s2l_gpu_create(device_, hbm_budget_, &ctx_);
        if (status == S2L_OK)
            status = s2l_gpu_setup_begin(ctx_, n_, np_, one_level_code(cfg), coarse ? coarse_code(cfg) : S2L_COARSE_NONE,
                                         sd.booleanPou() ? S2L_POU_BOOLEAN : S2L_POU_MULTIPLICITY, &setup_);
        std::vector<int64_t> grp(1, 0), gcol;
        std::vector<double> gval;
        // coarse basis triplets for E
        std::vector<Eigen::Triplet<double, int64_t>> wt;
        std::vector<int64_t> offsets(np_ + 1, 0);
        for (int p = 0; p < np_; ++p) {
            std::vector<char> in;
            if (p == 0) {
                in.swap(blob.b);
            } else {
                long long sz = 0;
                MPI_Recv(&sz, 1, MPI_LONG_LONG, p, tag, comm_, MPI_STATUS_IGNORE);
                in.resize((size_t)sz);
                MPI_Recv(in.data(), (int)sz, MPI_CHAR, p, tag + 1, comm_, MPI_STATUS_IGNORE);
            }
            Reader rd{in.data()};
            const auto meta = rd.get<int64_t>();
            const int64_t begin = meta[0];
            const int nI = (int)meta[1], nG = (int)meta[2], nl = nI + nG;
            const auto rp = rd.get<int64_t>();
            const auto col = rd.get<int64_t>();
            const auto val = rd.get<double>();
            for (int r = 0; r < nI; ++r) grp.push_back(grp.back() + (rp[r + 1] - rp[r]));
            nnz_displs_.push_back((int)gval.size());
            nnz_counts_.push_back((int)val.size());
            gcol.insert(gcol.end(), col.begin(), col.end());
            gval.insert(gval.end(), val.begin(), val.end());
            const auto ghosts = rd.get<int64_t>();
            const auto D = rd.get<double>();
            const auto fmeta = rd.get<int64_t>();
            if (fmeta[0] < 0) {  // AMG levels
                const int sweeps = (int)fmeta[1], nlev = (int)fmeta[2];
                const int64_t nc = fmeta[3];
                std::vector<std::vector<int64_t>> rps(3 * (size_t)nlev);
                std::vector<std::vector<int32_t>> cis(3 * (size_t)nlev);
                std::vector<std::vector<double>> vs(3 * (size_t)nlev);
                std::vector<int32_t> nrow((size_t)std::max(nlev, 1), 0);
                for (int l = 0; l < nlev; ++l)
                    for (int which = 0; which < 3; ++which) {
                        const size_t k = 3 * (size_t)l + which;
                        const auto shape = rd.get<int64_t>();
                        if (which == 0) nrow[l] = (int32_t)shape[0];
                        rps[k] = rd.get<int64_t>();
                        cis[k] = rd.get<int32_t>();
                        vs[k] = rd.get<double>();
                    }
                const auto dense = rd.get<double>();
                std::vector<const int64_t*> Arp(nlev), Prp(nlev), Rrp(nlev);
                std::vector<const int32_t*> Aci(nlev), Pci(nlev), Rci(nlev);
                std::vector<const double*> Av(nlev), Pv(nlev), Rv(nlev);
                for (int l = 0; l < nlev; ++l) {
                    auto ptrs = [&](int which, const int64_t*& r, const int32_t*& c, const double*& v) {
                        const size_t k = 3 * (size_t)l + which;
                        r = rps[k].empty() ? nullptr : rps[k].data();
                        c = cis[k].empty() ? nullptr : cis[k].data();
                        v = vs[k].empty() ? nullptr : vs[k].data();
                        // an empty operator still passes valid (empty) arrays when it has rows
                        static const int32_t no_ci = 0;
                        static const double no_v = 0.0;
                        if (r && !c) c = &no_ci;
                        if (r && !v) v = &no_v;
                    };
                    ptrs(0, Arp[l], Aci[l], Av[l]);
                    ptrs(1, Prp[l], Pci[l], Pv[l]);
                    ptrs(2, Rrp[l], Rci[l], Rv[l]);
                }
                const auto vm = rd.get<int64_t>();
                const int m = (int)vm[0];
                const auto V = rd.get<double>();
                offsets[p + 1] = offsets[p] + (coarse ? m : 0);
                if (coarse)
                    for (int a = 0; a < m; ++a)
                        for (int j = 0; j < nl; ++j) {
                            const double v = V[(size_t)a * nl + j];
                            if (v != 0.0) wt.emplace_back(j < nI ? begin + j : ghosts[j - nI], offsets[p] + a, v);
                        }
                if (status == S2L_OK)
                    status = s2l_gpu_add_subdomain_amg(setup_, p, begin, nI, nG, ghosts.data(), D.data(), nlev, sweeps,
                                                       nrow.data(), Arp.data(), Aci.data(), Av.data(), Prp.data(),
                                                       Pci.data(), Pv.data(), Rrp.data(), Rci.data(), Rv.data(), (int)nc,
                                                       nc ? dense.data() : nullptr, coarse ? m : 0,
                                                       coarse ? V.data() : nullptr);
                continue;
            }
            const int kind = (int)fmeta[0], single = (int)fmeta[1];
            const auto pin = rd.get<int32_t>();
            const auto pout = rd.get<int32_t>();
            const auto Lrp = rd.get<int64_t>();
            const auto Lci = rd.get<int32_t>();
            std::vector<char> Lv, Uv, dv;
            std::vector<int64_t> Urp;
            std::vector<int32_t> Uci;
            auto getv = [&](std::vector<char>& dst) {
                if (single) {
                    auto v = rd.get<float>();
                    dst.assign((const char*)v.data(), (const char*)v.data() + v.size() * sizeof(float));
                } else {
                    auto v = rd.get<double>();
                    dst.assign((const char*)v.data(), (const char*)v.data() + v.size() * sizeof(double));
                }
            };
            getv(Lv);
            if (kind == S2L_FACTOR_LU) {
                Urp = rd.get<int64_t>();
                Uci = rd.get<int32_t>();
                getv(Uv);
            }
            if (kind == S2L_FACTOR_LDLT) getv(dv);
            const auto vm = rd.get<int64_t>();
            const int m = (int)vm[0];
            const auto V = rd.get<double>();
            offsets[p + 1] = offsets[p] + (coarse ? m : 0);
            if (coarse)
                for (int a = 0; a < m; ++a)
                    for (int j = 0; j < nl; ++j) {
                        const double v = V[(size_t)a * nl + j];
                        if (v != 0.0) wt.emplace_back(j < nI ? begin + j : ghosts[j - nI], offsets[p] + a, v);
                    }
            if (status == S2L_OK)
                status = s2l_gpu_add_subdomain(setup_, p, begin, nI, nG, ghosts.data(), D.data(), kind,
                                               single ? S2L_REAL_F32 : S2L_REAL_F64, pin.data(), pout.data(),
                                               Lrp.data(), Lci.data(), Lv.data(), Urp.empty() ? nullptr : Urp.data(),
                                               Uci.empty() ? nullptr : Uci.data(), Uv.empty() ? nullptr : Uv.data(),
                                               dv.empty() ? nullptr : dv.data(), coarse ? m : 0,
                                               coarse ? V.data() : nullptr);
        }
        if (status == S2L_OK) status = s2l_gpu_set_matrix(setup_, grp.data(), gcol.data(), gval.data());
        if (status == S2L_OK && coarse) {
            const int64_t n0 = offsets[np_];
            Eigen::SparseMatrix<double, Eigen::ColMajor, int64_t> W(n_, n0);
            W.setFromTriplets(wt.begin(), wt.end());
            Eigen::SparseMatrix<double, Eigen::RowMajor, int64_t> A(n_, n_);
            {
                std::vector<Eigen::Triplet<double, int64_t>> at;
                at.reserve(gval.size());
                for (int64_t r = 0; r < n_; ++r)
                    for (int64_t e = grp[r]; e < grp[r + 1]; ++e) at.emplace_back(r, gcol[e], gval[e]);
                A.setFromTriplets(at.begin(), at.end());
            }
            Eigen::SparseMatrix<double, Eigen::ColMajor, int64_t> AW = A * W;
            Eigen::MatrixXd E = Eigen::MatrixXd(Eigen::SparseMatrix<double, Eigen::ColMajor, int64_t>(W.transpose()) * AW);
            Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> Er = E;
            status = s2l_gpu_set_coarse(setup_, n0, offsets.data(), Er.data());
        }
        // factors are refactorized on the device; AMG hierarchies on the host, then uploaded again
        if (status == S2L_OK && refactorize_ && !amg_on_) status = s2l_gpu_setup_option(setup_, "refactor", 1.0);
        if (status == S2L_OK && amg_on_ && cfg_.local_precision == "single")
            status = s2l_gpu_setup_option(setup_, "amg_single", 1.0);  // V-cycle in float
        if (status == S2L_OK) status = s2l_gpu_setup_end(setup_);
        if (status != S2L_OK) msg = ctx_ ? s2l_gpu_last_error(ctx_) : "no CUDA device";
    }
    check(status, (std::string("GPU setup: ") + msg).c_str());
}

GpuSolvePhase::~GpuSolvePhase()
{
    if (setup_) s2l_gpu_setup_destroy(setup_);
    if (ctx_) s2l_gpu_destroy(ctx_);
    if (amg_) s2l_amg_free(amg_);
}

void GpuSolvePhase::check(int status, const char* what) const
{
    int st = status;
    MPI_Bcast(&st, 1, MPI_INT, 0, comm_);
    if (st == S2L_OK) return;
    std::string m = what;
    if (rank_ == 0 && ctx_) m += std::string(": ") + s2l_gpu_last_error(ctx_);
    if (st == S2L_ERR_BADARG) throw std::invalid_argument(m);
    if (st == S2L_ERR_STATE) throw std::logic_error(m);
    throw std::runtime_error(m);
}

void GpuSolvePhase::gather(const core::Vec& owned, std::vector<double>& global) const
{
    if (rank_ == 0) global.resize((size_t)n_);
    MPI_Gatherv(owned.data(), (int)owned.size(), MPI_DOUBLE, rank_ == 0 ? global.data() : nullptr, counts_.data(),
                displs_.data(), MPI_DOUBLE, 0, comm_);
}

void GpuSolvePhase::scatter(const std::vector<double>& global, core::Vec& owned) const
{
    owned.resize(counts_[rank_]);
    MPI_Scatterv(rank_ == 0 ? global.data() : nullptr, counts_.data(), displs_.data(), MPI_DOUBLE, owned.data(),
                 counts_[rank_], MPI_DOUBLE, 0, comm_);
}

bool GpuSolvePhase::operatorCurrent() const { return op_version_ == sd_->valuesVersion(); }

bool GpuSolvePhase::preconditionerCurrent() const { return prec_version_ == sd_->valuesVersion(); }

void GpuSolvePhase::pushValues(prec::UpdateLevel level)
{
    const bool refac = level == prec::UpdateLevel::Refactorize;
    if (refac && amg_on_) {  // AMG local solvers: the hierarchies again on the host, a new setup
        buildAmg(cfg_.amg_reuse);
        upload();
        op_version_ = prec_version_ = sd_->valuesVersion();
        return;
    }
    const std::vector<core::Scalar>& v = sd_->system().val;
    std::vector<double> all;
    if (rank_ == 0) all.resize(nnz_counts_.empty() ? 0 : (size_t)nnz_displs_.back() + nnz_counts_.back());
    MPI_Gatherv(v.data(), (int)v.size(), MPI_DOUBLE, rank_ == 0 ? all.data() : nullptr,
                rank_ == 0 ? nnz_counts_.data() : nullptr, rank_ == 0 ? nnz_displs_.data() : nullptr, MPI_DOUBLE, 0,
                comm_);
    int st = S2L_OK;
    if (rank_ == 0)
        st = refac ? s2l_gpu_refactor(setup_, all.data(), S2L_PTR_HOST)
                   : s2l_gpu_update_matrix(setup_, all.data(), S2L_PTR_HOST);
    check(st, refac ? "GPU refactorization" : "GPU matrix update");
    op_version_ = sd_->valuesVersion();
    if (refac) prec_version_ = op_version_;
}

// ------------------------------------------------------------------------- GpuTwoLevelSchwarz
prec::UpdateLevel GpuTwoLevelSchwarz::update(prec::UpdateLevel requested)
{
    requested = prec::agree(requested, phase_->comm());
    if (requested == prec::UpdateLevel::Rebuild)
        throw std::logic_error("GpuTwoLevelSchwarz: Rebuild recomputes the coarse basis on the host; build a new "
                               "GpuSolvePhase from the rebuilt reference preconditioner");
    if (requested == prec::UpdateLevel::Refactorize && !phase_->preconditionerCurrent()) {
        phase_->pushValues(prec::UpdateLevel::Refactorize);
        return prec::UpdateLevel::Refactorize;
    }
    if (!phase_->operatorCurrent()) phase_->pushValues(prec::UpdateLevel::Reuse);
    return prec::UpdateLevel::Reuse;
}

void GpuTwoLevelSchwarz::apply(const core::Vec& r, core::Vec& z) const
{
    std::vector<double> rg, zg;
    phase_->gather(r, rg);
    int st = S2L_OK;
    if (phase_->rank() == 0) {
        zg.resize(rg.size());
        st = s2l_gpu_apply(phase_->setup(), rg.data(), zg.data(), S2L_PTR_HOST);
    }
    phase_->check(st, "GPU apply");
    phase_->scatter(zg, z);
}

// ------------------------------------------------------------------------- GpuKrylov
solv::KrylovResult GpuKrylov::solve(const linalg::DistributedMatrix&, const prec::Preconditioner& M, const core::Vec& b,
                                    core::Vec& x) const
{
    const auto* gm = dynamic_cast<const GpuTwoLevelSchwarz*>(&M);
    if (!gm) throw std::invalid_argument("GpuKrylov needs a GpuTwoLevelSchwarz preconditioner");
    const GpuSolvePhase& ph = *gm->phase();
    if (x.size() != b.size()) x = core::Vec::Zero(b.size());
    std::vector<double> bg, xg;
    ph.gather(b, bg);
    ph.gather(x, xg);
    s2l_result res{};
    std::vector<double> hist((size_t)maxit_ + 8);
    double meta[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int st = S2L_OK;
    if (ph.rank() == 0) {
        s2l_krylov_opts o{restart_, rtol_, maxit_, flexible_ ? 1 : 0, strict_ ? 1 : 0, (int)hist.size(),
                          stop_ == solv::StopNorm::OpenFOAM ? S2L_STOP_OPENFOAM : S2L_STOP_L2, atol_};
        res.history = hist.data();
        st = method_ == "bicgstab" ? s2l_gpu_bicgstab(ph.setup(), bg.data(), xg.data(), S2L_PTR_HOST, &o, &res)
                                   : s2l_gpu_gmres(ph.setup(), bg.data(), xg.data(), S2L_PTR_HOST, &o, &res);
        meta[0] = res.converged;
        meta[1] = res.breakdown;
        meta[2] = res.iterations;
        meta[3] = res.restarts;
        meta[4] = res.rel_residual;
        meta[5] = res.true_rel_residual;
        meta[6] = res.initial_residual_of;
        meta[7] = res.final_residual_of;
    }
    ph.check(st, "GPU Krylov solve");
    int hl = res.history_len;
    MPI_Bcast(meta, 8, MPI_DOUBLE, 0, ph.comm());
    MPI_Bcast(&hl, 1, MPI_INT, 0, ph.comm());
    MPI_Bcast(hist.data(), hl, MPI_DOUBLE, 0, ph.comm());
    ph.scatter(xg, x);
    solv::KrylovResult out;
    out.converged = meta[0] != 0.0;
    out.breakdown = meta[1] != 0.0;
    out.iterations = (int)meta[2];
    out.restarts = (int)meta[3];
    out.rel_residual = meta[4];
    out.true_rel_residual = meta[5];
    out.initial_residual_of = meta[6];
    out.final_residual_of = meta[7];
    out.history.assign(hist.begin(), hist.begin() + hl);
    return out;
}

std::string GpuKrylov::name() const
{
    if (method_ == "bicgstab") return "BiCGStab (B200)";
    return (flexible_ ? "FGMRES(" : "GMRES(") + std::to_string(restart_) + ") (B200)";
}

std::unique_ptr<solv::KrylovSolver> makeGpuKrylovSolver(const core::SolverConfig& cfg, double rtol, double atol)
{
    const solv::StopNorm stop = solv::parseStopNorm(cfg.stop_norm);
    if (atol > 0.0 && stop != solv::StopNorm::OpenFOAM)
        throw std::invalid_argument("an absolute tolerance needs the OpenFOAM stopping norm");
    if (cfg.krylov != "gmres" && cfg.krylov != "bicgstab") throw std::invalid_argument("unknown Krylov solver " + cfg.krylov);
    const bool single = cfg.local_precision == "single";
    return std::make_unique<GpuKrylov>(cfg.krylov, cfg.restart, rtol, cfg.maxit, single && cfg.krylov == "gmres", single,
                                       stop, atol);
}

std::unique_ptr<solv::KrylovSolver> makeGpuKrylovSolver(const core::SolverConfig& cfg)
{
    return makeGpuKrylovSolver(cfg, cfg.rtol, cfg.atol);
}

}  // namespace s2l::dropin
