// Driver around the reference library (compiled from its own sources with the thread-rank MPI
// stand-in).  TEST INFRASTRUCTURE ONLY: it produces the golden fixtures that pin the oracle and the
// GPU path, and times the reference for the benchmark's reference arm.
//
//   s2l_ref_dump  <reference flags> --dump-dir DIR [--napply K]
//       decomposes, builds the reference's preconditioner and writes, per rank, the data the
//       solve phase consumes (ghosts, D, V, the exact local factors), plus the reference's own
//       outputs: SpMV, coarse/one-level/two-level applies of seeded vectors, the local solves, and
//       a full Krylov solve (iterations, residual history, solution).
//   s2l_ref_bench <reference flags> --bench-steps K --bench-warmup W
//       setup, then W untimed and K timed solves; rank 0 prints one JSON line.
//
// The reference flags are parsed by its own SolverConfig::fromCommandLine (src/core/config.cpp).
// The local factors are recomputed here with the same Eigen solver class, precision and input the
// reference's LocalSolver used (src/linalg/local_solver.cpp:95-153, 400-451): Eigen's
// factorizations are deterministic, so they are the reference's factors; every export is checked
// against a solve of the reference's own LocalSolver before it is written.
#include "config.hpp"
#include "distributed_matrix.hpp"
#include "domain_decomposer.hpp"
#include "krylov.hpp"
#include "local_solver.hpp"
#include "mpi_utils.hpp"
#include "one_level_schwarz.hpp"
#include "subdomain.hpp"
#include "two_level_schwarz.hpp"

#include <Eigen/SparseCholesky>
#include <Eigen/SparseLU>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>

using namespace schwarz2lvl;

namespace {

struct Extra {
    std::string dump;
    int steps = 0, warmup = 0, napply = 2;
};

// ---------------------------------------------------------------------------------- writing
struct Writer {
    std::string dir;
    std::ofstream manifest;
    Writer(const std::string& d, int rank) : dir(d)
    {
        manifest.open(dir + "/manifest_rank" + std::to_string(rank) + ".txt");
    }
    template <typename T>
    void put(const std::string& name, const char* dtype, const T* p, size_t count)
    {
        std::ofstream f(dir + "/" + name + ".bin", std::ios::binary);
        f.write(reinterpret_cast<const char*>(p), (std::streamsize)(count * sizeof(T)));
        manifest << name << " " << dtype << " " << count << "\n";
    }
    void vec(const std::string& n, const std::vector<double>& v) { put(n, "f64", v.data(), v.size()); }
    void vec(const std::string& n, const core::Vec& v) { put(n, "f64", v.data(), (size_t)v.size()); }
    void i64(const std::string& n, const std::vector<int64_t>& v) { put(n, "i64", v.data(), v.size()); }
    void i32(const std::string& n, const std::vector<int32_t>& v) { put(n, "i32", v.data(), v.size()); }
    void scalar(const std::string& n, double v) { put(n, "f64", &v, 1); }
};

// ---------------------------------------------------------------------------------- factors
template <typename Real>
struct Csr {
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<Real> v;
};

template <typename Real>
using SpMatT = Eigen::SparseMatrix<Real, Eigen::ColMajor, core::LocalIndex>;

// column-major triplets (row, col, value) -> CSR with sorted columns, exact zeros dropped
template <typename Real>
Csr<Real> to_csr(int n, const std::vector<Eigen::Triplet<Real, int>>& t)
{
    Eigen::SparseMatrix<Real, Eigen::RowMajor, int> M(n, n);
    M.setFromTriplets(t.begin(), t.end());
    M.makeCompressed();
    Csr<Real> c;
    c.rp.assign(n + 1, 0);
    for (int r = 0; r < n; ++r) {
        for (typename Eigen::SparseMatrix<Real, Eigen::RowMajor, int>::InnerIterator it(M, r); it; ++it) {
            if (it.value() == Real(0) && it.col() != r) continue;
            c.ci.push_back(it.col());
            c.v.push_back(it.value());
        }
        c.rp[r + 1] = (int64_t)c.ci.size();
    }
    return c;
}

struct Factor {
    int kind = 0;  // 0 LU, 1 LLT, 2 LDLT (include/linalg/local_solver.hpp:51-52 order differs: ours)
    std::vector<int32_t> pin, pout;
    Csr<double> L, U;        // values widened (exact) for checking
    std::vector<double> d;
    bool single = false;
};

// t = b[pin]; L u = t; U v = u (U = L^T / D L^T for LLT / LDLT); x = v[pout]
std::vector<double> factor_solve(const Factor& F, const std::vector<double>& b)
{
    const int n = (int)F.pin.size();
    std::vector<double> t(n), x(n);
    for (int k = 0; k < n; ++k) t[k] = b[F.pin[k]];
    for (int r = 0; r < n; ++r) {
        double acc = t[r], dg = 1.0;
        for (int64_t e = F.L.rp[r]; e < F.L.rp[r + 1]; ++e) {
            const int c = F.L.ci[e];
            if (c < r) acc -= F.L.v[e] * t[c];
            else if (c == r) dg = F.L.v[e];
        }
        t[r] = F.kind == 1 ? acc / dg : acc;
    }
    if (F.kind == 0) {
        for (int r = n - 1; r >= 0; --r) {
            double acc = t[r], dg = 1.0;
            for (int64_t e = F.U.rp[r]; e < F.U.rp[r + 1]; ++e) {
                const int c = F.U.ci[e];
                if (c > r) acc -= F.U.v[e] * t[c];
                else if (c == r) dg = F.U.v[e];
            }
            t[r] = acc / dg;
        }
    } else {
        if (F.kind == 2)
            for (int r = 0; r < n; ++r) t[r] /= F.d[r];
        for (int r = n - 1; r >= 0; --r) {
            double dg = 1.0;
            if (F.kind == 1)
                for (int64_t e = F.L.rp[r]; e < F.L.rp[r + 1]; ++e)
                    if (F.L.ci[e] == r) dg = F.L.v[e];
            t[r] /= dg;
            for (int64_t e = F.L.rp[r]; e < F.L.rp[r + 1]; ++e) {
                const int c = F.L.ci[e];
                if (c < r) t[c] -= F.L.v[e] * t[r];
            }
        }
    }
    for (int j = 0; j < n; ++j) x[j] = t[F.pout[j]];
    return x;
}

template <typename Real>
Csr<double> widen(const Csr<Real>& c)
{
    return {c.rp, c.ci, std::vector<double>(c.v.begin(), c.v.end())};
}

// Eigen permutation P applied as (P v)[P.indices()[i]] = v[i]: t = P b  =>  t[k] = b[Pinv[k]].
template <typename Perm>
std::vector<int32_t> inverse_indices(const Perm& P)
{
    const int n = (int)P.indices().size();
    std::vector<int32_t> inv(n);
    for (int i = 0; i < n; ++i) inv[P.indices()[i]] = i;
    return inv;
}
template <typename Perm>
std::vector<int32_t> indices(const Perm& P)
{
    const int n = (int)P.indices().size();
    std::vector<int32_t> v(n);
    for (int i = 0; i < n; ++i) v[i] = P.indices()[i];
    return v;
}

template <typename Real, typename Raw>
void export_factor(const core::SpMat& A, linalg::Factorization f, Factor& F, Raw& raw)
{
    const int n = (int)A.rows();
    SpMatT<Real> M = A.template cast<Real>();
    F.single = !std::is_same_v<Real, double>;
    using Tr = Eigen::Triplet<Real, int>;
    if (f == linalg::Factorization::Cholesky || f == linalg::Factorization::LDLT) {
        std::vector<Tr> t;
        if (f == linalg::Factorization::Cholesky) {
            Eigen::SimplicialLLT<SpMatT<Real>> s(M);
            if (s.info() != Eigen::Success) throw std::runtime_error("export: Cholesky failed");
            SpMatT<Real> L = s.matrixL();
            for (int c = 0; c < n; ++c)
                for (typename SpMatT<Real>::InnerIterator it(L, c); it; ++it) t.emplace_back((int)it.row(), c, it.value());
            F.kind = 1;
            F.pin = inverse_indices(s.permutationP());
            F.pout = indices(s.permutationP());
        } else {
            Eigen::SimplicialLDLT<SpMatT<Real>> s(M);
            if (s.info() != Eigen::Success) throw std::runtime_error("export: LDLT failed");
            SpMatT<Real> L = s.matrixL();
            for (int c = 0; c < n; ++c) {
                t.emplace_back(c, c, Real(1));
                for (typename SpMatT<Real>::InnerIterator it(L, c); it; ++it)
                    if (it.row() > c) t.emplace_back((int)it.row(), c, it.value());
            }
            F.kind = 2;
            auto D = s.vectorD();
            F.d.assign(D.data(), D.data() + n);
            F.pin = inverse_indices(s.permutationP());
            F.pout = indices(s.permutationP());
        }
        raw.L = to_csr<Real>(n, t);
        F.L = widen(raw.L);
        return;
    }
    // SparseLU (supernodal): L's supernodes hold the diagonal blocks of U as well
    Eigen::SparseLU<SpMatT<Real>, Eigen::COLAMDOrdering<core::LocalIndex>> s;
    s.analyzePattern(M);
    s.factorize(M);
    if (s.info() != Eigen::Success) throw std::runtime_error("export: SparseLU failed");
    std::vector<Tr> tl, tu;
    auto Lr = s.matrixL();
    const auto& Lm = Lr.m_mapL;
    using SC = typename std::decay<decltype(Lm)>::type;
    for (int c = 0; c < n; ++c) {
        tl.emplace_back(c, c, Real(1));
        for (typename SC::InnerIterator it(Lm, c); it; ++it) {
            const int r = (int)it.row();
            if (r > c) tl.emplace_back(r, c, it.value());
            else tu.emplace_back(r, c, it.value());
        }
    }
    auto Ur = s.matrixU();
    const auto& Um = Ur.m_mapU;
    using MU = typename std::decay<decltype(Um)>::type;
    for (int c = 0; c < n; ++c)
        for (typename MU::InnerIterator it(Um, c); it; ++it) tu.emplace_back((int)it.row(), c, it.value());
    raw.L = to_csr<Real>(n, tl);
    raw.U = to_csr<Real>(n, tu);
    F.kind = 0;
    F.L = widen(raw.L);
    F.U = widen(raw.U);
    F.pin = inverse_indices(s.rowsPermutation());
    F.pout = indices(s.colsPermutation());
}

template <typename Real>
struct Raw {
    Csr<Real> L, U;
};

template <typename Real>
void write_factor(Writer& w, const std::string& p, const Factor& F, const Raw<Real>& raw)
{
    const char* dt = std::is_same_v<Real, double> ? "f64" : "f32";
    std::vector<int64_t> meta = {F.kind, F.single ? 1 : 0};
    w.i64(p + "fmeta", meta);
    w.i32(p + "pin", F.pin);
    w.i32(p + "pout", F.pout);
    w.i64(p + "L_rp", raw.L.rp);
    w.i32(p + "L_ci", raw.L.ci);
    w.put(p + "L_v", dt, raw.L.v.data(), raw.L.v.size());
    if (F.kind == 0) {
        w.i64(p + "U_rp", raw.U.rp);
        w.i32(p + "U_ci", raw.U.ci);
        w.put(p + "U_v", dt, raw.U.v.data(), raw.U.v.size());
    }
    if (F.kind == 2) {
        std::vector<Real> d(F.d.begin(), F.d.end());
        w.put(p + "d", dt, d.data(), d.size());
    }
}

std::vector<double> seeded(size_t n, unsigned long long seed)
{
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> v(n);
    for (auto& x : v) x = u(g);
    return v;
}

core::Vec owned_part(const std::vector<double>& g, const core::LocalSystem& sys)
{
    const auto b = sys.rowBegin();
    core::Vec v(sys.nOwned());
    for (int i = 0; i < sys.nOwned(); ++i) v[i] = g[(size_t)(b + i)];
    return v;
}

Extra strip(int argc, char** argv, std::vector<char*>& keep)
{
    Extra e;
    keep.push_back(argv[0]);
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&](void) -> std::string {
            if (i + 1 >= argc) throw std::invalid_argument(a + " needs a value");
            return argv[++i];
        };
        if (a == "--dump-dir") e.dump = val();
        else if (a == "--bench-steps") e.steps = std::stoi(val());
        else if (a == "--bench-warmup") e.warmup = std::stoi(val());
        else if (a == "--napply") e.napply = std::stoi(val());
        else keep.push_back(argv[i]);
    }
    return e;
}

}  // namespace

int main(int argc, char** argv)
{
    MPI_Init(&argc, &argv);
    MPI_Comm comm = MPI_COMM_WORLD;
    const int rank = core::mpiRank(comm), np = core::mpiSize(comm);
    try {
        std::vector<char*> keep;
        const Extra ex = strip(argc, argv, keep);
        core::SolverConfig cfg = core::SolverConfig::fromCommandLine((int)keep.size(), keep.data());
        part::DecompositionInfo info;
        info.keep_global = !ex.dump.empty();
        core::LocalSystem sys = part::DomainDecomposer::decompose(cfg, comm, info);
        if (ex.steps == 0 && ex.dump.empty()) {
            // same warm-up as the reference driver (src/main.cpp:122-130), untimed
            linalg::LocalSolverSpec ws;
            ws.backend = cfg.local_solver;
            ws.factorization = cfg.local_factorization;
            linalg::warmUpLocalSolver(ws);
        }
        MPI_Barrier(comm);
        const double t_setup0 = MPI_Wtime();
        part::Subdomain sd(sys, cfg.pou);
        linalg::DistributedMatrix A(sd);
        std::unique_ptr<prec::Preconditioner> M;
        const prec::TwoLevelSchwarz* two = nullptr;
        const prec::OneLevelSchwarz* one = nullptr;
        if (cfg.coarse == "none") {
            auto p = std::make_unique<prec::OneLevelSchwarz>(
                sd, cfg.one_level == "asm" ? prec::OneLevelSchwarz::Variant::ASM : prec::OneLevelSchwarz::Variant::RAS,
                prec::localSolverSpec(cfg, sys.symmetric));
            one = p.get();
            M = std::move(p);
        } else {
            auto p = std::make_unique<prec::TwoLevelSchwarz>(sd, A, cfg);
            two = p.get();
            one = &p->oneLevel();
            M = std::move(p);
        }
        MPI_Barrier(comm);
        const double t_setup = MPI_Wtime() - t_setup0;
        const core::Vec b = Eigen::Map<const core::Vec>(sys.rhs.data(), (Eigen::Index)sys.rhs.size());
        auto krylov = solv::makeKrylovSolver(cfg);

        // ------------------------------------------------------------------ timing mode
        if (ex.steps > 0) {
            solv::KrylovResult res;
            for (int k = 0; k < ex.warmup; ++k) {
                core::Vec x = core::Vec::Zero(b.size());
                res = krylov->solve(A, *M, b, x);
            }
            std::vector<double> times;
            for (int k = 0; k < ex.steps; ++k) {
                core::Vec x = core::Vec::Zero(b.size());
                MPI_Barrier(comm);
                const double t0 = MPI_Wtime();
                res = krylov->solve(A, *M, b, x);
                MPI_Barrier(comm);
                times.push_back(MPI_Wtime() - t0);
            }
            if (rank == 0) {
                std::ostringstream s;
                s << std::setprecision(17) << "{\"solve_s\": [";
                for (size_t k = 0; k < times.size(); ++k) s << (k ? ", " : "") << times[k];
                s << "], \"iterations\": " << res.iterations << ", \"converged\": " << (res.converged ? "true" : "false")
                  << ", \"true_rel_residual\": " << res.true_rel_residual << ", \"setup_s\": " << t_setup
                  << ", \"ranks\": " << np << ", \"n0\": " << (two ? two->stats().n0 : 0) << "}";
                std::cout << s.str() << std::endl;
            }
            MPI_Finalize();
            return 0;
        }

        // ------------------------------------------------------------------ dump mode
        Writer w(ex.dump, rank);
        const std::string p = "sub" + std::to_string(rank) + "_";
        const int64_t n = sys.n_global;
        {
            std::vector<int64_t> meta = {(int64_t)sys.rowBegin(), (int64_t)sd.nOwned(), (int64_t)sd.nGhost(),
                                         two ? (int64_t)two->coarse().localDimension() : 0};
            w.i64(p + "meta", meta);
            w.i64(p + "ghosts", sd.ghosts());
            w.vec(p + "D", sd.pou());
            if (two) {
                const core::Mat& V = two->coarse().basis();
                w.put(p + "V", "f64", V.data(), (size_t)V.size());  // column-major n_local x m
            }
            // exact local factors
            const auto& ls = one->localSolver();
            const bool single = cfg.local_precision == "single";
            Factor F;
            if (single) {
                Raw<float> raw;
                export_factor<float>(sd.Aii(), ls.factorization(), F, raw);
                write_factor(w, p, F, raw);
            } else {
                Raw<double> raw;
                export_factor<double>(sd.Aii(), ls.factorization(), F, raw);
                write_factor(w, p, F, raw);
            }
            // the export reproduces the reference's own local solve
            const std::vector<double> bl = seeded((size_t)sd.nLocal(), 777 + (unsigned long long)rank);
            core::Vec bv = Eigen::Map<const core::Vec>(bl.data(), (Eigen::Index)bl.size()), xv;
            ls.solve(bv, xv);
            const std::vector<double> xe = factor_solve(F, bl);
            double num = 0, den = 0;
            for (size_t k = 0; k < xe.size(); ++k) {
                num += (xe[k] - xv[(Eigen::Index)k]) * (xe[k] - xv[(Eigen::Index)k]);
                den += xv[(Eigen::Index)k] * xv[(Eigen::Index)k];
            }
            const double rel = std::sqrt(num / std::max(den, 1e-300));
            if (rel > (single ? 1e-4 : 1e-10)) {
                std::ostringstream m;
                m << "factor export of rank " << rank << " disagrees with LocalSolver::solve: " << rel;
                throw std::runtime_error(m.str());
            }
            w.vec(p + "ls_b", bl);
            w.vec(p + "ls_x", xv);
            w.scalar(p + "ls_export_rel", rel);
            // Aii (column-major CSC as stored by the reference)
            std::vector<int64_t> cp(sd.Aii().outerIndexPtr(), sd.Aii().outerIndexPtr() + sd.nLocal() + 1);
            std::vector<int32_t> ri(sd.Aii().innerIndexPtr(), sd.Aii().innerIndexPtr() + sd.Aii().nonZeros());
            std::vector<double> av(sd.Aii().valuePtr(), sd.Aii().valuePtr() + sd.Aii().nonZeros());
            w.i64(p + "Aii_cp", cp);
            w.i32(p + "Aii_ri", ri);
            w.vec(p + "Aii_v", av);
        }
        if (rank == 0) {
            w.i64("global_ownership", sys.ownership);
            w.i64("global_A_rp", info.A_perm.row_ptr);
            w.i64("global_A_ci", info.A_perm.col);
            w.vec("global_A_v", info.A_perm.val);
            w.vec("global_b", info.b_perm);
            std::vector<int32_t> part(info.part.begin(), info.part.end());
            w.i32("global_part", part);
            w.i64("global_new_to_old", info.new_to_old);
            std::vector<int64_t> meta = {n, np, sys.symmetric ? 1 : 0, two ? (int64_t)two->stats().n0 : 0};
            w.i64("global_meta", meta);
            if (two) w.i64("global_coarse_offsets", two->coarse().offsets());
        }
        // reference outputs: SpMV and applies of seeded vectors (renumbered ordering)
        for (int k = 0; k < ex.napply; ++k) {
            const std::vector<double> rg = seeded((size_t)n, 1000 + (unsigned long long)k);
            const core::Vec r = owned_part(rg, sys);
            core::Vec y, z, z1, x0;
            A.apply(r, y);
            M->apply(r, z);
            one->apply(r, z1);
            if (two && two->coarse().dimension() > 0) two->coarse().apply(r, x0);
            const auto gy = part::DomainDecomposer::gather(sys, y);
            const auto gz = part::DomainDecomposer::gather(sys, z);
            const auto gz1 = part::DomainDecomposer::gather(sys, z1);
            std::vector<double> gx0;
            if (two && two->coarse().dimension() > 0) gx0 = part::DomainDecomposer::gather(sys, x0);
            if (rank == 0) {
                const std::string q = "apply" + std::to_string(k) + "_";
                w.vec(q + "r", rg);
                w.vec(q + "spmv", gy);
                w.vec(q + "z", gz);
                w.vec(q + "one_level", gz1);
                if (!gx0.empty()) w.vec(q + "coarse", gx0);
            }
        }
        // a full Krylov solve
        core::Vec x = core::Vec::Zero(b.size());
        const solv::KrylovResult res = krylov->solve(A, *M, b, x);
        const auto gx = part::DomainDecomposer::gather(sys, x);
        if (rank == 0) {
            w.vec("krylov_x", gx);
            w.vec("krylov_history", res.history);
            std::vector<double> meta = {(double)res.iterations,  res.converged ? 1.0 : 0.0, res.rel_residual,
                                        res.true_rel_residual,   (double)res.restarts,   res.breakdown ? 1.0 : 0.0,
                                        res.initial_residual_of, res.final_residual_of};
            w.vec("krylov_meta", meta);
        }
    } catch (const std::exception& e) {
        std::cerr << "[rank " << rank << "] error: " << e.what() << std::endl;
        MPI_Abort(comm, 1);
    }
    MPI_Finalize();
    return 0;
}
