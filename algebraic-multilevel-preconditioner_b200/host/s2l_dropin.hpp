/**
 * @file s2l_dropin.hpp
 * @brief Drop-in classes that move the solve phase of schwarz2lvl onto one B200.
 *
 * Compiled inside the reference's build (they derive from its classes):
 *  - GpuTwoLevelSchwarz replaces prec::TwoLevelSchwarz / prec::OneLevelSchwarz as the
 *    prec::Preconditioner of the solve (include/preconditioner/preconditioner.hpp:64-96);
 *  - GpuKrylov replaces solv::Gmres / solv::BiCgStab as the solv::KrylovSolver
 *    (include/solver/krylov.hpp:60-76), built by makeGpuKrylovSolver() in place of
 *    solv::makeKrylovSolver() (src/solver/krylov.cpp:23-36).
 *
 * Construction is collective: every rank hands over its subdomain, its set-up reference
 * preconditioner (local factors, coarse basis) and its owned rows; rank 0 gathers them and owns
 * the device copy (all subdomains resident on one GPU), through the C ABI of include/s2l_gpu.h.
 * apply() and solve() keep the reference's conventions: owned entries in, owned entries out,
 * collective over the communicator, errors as exceptions (std::invalid_argument for bad
 * arguments, std::runtime_error for numerical or device failures, std::logic_error for misuse).
 */
#ifndef S2L_DROPIN_HPP
#define S2L_DROPIN_HPP

#include "config.hpp"
#include "distributed_matrix.hpp"
#include "krylov.hpp"
#include "one_level_schwarz.hpp"
#include "preconditioner.hpp"
#include "subdomain.hpp"
#include "two_level_schwarz.hpp"

#include "s2l_gpu.h"

#include <memory>
#include <string>
#include <vector>

namespace s2l::dropin {

/// @brief The device copy of one matrix's setup, shared by the preconditioner and the solver.
class GpuSolvePhase {
public:
    /**
     * @brief Gathers every rank's subdomain on rank 0 and uploads it (collective).
     * @param sd     Subdomain of the calling rank.
     * @param one    Its one-level preconditioner (the local factors are those of one.localSolver()).
     * @param two    Its two-level preconditioner (coarse basis and offsets), or nullptr (one level).
     * @param cfg    Configuration (variants, precision).
     * @param device CUDA device of rank 0.
     * @param hbm_budget Device bytes the setup may use (0 = no limit).
     * @param refactorize Keep the factor patterns on the device so that update(Refactorize) can
     *                    refactorize there (setup option "refactor").
     * With --local-approx amg every rank builds the AMG hierarchy of its A_ii with the library's
     * host setup (s2l_amg_build, the reference's AMGCL setup restated; FP64 only), and
     * update(Refactorize) builds it again (or, with --amg-reuse, keeps its transfer operators) and
     * uploads the setup anew with the kept coarse basis.
     */
    GpuSolvePhase(const schwarz2lvl::part::Subdomain& sd, const schwarz2lvl::prec::OneLevelSchwarz& one,
                  const schwarz2lvl::prec::TwoLevelSchwarz* two, const schwarz2lvl::core::SolverConfig& cfg,
                  int device = 0, size_t hbm_budget = 0, bool refactorize = false);
    ~GpuSolvePhase();
    GpuSolvePhase(const GpuSolvePhase&) = delete;
    GpuSolvePhase& operator=(const GpuSolvePhase&) = delete;

    MPI_Comm comm() const { return comm_; }
    int rank() const { return rank_; }
    /// @brief Global vector on rank 0 from the owned entries of every rank (collective).
    void gather(const schwarz2lvl::core::Vec& owned, std::vector<double>& global) const;
    /// @brief Owned entries from a global vector held by rank 0 (collective).
    void scatter(const std::vector<double>& global, schwarz2lvl::core::Vec& owned) const;
    /// @brief Device setup (rank 0 only; nullptr elsewhere).
    s2l_setup* setup() const { return setup_; }
    /// @brief Throws the exception type of a failed status (rank 0), agreed on by every rank.
    void check(int status, const char* what) const;
    /// @brief The matrix values of every rank's rows (Subdomain::system(), after
    ///        Subdomain::updateValues) to the device (collective): Reuse gives the operator its new
    ///        values and keeps the preconditioner (s2l_gpu_update_matrix); Refactorize also
    ///        refactorizes the local factors and refreshes E on the device (s2l_gpu_refactor).
    void pushValues(schwarz2lvl::prec::UpdateLevel level);
    /// @brief The device operator holds the subdomain's current values.
    bool operatorCurrent() const;
    /// @brief The device preconditioner was built (or refactorized) from the current values.
    bool preconditionerCurrent() const;

private:
    /// @brief This rank's part (rows, ghosts, D, local factors or AMG levels, V) to rank 0, which
    ///        uploads every part as a new device setup (collective).
    void upload();
    /// @brief This rank's AMG hierarchy of sd.Aii() (collective: every rank agrees on the status).
    void buildAmg(bool keep_transfer);

    MPI_Comm comm_;
    int rank_ = 0, np_ = 1;
    schwarz2lvl::core::GlobalIndex n_ = 0;
    std::vector<int> counts_, displs_;
    s2l_ctx* ctx_ = nullptr;
    s2l_setup* setup_ = nullptr;
    const schwarz2lvl::part::Subdomain* sd_ = nullptr;
    std::vector<int> nnz_counts_, nnz_displs_;  // matrix values per rank (rank 0)
    long op_version_ = 0, prec_version_ = 0;     // Subdomain::valuesVersion() of the device copies
    // what upload() needs again after a refactorization of AMG local solvers
    schwarz2lvl::core::SolverConfig cfg_;
    int device_ = 0;
    size_t hbm_budget_ = 0;
    bool refactorize_ = false, coarse_ = false, amg_on_ = false;
    int factorization_ = 0;     // linalg::Factorization of the reference's local solver (factors)
    std::vector<double> V_;     // this rank's coarse basis (column-major, n_local x m_)
    int m_ = 0;
    s2l_amg* amg_ = nullptr;    // this rank's AMG hierarchy (--local-approx amg)
};

/// @brief z = M^{-1} r on the GPU: the two-level (or one-level) Schwarz apply of the reference.
class GpuTwoLevelSchwarz final : public schwarz2lvl::prec::Preconditioner {
public:
    GpuTwoLevelSchwarz(std::shared_ptr<GpuSolvePhase> phase, std::string name)
        : phase_(std::move(phase)), name_(std::move(name)) {}
    void apply(const schwarz2lvl::core::Vec& r, schwarz2lvl::core::Vec& z) const override;
    /// @brief The reference's update contract (include/preconditioner/preconditioner.hpp:64-96,
    ///        src/preconditioner/two_level_schwarz.cpp:30-41), collective: Reuse keeps the
    ///        preconditioner (the device operator takes the new values), Refactorize refactorizes on
    ///        the device (AMG local solvers: on the host, then uploaded; returns Reuse when already
    ///        up to date); Rebuild recomputes the coarse basis
    ///        on the host and needs a new GpuSolvePhase (std::logic_error).
    schwarz2lvl::prec::UpdateLevel update(schwarz2lvl::prec::UpdateLevel requested) override;
    bool upToDate() const override { return phase_->preconditionerCurrent(); }
    std::string name() const override { return name_ + " (B200)"; }
    const std::shared_ptr<GpuSolvePhase>& phase() const { return phase_; }

private:
    std::shared_ptr<GpuSolvePhase> phase_;
    std::string name_;
};

/// @brief Right-preconditioned GMRES(m) or BiCGStab with every step on the GPU.
class GpuKrylov final : public schwarz2lvl::solv::KrylovSolver {
public:
    GpuKrylov(std::string method, int restart, double rtol, int maxit, bool flexible, bool strict,
              schwarz2lvl::solv::StopNorm stop = schwarz2lvl::solv::StopNorm::L2, double atol = 0.0)
        : method_(std::move(method)), restart_(restart), rtol_(rtol), maxit_(maxit), flexible_(flexible),
          strict_(strict), stop_(stop), atol_(atol) {}
    /// @brief M must be a GpuTwoLevelSchwarz (std::invalid_argument otherwise).
    schwarz2lvl::solv::KrylovResult solve(const schwarz2lvl::linalg::DistributedMatrix& A,
                                          const schwarz2lvl::prec::Preconditioner& M,
                                          const schwarz2lvl::core::Vec& b, schwarz2lvl::core::Vec& x) const override;
    std::string name() const override;

private:
    std::string method_;
    int restart_;
    double rtol_;
    int maxit_;
    bool flexible_, strict_;
    schwarz2lvl::solv::StopNorm stop_;
    double atol_;
};

/// @brief The GPU counterpart of solv::makeKrylovSolver(cfg) (src/solver/krylov.cpp:23-36):
///        --krylov gmres|bicgstab, --restart, --rtol, --atol, --maxit, --stop-norm l2|openfoam; FP32
///        local factors (--local-precision single) select flexible GMRES with an FP64 true-residual
///        acceptance.
std::unique_ptr<schwarz2lvl::solv::KrylovSolver> makeGpuKrylovSolver(const schwarz2lvl::core::SolverConfig& cfg);
/// @brief Same, with the tolerances @p rtol and @p atol instead of those of @p cfg (e.g. the last
///        corrector), as solv::makeKrylovSolver(cfg, rtol, atol).
std::unique_ptr<schwarz2lvl::solv::KrylovSolver> makeGpuKrylovSolver(const schwarz2lvl::core::SolverConfig& cfg,
                                                                     double rtol, double atol);

}  // namespace s2l::dropin

#endif
