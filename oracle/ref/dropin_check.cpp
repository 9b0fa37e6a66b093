// Checks the C++ drop-in (algebraic-multilevel-preconditioner_b200/host/s2l_dropin.*) against the
// reference itself.  TEST INFRASTRUCTURE ONLY (run by tests/test_gpu_dropin.py on the GPU host).
//
// With the reference's flags it builds, on S2L_NP thread-ranks, the reference's own
// preconditioner and Krylov solver and the drop-in GpuTwoLevelSchwarz / GpuKrylov from the same
// set-up objects, then compares: Preconditioner::apply of seeded vectors (relative difference), and
// KrylovSolver::solve (iterations, convergence, true residual, solution).  With S2L_DROPIN_UPDATE
// set to "reuse" or "refactorize" it then gives the matrix new values (D A D, same pattern,
// Subdomain::updateValues), calls update() with that level on both preconditioners and compares
// again.  Rank 0 prints one JSON line; the exit code is 0 when every comparison is within tolerance.
#include "s2l_dropin.hpp"

#include "domain_decomposer.hpp"
#include "mpi_utils.hpp"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>

using namespace schwarz2lvl;

int main(int argc, char** argv)
{
    MPI_Init(&argc, &argv);
    MPI_Comm comm = MPI_COMM_WORLD;
    const int rank = core::mpiRank(comm);
    int code = 0;
    try {
        const core::SolverConfig cfg = core::SolverConfig::fromCommandLine(argc, argv);
        part::DecompositionInfo info;
        core::LocalSystem sys = part::DomainDecomposer::decompose(cfg, comm, info);
        const char* upd = std::getenv("S2L_DROPIN_UPDATE");
        const std::string update_level = upd ? upd : "";
        part::Subdomain sd(sys, cfg.pou);
        linalg::DistributedMatrix A(sd);
        std::unique_ptr<prec::Preconditioner> M;
        const prec::OneLevelSchwarz* one = nullptr;
        const prec::TwoLevelSchwarz* two = nullptr;
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
        auto phase = std::make_shared<s2l::dropin::GpuSolvePhase>(sd, *one, two, cfg, 0, 0,
                                                                  update_level == "refactorize");
        s2l::dropin::GpuTwoLevelSchwarz G(phase, M->name());
        // apply parity on seeded vectors (U[-1,1], owned part of a global renumbered vector)
        auto apply_diff = [&]() {
            double worst = 0.0;
            for (int k = 0; k < 3; ++k) {
                std::mt19937_64 g(4242 + k);
                std::uniform_real_distribution<double> u(-1.0, 1.0);
                std::vector<double> rg((size_t)sys.n_global);
                for (auto& v : rg) v = u(g);
                core::Vec r(sys.nOwned()), z1, z2;
                for (int i = 0; i < sys.nOwned(); ++i) r[i] = rg[(size_t)(sys.rowBegin() + i)];
                M->apply(r, z1);
                G.apply(r, z2);
                double num = (z1 - z2).squaredNorm(), den = z1.squaredNorm();
                double gn = 0.0, gd = 0.0;
                MPI_Allreduce(&num, &gn, 1, MPI_DOUBLE, MPI_SUM, comm);
                MPI_Allreduce(&den, &gd, 1, MPI_DOUBLE, MPI_SUM, comm);
                worst = std::max(worst, std::sqrt(gn / gd));
            }
            return worst;
        };
        double worst = apply_diff();
        // the two parts of the apply on their own (the drop-in's device setup through the C ABI on
        // rank 0): the one-level apply (local solves, exact factors on both sides) and the coarse
        // correction (E solved by the reference's factorization, by the explicit inverse on the GPU)
        auto part_diff = [&](bool coarse_part) {
            std::mt19937_64 g(777);
            std::uniform_real_distribution<double> u(-1.0, 1.0);
            std::vector<double> rg((size_t)sys.n_global);
            for (auto& v : rg) v = u(g);
            core::Vec r(sys.nOwned()), z1, z2;
            for (int i = 0; i < sys.nOwned(); ++i) r[i] = rg[(size_t)(sys.rowBegin() + i)];
            if (coarse_part) two->coarse().apply(r, z1);
            else one->apply(r, z1);
            std::vector<double> rgl, zgl;
            phase->gather(r, rgl);
            int st = 0;
            if (rank == 0) {
                zgl.assign(rgl.size(), 0.0);
                st = coarse_part ? s2l_gpu_coarse_apply(phase->setup(), rgl.data(), zgl.data(), S2L_PTR_HOST)
                                 : s2l_gpu_one_level_apply(phase->setup(), rgl.data(), zgl.data(), S2L_PTR_HOST);
            }
            phase->check(st, "component apply");
            phase->scatter(zgl, z2);
            double num = (z1 - z2).squaredNorm(), den = z1.squaredNorm(), gn = 0.0, gd = 0.0;
            MPI_Allreduce(&num, &gn, 1, MPI_DOUBLE, MPI_SUM, comm);
            MPI_Allreduce(&den, &gd, 1, MPI_DOUBLE, MPI_SUM, comm);
            return std::sqrt(gn / gd);
        };
        const double one_diff = part_diff(false);
        const double coarse_diff = (two && cfg.coarse != "none" && two->coarse().dimension() > 0) ? part_diff(true) : 0.0;
        std::string level_out;
        if (!update_level.empty()) {
            // new values D A D with d(g) = 1 + 0.1 sin(1 + 0.37 g) (same pattern, symmetric kept)
            auto d = [](int64_t g) { return 1.0 + 0.1 * std::sin(1.0 + 0.37 * (double)g); };
            for (int i = 0; i < sys.nOwned(); ++i)
                for (int64_t e = sys.row_ptr[i]; e < sys.row_ptr[i + 1]; ++e)
                    sys.val[e] *= d(sys.rowBegin() + i) * d(sys.col[e]);
            sd.updateValues();
            const prec::UpdateLevel want =
                update_level == "refactorize" ? prec::UpdateLevel::Refactorize : prec::UpdateLevel::Reuse;
            const prec::UpdateLevel l1 = M->update(want);
            const prec::UpdateLevel l2 = G.update(want);
            if (l1 != l2) throw std::runtime_error("update levels differ");
            level_out = prec::toString(l2);
            if (G.upToDate() != M->upToDate()) throw std::runtime_error("upToDate differs");
            worst = std::max(worst, apply_diff());
        }
        // solves: the reference's Krylov solver with its preconditioner, the GPU's with the drop-in
        const core::Vec b = Eigen::Map<const core::Vec>(sys.rhs.data(), (Eigen::Index)sys.rhs.size());
        core::Vec x1 = core::Vec::Zero(b.size()), x2 = core::Vec::Zero(b.size());
        const solv::KrylovResult r1 = solv::makeKrylovSolver(cfg)->solve(A, *M, b, x1);
        auto gk = s2l::dropin::makeGpuKrylovSolver(cfg);
        const solv::KrylovResult r2 = gk->solve(A, G, b, x2);
        double num = (x1 - x2).squaredNorm(), den = x1.squaredNorm(), gn = 0, gd = 0;
        MPI_Allreduce(&num, &gn, 1, MPI_DOUBLE, MPI_SUM, comm);
        MPI_Allreduce(&den, &gd, 1, MPI_DOUBLE, MPI_SUM, comm);
        const double xdiff = std::sqrt(gn / gd);
        // residual histories (||r|| / ||b|| after every application of M^-1), common prefix
        double hdiff = 0.0;
        const size_t nh = std::min(r1.history.size(), r2.history.size());
        for (size_t i = 0; i < nh; ++i)
            hdiff = std::max(hdiff, std::abs(r1.history[i] - r2.history[i]) / std::max(std::abs(r1.history[i]), 1e-300));
        const bool single = cfg.local_precision == "single";
        const double tol = single ? 1e-5 : 1e-12;
        const bool of = cfg.stop_norm == "openfoam";
        // L2: the true residual meets rtol (10% slack); OpenFOAM: the normalised residual meets
        // max(rtol x initial, atol) and the initial one is the reference's
        const bool met = of ? (r2.final_residual_of <= 1.1 * std::max(cfg.rtol * r2.initial_residual_of, cfg.atol) &&
                               std::abs(r2.initial_residual_of - r1.initial_residual_of) <=
                                   1e-10 * r1.initial_residual_of)
                            : r2.true_rel_residual <= 1.1 * cfg.rtol;
        const bool ok = worst <= tol && r2.converged && met && std::abs(r1.iterations - r2.iterations) <= (single ? 3 : 1);
        if (rank == 0) {
            std::ostringstream s;
            s << std::setprecision(6) << "{\"apply_rel_diff\": " << worst << ", \"ref_iterations\": " << r1.iterations
              << ", \"gpu_iterations\": " << r2.iterations << ", \"gpu_converged\": " << (r2.converged ? "true" : "false")
              << ", \"gpu_true_rel_residual\": " << r2.true_rel_residual << ", \"ref_true_rel_residual\": "
              << r1.true_rel_residual << ", \"gpu_final_residual_of\": " << r2.final_residual_of
              << ", \"ref_final_residual_of\": " << r1.final_residual_of << ", \"x_rel_diff\": " << xdiff
              << ", \"history_rel_diff\": " << hdiff << ", \"one_level_rel_diff\": " << one_diff
              << ", \"coarse_rel_diff\": " << coarse_diff
              << ", \"gpu_solver\": \"" << gk->name() << "\", \"update\": \"" << level_out
              << "\", \"ok\": " << (ok ? "true" : "false") << "}";
            std::cout << s.str() << std::endl;
        }
        code = ok ? 0 : 1;
    } catch (const std::exception& e) {
        std::cerr << "[rank " << rank << "] error: " << e.what() << std::endl;
        code = 2;
    }
    MPI_Finalize();
    return code;
}
