// Applies the reference's AMG local solver (LocalSolver from makeInexactSolver, AMGCL smoothed
// aggregation + Gauss-Seidel, one V-cycle from x = 0) to given vectors.  TEST INFRASTRUCTURE ONLY:
// tests/golden/make_amg_golden.py runs it to pin the AMG restatement of the setup code and of the
// oracle (src/linalg/inexact_solver.cpp:45-178).
//
// Usage: amg_dump <in.bin> <out.bin> <coarse_enough> <sweeps> <coarsening sa|rs> [<next.bin> <reuse 0|1>]
// in.bin : int64 n, int64 nnz, int64 nvec, int64 rowptr[n + 1], int64 col[nnz], double val[nnz],
//          double vectors[nvec][n]          (CSR of A_ii, sorted columns)
// next.bin: the same layout with nvec = 0: new values of A_ii; the solver is then refactorize()d
//          with them (AmgOptions::reuse: keep the transfer operators, else a new hierarchy)
// out.bin: double results[nvec][n]          (the solver's solve() of each vector)
// S2L_AMG_SINGLE=1 in the environment: the solver in single precision (--local-precision single)
#include "inexact_solver.hpp"

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

using namespace schwarz2lvl;

static bool read_matrix(const char* path, core::SpMat& A, int64_t& n, int64_t& nvec, std::vector<double>& x)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    int64_t hdr[3];
    if (std::fread(hdr, sizeof(int64_t), 3, f) != 3) {
        std::fclose(f);
        return false;
    }
    n = hdr[0];
    const int64_t nnz = hdr[1];
    nvec = hdr[2];
    std::vector<int64_t> rp(n + 1), ci(nnz);
    std::vector<double> v(nnz);
    x.assign((size_t)(n * nvec), 0.0);
    const bool ok = std::fread(rp.data(), sizeof(int64_t), n + 1, f) == (size_t)(n + 1) &&
                    std::fread(ci.data(), sizeof(int64_t), nnz, f) == (size_t)nnz &&
                    std::fread(v.data(), sizeof(double), nnz, f) == (size_t)nnz &&
                    std::fread(x.data(), sizeof(double), n * nvec, f) == (size_t)(n * nvec);
    std::fclose(f);
    if (!ok) return false;
    std::vector<Eigen::Triplet<double, core::LocalIndex>> t;
    t.reserve(nnz);
    for (int64_t r = 0; r < n; ++r)
        for (int64_t e = rp[r]; e < rp[r + 1]; ++e) t.emplace_back((core::LocalIndex)r, (core::LocalIndex)ci[e], v[e]);
    A.resize(n, n);
    A.setFromTriplets(t.begin(), t.end());
    A.makeCompressed();
    return true;
}

int s2l_rank_main(int argc, char** argv)
{
    if (argc < 6) {
        std::cerr << "usage: amg_dump in.bin out.bin coarse_enough sweeps sa|rs [next.bin reuse]\n";
        return 1;
    }
    int64_t n = 0, nvec = 0;
    std::vector<double> x;
    core::SpMat A;
    if (!read_matrix(argv[1], A, n, nvec, x)) return 1;
    linalg::LocalSolverSpec spec;
    spec.approx = "amg";
    spec.amg.coarse_enough = std::atoi(argv[3]);
    spec.amg.sweeps = std::atoi(argv[4]);
    spec.amg.coarsening = argv[5];
    spec.amg.reuse = argc >= 8 && std::atoi(argv[7]) != 0;
    const char* single = std::getenv("S2L_AMG_SINGLE");  // 1: --local-precision single (AMGCL in float)
    spec.single = single && std::atoi(single) != 0;
    auto solver = linalg::makeInexactSolver(spec);
    if (!solver->factorize(A)) {
        std::cerr << "AMG setup failed: " << solver->lastError() << "\n";
        return 2;
    }
    if (argc >= 8) {
        core::SpMat A1;
        int64_t n1 = 0, nv1 = 0;
        std::vector<double> none;
        if (!read_matrix(argv[6], A1, n1, nv1, none) || n1 != n) return 1;
        if (!solver->refactorize(A1)) {
            std::cerr << "AMG refactorization failed: " << solver->lastError() << "\n";
            return 2;
        }
    }
    std::cerr << solver->name() << "\n";
    std::vector<double> out((size_t)(n * nvec));
    for (int64_t k = 0; k < nvec; ++k) {
        core::Vec b = Eigen::Map<core::Vec>(x.data() + k * n, n), y;
        solver->solve(b, y);
        for (int64_t i = 0; i < n; ++i) out[(size_t)(k * n + i)] = y[i];
    }
    FILE* g = std::fopen(argv[2], "wb");
    if (!g) return 1;
    std::fwrite(out.data(), sizeof(double), out.size(), g);
    std::fclose(g);
    return 0;
}
