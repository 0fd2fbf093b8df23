// cg front end.  Keeps the reference binary's surface (CG/src/main.cu:23-278):
// the version table and indices, -v (comma list), -s, -niter (default
// 10000), -num_runs, -matrix_path, -compare-single-gpu, -compare-cpu; the
// default matrix is the reference's random tridiagonal one with
// n = 20,971,520 (CG/src/main.cu:118-129), b = ones, x0 = 0, a fixed
// iteration count, and "Execution time: %8.4f s" per run.
// Additive flags:
//   -problem tridiag|poisson   matrix (poisson: 7-point Dirichlet Poisson CSR)
//   -grid G                    poisson grid side (default 128 -> n = G^3)
//   -tol T                     stop at ||b-Ax||/||b|| <= T (with -maxiter cap)
//   -maxiter M                 iteration cap in tolerance mode (default 20000)
//   -seed S                    poisson: x* ~ U[-1,1) from Philox(S), b = A x*
#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

#include "cfm.h"
#include "cli_common.h"

int main(int argc, char **argv) {
    using cli::Version;
    const char *multi = nullptr;
    const std::vector<Version> versions = {
        {"Baseline Discrete Standard", CFM_CG_DISCRETE, multi},
        {"Baseline Discrete Pipelined", CFM_CG_DISCRETE, multi},
        {"Single Stream Standard", CFM_CG_PERSISTENT, multi},
        {"Single Stream Pipelined", CFM_CG_PERSISTENT_PIPELINED, multi},
        {"Single Stream Pipelined Multi Overlap", CFM_CG_PERSISTENT_PIPELINED, multi},
        {"Single Stream Standard Saxpy Overlap", CFM_CG_PERSISTENT, multi},
        {"Profiling Discrete Standard", CFM_CG_DISCRETE, multi},
        {"Profiling Discrete Pipelined", CFM_CG_DISCRETE, multi},
        {"Single GPU Discrete Standard", CFM_CG_DISCRETE, multi},
        {"Single Stream Pipelined Gather", CFM_CG_PERSISTENT_PIPELINED, multi},
    };
    const std::string vlist = cli::argval<std::string>(argc, argv, "-v", "0");
    const bool silent = cli::has(argc, argv, "-s");
    const int niter = cli::argval<int>(argc, argv, "-niter", 10000);
    const int num_runs = cli::argval<int>(argc, argv, "-num_runs", 1);
    const std::string matrix_path = cli::argval<std::string>(argc, argv, "-matrix_path", "");
    const bool cmp_sgpu = cli::has(argc, argv, "-compare-single-gpu");
    const bool cmp_cpu = cli::has(argc, argv, "-compare-cpu");
    const std::string problem = cli::argval<std::string>(argc, argv, "-problem", "tridiag");
    const int grid = cli::argval<int>(argc, argv, "-grid", 128);
    const double tol = cli::argval<double>(argc, argv, "-tol", 0.0);
    const int maxiter = cli::argval<int>(argc, argv, "-maxiter", 20000);
    const unsigned long long seed = cli::argval<unsigned long long>(argc, argv, "-seed", 0ULL);

    std::vector<int> sel;
    {
        std::stringstream ss(vlist);
        std::string tok;
        while (std::getline(ss, tok, ',')) {
            try {
                sel.push_back(std::stoi(tok));
            } catch (...) {
                std::fprintf(stderr, "ERROR: bad -v entry '%s'\n", tok.c_str());
                return 1;
            }
        }
    }
    for (int v : sel)
        if (v < 0 || v >= (int)versions.size()) {
            std::fprintf(stderr, "ERROR: -v %d out of range [0, %zu)\n", v, versions.size());
            return 1;
        }
    if (cmp_cpu)
        std::fprintf(stderr,
                     "NOTE: -compare-cpu ignored: the reference's CPU CG never writes its SpMV "
                     "output (CG/src/common.cu:784-798); use -compare-single-gpu\n");

    // ---- matrix and right-hand side
    int n = 0;
    std::vector<int> rowptr, col;
    std::vector<double> val, b;
    if (!matrix_path.empty()) {
        // MatrixMarket file, as the reference's -matrix_path (b = ones)
        int m = 0, nn = 0;
        long long nnz = 0;
        int st = cfm_mm_read(matrix_path.c_str(), &m, &nn, &nnz, nullptr, nullptr, nullptr);
        if (st) return cli::fail("cfm_mm_read", st);
        if (m != nn) {
            std::fprintf(stderr, "ERROR: -matrix_path: the matrix is %d x %d, not square\n", m, nn);
            return 1;
        }
        n = m;
        rowptr.resize(n + 1);
        col.resize(nnz);
        val.resize(nnz);
        if ((st = cfm_mm_read(matrix_path.c_str(), &m, &nn, &nnz, rowptr.data(), col.data(), val.data())))
            return cli::fail("cfm_mm_read", st);
    } else if (problem == "tridiag") {
        n = 10485760 * 2;
        const long long nnz = (long long)(n - 2) * 3 + 4;
        rowptr.resize(n + 1);
        col.resize(nnz);
        val.resize(nnz);
        cfm_tridiag_csr(n, rowptr.data(), col.data(), val.data());
    } else if (problem == "poisson") {
        const long long nnz = cfm_poisson3d_nnz(grid, grid, grid);
        n = grid * grid * grid;
        rowptr.resize(n + 1);
        col.resize(nnz);
        val.resize(nnz);
        int st = cfm_poisson3d_csr(grid, grid, grid, rowptr.data(), col.data(), val.data());
        if (st) return cli::fail("poisson matrix", st);
    } else {
        std::fprintf(stderr, "ERROR: -problem must be tridiag or poisson\n");
        return 1;
    }
    cfm_csr *A = nullptr;
    int st = cfm_csr_create(n, (long long)val.size(), rowptr.data(), col.data(), val.data(), &A);
    if (st) return cli::fail("cfm_csr_create", st);
    if (problem == "poisson") {
        std::vector<double> xs(n);
        cfm_uniform(seed, n, -1.0, 1.0, xs.data());
        b.resize(n);
        if ((st = cfm_csr_spmv_host(A, xs.data(), b.data()))) return cli::fail("b = A x*", st);
    }
    const double *bptr = b.empty() ? nullptr : b.data();

    cfm_cg_params base{};
    base.maxiter = tol > 0 ? maxiter : niter;
    base.tol = tol;

    std::vector<double> x_ref;
    double t_ref = -1;
    if (cmp_sgpu) {
        cfm_cg_params pr = base;
        pr.impl = CFM_CG_DISCRETE;
        cfm_cg *hr = nullptr;
        if ((st = cfm_cg_create(A, &pr, &hr))) return cli::fail("reference create", st);
        x_ref.resize(n);
        cfm_stats s{};
        st = cfm_cg_solve(hr, bptr, x_ref.data(), &s);
        if (st && st != CFM_NOT_CONVERGED) return cli::fail("reference solve", st);
        t_ref = s.seconds;
        cfm_cg_destroy(hr);
    }

    int rc = 0;
    std::vector<double> x(n);
    for (int v : sel) {
        const Version &ver = versions[v];
        if (!silent) {
            cli::print_versions(versions);
            std::printf("Running %s\n\n", ver.name);
        }
        cfm_cg_params pp = base;
        pp.impl = ver.impl;
        cfm_cg *h = nullptr;
        if ((st = cfm_cg_create(A, &pp, &h))) return cli::fail("cfm_cg_create", st);
        for (int run = 1; run <= num_runs; ++run) {
            cfm_stats s{};
            st = cfm_cg_solve(h, bptr, x.data(), &s);
            if (st && st != CFM_NOT_CONVERGED) return cli::fail("cfm_cg_solve", st);
            bool ok = true;
            if (cmp_sgpu && run == 1) {
                for (int i = 0; i < n; ++i)
                    if (std::fabs(x_ref[i] - x[i]) > 1e-5 || std::isnan(x[i]) ||
                        std::isnan(x_ref[i])) {
                        std::fprintf(stderr,
                                     "ERROR: x[%d] = %.8f does not match %.8f (Single GPU "
                                     "reference)\n",
                                     i, x[i], x_ref[i]);
                        ok = false;
                        rc = 3;
                        break;
                    }
            }
            if (ok) {
                std::printf("Execution time: %8.4f s\n", s.seconds);
                if (cmp_sgpu && run == 1)
                    std::printf(
                        "Non-persistent kernel - 1 GPU: %8.4f s, 1 GPUs: %8.4f s, speedup: "
                        "%8.2f, efficiency: %8.2f \n",
                        t_ref, s.seconds, t_ref / s.seconds, t_ref / s.seconds * 100);
            }
            std::printf("Iterations: %lld, restarts: %d, true relative residual: %.3e, %.1f GB/s, "
                        "%d launches%s\n",
                        s.iterations, s.refinements, s.residual, s.gbs, s.launches,
                        st == CFM_NOT_CONVERGED ? " (not converged)" : "");
        }
        cfm_cg_destroy(h);
    }
    cfm_csr_destroy(A);
    return rc;
}
