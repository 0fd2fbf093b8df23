// jacobi2D / jacobi3D front end (compiled twice, CFM_DIMS = 2 or 3).
//
// Keeps the reference binaries' surface (Stencil/jacobi2D/src/main.cu:24-68,
// Stencil/jacobi3D/src/main.cu:30-72): the same version table and indices,
// -v/-s/-nx/-ny/-nz/-niter/-compare with the same defaults, and
// "Execution time: %8.4f s" as the first line after the version banner
// (the bench scripts take the first float they see, Scripts/bench.py:85).
// Additive flags (after the reference's, never changing the first float):
//   -precision fp32|fp64   grid type (reference: fp32, `typedef float real`)
//   -problem ref|config    initial state, see cfm.h (3D config is y-periodic)
//   -out FILE              write the final grid (raw, row-major) to FILE
//   -boundary dirichlet|mirror
//                          2D x boundary, see cfm_boundary in cfm.h.  Default:
//                          mirror for PERKS, whose reference run is checked
//                          against the mirror sweep (Stencil/jacobi2D/src/
//                          PERKS/multi-stream-perks.cu:225-226), dirichlet for
//                          every other version and for 3D
#include <cstdio>
#include <string>
#include <vector>

#include "cfm.h"
#include "cli_common.h"

#ifndef CFM_DIMS
#define CFM_DIMS 3
#endif

int main(int argc, char **argv) {
    using cli::Version;
    const char *nocomp =
        "measures multi-GPU halo communication only (no stencil); there is no halo exchange on one GPU";
    const std::vector<Version> versions = {
        {"Baseline Copy", CFM_JACOBI_HOST_LOOP, nullptr},
        {"Baseline Overlap", CFM_JACOBI_HOST_LOOP, nullptr},
        {"Baseline P2P", CFM_JACOBI_HOST_LOOP_INKERNEL_HALO, nullptr},
        {"Design 1", CFM_JACOBI_PERSISTENT, nullptr},
        {"Design 2", CFM_JACOBI_PERSISTENT, nullptr},
        {"PERKS", CFM_JACOBI_RESIDENT, nullptr},
        {"Baseline Copy (No computation)", -1, nocomp},
        {"Baseline Overlap (No Computation)", -1, nocomp},
        {"Baseline P2P (No Computation)", -1, nocomp},
        {"Design 1 (No Computation)", -1, nocomp},
        {"Design 2 (No Computation)", -1, nocomp},
    };
    const int sel = cli::argval<int>(argc, argv, "-v", 0);
    const bool silent = cli::has(argc, argv, "-s");
    if (sel < 0 || sel >= (int)versions.size()) {
        std::fprintf(stderr, "ERROR: -v %d out of range [0, %zu)\n", sel, versions.size());
        return 1;
    }
    const Version &v = versions[sel];
    if (!silent) {
        cli::print_versions(versions);
        std::printf("Running %s\n\n", v.name);
    }
    if (v.impl < 0) {
        std::fprintf(stderr, "ERROR: version %d (%s) %s\n", sel, v.name, v.why);
        return 2;
    }

    cfm_jacobi_params p{};
    p.dims = CFM_DIMS;
    const int niter = cli::argval<int>(argc, argv, "-niter", 1000);
    p.nx = cli::argval<int>(argc, argv, "-nx", CFM_DIMS == 2 ? 16384 : 512);
    p.ny = cli::argval<int>(argc, argv, "-ny", CFM_DIMS == 2 ? 16384 : 512);
    p.nz = CFM_DIMS == 3 ? cli::argval<int>(argc, argv, "-nz", 512) : 1;
    const bool compare = cli::has(argc, argv, "-compare");
    const std::string prec = cli::argval<std::string>(argc, argv, "-precision", "fp32");
    const std::string prob = cli::argval<std::string>(argc, argv, "-problem", "ref");
    const std::string out = cli::argval<std::string>(argc, argv, "-out", "");
    const std::string bnd = cli::argval<std::string>(
        argc, argv, "-boundary",
        (CFM_DIMS == 2 && v.impl == CFM_JACOBI_RESIDENT) ? "mirror" : "dirichlet");
    if (bnd != "dirichlet" && (bnd != "mirror" || CFM_DIMS != 2)) {
        std::fprintf(stderr, "ERROR: -boundary must be dirichlet%s\n", CFM_DIMS == 2 ? " or mirror" : "");
        return 1;
    }
    const int boundary = bnd == "mirror" ? CFM_BOUNDARY_MIRROR : CFM_BOUNDARY_DIRICHLET;
    if (prec != "fp32" && prec != "fp64") {
        std::fprintf(stderr, "ERROR: -precision must be fp32 or fp64\n");
        return 1;
    }
    if (prob != "ref" && prob != "config") {
        std::fprintf(stderr, "ERROR: -problem must be ref or config\n");
        return 1;
    }
    p.precision = prec == "fp64" ? CFM_FP64 : CFM_FP32;
    const int problem = prob == "config" ? CFM_PROBLEM_CONFIG : CFM_PROBLEM_REF;
    p.periodic_y = (CFM_DIMS == 3 && problem == CFM_PROBLEM_CONFIG) ? 1 : 0;
    p.impl = v.impl;

    cfm_jacobi *h = nullptr;
    int st = cfm_jacobi_create(&p, &h);
    if (st) return cli::fail("cfm_jacobi_create", st);
    if ((st = cfm_jacobi_set_boundary(h, boundary))) return cli::fail("boundary", st);
    if ((st = cfm_jacobi_load_problem(h, problem))) return cli::fail("load problem", st);
    cfm_stats s{};
    st = cfm_jacobi_run(h, niter, &s);
    if (st) return cli::fail("cfm_jacobi_run", st);

    const size_t n = (size_t)p.nx * p.ny * (CFM_DIMS == 3 ? p.nz : 1);
    const size_t es = p.precision == CFM_FP64 ? 8 : 4;
    std::vector<unsigned char> grid(n * es);
    if ((st = cfm_jacobi_download(h, grid.data()))) return cli::fail("download", st);

    bool mismatch = false;
    cfm_stats sref{};
    if (compare) {
        // -compare: the reference reruns its host-loop single_gpu() on the same
        // device and compares interior points at tol 1e-7 (Stencil/jacobi2D/src/
        // common.cu:344-361); mismatches are reported on stderr.
        cfm_jacobi_params pr = p;
        pr.impl = CFM_JACOBI_HOST_LOOP;
        cfm_jacobi *hr = nullptr;
        if ((st = cfm_jacobi_create(&pr, &hr))) return cli::fail("compare create", st);
        if ((st = cfm_jacobi_set_boundary(hr, boundary))) return cli::fail("compare boundary", st);
        if ((st = cfm_jacobi_load_problem(hr, problem))) return cli::fail("compare load", st);
        if ((st = cfm_jacobi_run(hr, niter, &sref))) return cli::fail("compare run", st);
        std::vector<unsigned char> ref(n * es);
        if ((st = cfm_jacobi_download(hr, ref.data()))) return cli::fail("compare download", st);
        cfm_jacobi_destroy(hr);
        long long bad = 0;
        const int nz = CFM_DIMS == 3 ? p.nz : 3;
        for (int z = 1; z < nz - 1; ++z)
            for (int y = 1; y < p.ny - 1; ++y)
                for (int x = 1; x < p.nx - 1; ++x) {
                    const size_t i = ((size_t)(CFM_DIMS == 3 ? z : 0) * p.ny + y) * p.nx + x;
                    const double a = es == 8 ? ((double *)grid.data())[i] : ((float *)grid.data())[i];
                    const double r = es == 8 ? ((double *)ref.data())[i] : ((float *)ref.data())[i];
                    if (std::fabs(a - r) > 1.0e-7) {
                        if (bad < 10)
                            std::fprintf(stderr, "ERROR: a[%zu] = %.8f does not match %.8f (reference)\n",
                                         i, a, r);
                        ++bad;
                    }
                }
        if (bad) {
            std::fprintf(stderr, "ERROR: %lld interior points differ from the host-loop run\n", bad);
            mismatch = true;
        }
    }

    std::printf("Execution time: %8.4f s\n", s.seconds);
    if (compare && !mismatch) {
        std::printf(
            "Non-persistent kernel - %dx%d%s: 1 GPU: %8.4f s, 1 GPUs: %8.4f s, speedup: %8.2f, "
            "efficiency: %8.2f \n",
            p.nx, p.ny, CFM_DIMS == 3 ? ("x" + std::to_string(p.nz)).c_str() : "", sref.seconds,
            s.seconds, sref.seconds / s.seconds, sref.seconds / s.seconds * 100);
    }
    double norm;
    if (es == 8) {
        const double *g = (const double *)grid.data();
        norm = cli::l2_norm(std::vector<double>(g, g + n));
    } else {
        const float *g = (const float *)grid.data();
        norm = cli::l2_norm(std::vector<float>(g, g + n));
    }
    std::printf("Throughput: %.3f GLUP/s, %.1f GB/s (%s, %d launches, %lld sweeps)\n", s.glups,
                s.gbs, prec.c_str(), s.launches, s.iterations);
    std::printf("Final grid L2 norm: %.17g\n", norm);
    if (!out.empty()) {
        FILE *f = std::fopen(out.c_str(), "wb");
        if (!f || std::fwrite(grid.data(), 1, grid.size(), f) != grid.size()) {
            std::fprintf(stderr, "ERROR: cannot write %s\n", out.c_str());
            if (f) std::fclose(f);
            return 1;
        }
        std::fclose(f);
    }
    cfm_jacobi_destroy(h);
    return mismatch ? 3 : 0;
}
