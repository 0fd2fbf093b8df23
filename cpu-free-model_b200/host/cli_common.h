// Argument helpers and reporting shared by the jacobi2D / jacobi3D / cg
// command-line front ends.  Flags are scanned the way the reference scans
// them (Stencil/jacobi2D/include/common.h:28-39): "-flag value" anywhere in
// argv, last-definition-irrelevant, missing value -> default.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "cfm.h"

namespace cli {

template <typename T>
T argval(int argc, char **argv, const char *flag, T dflt) {
    for (int i = 1; i + 1 < argc; ++i)
        if (std::strcmp(argv[i], flag) == 0) {
            std::istringstream in(argv[i + 1]);
            T v = dflt;
            in >> v;
            return v;
        }
    return dflt;
}

inline bool has(int argc, char **argv, const char *flag) {
    for (int i = 1; i < argc; ++i)
        if (std::strcmp(argv[i], flag) == 0) return true;
    return false;
}

inline int fail(const char *what, int status) {
    std::fprintf(stderr, "ERROR: %s failed: %s (%s)\n", what, cfm_status_string(status),
                 cfm_last_error());
    return 1;
}

struct Version {
    const char *name;
    int impl;       // library implementation, or -1 when not provided on one GPU
    const char *why;  // reason when impl < 0
};

inline void print_versions(const std::vector<Version> &v) {
    std::printf("Versions (select with -v):\n");
    for (size_t i = 0; i < v.size(); ++i) std::printf("%zu:\t%s\n", i, v[i].name);
    std::printf("\n");
}

template <typename T>
double l2_norm(const std::vector<T> &a) {
    long double s = 0;
    for (const T &v : a) s += (long double)v * (long double)v;
    return std::sqrt((double)s);
}

}  // namespace cli
