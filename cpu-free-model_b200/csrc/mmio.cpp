// MatrixMarket coordinate reader with the behaviour of the reference's
// loadMMSparseMatrix (CG/src/mmio_wrapper.cpp:170-378), written from the
// NIST MatrixMarket format description:
//  - "coordinate" matrices of field real or integer; array (dense), pattern
//    and complex files are rejected;
//  - symmetric / hermitian / skew-symmetric files are expanded to the full
//    pattern (the mirrored off-diagonal entry negated for skew);
//  - entries are sorted by (row, column) and compressed to CSR;
//  - the index base is 1 when some index equals the dimension, 0 when some
//    index is 0 (both: error), and is kept in the output like the reference
//    keeps it (rowptr[0] = base; cfm_csr_create reads the base from there);
//  - rows must end up with strictly increasing columns (duplicates: error).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cfm.h"
#include "cfm_internal.h"

namespace {

struct Entry {
    int i, j;
    double v;
};

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

int read_mm(const char *path, int *m_out, int *n_out, std::vector<Entry> &e, int *base_out) {
    FILE *f = std::fopen(path, "r");
    if (!f) {
        cfm::set_error("cannot open '%s'", path);
        return CFM_BAD_ARG;
    }
    struct Closer {
        FILE *f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    char line[4096];
    if (!std::fgets(line, sizeof line, f)) {
        cfm::set_error("'%s': empty file", path);
        return CFM_BAD_ARG;
    }
    char b0[64] = {0}, b1[64] = {0}, b2[64] = {0}, b3[64] = {0}, b4[64] = {0};
    if (std::sscanf(line, "%63s %63s %63s %63s %63s", b0, b1, b2, b3, b4) != 5 ||
        lower(b0) != "%%matrixmarket" || lower(b1) != "matrix") {
        cfm::set_error("'%s': missing %%%%MatrixMarket matrix banner", path);
        return CFM_BAD_ARG;
    }
    const std::string fmt = lower(b2), field = lower(b3), sym = lower(b4);
    if (fmt != "coordinate") {
        cfm::set_error("'%s': dense (array) matrices are not supported", path);
        return CFM_UNSUPPORTED;
    }
    if (field != "real" && field != "integer" && field != "double") {
        cfm::set_error("'%s': field '%s' not supported (real or integer only)", path, b3);
        return CFM_UNSUPPORTED;
    }
    const bool symmetric = sym == "symmetric" || sym == "hermitian";
    const bool skew = sym == "skew-symmetric";
    if (!symmetric && !skew && sym != "general") {
        cfm::set_error("'%s': unknown symmetry '%s'", path, b4);
        return CFM_BAD_ARG;
    }
    long long m = 0, n = 0, nz = 0;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        bool blank = true;
        for (char *c = line; *c; ++c)
            if (!std::isspace((unsigned char)*c)) blank = false;
        if (blank) continue;
        if (std::sscanf(line, "%lld %lld %lld", &m, &n, &nz) != 3) {
            cfm::set_error("'%s': bad size line", path);
            return CFM_BAD_ARG;
        }
        break;
    }
    if (m <= 0 || n <= 0 || nz < 0 || m > 2147483646LL || n > 2147483646LL) {
        cfm::set_error("'%s': bad sizes %lld x %lld, %lld entries", path, m, n, nz);
        return CFM_BAD_ARG;
    }
    e.clear();
    e.reserve((size_t)nz * ((symmetric || skew) ? 2 : 1));
    for (long long k = 0; k < nz; ++k) {
        long long i, j;
        double v;
        if (std::fscanf(f, "%lld %lld %lf", &i, &j, &v) != 3) {
            cfm::set_error("'%s': entry %lld unreadable", path, k + 1);
            return CFM_BAD_ARG;
        }
        e.push_back({(int)i, (int)j, v});
        if ((symmetric || skew) && i != j) e.push_back({(int)j, (int)i, skew ? -v : v});
    }
    std::sort(e.begin(), e.end(),
              [](const Entry &a, const Entry &b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });
    bool base0 = false, base1 = false;
    for (const Entry &x : e) {
        if (x.i == 0 || x.j == 0) base0 = true;
        if (x.i == m || x.j == n) base1 = true;
    }
    if (base0 && base1) {
        cfm::set_error("'%s': indices are both 0-based and 1-based", path);
        return CFM_BAD_ARG;
    }
    const int base = base1 ? 1 : 0;
    for (size_t k = 0; k < e.size(); ++k) {
        const Entry &x = e[k];
        if (x.i < base || x.i >= m + base || x.j < base || x.j >= n + base) {
            cfm::set_error("'%s': index (%d, %d) out of range", path, x.i, x.j);
            return CFM_BAD_ARG;
        }
        if (k > 0 && e[k - 1].i == x.i && e[k - 1].j >= x.j) {
            cfm::set_error("'%s': duplicate entry (%d, %d)", path, x.i, x.j);
            return CFM_BAD_ARG;
        }
    }
    *m_out = (int)m;
    *n_out = (int)n;
    *base_out = base;
    return CFM_OK;
}

}  // namespace

extern "C" int cfm_mm_read(const char *path, int *m, int *n, long long *nnz, int *rowptr,
                           int *col, double *val) {
    CFM_ARG_CHECK(path && m && n && nnz, "null argument");
    std::vector<Entry> e;
    int base = 0;
    int st = read_mm(path, m, n, e, &base);
    if (st) return st;
    *nnz = (long long)e.size();
    if (!rowptr) return CFM_OK;  // size query
    CFM_ARG_CHECK(col && val, "col/val are null");
    std::vector<long long> cnt((size_t)*m + 1, 0);
    for (const Entry &x : e) cnt[(size_t)(x.i - base) + 1]++;
    rowptr[0] = base;
    long long acc = base;
    for (int r = 0; r < *m; ++r) {
        acc += cnt[(size_t)r + 1];
        rowptr[r + 1] = (int)acc;
    }
    for (size_t k = 0; k < e.size(); ++k) {
        col[k] = e[k].j;
        val[k] = e[k].v;
    }
    return CFM_OK;
}
