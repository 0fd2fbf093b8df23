"""A foreign C host: a C99 program that includes include/cfm.h and links
libcfm.so (-I include -L lib -lcfm, as a foreign build would) compiles, runs, and gets status codes
back (never an exit) for bad arguments.  No GPU needed: device-side calls on a
machine without a GPU must return a status too."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cpu-free-model_b200", "lib")

SRC = r"""
#include <stdio.h>
#include "cfm.h"

int main(void) {
    printf("ok=%s\n", cfm_status_string(CFM_OK));
    cfm_jacobi_params bad = {4, 8, 8, 8, CFM_FP64, 1, CFM_JACOBI_PERSISTENT};
    cfm_jacobi *h = 0;
    int st = cfm_jacobi_create(&bad, &h);
    printf("bad_dims=%d handle_null=%d msg=%s\n", st, h == 0, cfm_last_error());
    cfm_csr *A = 0;
    int rowptr[3] = {0, 1, 2}, col[2] = {0, 1};
    double val[2] = {2.0, 2.0};
    st = cfm_csr_create(2, 5, rowptr, col, val, &A);
    printf("bad_nnz=%d\n", st);
    cfm_jacobi_params good = {3, 16, 16, 16, CFM_FP64, 1, CFM_JACOBI_PERSISTENT};
    st = cfm_jacobi_create(&good, &h);
    printf("create=%d\n", st);
    if (st == CFM_OK) cfm_jacobi_destroy(h);
    return 0;
}
"""


def test_c99_host_compiles_links_and_gets_status_codes(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libcfm.so")):
        pytest.fail("libcfm.so is missing: build it first (no CPU fallback)")
    src = tmp_path / "host.c"
    src.write_text(SRC)
    exe = tmp_path / "host"
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                         "-L", LIB, "-lcfm", "-Wl,-rpath," + LIB, "-o", str(exe)],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("ok=")
    assert "bad_dims=1 handle_null=1" in out.stdout
    assert "bad_nnz=1" in out.stdout
    create = int(out.stdout.split("create=")[1].split()[0])
    assert create in (0, 6)  # CFM_OK with a GPU, CFM_NO_DEVICE without one
