"""MatrixMarket input (the reference's -matrix_path, CG/src/mmio_wrapper.cpp:170-378):
the reader against SciPy's on general, symmetric, skew-symmetric and integer
files, its index-base rule, and the files it must refuse."""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

import cfm


def write(path, text):
    path.write_text(text)
    return str(path)


def csr_of(path):
    rowptr, col, val, m, n = cfm.mm_read(path)
    base = rowptr[0]
    return sp.csr_matrix((val, col - base, rowptr - base), shape=(m, n)), rowptr, col


def test_general_real_matches_scipy(tmp_path):
    rng = np.random.default_rng(3)
    A = sp.random(37, 29, density=0.2, random_state=4, format="coo")
    A.data = rng.normal(size=A.nnz)
    p = tmp_path / "g.mtx"
    scipy.io.mmwrite(str(p), A)
    got, rowptr, col = csr_of(str(p))
    want = scipy.io.mmread(str(p)).tocsr()
    assert got.shape == want.shape and rowptr[0] == 1
    np.testing.assert_array_equal(got.toarray(), want.toarray())
    for r in range(got.shape[0]):  # columns strictly increasing in each row
        c = col[rowptr[r] - 1:rowptr[r + 1] - 1]
        assert np.all(np.diff(c) > 0)


@pytest.mark.parametrize("symmetry", ["symmetric", "skew-symmetric"])
def test_symmetric_files_are_expanded(tmp_path, symmetry):
    n = 40
    rng = np.random.default_rng(5)
    L = sp.random(n, n, density=0.1, random_state=6, format="coo")
    L = sp.tril(L, k=-1 if symmetry == "skew-symmetric" else 0).tocoo()
    L.data = rng.normal(size=L.nnz)
    full = L + (-L.T if symmetry == "skew-symmetric" else L.T) - (sp.diags(L.diagonal()) if symmetry == "symmetric" else 0)
    p = tmp_path / "s.mtx"
    scipy.io.mmwrite(str(p), full.tocoo(), symmetry=symmetry)
    got, _, _ = csr_of(str(p))
    np.testing.assert_allclose(got.toarray(), full.toarray(), rtol=0, atol=0)


def test_integer_field_and_zero_base(tmp_path):
    p = write(tmp_path / "i.mtx", "%%MatrixMarket matrix coordinate integer general\n"
              "% comment\n\n3 3 4\n0 0 2\n1 1 3\n2 2 4\n0 2 -1\n")
    got, rowptr, _ = csr_of(p)
    assert rowptr[0] == 0
    np.testing.assert_array_equal(got.toarray(), [[2, 0, -1], [0, 3, 0], [0, 0, 4]])


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n",
    "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",
])
def test_unsupported_files(tmp_path, text):
    with pytest.raises(cfm.CfmError) as e:
        cfm.mm_read(write(tmp_path / "u.mtx", text))
    assert e.value.status == cfm.UNSUPPORTED


@pytest.mark.parametrize("text", [
    "not a banner\n2 2 1\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n1 1 2\n",   # duplicate
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",          # out of range
    "%%MatrixMarket matrix coordinate real general\n3 3 2\n0 0 1\n3 3 1\n",   # both bases
    "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n",          # truncated
])
def test_malformed_files(tmp_path, text):
    with pytest.raises(cfm.CfmError) as e:
        cfm.mm_read(write(tmp_path / "m.mtx", text))
    assert e.value.status == cfm.BAD_ARG


def test_missing_file(tmp_path):
    with pytest.raises(cfm.CfmError):
        cfm.mm_read(str(tmp_path / "nope.mtx"))
