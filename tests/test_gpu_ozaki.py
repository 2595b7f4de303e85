"""GPU tests of the FP64 trailing update on the integer tensor pipe (digit
splitting, ozaki_update.cu): a dense front through pardiso_64 against numpy, every
variant of the golden models with every trailing update forced onto that path
(TDEM_OZAKI_ALL=1: small fronts, partial tiles, panels shorter than 512 columns)
against the reference's goldens, and the 40^3 model, where the analysis picks the
path for its large panels by itself, against the FP64 tensor-pipe factorization."""
import os
import sys

import numpy as np
import pytest

from conftest import FP64_TOL, GOLDEN

pytestmark = pytest.mark.gpu


def _upper(A):
    import scipy.sparse as sp
    U = sp.triu(sp.csr_matrix(A)).tocsr()
    U.sort_indices()
    return U.data.copy(), (U.indptr + 1).astype(np.int64), (U.indices + 1).astype(np.int64)


def test_dense_front_on_the_integer_pipe(pkg):
    """3,000 pivots in one front: rank-512 trailing updates of 2,488 and 1,976 rows
    go through the digit path; the solution matches numpy's to FP64 accuracy."""
    n = 3000
    rng = np.random.default_rng(17)
    G = rng.standard_normal((n, n))
    # a wide spread of row scales, so that the per-row exponents matter
    D = np.diag(10.0 ** rng.uniform(-3, 3, n))
    A = D @ (G @ G.T / n + np.eye(n)) @ D
    a, ia, ja = _upper(A)
    h = np.zeros(64, dtype=np.int64)
    assert pkg.pardiso_64(h, 12, a, ia, ja, nrhs=2) == 0
    b = rng.standard_normal((2, n))
    x = np.zeros_like(b)
    assert pkg.pardiso_64(h, 33, a, ia, ja, nrhs=2, b=b, x=x) == 0
    xr = np.linalg.solve(A, b.T).T
    assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()
    pkg.pardiso_64(h, -1, a, ia, ja)


def test_large_dense_front_on_the_integer_pipe(pkg):
    """12,000 pivots in one front: the first trailing update (11,488 rows, K = 512,
    8,190 output tiles of 128 x 64 for 148 persistent CTAs) has the shape of the
    large 80^3 updates, so this is also the case the kernel is profiled on.  The
    matrix is D (3 I + (B + B^T) / sqrt(2 n)) D with Gaussian B (eigenvalues of the
    inner matrix within about [1, 5]) and row scales over six decades; the check is
    the componentwise-scaled residual, which an FP64 backward-stable solve keeps
    near n u."""
    n = 12000
    rng = np.random.default_rng(23)
    A = rng.standard_normal((n, n))
    A += A.T
    A *= 1.0 / np.sqrt(2.0 * n)
    A[np.diag_indices(n)] += 3.0
    dsc = 10.0 ** rng.uniform(-3, 3, n)
    A *= dsc[:, None]
    A *= dsc[None, :]
    # 1-based upper CSR, row by row (a dense 12,000^2 matrix through scipy.sparse
    # would need several copies of it)
    counts = np.arange(n, 0, -1, dtype=np.int64)
    ia = np.empty(n + 1, dtype=np.int64)
    ia[0] = 1
    np.cumsum(counts, out=ia[1:])
    ia[1:] += 1
    a = np.empty(ia[-1] - 1)
    ja = np.empty(ia[-1] - 1, dtype=np.int64)
    cols = np.arange(1, n + 1, dtype=np.int64)
    for i in range(n):
        a[ia[i] - 1:ia[i + 1] - 1] = A[i, i:]
        ja[ia[i] - 1:ia[i + 1] - 1] = cols[i:]
    h = np.zeros(64, dtype=np.int64)
    assert pkg.pardiso_64(h, 12, a, ia, ja, nrhs=1) == 0
    b = rng.standard_normal((1, n))
    x = np.zeros_like(b)
    assert pkg.pardiso_64(h, 33, a, ia, ja, nrhs=1, b=b, x=x) == 0
    pkg.pardiso_64(h, -1, a, ia, ja)
    r = A @ x[0] - b[0]
    scale = np.abs(A) @ np.abs(x[0]) + np.abs(b[0])
    assert np.max(np.abs(r) / scale) <= 1e-11


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
@pytest.mark.parametrize("case", ["cube8_block", "cube8_two_wires"])
def test_every_trailing_update_on_the_integer_pipe(pkg, golden, outs, tmp_path, monkeypatch, case, variant):
    monkeypatch.setenv("TDEM_OZAKI_ALL", "1")
    d = str(tmp_path / "g")
    golden.write_case_inputs(case, d)
    p = pkg.plan(d, variant[0], int(variant[1]))
    assert p["ozaki_flops"] > 0
    with pkg.Solver(d, variant[0], int(variant[1])) as s:
        s.run()
        s.write_outputs()
    npls = golden.CASES[case].get("n_sources", 1)
    for o in golden.OUTPUTS:
        for q in range(1, npls + 1):
            err = outs.compare_files(os.path.join(d, "%s.%d" % (o, q)),
                                     os.path.join(GOLDEN, case, "%s_%s.%d" % (variant, o, q)))
            assert err <= FP64_TOL, (o, q, err)


def test_integer_pipe_matches_fp64_pipe_at_40_cubed(pkg, outs, tmp_path, monkeypatch):
    sys.path.insert(0, GOLDEN)
    import make_scale_golden as sg
    res = {}
    for oz in ("1", "0"):
        monkeypatch.setenv("TDEM_OZAKI", oz)
        d = str(tmp_path / ("oz" + oz))
        sg.write_case_inputs("c1", d)
        if oz == "1":
            assert pkg.plan(d, "A", 2)["ozaki_flops"] > 0
        with pkg.Solver(d, "A", 2) as s:
            s.run()
            s.write_outputs()
            res[oz] = s.results()
        for o in sg.OUTPUTS:
            assert outs.compare_files(os.path.join(d, o + ".1"),
                                      os.path.join(GOLDEN, "scale", "c1", "A2_%s.1" % o)) <= FP64_TOL
    # the two factorizations give the same transients to well inside the tolerance
    for a, b in zip(res["1"], res["0"]):
        sc = np.abs(b).max()
        assert np.abs(a - b).max() <= 1e-9 * sc
