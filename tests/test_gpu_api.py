"""GPU tests of the C-ABI behaviour: results vs files, determinism, errors,
cancellation, and the GPU-backed pardiso_64."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_results_match_files_and_repeat_bitwise(pkg, golden, outs, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    with pkg.Solver(d, "A", 3) as s:
        s.run()
        e1, m1, b1 = s.results()
        s.write_outputs()
        s.run()
        e2, m2, b2 = s.results()
    assert np.array_equal(e1, e2) and np.array_equal(m1, m2) and np.array_equal(b1, b2)
    tab = outs.read_transients(os.path.join(d, "eall_anom.1"))
    for i, (_, t) in enumerate(tab):
        assert np.allclose(t[:, 1:], e1[:, :, i], rtol=1e-15, atol=0)
    tab = outs.read_transients(os.path.join(d, "edsall_anom.1"))
    for i, (_, t) in enumerate(tab):
        assert np.allclose(t[:, 1:], m1[:, :, i], rtol=1e-15, atol=0)


def test_missing_input_is_an_input_error(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube6", d)
    os.unlink(os.path.join(d, "edges.dat"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.Solver(d, "A", 2)
    assert ei.value.status == 2 and "edges.dat" in str(ei.value)


def test_truncated_mesh_file_is_an_input_error(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube6", d)
    p = os.path.join(d, "xyz.dat")
    data = open(p, "rb").read()
    open(p, "wb").write(data[: len(data) // 2])
    with pytest.raises(pkg.TdemError) as ei:
        pkg.Solver(d, "E", 3)
    assert ei.value.status == 2


def test_bad_arguments(pkg, tmp_path):
    with pytest.raises(ValueError):
        pkg.Solver(str(tmp_path), "X", 2)
    lib = pkg.load_library()
    import ctypes
    h = ctypes.c_void_p()
    assert lib.tdem_solver_create(os.fsencode(str(tmp_path)), 0, 4, 0, ctypes.byref(h)) == 1


def test_cancel_before_run(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    with pkg.Solver(d, "A", 2) as s:
        s.cancel()
        with pytest.raises(pkg.TdemError) as ei:
            s.run()
        assert ei.value.status == 5
        s.run()  # the flag is consumed by the cancelled run
        assert s.info()["steps"] > 0


def _spd(n, seed, density=0.003):
    import scipy.sparse as sp
    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    return (A + A.T + sp.identity(n) * (abs(A).sum(1).max() + 1.0)).tocsr()


def _upper(A):
    import scipy.sparse as sp
    U = sp.triu(A).tocsr()
    U.sort_indices()
    return U.data.copy(), (U.indptr + 1).astype(np.int64), (U.indices + 1).astype(np.int64)


def test_pardiso_gpu_multi_rhs_and_refactor(pkg):
    n = 2500
    A = _spd(n, 7)
    a, ia, ja = _upper(A)
    h = np.zeros(64, dtype=np.int64)
    assert pkg.pardiso_64(h, 12, a, ia, ja) == 0
    b = np.random.default_rng(1).standard_normal((4, n))
    x = np.zeros_like(b)
    assert pkg.pardiso_64(h, 33, a, ia, ja, nrhs=4, b=b, x=x) == 0
    xr = np.linalg.solve(A.toarray(), b.T).T
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    # same pattern, new values: analysis reused, new factorization
    A2 = A.copy()
    A2.data *= 2.0
    a2, _, _ = _upper(A2)
    assert pkg.pardiso_64(h, 12, a2, ia, ja) == 0
    assert pkg.pardiso_64(h, 33, a2, ia, ja, nrhs=4, b=b, x=x) == 0
    assert np.abs(x - xr / 2).max() <= 1e-12 * np.abs(xr).max()
    assert pkg.pardiso_64(h, -1, a2, ia, ja) == 0
    assert h[0] == 0


def test_pardiso_gpu_dense_front(pkg):
    """A dense SPD matrix is one front of 1,300 pivots: five outer panels of 256
    columns, each ending in a rank-256 trailing update of the rest."""
    n = 1300
    rng = np.random.default_rng(5)
    G = rng.standard_normal((n, n))
    Ad = G @ G.T / n + np.eye(n)
    import scipy.sparse as sp
    a, ia, ja = _upper(sp.csr_matrix(Ad))
    h = np.zeros(64, dtype=np.int64)
    assert pkg.pardiso_64(h, 12, a, ia, ja) == 0
    b = rng.standard_normal((2, n))
    x = np.zeros_like(b)
    assert pkg.pardiso_64(h, 33, a, ia, ja, nrhs=2, b=b, x=x) == 0
    xr = np.linalg.solve(Ad, b.T).T
    assert np.abs(x - xr).max() <= 1e-11 * np.abs(xr).max()
    pkg.pardiso_64(h, -1, a, ia, ja)


@pytest.mark.parametrize("nrhs", [1, 2, 3, 8, 16, 31, 32, 64])
def test_pardiso_gpu_block_solves(pkg, nrhs):
    """All right-hand sides in one solve: the streaming level solves (1-2 columns)
    and the tensor-pipe block kernels (3-64 columns) on a dense 1,300-pivot front
    (chain, chunk and partial-sum paths) and on a sparse matrix (many fronts)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(40 + nrhs)
    n = 1300
    G = rng.standard_normal((n, n))
    Ad = G @ G.T / n + np.eye(n)
    for A in (sp.csr_matrix(Ad), _spd(3000, 11)):
        a, ia, ja = _upper(A)
        h = np.zeros(64, dtype=np.int64)
        assert pkg.pardiso_64(h, 12, a, ia, ja, nrhs=nrhs) == 0
        b = rng.standard_normal((nrhs, A.shape[0]))
        x = np.zeros_like(b)
        assert pkg.pardiso_64(h, 33, a, ia, ja, nrhs=nrhs, b=b, x=x) == 0
        xr = np.linalg.solve(A.toarray(), b.T).T
        assert np.abs(x - xr).max() <= 1e-11 * np.abs(xr).max()
        pkg.pardiso_64(h, -1, a, ia, ja)


def test_pardiso_gpu_not_positive_definite(pkg):
    n = 400
    A = _spd(n, 9)
    A = A - 10.0 * abs(A).sum(1).max() * __import__("scipy.sparse", fromlist=["identity"]).identity(n)
    a, ia, ja = _upper(A.tocsr())
    h = np.zeros(64, dtype=np.int64)
    assert pkg.pardiso_64(h, 12, a, ia, ja) == -4
    pkg.pardiso_64(h, -1, a, ia, ja)


@pytest.mark.parametrize("form,scheme", [("A", 3), ("E", 2)])
def test_factor_ahead_matches_sequential_bitwise(pkg, golden, tmp_path, form, scheme):
    """Two factor slots (the next factorization overlapped with the current
    decade's steps on a second stream) give bit-identical transients."""
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    out = {}
    for slots in (1, 2):
        with pkg.Solver(d, form, scheme, factor_slots=slots) as s:
            s.run()
            out[slots] = s.results()
            info = s.info()
            assert info["factor_slots"] == slots
            assert info["factorizations"] >= 2
            s.run()
            again = s.results()
        for a, b in zip(out[slots], again):
            assert np.array_equal(a, b)
    for a, b in zip(out[1], out[2]):
        assert np.array_equal(a, b)


def test_factor_slots_out_of_range_is_rejected(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube6", d)
    with pytest.raises(pkg.TdemError) as ei:
        pkg.Solver(d, "A", 2, factor_slots=3)
    assert ei.value.status == 1
