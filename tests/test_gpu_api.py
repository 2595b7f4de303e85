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


def test_pardiso_gpu_zeroed_pt_reuses_its_handle(pkg):
    """The reference zeroes pt before every phase 12 (pardiso_solver::init) and
    releases it once at the end: every refactorization must reuse the handle kept
    for that pt array, holding one factor on the device, not one per call."""
    import torch
    lib = pkg.load_library()
    n = 3000
    A = _spd(n, 13)
    a, ia, ja = _upper(A)
    h = np.zeros(64, dtype=np.int64)
    before = lib.tdem_pardiso_handles()
    rng = np.random.default_rng(3)
    b = rng.standard_normal((8, n))
    x = np.zeros_like(b)
    xr = np.linalg.solve(A.toarray(), b.T).T
    free = []
    for k in range(4):
        h[:] = 0  # what pardiso_solver::factorize does before each phase 12
        scale = 1.0 + k
        a2 = a * scale
        assert pkg.pardiso_64(h, 12, a2, ia, ja) == 0  # analysed with nrhs = 1, as the reference does
        assert lib.tdem_pardiso_handles() == before + 1
        x[:] = 0
        assert pkg.pardiso_64(h, 33, a2, ia, ja, nrhs=8, b=b, x=x) == 0  # widens to 8 columns once
        assert np.abs(x - xr / scale).max() <= 1e-11 * np.abs(xr).max()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    # no factor, stream or workspace accumulates across refactorizations
    assert free[-1] >= free[1] - (1 << 20)
    assert pkg.pardiso_64(h, -1, a, ia, ja) == 0
    assert h[0] == 0 and lib.tdem_pardiso_handles() == before


def test_pardiso_gpu_dense_front(pkg):
    """A dense SPD matrix is one front of 1,300 pivots: three outer panels of up
    to 512 columns, the first two ending in a rank-512 trailing update of the rest."""
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


def test_stop_file_ends_the_drop_in_run(pkg, golden, tmp_path):
    """A `stop` file in the run directory ends the module run before any output is
    written, as the reference's CheckStop does (TaskSP.cpp:462)."""
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube6", d)
    open(os.path.join(d, "stop"), "w").close()
    with pytest.raises(pkg.TdemError) as ei:
        pkg.run_directory(d, "A", 2)
    assert ei.value.status == 5
    assert not os.path.exists(os.path.join(d, "eall_anom.1"))
    os.unlink(os.path.join(d, "stop"))
    pkg.run_directory(d, "A", 2)
    assert os.path.exists(os.path.join(d, "eall_anom.1"))


@pytest.mark.parametrize("form,scheme", [("A", 2), ("E", 3)])
def test_time_watcher_log_has_the_reference_phases(pkg, golden, tmp_path, form, scheme):
    """The module run appends the reference's TimeWatcher labels, one per phase,
    in time order: one factorization mark pair per factorization, one solve and
    one receiver pair per step."""
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    pkg.run_directory(d, form, scheme)
    with pkg.Solver(d, form, scheme) as s:  # counts of the same run (no log here)
        s.run()
        info = s.info()
    lines = [ln.rstrip("\n").split("\t", 1) for ln in open(os.path.join(d, "TimeWatcher.log"))]
    ticks = [int(t) for t, _ in lines]
    labels = [lab for _, lab in lines]
    assert labels[:2] == ["Start CalcSP", "Start Prepare_To_Schema"]
    assert "Finish Prepare_To_Schema" in labels
    assert ticks == sorted(ticks)
    assert labels.count("Start factorization") == info["factorizations"]
    assert labels.count("Finish factorization") == info["factorizations"]
    assert labels.count("Start prepare matrix for new decade") == info["factorizations"]
    assert labels.count("Start Direct-Inverse") == info["steps"]
    assert labels.count("Finish Direct-Inverse") == info["steps"]
    n_dec = labels.count("Start schema iDec= 0") and sum(1 for x in labels if x.startswith("Start decade iDec="))
    assert n_dec >= 2 and n_dec == sum(1 for x in labels if x.startswith("Finish decade iDec="))
    assert labels[-1] == "Finish decade iDec= %d" % (n_dec - 1)
    # every factorization finishes after it starts
    for a, b in zip([i for i, x in enumerate(labels) if x == "Start factorization"],
                    [i for i, x in enumerate(labels) if x == "Finish factorization"]):
        assert a < b
