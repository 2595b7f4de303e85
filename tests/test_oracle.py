"""Pins of the oracle (test infrastructure) against the reference.

  * element matrices: quadrature of the edge basis vs the reference's closed-form
    entries (T_Brick.cpp:142-474) and the curl-curl null space;
  * the numpy restatement of the whole transient vs the golden outputs of the
    reference's own CalcNonstat3DLine built from source;
  * the reference build in this checkout (oracle/_ref) reproduces the goldens;
  * the CPU Cholesky behind the pardiso_64 stand-in vs a dense solve.
"""
import ctypes
import os
import sys
import shutil

import numpy as np
import pytest

import tdem_oracle
from conftest import FP64_TOL, GOLDEN, ROOT


def closed_form_entries(hx, hy, hz):
    """Selected entries of the reference's closed-form B and C (T_Brick.cpp:147-174, 316-332)."""
    mx, my, mz = 2 * hx / (hy * hz), 2 * hy / (hx * hz), 2 * hz / (hx * hy)
    cx = hy * hz / (2 * hx)
    return {
        ("B", 0, 0): 2.0 / 3.0 * (my + mz),
        ("B", 0, 1): my / 3.0 - 2.0 / 3.0 * mz,
        ("B", 0, 3): -(my + mz) / 3.0,
        ("B", 0, 4): -2.0 / 3.0 * mz,
        ("B", 0, 8): -2.0 / 3.0 * my,
        ("B", 4, 8): -2.0 / 3.0 * mx,
        ("B", 8, 11): -(mx + my) / 3.0,
        ("C", 0, 0): 8.0 / 9.0 * cx,
        ("C", 0, 1): 4.0 / 9.0 * cx,
        ("C", 0, 3): 2.0 / 9.0 * cx,
        ("C", 0, 4): 0.0,
    }


@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (10.0, 20.0, 5.0), (3.7, 120.0, 0.8)])
def test_element_matrices_known_answer(h):
    B, C = tdem_oracle.local_matrices(np.array(h))
    for (kind, i, j), v in closed_form_entries(*h).items():
        got = (B if kind == "B" else C)[i, j]
        assert abs(got - v) <= 1e-13 * max(1.0, abs(v)), (kind, i, j, got, v)
    assert np.allclose(B, B.T, rtol=0, atol=1e-13 * abs(B).max())
    assert np.all(np.linalg.eigvalsh(C) > 0)
    # gradients of nodal functions lie in the curl-curl null space: edge DOF of
    # grad(phi) is (phi(upper) - phi(lower)) / 2
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 2), (4, 6), (1, 3), (5, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
    G = np.zeros((12, 8))
    for k, (a, b) in enumerate(pairs):
        G[k, a], G[k, b] = -0.5, 0.5
    assert np.abs(B @ G).max() <= 1e-12 * abs(B).max()


def _golden_case_dir(golden, name, tmp_path):
    d = str(tmp_path / name)
    golden.write_case_inputs(name, d)
    return d


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
@pytest.mark.parametrize("case", ["cube6", "cube8_block", "cube8_two_wires"])
def test_numpy_oracle_matches_reference_goldens(golden, outs, tmp_path, case, variant):
    d = _golden_case_dir(golden, case, tmp_path)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    npls = golden.CASES[case].get("n_sources", 1)
    for o in golden.OUTPUTS:
        for p in range(1, npls + 1):
            err = outs.compare_files(os.path.join(d, "%s.%d" % (o, p)),
                                     os.path.join(GOLDEN, case, "%s_%s.%d" % (variant, o, p)))
            assert err <= FP64_TOL, (o, p, err)


def test_reference_build_reproduces_goldens(golden, outs, tmp_path):
    import run_ref
    if not run_ref.available("CalcNonstat3DLine_A3"):
        pytest.skip("oracle/_ref not built")
    d = _golden_case_dir(golden, "cube8_block", tmp_path)
    run_ref.run_transient(d, "A3")
    for o in golden.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, "cube8_block", "A3_%s.1" % o))
        assert err <= FP64_TOL


def test_cpu_cholesky_pardiso_stand_in():
    lib_path = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
    if not os.path.exists(lib_path):
        pytest.skip("oracle library not built")
    import scipy.sparse as sp
    lib = ctypes.CDLL(lib_path)
    n = 700
    A = sp.random(n, n, density=0.01, random_state=3, format="csr")
    A = (A + A.T + sp.identity(n) * (abs(A).sum(1).max() + 1.0)).tocsr()
    U = sp.triu(A).tocsr()
    U.sort_indices()
    ia = (U.indptr + 1).astype(np.int64)
    ja = (U.indices + 1).astype(np.int64)
    a = U.data.astype(np.float64)
    pt = np.zeros(64, dtype=np.int64)
    iparm = np.zeros(64, dtype=np.int64)
    perm = np.zeros(n, dtype=np.int64)
    b = np.random.default_rng(0).standard_normal((3, n))
    x = np.zeros_like(b)
    err = ctypes.c_longlong(0)
    P = ctypes.POINTER(ctypes.c_longlong)

    def ll(v):
        return ctypes.byref(ctypes.c_longlong(v))

    for phase in (12, 33, -1):
        lib.pardiso_64(pt.ctypes.data_as(ctypes.c_void_p), ll(1), ll(1), ll(2), ll(phase), ll(n),
                       a.ctypes.data_as(ctypes.c_void_p), ia.ctypes.data_as(P), ja.ctypes.data_as(P),
                       perm.ctypes.data_as(P), ll(3), iparm.ctypes.data_as(P), ll(0),
                       b.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), ctypes.byref(err))
        assert err.value == 0
    xr = np.linalg.solve(A.toarray(), b.T).T
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()


def test_decade_logic():
    t = np.concatenate([np.arange(0, 5) * 1.0, 4 + np.arange(1, 5) * 2.0, 12 + np.arange(1, 4) * 4.0])
    assert tdem_oracle.decade_starts(t) == [0, 5, 9, 12]
    assert tdem_oracle.find_layer(t, 6.0) == 5
    assert tdem_oracle.find_layer(t, 0.0) == 0
    assert tdem_oracle.find_layer(t, 5.5) == -1


def test_reference_build_reproduces_primary_secondary_goldens(outs, tmp_path):
    """The primary-secondary fixtures come from the reference reading the normal field
    through its named-shared-memory calls (served from files by the oracle build)."""
    import run_ref
    import sys
    sys.path.insert(0, GOLDEN)
    import make_ps_golden as ps
    if not run_ref.available("CalcNonstat3DLine_A2"):
        pytest.skip("oracle/_ref not built")
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d)
    run_ref.run_transient(d, "A2")
    for o in ps.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, ps.CASE, "A2_%s.1" % o))
        assert err <= 1e-12, (o, err)
    # without the anomalous-edge list the normal field is not read and the result differs
    os.unlink(os.path.join(d, "mtrsizeforE0"))
    run_ref.run_transient(d, "A2")
    assert outs.compare_files(os.path.join(d, "eall_anom.1"), os.path.join(GOLDEN, ps.CASE, "A2_eall_anom.1")) > 0.1


@pytest.mark.parametrize("case,variant", [("cube8_block_ps", v) for v in ("A2", "A3", "E2", "E3")] +
                         [("cube8_block_ps_ia", v) for v in ("A2", "E3")])
def test_numpy_oracle_primary_secondary_matches_reference(outs, tmp_path, case, variant):
    """The restatement of the primary-secondary source against the reference: C_dsigma
    times the normal field's edge values (A, time_approx.cpp:671-683, 1263-1348) or
    times minus their time derivative, layer 0 from the normal potential (E,
    E2/time_approx.cpp:1384-1431, E3/time_approx.cpp:1400-1460)."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_ps_golden as ps
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d, case)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    for o in ps.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, case, "%s_%s.1" % (variant, o)))
        assert err <= FP64_TOL, (o, err)


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
def test_numpy_oracle_wire_beyond_the_mesh_matches_reference(outs, tmp_path, variant):
    """A wire that runs past the mesh edge: the dipoles no element holds go to the nearest
    element with local coordinates outside [0, 1] (vec_prep_data.cpp:878-980); the
    restatement against the reference's outputs, and (E-form, whose step-off source reads
    every dipole) against a run that drops those dipoles."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_beyond_golden as bg
    d = str(tmp_path / "beyond")
    bg.write_case_inputs(d)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    for o in bg.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, bg.CASE, "%s_%s.1" % (variant, o)))
        assert err <= FP64_TOL, (o, err)
    if variant == "E2":
        # the wire cut at the mesh edge, x = 600 .. 1000 m with the same dipole length
        with open(os.path.join(d, "sours"), "w") as f:
            f.write("600.0 0.0 0.0\n1000.0 0.0 0.0\n")
        with open(os.path.join(d, "nSrsRazb"), "w") as f:
            f.write("50\n")
        tdem_oracle.run(d, "E", 2)
        assert outs.compare_files(os.path.join(d, "eall_anom.1"),
                                  os.path.join(GOLDEN, bg.CASE, "E2_eall_anom.1")) > 1e-3


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
@pytest.mark.parametrize("case,npls", [("cube8_receivers_on_nodes", 1), ("cube8_two_wires_ragged", 2),
                                       ("cube6_no_b_receivers", 1), ("cube8_neib1_window", 1),
                                       ("cube8_permeable_block", 1)])
def test_numpy_oracle_receivers_on_element_boundaries_match_reference(outs, tmp_path, case, npls, variant):
    """Receivers on mesh nodes, edges and faces, some on the conductive block's surface:
    the first element in element order holds each (and, for field values, its material
    picks the smoothing subdomain), as in the reference (OutputResultant3d.cpp:572-712);
    two sources with ragged receiver lists (recvsb 2 and 5, recvse 3 and 1); no B
    receivers at all (empty emf and B files); a one-level receiver neighbourhood with a
    printed window inside the time grid; and a permeable block (relative mu 20)."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_nodes_golden as ng
    d = str(tmp_path / "nodes")
    ng.write_case_inputs(d, case)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    for o in ng.OUTPUTS:
        for p in range(1, npls + 1):
            err = outs.compare_files(os.path.join(d, "%s.%d" % (o, p)),
                                     os.path.join(GOLDEN, case, "%s_%s.%d" % (variant, o, p)))
            assert err <= FP64_TOL, (o, p, err)


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
def test_numpy_oracle_ramped_current_matches_reference(outs, tmp_path, variant):
    """A current that ramps down over four layers with an undershoot: the A-form source
    J(t) on every layer where it is non-zero, the E-form source -dJ/dt from the layers'
    differences (time_approx.cpp:1039-1076, E2/time_approx.cpp:1057-1105); measured up to
    2.5e-10 of the peak (A2), 7e-12 (E-form)."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_beyond_golden as bg
    d = str(tmp_path / "ramp")
    bg.write_case_inputs(d, bg.CASE_RAMP)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    for o in bg.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"),
                                 os.path.join(GOLDEN, bg.CASE_RAMP, "%s_%s.1" % (variant, o)))
        assert err <= FP64_TOL, (o, err)


def test_reference_zeroes_receivers_when_the_print_window_ends_inside_a_decade(golden, outs, tmp_path):
    """The one known divergence from the reference's outputs, shown on the reference itself:
    it projects a decade's receivers when that decade's last layer passes the receiver step
    (OutputResultant3d.cpp:432-474), and that step skips layers past the printed window
    (give_out_vec_loop.cpp:234). So with a window ending inside a decade, every printed
    layer of that decade holds zeros in B (and a jump in E). The restatement, like the
    drop-in, prints the computed values there; it agrees everywhere else."""
    import run_ref
    if not run_ref.available("CalcNonstat3DLine_A2"):
        pytest.skip("oracle/_ref not built")
    d = str(tmp_path / "w")
    golden.write_case_inputs("cube8_block", d)
    with open(os.path.join(d, "timeintervalforprint"), "w") as f:
        f.write("1.5000000000000e-04 6.0000000000000e-04\n")  # ends inside the third decade
    r, o = os.path.join(d, "ref"), os.path.join(d, "oracle")
    run_ref.copy_inputs(d, r)
    run_ref.copy_inputs(d, o)
    run_ref.run_transient(r, "A2")
    tdem_oracle.run(o, "A", 2)
    for (_, ref), (_, ora) in zip(outs.read_transients(os.path.join(r, "ball_anom.1")),
                                  outs.read_transients(os.path.join(o, "ball_anom.1"))):
        late = ref[:, 0] > 0.5  # ms: layers 5.24e-4 and 6.19e-4 s, the third decade
        assert late.sum() == 2 and np.all(ref[late, 1:] == 0.0) and np.any(ora[late, 1:] != 0.0)
        scale = np.abs(ref[~late, 1:]).max()
        assert np.abs(ref[~late, 1:] - ora[~late, 1:]).max() <= FP64_TOL * scale


def test_three_point_formulas_exact_for_quadratics():
    """Known answers of the time discretisation (reference math, no reference run):
    the BDF2 step coefficients (A3/time_approx.cpp:943-945) and the three-point
    derivative used for outputs and the E-form sources (E3/time_approx.cpp:1434-1460)
    differentiate quadratics exactly on non-uniform steps."""
    rng = np.random.default_rng(5)
    for _ in range(50):
        a, b, c = rng.standard_normal(3)
        u = lambda t: a + b * t + c * t * t
        du = lambda t: b + 2 * c * t
        tj2 = rng.uniform(0, 1)
        tj1 = tj2 + rng.uniform(0.1, 1)
        tj = tj1 + rng.uniform(0.1, 1)
        dt, dt0, dt1 = tj - tj2, tj - tj1, tj1 - tj2
        mult = (dt + dt0) / (dt * dt0)
        m1 = dt / (dt1 * dt0)
        m2 = -dt0 / (dt * dt1)
        # the step solves (C mult + B) u_j = C (m1 u_j1 + m2 u_j2) + ...: mult u_j - m1 u_j1 - m2 u_j2 = du/dt
        assert abs(mult * u(tj) - m1 * u(tj1) - m2 * u(tj2) - du(tj)) <= 1e-9 * (1 + abs(du(tj)))
        for t in (tj2, tj1, tj, 0.5 * (tj1 + tj)):
            got = tdem_oracle._dA_dt(t, u(tj), u(tj1), u(tj2), dt, dt0, dt1, tj, tj1, tj2)
            assert abs(got - du(t)) <= 1e-9 * (1 + abs(du(t)))


@pytest.mark.parametrize("variant", ["A3", "E3"])
def test_numpy_oracle_matches_32_wire_golden(outs, tmp_path, variant):
    """The restatement on the 32-wire block case of tests/golden/scale (12^3, 32
    right-hand sides per step, made by the reference's own CalcNonstat3DLine)."""
    sys.path.insert(0, GOLDEN)
    import make_scale_golden as sg
    d = str(tmp_path / "w")
    sg.write_case_inputs("wires32", d)
    tdem_oracle.run(d, variant[0], int(variant[1]))
    for o in sg.OUTPUTS:
        for p in range(1, 33):
            err = outs.compare_files(os.path.join(d, "%s.%d" % (o, p)),
                                     os.path.join(GOLDEN, "scale", "wires32", "%s_%s.%d" % (variant, o, p)))
            assert err <= FP64_TOL, (o, p, err)
