"""Host-only planning (tdem_solver_plan, no GPU): the input reading, nested
dissection, assembly tree and launch plans of a forward solve, including the
replay that every level-solve unit waits only for units queued before it, on
models of several sizes, formulations and schemes."""
import os
import sys

import numpy as np
import pytest


def _counts_consistent(p):
    assert 0 < p["n_interior"] < p["n_edges"]
    # the factor holds at least the lower triangle of the interior system
    assert p["nnz_factor"] >= (p["nnz_matrix"] * p["n_interior"] // p["n_edges"] + p["n_interior"]) // 2
    assert p["device_bytes"] > 8 * p["nnz_factor"]
    assert p["factor_slot_bytes"] >= 8 * p["nnz_factor"]
    assert p["factor_flops"] > 0 and p["solve_units"] > 0
    assert p["n_fronts"] > 0 and p["tree_levels"] >= 1
    # one dependent 64-wide link per level at least, never more than all pivot blocks
    assert p["tree_levels"] <= p["solve_chain"] <= p["n_interior"] // 64 + p["n_fronts"]


@pytest.mark.parametrize("cells,form,scheme", [(8, "A", 2), (10, "E", 3), (14, "A", 3), (16, "E", 2)])
def test_plan_small_models(pkg, mg, tmp_path, cells, form, scheme):
    d = str(tmp_path / "m")
    spec = mg.small_model(cells=cells, n_dec=2, steps_per_dec=4)
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    p = pkg.plan(d, form, scheme)
    _counts_consistent(p)
    assert p["n_sources"] == 1
    # leaf size changes the ordering but not the system
    q = pkg.plan(d, form, scheme, leaf_size=48)
    _counts_consistent(q)
    assert (q["n_interior"], q["nnz_matrix"]) == (p["n_interior"], p["nnz_matrix"])


def test_plan_two_wires_and_fp32(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_two_wires", d)
    p64 = pkg.plan(d, "A", 3)
    assert p64["n_sources"] == 2
    p32 = pkg.plan(d, "A", 3, precision=32)
    # the FP32 factor halves the factor slot; the FP64 system copy for the CG is extra
    assert p32["factor_slot_bytes"] * 2 == p64["factor_slot_bytes"]
    assert p64["factor_flops"] == p32["factor_flops"]


def test_plan_missing_input_is_an_input_error(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube6", d)
    os.unlink(os.path.join(d, "edges.dat"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(d, "A", 2)
    assert ei.value.status == 2 and "edges.dat" in str(ei.value)


def test_plan_receiver_outside_the_mesh_is_an_input_error(pkg, mg, tmp_path):
    """A receiver that no element holds stops the run, as the reference does ("There are
    no elements for receiver(s)", OutputResultant3d.cpp:724-749, which has no nearest-element
    rule for receivers); a wire past the mesh edge does not (its outer dipoles go to the
    nearest element)."""
    import dataclasses
    base = mg.small_model(cells=8, n_dec=2, steps_per_dec=4)
    far = float(base.x[-1]) + 500.0
    spec = dataclasses.replace(base, receivers_b=[[(0.0, 10.0, 0.0), (far, 0.0, 0.0)]],
                               receivers_e=[[(0.0, 10.0, 0.0)]])
    d = str(tmp_path / "rec")
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(d, "A", 2)
    assert ei.value.status == 2 and "receiver outside the mesh" in str(ei.value)
    spec = dataclasses.replace(base, sources=[((far - 900.0, 0.0, 0.0), (far, 0.0, 0.0))])
    d = str(tmp_path / "wire")
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    assert pkg.plan(d, "E", 2)["n_sources"] == 1


def test_plan_bad_arguments(pkg, tmp_path):
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(str(tmp_path), "A", 4)
    assert ei.value.status == 1
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(str(tmp_path), "A", 2, factor_slots=3)
    assert ei.value.status == 1


def test_plan_digest_independent_of_host_threads(pkg, mg, tmp_path, monkeypatch):
    # large enough that the dissection forks and every parallel pass cuts several ranges
    d = str(tmp_path / "m")
    spec = mg.small_model(cells=28, n_dec=2, steps_per_dec=4)
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    digests = {}
    for t in ("1", "3", "8"):
        monkeypatch.setenv("TDEM_HOST_THREADS", t)
        p = pkg.plan(d, "E", 2)
        _counts_consistent(p)
        assert p["plan_seconds"] > 0
        digests[t] = p["digest"]
    assert p["n_interior"] > 40000
    assert len(set(digests.values())) == 1, digests
    # the digest does see a different ordering
    assert pkg.plan(d, "E", 2, leaf_size=48)["digest"] != digests["1"]


def test_plan_primary_secondary_mode(pkg, tmp_path):
    """fdirect 0 with anomalous edges: both formulations plan (the normal field is read
    per step); the E-formulation also needs the normal potential v3n.dat (layer 0)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_ps_golden as ps
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d)
    for form, scheme in (("A", 3), ("E", 2)):
        _counts_consistent(pkg.plan(d, form, scheme))
    os.unlink(os.path.join(d, "v3n.dat"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(d, "E", 3)
    assert ei.value.status == 2 and "v3n.dat" in str(ei.value)
    pkg.plan(d, "A", 2)  # the A-formulation does not read it
    os.unlink(os.path.join(d, "PName"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(d, "A", 2)
    assert "PName" in str(ei.value)


def test_plan_anomaly_index_required_with_anomal_type(pkg, tmp_path):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_ps_golden as ps
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d, ps.CASE_IA)
    _counts_consistent(pkg.plan(d, "E", 3))
    os.unlink(os.path.join(d, "ia"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.plan(d, "A", 2)
    assert ei.value.status == 2 and "ia" in str(ei.value)


def test_element_colouring_is_valid_and_greedy(pkg, mg, tmp_path):
    """Assembly colours (host): conflict-free, ascending per colour, greedy (CPU driver
    compiled against the library)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "colouring")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    os.path.join(here, "native", "colouring.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    d = str(tmp_path / "m")
    spec = mg.small_model(cells=12, n_dec=2, steps_per_dec=4, block=True)
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout


def test_models_of_one_mesh_merge_for_batched_serving(pkg, mg, tmp_path):
    """merge_models / plan_merged (host): directories of one mesh with different wires
    and receivers merge in order, each keeping its receivers' ranges and its initial
    field; a directory with another mesh is refused (CPU driver compiled against the
    library)."""
    import dataclasses
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "merge")
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    "-I", os.path.join(os.path.dirname(here), "include"), "-I", cuda_inc,
                    os.path.join(here, "native", "merge_models.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    base = mg.small_model(cells=8, n_dec=2, steps_per_dec=4)
    dirs = []
    for i, wires in enumerate([[((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0))],
                               [((-30.0, 20.0, 0.0), (30.0, 20.0, 0.0)), ((0.0, -40.0, 0.0), (0.0, 20.0, 0.0))],
                               [((-20.0, -20.0, 0.0), (40.0, -20.0, 0.0))]]):
        rec = [(0.0, 15.0 + 5.0 * i + 25.0 * k, 0.0) for k in range(3 + i)]
        spec = dataclasses.replace(base, sources=wires, receivers_b=[rec] * len(wires),
                                   receivers_e=[rec] * len(wires))
        d = str(tmp_path / ("tx%d" % i))
        mg.write_model(d, spec)
        mg.write_analytic_initial_field(d, spec)
        dirs.append(d)
    other = str(tmp_path / "other")
    spec = mg.small_model(cells=10, n_dec=2, steps_per_dec=4)
    mg.write_model(other, spec)
    mg.write_analytic_initial_field(other, spec)
    r = subprocess.run([exe] + dirs + [other], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok 4 sources"), r.stdout + r.stderr
    # the other checks: materials, time grid, current function, source settings
    import shutil as sh
    for name, edit, message in (
            ("mat", _scale_sigma, "the materials differ"),
            ("grid", _shift_time, "the time grids differ"),
            ("srs", _set_dipole_count, "the source or receiver settings differ")):
        d = str(tmp_path / ("bad_" + name))
        sh.copytree(dirs[0], d)
        edit(d)
        r = subprocess.run([exe, "--expect", dirs[1], d, message], capture_output=True, text=True)
        assert r.returncode == 0, (name, r.stdout + r.stderr)


def _set_dipole_count(d):
    with open(os.path.join(d, "nSrsRazb"), "w") as f:
        f.write("7\n")


def _scale_sigma(d):
    rows = [line.split() for line in open(os.path.join(d, "sig3d")) if line.strip()]
    with open(os.path.join(d, "sig3d"), "w") as f:
        f.write("".join("%s\t%.7e\t%.7e\n" % (r[0], 2 * float(r[1]), 2 * float(r[2])) for r in rows))


def _shift_time(d):
    with open(os.path.join(d, "infite.0")) as f:
        head, body = f.read().split("T I M E :", 1)
    last = body.replace(";", " ").split()[-1]
    with open(os.path.join(d, "infite.0"), "w") as f:
        f.write(head + "T I M E :" + body.replace(last, "%.13e" % (1.5 * float(last))))


def test_point_location_and_threaded_receiver_smoothing(pkg, mg, tmp_path):
    """The element grid used to place dipoles and receivers finds the same element as a
    scan over all elements (graded tensor mesh with points on nodes and faces, random
    overlapping boxes, a model's dipoles, a wire half past the mesh edge whose outer
    dipoles go to the nearest element), and the receiver operators built on 1 and on 3
    host threads are byte-identical (CPU driver compiled against the library)."""
    import dataclasses
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "locate")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    "-I", os.path.join(os.path.dirname(here), "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(here, "native", "point_location.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    base = mg.small_model(cells=10, n_dec=2, steps_per_dec=4)
    x_max = float(base.x[-1])
    wires = [((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0)), ((-30.0, 20.0, 0.0), (30.0, 20.0, 0.0)),
             ((0.0, -40.0, 0.0), (0.0, 20.0, 0.0)),
             ((x_max - 400.0, 0.0, 0.0), (x_max + 400.0, 0.0, 0.0))]  # half of it past the mesh edge
    rec = [(0.0, 10.0 + 12.5 * k, 0.0) for k in range(6)] + [(-20.0, -20.0, 0.0)]
    spec = dataclasses.replace(base, sources=wires, receivers_b=[rec] * 4, receivers_e=[rec] * 4)
    d = str(tmp_path / "m")
    mg.write_model(d, spec)
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    assert "(0 outside" not in r.stdout, r.stdout


def _read_operator(path):
    b = open(path, "rb").read()
    nrec, nrows, nnz = (int(v) for v in np.frombuffer(b, "<i8", 3))
    off = 24
    rowptr = np.frombuffer(b, "<i8", nrows + 1, off)
    off += 8 * (nrows + 1)
    col = np.frombuffer(b, "<i4", nnz, off)
    off += 4 * nnz
    val = np.frombuffer(b, "<f8", nnz, off)
    off += 8 * nnz
    src = np.frombuffer(b, "<i4", nrows, off)
    return nrec, rowptr, col, val, src


@pytest.mark.parametrize("case,form", [("cube8_two_wires", "A"), ("cube8_two_wires", "E"),
                                       ("cube6_wire_beyond", "E"), ("cube8_receivers_on_nodes", "E"),
                                       ("cube8_two_wires_ragged", "A"), ("cube6_no_b_receivers", "A"),
                                       ("cube8_neib1_window", "E"), ("cube6_ramp_current", "A"),
                                       ("cube8_permeable_block", "E")])
def test_host_plan_products_match_the_oracle(pkg, golden, tmp_path, case, form):
    """The host half of a solve (TransientSolve::plan, no device) against the numpy oracle,
    which the reference's goldens pin: the source vectors and the initial field that go to
    the device, and each receiver operator applied to a random field against the oracle's
    smoothing of that field (ReceiverSet: the subdomain mass-matrix solve per time layer
    that the operator folds into one row per receiver)."""
    import shutil
    import subprocess
    import tdem_oracle
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "dump")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    "-I", os.path.join(os.path.dirname(here), "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(here, "native", "host_plan_dump.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    d = str(tmp_path / case)
    if case in ("cube6_wire_beyond", "cube8_receivers_on_nodes", "cube8_two_wires_ragged", "cube6_no_b_receivers",
                "cube8_neib1_window", "cube6_ramp_current", "cube8_permeable_block"):
        sys.path.insert(0, os.path.join(here, "golden"))
        import make_beyond_golden as bg
        import make_nodes_golden as ng
        if case in ("cube6_wire_beyond", "cube6_ramp_current"):
            bg.write_case_inputs(d, case)
        else:
            ng.write_case_inputs(d, case)
    else:
        golden.write_case_inputs(case, d)
    out = str(tmp_path / "plan")
    r = subprocess.run([exe, d, "1" if form == "E" else "0", out], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    m = tdem_oracle.read_model(d)
    n, npls = m["n"], m["npls"]
    eform = form == "E"
    S = np.fromfile(out + ".S").reshape(npls, n).T
    u0 = np.fromfile(out + ".u0").reshape(npls, n).T
    have_src = m["fdirect"] and (eform or np.any(m["cf"][1:] != 0)) and m["nsrs"] > 0
    S_or = tdem_oracle.source_vectors(m) if have_src else np.zeros((n, npls))
    assert np.abs(S - S_or).max() <= 1e-13 * max(np.abs(S_or).max(), 1e-300)
    u0_or = tdem_oracle.initial_field(m, eform)
    assert np.abs(u0 - u0_or).max() <= 1e-13 * max(np.abs(u0_or).max(), 1e-300)
    u = np.random.default_rng(1).standard_normal((n, npls))
    for key, pts, curl, ig in (("rb", m["rec_b"], True, m["ig_b"]), ("re", m["rec_e"], False, m["ig_e"])):
        nrec, rowptr, col, val, src = _read_operator(out + "." + key)
        assert nrec == len(pts)
        if nrec == 0:
            assert len(rowptr) == 1 and len(col) == 0
            continue
        got = np.array([val[rowptr[k]:rowptr[k + 1]] @ u[col[rowptr[k]:rowptr[k + 1]], src[k]]
                        for k in range(3 * nrec)]).reshape(3, nrec)
        own = np.zeros(nrec, int)
        for p in range(npls):
            own[ig[p]:ig[p + 1]] = p
        want = tdem_oracle.ReceiverSet(m, np.asarray(pts), curl).evaluate(u, own)
        # CG to 1e-15 against a direct solve: measured up to 2.5e-15 of the peak
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), (key, np.abs(got - want).max())


def test_merged_host_plan_is_the_parts_side_by_side(pkg, mg, tmp_path):
    """plan_merged (the serving loop's batched time steps), host half: the source vectors
    and initial fields of three directories over one mesh are their solo plans' columns
    side by side, and every receiver row is its solo plan's row (each directory's receivers
    smoothed on their own neighbourhood), placed component-major over all receivers and
    sampling the directory's shifted source column."""
    import dataclasses
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "dump")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    "-I", os.path.join(os.path.dirname(here), "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(here, "native", "host_plan_dump.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    base = mg.small_model(cells=8, n_dec=2, steps_per_dec=4)
    dirs = []
    for i, wires in enumerate([[((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0))],
                               [((-30.0, 20.0, 0.0), (30.0, 20.0, 0.0)), ((0.0, -40.0, 0.0), (0.0, 20.0, 0.0))],
                               [((-20.0, -20.0, 0.0), (40.0, -20.0, 0.0))]]):
        rec = [(0.0, 15.0 + 5.0 * i + 25.0 * k, 0.0) for k in range(3 + i)]
        spec = dataclasses.replace(base, sources=wires, receivers_b=[rec] * len(wires),
                                   receivers_e=[rec] * len(wires))
        d = str(tmp_path / ("tx%d" % i))
        mg.write_model(d, spec)
        mg.write_analytic_initial_field(d, spec)
        dirs.append(d)
    for form in ("0", "1"):
        solo = []
        for k, d in enumerate(dirs):
            out = str(tmp_path / ("solo%d_%s" % (k, form)))
            r = subprocess.run([exe, d, form, out], capture_output=True, text=True)
            assert r.returncode == 0, r.stdout + r.stderr
            solo.append((out, int(r.stdout.split()[2])))
        out = str(tmp_path / ("merged_" + form))
        r = subprocess.run([exe, "--merged", form, out] + dirs, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        n, npls = (int(v) for v in r.stdout.split()[1:3])
        assert npls == sum(p for _, p in solo)
        for ext in (".S", ".u0"):
            want = np.concatenate([np.fromfile(o + ext) for o, _ in solo])
            assert np.array_equal(np.fromfile(out + ext), want), ext
        for key in ("rb", "re"):
            nrec, rp, col, val, src = _read_operator(out + "." + key)
            parts = [_read_operator(o + "." + key) for o, _ in solo]
            assert nrec == sum(p[0] for p in parts)
            for c in range(3):
                roff = coff = 0
                for (nr, prp, pcol, pval, psrc), (_, pn) in zip(parts, solo):
                    for i in range(nr):
                        a, b = c * nrec + roff + i, c * nr + i
                        assert np.array_equal(col[rp[a]:rp[a + 1]], pcol[prp[b]:prp[b + 1]])
                        assert np.array_equal(val[rp[a]:rp[a + 1]], pval[prp[b]:prp[b + 1]])
                        assert src[a] == psrc[b] + coff
                    roff += nr
                    coff += pn


def test_stationary_source_points_match_a_scan(pkg, golden, tmp_path):
    """The stationary module's electrodes and dipoles (stationary_source_points, host only)
    against a scan over all earth elements with the nearest-element rule, restated in the
    driver: bitwise equal elements and local coordinates, on cube8_two_wires and on the wire
    half past the mesh edge (51 points outside the mesh)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    here = os.path.dirname(os.path.abspath(__file__))
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "points")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    "-I", os.path.join(os.path.dirname(here), "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(here, "native", "stationary_points.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_beyond_golden as bg
    a, b = str(tmp_path / "two"), str(tmp_path / "beyond")
    golden.write_case_inputs("cube8_two_wires", a)
    bg.write_case_inputs(b)
    for d, outside in ((a, 0), (b, 51)):
        r = subprocess.run([exe, d], capture_output=True, text=True)
        assert r.returncode == 0 and r.stdout.strip().endswith("(%d outside)" % outside), r.stdout + r.stderr
