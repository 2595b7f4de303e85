"""GPU tests of the grounded-wire stationary initial field (tdem_stationary_directory,
the drop-in for CalcStat3D_3T_A): v3a.dat / a0.dat against the reference's own
outputs stored in tests/golden (CalcStat3D_3T_A built from source), the full
stationary -> transient chain against the golden transients, the drop-in
executable under the module's name, and the reference binary at a larger size
when oracle/_ref is present."""
import os
import subprocess

import numpy as np
import pytest

from conftest import FP64_TOL, GOLDEN, ROOT

pytestmark = pytest.mark.gpu

# two FP64 direct solves (different orderings) of the nodal systems; the 1e30
# boundary penalty and the point electrodes keep the systems far from singular
STAT_TOL = 1e-10


def _fields(d, n_nodes, npls):
    v = np.fromfile(os.path.join(d, "v3a.dat")).reshape(npls, n_nodes)
    a = np.fromfile(os.path.join(d, "a0.dat")).reshape(npls, n_nodes, 3)
    z = np.fromfile(os.path.join(d, "v3n.dat"))
    return v, a, z


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _write_model(golden, mg, name, d):
    spec = mg.small_model(**golden.CASES[name])
    mg.write_model(d, spec)
    return spec


@pytest.mark.parametrize("name", ["cube6", "cube8_block", "cube8_two_wires"])
def test_stationary_matches_reference_goldens(pkg, golden, mg, name, tmp_path):
    d = str(tmp_path / name)
    spec = _write_model(golden, mg, name, d)
    pkg.stationary_directory(d)
    npls, nn = len(spec.sources), spec.n_nodes
    v, a, z = _fields(d, nn, npls)
    vr, ar, zr = _fields(os.path.join(GOLDEN, name), nn, npls)
    assert z.shape == zr.shape and not z.any()
    for p in range(npls):
        assert _rel(v[p], vr[p]) <= STAT_TOL
        for c in range(3):
            if np.abs(ar[p, :, c]).max() > 0:
                assert _rel(a[p, :, c], ar[p, :, c]) <= STAT_TOL, (p, c, _rel(a[p, :, c], ar[p, :, c]))


def test_stationary_then_transient_matches_golden_chain(pkg, golden, mg, outs, tmp_path):
    """GPU stationary field feeding the GPU transient reproduces the reference's
    stationary -> transient chain."""
    name = "cube8_block"
    d = str(tmp_path / name)
    _write_model(golden, mg, name, d)
    pkg.stationary_directory(d)
    for v in ("A3", "E2"):
        pkg.run_directory(d, v[0], int(v[1]))
        for o in ("eall_anom", "edsall_anom"):
            ref = os.path.join(GOLDEN, name, "%s_%s.1" % (v, o))
            err = outs.compare_files(os.path.join(d, "%s.1" % o), ref)
            assert err <= FP64_TOL, (v, o, err)


def test_stationary_drop_in_executable(pkg, golden, mg, tmp_path):
    name = "cube6"
    d = str(tmp_path / name)
    spec = _write_model(golden, mg, name, d)
    exe = os.path.join(os.path.dirname(pkg.LIB_PATH), "tdem_calcnonstat3dline")
    link = str(tmp_path / "CalcStat3D_3T_A")
    os.symlink(exe, link)
    r = subprocess.run([link, d], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v, _, _ = _fields(d, spec.n_nodes, 1)
    vr, _, _ = _fields(os.path.join(GOLDEN, name), spec.n_nodes, 1)
    assert _rel(v[0], vr[0]) <= STAT_TOL


def test_stationary_missing_input_is_an_input_error(pkg, golden, mg, tmp_path):
    d = str(tmp_path / "m")
    _write_model(golden, mg, "cube6", d)
    os.unlink(os.path.join(d, "sours"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.stationary_directory(d)
    assert ei.value.status == 2 and "sours" in str(ei.value)


def test_stationary_matches_reference_binary_16(pkg, mg, tmp_path):
    """16^3 cells (fronts of several 256-column outer panels) against the
    reference CalcStat3D_3T_A run here, when the oracle build is present."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import run_ref
    if not run_ref.available("CalcStat3D_3T_A"):
        pytest.skip("reference build (oracle/_ref) not present")
    spec = mg.small_model(cells=16, n_dec=2, steps_per_dec=4, n_sources=2)
    dr, dg = str(tmp_path / "ref"), str(tmp_path / "gpu")
    mg.write_model(dr, spec)
    mg.write_model(dg, spec)
    run_ref.run_stationary(dr)
    pkg.stationary_directory(dg)
    v, a, _ = _fields(dg, spec.n_nodes, 2)
    vr, ar, _ = _fields(dr, spec.n_nodes, 2)
    for p in range(2):
        assert _rel(v[p], vr[p]) <= STAT_TOL
        for c in range(3):
            if np.abs(ar[p, :, c]).max() > 0:
                assert _rel(a[p, :, c], ar[p, :, c]) <= STAT_TOL
