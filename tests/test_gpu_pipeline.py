"""GPU test of the direct-mode 3D-only module sequence (tdem_pipeline_directory,
the B200 stand-in for GeoCalculatorSP's CalcMainTask in direct mode) against the
reference's own modules run one after another in the same order (built from source
under oracle/_ref): TimeDirectSolver, CorrectTimeMesh, CalcStat3D_3T_A,
CalcNonstat3DLine, SumNonstat3DOnly."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from conftest import FP64_TOL, GOLDEN

pytestmark = pytest.mark.gpu

MODULES = ("TimeDirectSolver", "CorrectTimeMesh", "CalcStat3D_3T_A", "CalcNonstat3DLine_A2", "SumNonstat3DOnly")


def _numbers(path):
    vals = []
    for line in open(path):
        for tok in line.replace("\t", " ").split():
            try:
                vals.append(float(tok))
            except ValueError:
                pass
    return np.array(vals)


def test_pipeline_matches_the_reference_module_sequence(pkg, mg, outs, tmp_path):
    import run_ref
    if not all(run_ref.available(m) for m in MODULES):
        pytest.skip("oracle/_ref modules not built")
    sys.path.insert(0, GOLDEN)
    import make_timegrid_golden as tg
    src = str(tmp_path / "src")
    spec = mg.small_model(cells=8, n_dec=2, steps_per_dec=5, block=True, n_receivers=4)
    mg.write_model(src, spec)
    # a log-spaced time list for the time-grid modules to regularise
    tg.grid_case(src, tg.log_times(30, 1e-3, 5e-6), 2.0, 5)
    gdir, rdir = str(tmp_path / "gpu"), str(tmp_path / "ref")
    shutil.copytree(src, gdir)
    shutil.copytree(src, rdir)
    pkg.pipeline_directory(gdir, "A", 2)
    for name in ("TimeDirectSolver", "CorrectTimeMesh"):
        subprocess.run([run_ref.binary(name)], cwd=rdir, check=True, capture_output=True, timeout=300)
    run_ref.run_stationary(rdir)
    run_ref.run_transient(rdir, "A2")
    subprocess.run([run_ref.binary("SumNonstat3DOnly")], cwd=rdir, check=True, capture_output=True, timeout=300)
    # the time grid is byte-identical, the transients within the FP64 tolerance
    for name in ("infite.0", "currentfunction", "deltafunction"):
        assert open(os.path.join(gdir, name), "rb").read() == open(os.path.join(rdir, name), "rb").read(), name
    for o in ("eall_anom.1", "edsall_anom.1", "ball_anom.1"):
        assert outs.compare_files(os.path.join(gdir, o), os.path.join(rdir, o)) <= FP64_TOL, o
    # the component files: the same numbers up to the transients' tolerance
    for stem in ("Exall", "Eyall", "Ezall", "Bxall", "Byall", "Bzall", "Edsxall", "Edsyall", "Edsall"):
        a, b = _numbers(os.path.join(gdir, stem + ".1")), _numbers(os.path.join(rdir, stem + ".1"))
        assert a.shape == b.shape, stem
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-8 * scale, stem


def test_pipeline_stops_at_the_first_failing_module(pkg, mg, tmp_path):
    d = str(tmp_path / "m")
    spec = mg.small_model(cells=6, n_dec=2, steps_per_dec=5)
    mg.write_model(d, spec)
    os.unlink(os.path.join(d, "nver.dat"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.pipeline_directory(d, "A", 2)
    assert "CalcStat3D_3T_A" in str(ei.value)
    assert not os.path.exists(os.path.join(d, "eall_anom.1"))
