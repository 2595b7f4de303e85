"""Time-grid modules on the host (no GPU): TimeDirectSolver and CorrectTimeMesh
against the reference's own programs, byte for byte.

Golden fixtures (tests/golden/timegrid, made by make_timegrid_golden.py with the
reference compiled from source) pin every file the two modules leave behind; where
oracle/_ref holds the reference programs, seeded grids are compared live."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_timegrid_golden as tg  # noqa: E402


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def _stage(case, dst):
    for f in tg.INPUTS:
        shutil.copy(os.path.join(tg.FIXTURES, case, "in", f), os.path.join(dst, f))


def _run(pkg, d, direct):
    if direct:
        pkg.time_direct_solver(d)
    pkg.correct_time_mesh(d)


def _same_files(a, b):
    names = [f for f in tg.OUTPUTS if os.path.exists(os.path.join(b, f))]
    assert names
    for f in tg.OUTPUTS:
        assert os.path.exists(os.path.join(a, f)) == os.path.exists(os.path.join(b, f)), f
    for f in names:
        assert _read(os.path.join(a, f)) == _read(os.path.join(b, f)), f


@pytest.mark.parametrize("case", sorted(tg.CASES))
def test_matches_reference_golden(pkg, tmp_path, case):
    _stage(case, str(tmp_path))
    _run(pkg, str(tmp_path), tg.CASES[case][3])
    _same_files(str(tmp_path), os.path.join(tg.FIXTURES, case, "out"))


def test_correction_refills_the_short_decade(pkg, tmp_path):
    _stage("correct_only", str(tmp_path))
    pkg.correct_time_mesh(str(tmp_path))
    t = np.array([float(v) for v in _read(str(tmp_path / "infite.0")).decode().split("T I M E :")[1]
                  .replace(";", " ").split()])
    steps = np.diff(t)
    # 10 steps of 1e-6, then 2e-6 steps through the short decade's span, then 8e-6
    assert np.allclose(steps[:10], 1e-6, rtol=1e-6)
    assert np.allclose(steps[10:22], 2e-6, rtol=1e-6)
    assert np.allclose(steps[-6:], 8e-6, rtol=1e-6)


def test_drop_in_executables(pkg, tmp_path):
    d = tmp_path / "run"
    d.mkdir()
    _stage("log60", str(d))
    bindir = tmp_path / "bin"
    bindir.mkdir()
    exe = os.path.join(os.path.dirname(pkg.LIB_PATH), "tdem_calcnonstat3dline")
    for name in ("TimeDirectSolver", "CorrectTimeMesh"):
        os.symlink(exe, str(bindir / name))
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.dirname(pkg.LIB_PATH))
    for name in ("TimeDirectSolver", "CorrectTimeMesh"):
        subprocess.run([str(bindir / name)], cwd=str(d), check=True, env=env)
    _same_files(str(d), os.path.join(tg.FIXTURES, "log60", "out"))


@pytest.mark.parametrize("missing", ["tcff", "infite.0", "currentfunction", "deltafunction"])
def test_missing_input_is_an_input_error(pkg, tmp_path, missing):
    _stage("log60", str(tmp_path))
    os.unlink(str(tmp_path / missing))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.time_direct_solver(str(tmp_path))
    assert ei.value.status == 2 and missing in str(ei.value)


def test_one_time_is_refused_and_nothing_rewritten(pkg, tmp_path):
    d = str(tmp_path)
    tg.grid_case(d, [0.0, 1e-6, 3e-6], 2.0, 9)
    tg.write_infite(d, [0.0])
    before = {f: _read(os.path.join(d, f)) for f in tg.INPUTS}
    for run in (pkg.time_direct_solver, pkg.correct_time_mesh):
        with pytest.raises(pkg.TdemError) as ei:
            run(d)
        assert ei.value.status == 2 and "infite.0" in str(ei.value)
    assert {f: _read(os.path.join(d, f)) for f in tg.INPUTS} == before


REF_PROGRAMS = all(os.path.exists(os.path.join(tg.REF_BIN, n)) for n in ("TimeDirectSolver", "CorrectTimeMesh"))


@pytest.mark.skipif(not REF_PROGRAMS, reason="reference programs not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("seed", range(8))
def test_live_against_reference(pkg, tmp_path, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(5, 300))
    t_first = 10.0 ** rng.uniform(-8, -5)
    t_end = t_first * 10.0 ** rng.uniform(2, 7)
    times = tg.log_times(n, t_end, t_first)
    if seed % 2:
        times = np.concatenate([[0.0], np.sort(times[1:] * rng.uniform(0.9, 1.1, n))])
    tcff = float(rng.choice([1.5, 2.0, 2.5, 3.0]))
    ref, own = tmp_path / "ref", tmp_path / "own"
    tg.grid_case(str(ref), times, tcff, seed)
    shutil.copytree(str(ref), str(own))
    tg.run_reference(str(ref), True)
    _run(pkg, str(own), True)
    _same_files(str(own), str(ref))
