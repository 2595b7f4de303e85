"""Post-processing modules on the host (no GPU): SumNonstat3DOnly and SummatorEDMN
against the reference's own programs, byte for byte.

Golden fixtures (tests/golden/postprocess, made by make_postprocess_golden.py with
the reference compiled from source) pin the outputs; where oracle/_ref holds the
reference programs, further seeded cases are compared live."""
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_postprocess_golden as pg  # noqa: E402

CASES = sorted(pg.CASES)


def _stage(case, dst):
    src = os.path.join(pg.FIXTURES, case, "in")
    for f in os.listdir(src):
        shutil.copy(os.path.join(src, f), os.path.join(dst, f))


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def _calls(d):
    """The summator calls of a case: both WithDDV values for every transmitter."""
    npls = sum(1 for f in os.listdir(d) if f.startswith("eall_anom."))
    return npls, [(ddv, 1, p) for p in range(npls) for ddv in (0, 1)]


def _run_product(pkg, d, case):
    pkg.sum_nonstat_3d_only(d)
    npls, calls = _calls(d)
    params = pg.CASES[case]
    pg.prepare_summator(d, npls, bool(params and params["cut_last_newline"]))
    for ddv, prof, place in calls:
        pkg.summator_edmn(d, ddv, prof, place)


@pytest.mark.parametrize("case", CASES)
def test_outputs_match_reference_golden(pkg, tmp_path, case):
    d = str(tmp_path)
    _stage(case, d)
    _run_product(pkg, d, case)
    expected = os.path.join(pg.FIXTURES, case, "out")
    names = sorted(os.listdir(expected))
    assert any(n.startswith("edmoonall") for n in names) and any(n.startswith("Exall") for n in names)
    for f in names:
        assert _read(os.path.join(d, f)) == _read(os.path.join(expected, f)), f


def test_results_do_not_depend_on_host_threads(pkg, tmp_path, monkeypatch):
    monkeypatch.setenv("TDEM_HOST_THREADS", "1")
    d = str(tmp_path)
    _stage("chain", d)
    _run_product(pkg, d, "chain")
    expected = os.path.join(pg.FIXTURES, "chain", "out")
    for f in os.listdir(expected):
        assert _read(os.path.join(d, f)) == _read(os.path.join(expected, f)), f


def _exe(pkg):
    return os.path.join(os.path.dirname(pkg.LIB_PATH), "tdem_calcnonstat3dline")


def test_drop_in_executables(pkg, tmp_path):
    """The executable installed under the reference modules' names takes their
    command lines and writes the same files."""
    case = "mixed"
    d = tmp_path / "run"
    d.mkdir()
    _stage(case, str(d))
    bindir = tmp_path / "bin"
    bindir.mkdir()
    for name in ("SumNonstat3DOnly", "SummatorEDMN"):
        os.symlink(_exe(pkg), str(bindir / name))
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.dirname(pkg.LIB_PATH))
    subprocess.run([str(bindir / "SumNonstat3DOnly")], cwd=str(d), check=True, env=env)
    npls, calls = _calls(str(d))
    pg.prepare_summator(str(d), npls, False)
    for ddv, prof, place in calls:
        subprocess.run([str(bindir / "SummatorEDMN"), str(ddv), str(prof), str(place)], cwd=str(d), check=True,
                       env=env)
    expected = os.path.join(pg.FIXTURES, case, "out")
    for f in os.listdir(expected):
        assert _read(str(d / f)) == _read(os.path.join(expected, f)), f
    # the reference's argument check: three parameters are required
    r = subprocess.run([str(bindir / "SummatorEDMN"), "1", "1"], cwd=str(d), env=env, capture_output=True)
    assert r.returncode != 0


def test_no_lines_writes_nothing(pkg, tmp_path):
    d = str(tmp_path)
    _stage("mixed", d)
    with open(os.path.join(d, "xyzmn"), "w") as f:
        f.write("0\n")
    pkg.summator_edmn(d, 1, 1, 0)  # SummatorEDMN/main.cpp:282-291: nothing to do
    assert not any(f.startswith(("edmnall", "edmoonall")) for f in os.listdir(d))


@pytest.mark.parametrize("missing", ["group", "infite.0", "recvse", "eall_anom.2", "edsall_anom.1"])
def test_split_missing_input_is_an_input_error(pkg, tmp_path, missing):
    d = str(tmp_path)
    _stage("mixed", d)
    os.unlink(os.path.join(d, missing))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.sum_nonstat_3d_only(d)
    assert ei.value.status == 2 and missing in str(ei.value)


def test_split_truncated_results_are_an_input_error(pkg, tmp_path):
    d = str(tmp_path)
    _stage("mixed", d)
    fn = os.path.join(d, "eall_anom.1")
    with open(fn) as f:
        lines = f.read().splitlines(True)
    with open(fn, "w") as f:
        f.write("".join(lines[:-3]))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.sum_nonstat_3d_only(d)
    assert ei.value.status == 2 and "eall_anom.1" in str(ei.value)


def test_summator_missing_and_inconsistent_inputs(pkg, tmp_path):
    d = str(tmp_path)
    _stage("mixed", d)
    pkg.sum_nonstat_3d_only(d)
    pg.prepare_summator(d, 2, False)
    os.unlink(os.path.join(d, "ezall1_1"))
    with pytest.raises(pkg.TdemError) as ei:
        pkg.summator_edmn(d, 0, 1, 1)
    assert ei.value.status == 2 and "ezall1_1" in str(ei.value)
    # zero lines in the transmitter's own list: the reference divides by zero here
    with open(os.path.join(d, "xyzmn1_1"), "w") as f:
        f.write("0\n")
    with pytest.raises(pkg.TdemError):
        pkg.summator_edmn(d, 0, 1, 0)
    # a y curve shorter than its x curve (undefined in the reference) is refused
    fn = os.path.join(d, "eyall1_0")
    with open(fn) as f:
        lines = f.read().splitlines(True)
    with open(fn, "w") as f:
        f.write("".join(lines[:8]))
    with open(os.path.join(d, "xyzmn1_1"), "w") as f:
        f.write("2\n" + "0 0 0 1 1 1\n" * 2)
    with pytest.raises(pkg.TdemError) as ei:
        pkg.summator_edmn(d, 0, 1, 0)
    assert "fewer time rows" in str(ei.value)


REF_PROGRAMS = all(os.path.exists(os.path.join(pg.REF_BIN, n)) for n in ("SumNonstat3DOnly", "SummatorEDMN"))


@pytest.mark.skipif(not REF_PROGRAMS, reason="reference programs not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("seed,nb,ne,lines,cut", [
    (101, (4,), (10,), (2,), False),
    (102, (1, 2, 0), (5, 7, 12), (1, 2, 3), True),
    (103, (0, 0), (3, 4), (3, 4), False),   # one point per line (ddV split point 0)
    (104, (2,), (2,), (3,), False),         # fewer points than lines: no point per line
])
def test_live_against_reference(pkg, tmp_path, seed, nb, ne, lines, cut):
    ref, own = tmp_path / "ref", tmp_path / "own"
    meta = pg.synth_case(str(ref), seed=seed, nb=nb, ne=ne, lines=lines, nt=9, window=(1, 8), with_zeros=True,
                         cut_last_newline=cut)
    shutil.copytree(str(ref), str(own))
    pg.run_reference(str(ref), meta)
    pkg.sum_nonstat_3d_only(str(own))
    pg.prepare_summator(str(own), meta["npls"], cut)
    for ddv, prof, place in meta["calls"]:
        pkg.summator_edmn(str(own), ddv, prof, place)
    names = ["%s.%d" % (s, p + 1) for s in pg.SPLIT_OUTPUTS for p in range(meta["npls"])]
    names += pg.summator_outputs(meta["calls"])
    for f in names:
        assert _read(str(own / f)) == _read(str(ref / f)), f
