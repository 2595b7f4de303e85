"""Host side of the primary-secondary source of the E-formulation (no GPU): the
library's values of -dEn/dt for every kind of step (two-point, three-point, with and
without layer 0) are bit-identical to the oracle restatement, which is pinned to the
reference's own outputs (test_oracle.py)."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import tdem_oracle
from conftest import GOLDEN, ROOT

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("case", ["cube8_block_ps", "cube8_block_ps_ia"])
def test_normal_field_rate_matches_oracle(pkg, tmp_path, case):
    sys.path.insert(0, GOLDEN)
    import make_ps_golden as ps
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "rate")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    os.path.join(HERE, "native", "normal_field_rate.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d, case)
    m = tdem_oracle.read_model(d)
    steps = [(1, 0, -1, 0), (2, 1, 0, 0), (3, 2, 1, 1), (4, 3, 2, 1), (8, 6, 4, 1), (12, 10, 8, 1), (5, 4, 3, 0)]
    out = str(tmp_path / "rate.bin")
    subprocess.run([exe, d, out] + [str(x) for s in steps for x in s], check=True, capture_output=True)
    got = np.fromfile(out, "<f8").reshape(len(steps), m["npls"], m["n"])
    for k, (it, t1, t2, three) in enumerate(steps):
        ref = tdem_oracle.normal_field_rate(m, it, t1, t2, bool(three)).T
        assert np.array_equal(got[k], ref), (it, t1, t2, three)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_normal_field_errors(pkg, tmp_path):
    """A missing or short layer file and a missing normal potential are reported."""
    sys.path.insert(0, GOLDEN)
    import make_ps_golden as ps
    lib_dir = os.path.dirname(pkg.LIB_PATH)
    exe = str(tmp_path / "rate")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(pkg.__file__), "csrc"),
                    os.path.join(HERE, "native", "normal_field_rate.cpp"), "-L" + lib_dir, "-ltdem_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    d = str(tmp_path / "ps")
    ps.write_case_inputs(d)
    f3 = os.path.join(d, "m%s.enor.%04d" % (ps.PNAME, 3))
    with open(f3, "rb") as f:
        data = f.read()
    with open(f3, "wb") as f:
        f.write(data[:-4])
    r = subprocess.run([exe, d, str(tmp_path / "o.bin"), "3", "2", "1", "1"], capture_output=True, text=True)
    assert r.returncode != 0 and "too short" in r.stdout
    os.unlink(f3)
    r = subprocess.run([exe, d, str(tmp_path / "o.bin"), "3", "2", "1", "1"], capture_output=True, text=True)
    assert r.returncode != 0 and "cannot open the normal field" in r.stdout
    os.unlink(os.path.join(d, "v3n.dat"))
    r = subprocess.run([exe, d, str(tmp_path / "o.bin"), "2", "1", "0", "0"], capture_output=True, text=True)
    assert r.returncode != 0 and "v3n.dat" in r.stdout
