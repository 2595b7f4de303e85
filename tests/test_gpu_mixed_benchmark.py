"""GPU tests of precision 32 on the benchmark physics (air of 1e-8 S/m, as the
reference's mesh builder writes it): the factorization runs in FP64 and its factor
is held rounded to FP32; every time step solves with that FP32 factor inside an
FP64 preconditioned conjugate gradient on the FP64 system to a relative residual of
1e-10.  An FP32 factorization of these systems breaks down (their condition number
is beyond FP32), a rounded FP64 factor does not.  The transients are compared with
the reference's own (golden outputs) and with the FP64 GPU path."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

# acceptance level of the mixed-precision path against the FP64 oracle (receiver
# transients, relative to each receiver's peak)
MIXED_ACCEPT = 1e-5


@pytest.mark.parametrize("variant", ["A2", "A3", "E2", "E3"])
def test_mixed_matches_reference_goldens(pkg, golden, outs, tmp_path, variant):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    with pkg.Solver(d, variant[0], int(variant[1]), precision=32) as s:
        s.run()
        s.write_outputs()
        info = s.info()
    assert info["precision"] == 32 and info["refine_worst"] <= 1e-10
    assert 0 < info["refine_iters_max"] <= 20, info["refine_iters_max"]
    for o in golden.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, "cube8_block", "%s_%s.1" % (variant, o)))
        assert err <= MIXED_ACCEPT, (o, err)


def test_mixed_full_c1_transient_matches_reference(pkg, outs, tmp_path):
    """The 40^3 half-space, all 120 steps, against the reference's FP64 transient."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_scale_golden as sg
    d = str(tmp_path / "c1")
    sg.write_case_inputs("c1", d)
    with pkg.Solver(d, "A", 2, precision=32) as s:
        s.run()
        s.write_outputs()
        info = s.info()
    assert info["refine_worst"] <= 1e-10
    for o in sg.OUTPUTS:
        err = outs.compare_files(os.path.join(d, o + ".1"), os.path.join(GOLDEN, "scale", "c1", "A2_%s.1" % o))
        assert err <= MIXED_ACCEPT, (o, err)


def test_mixed_factor_ahead_is_bitwise_sequential(pkg, golden, tmp_path):
    d = str(tmp_path / "m")
    golden.write_case_inputs("cube8_block", d)
    out = {}
    for slots in (1, 2):
        with pkg.Solver(d, "E", 3, precision=32, factor_slots=slots) as s:
            s.run()
            out[slots] = s.results()
            assert s.info()["factor_slots"] == slots
    for a, b in zip(out[1], out[2]):
        assert np.array_equal(a, b)
