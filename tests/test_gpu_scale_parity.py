"""GPU parity at the benchmark's scales against the reference's own
CalcNonstat3DLine (golden outputs in tests/golden/scale, made by
tests/golden/make_scale_golden.py from the reference built from source):

  * the plain-method configuration in full: 40^3 half-space, A-formulation,
    backward Euler, all 120 steps (6 factorizations);
  * 32 wires solved as one n x 32 block per step (the batched path), A- and
    E-formulation with the three-point scheme, every transmitter's three files.
"""
import os
import sys

import pytest

from conftest import FP64_TOL, GOLDEN

pytestmark = pytest.mark.gpu

sys.path.insert(0, GOLDEN)
import make_scale_golden as sg  # noqa: E402

SCALE = os.path.join(GOLDEN, "scale")


def _compare(outs, d, case, variant, npls):
    worst = 0.0
    for o in sg.OUTPUTS:
        for p in range(1, npls + 1):
            err = outs.compare_files(os.path.join(d, "%s.%d" % (o, p)),
                                     os.path.join(SCALE, case, "%s_%s.%d" % (variant, o, p)))
            assert err <= FP64_TOL, (o, p, err)
            worst = max(worst, err)
    return worst


def test_c1_full_transient_matches_reference(pkg, outs, tmp_path):
    d = str(tmp_path / "c1")
    sg.write_case_inputs("c1", d)
    with pkg.Solver(d, "A", 2) as s:
        s.run()
        s.write_outputs()
        info = s.info()
    assert info["steps"] == 120 and info["factorizations"] == 6 and info["n_edges"] == 201720
    _compare(outs, d, "c1", "A2", 1)


@pytest.mark.parametrize("variant", ["A3", "E3"])
def test_32_wires_as_one_block_match_reference(pkg, outs, tmp_path, variant):
    d = str(tmp_path / "w")
    sg.write_case_inputs("wires32", d)
    with pkg.Solver(d, variant[0], int(variant[1])) as s:
        s.run()
        s.write_outputs()
        assert s.info()["n_sources"] == 32
    _compare(outs, d, "wires32", variant, 32)


def test_solve_autotuner_measures_every_schedule(pkg, outs, tmp_path, monkeypatch):
    """The 32-column step solve is tuned on the first step: nine schedules (fused,
    panel or persistent fused solves, the columns in 1, 2 or 4 groups) are timed
    and the fastest kept;
    the transients stay within the FP64 tolerance of the reference whichever wins,
    and with the tuner off (fused, one group) as well."""
    d = str(tmp_path / "w")
    sg.write_case_inputs("wires32", d)
    with pkg.Solver(d, "A", 3) as s:
        s.run()
        s.write_outputs()
        info = s.info()
        log = s.tune_log()
    assert info["solve_candidates"] == 9 and info["solve_tuned_ms"] > 0
    assert len(log) == 9 and min(ms for _, _, ms in log) == pytest.approx(info["solve_tuned_ms"])
    assert info["solve_schedule"] in (0, 1, 2) and info["solve_split"] in (1, 2, 4)
    _compare(outs, d, "wires32", "A3", 32)
    monkeypatch.setenv("TDEM_SOLVE_AUTOTUNE", "0")
    d2 = str(tmp_path / "w2")
    sg.write_case_inputs("wires32", d2)
    with pkg.Solver(d2, "A", 3) as s:
        s.run()
        s.write_outputs()
        info = s.info()
    assert info["solve_candidates"] == 0 and info["solve_schedule"] == 0 and info["solve_split"] == 1
    _compare(outs, d2, "wires32", "A3", 32)


@pytest.mark.parametrize("schedule", ["0,1", "1,1", "2,1", "2,2", "2,4", "0,4"])
@pytest.mark.parametrize("variant", ["A3", "E3"])
def test_every_solve_schedule_matches_reference(pkg, outs, tmp_path, monkeypatch, schedule, variant):
    """Each schedule the autotuner chooses among, forced for the whole run."""
    monkeypatch.setenv("TDEM_SOLVE_SCHEDULE", schedule)
    d = str(tmp_path / "w")
    sg.write_case_inputs("wires32", d)
    with pkg.Solver(d, variant[0], int(variant[1])) as s:
        s.run()
        s.write_outputs()
        info = s.info()
    kind, split = (int(v) for v in schedule.split(","))
    assert info["solve_schedule"] == kind and info["solve_split"] == split
    _compare(outs, d, "wires32", variant, 32)


def test_persistent_schedule_is_bitwise_the_one_unit_per_cta_schedule(pkg, tmp_path, monkeypatch):
    """The persistent many-column kernels take the same products in the same order
    as the one-unit-per-CTA kernels: identical transients, bit for bit."""
    import numpy as np
    out = {}
    for sched in ("0,1", "2,1"):
        monkeypatch.setenv("TDEM_SOLVE_SCHEDULE", sched)
        d = str(tmp_path / sched.replace(",", "_"))
        sg.write_case_inputs("wires32", d)
        with pkg.Solver(d, "E", 3) as s:
            s.run()
            out[sched] = s.results()
    for a, b in zip(out["0,1"], out["2,1"]):
        assert np.array_equal(a, b)
