"""Size-independent properties at the 40^3 workload size (the oracle would take
minutes there): linearity in the initial field and multi-source consistency."""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_linearity_in_initial_field_40cubed(pkg, mg, tmp_path):
    spec = mg.halfspace_model(n_dec=3, steps_per_dec=10, t_end=2e-3)
    d1, d2 = str(tmp_path / "a"), str(tmp_path / "b")
    for d in (d1, d2):
        mg.write_model(d, spec)
        mg.write_analytic_initial_field(d, spec)
    a0 = np.fromfile(os.path.join(d2, "a0.dat"), "<f8")
    (3.0 * a0).tofile(os.path.join(d2, "a0.dat"))
    with pkg.Solver(d1, "A", 2) as s:
        s.run()
        e1, m1, b1 = s.results()
    with pkg.Solver(d2, "A", 2) as s:
        s.run()
        e3, m3, b3 = s.results()
    for x, y in ((e1, e3), (m1, m3), (b1, b3)):
        assert np.abs(3.0 * x - y).max() <= 1e-9 * np.abs(y).max()


def test_two_sources_match_single_source_runs(pkg, mg, tmp_path):
    w1 = ((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0))
    w2 = ((-30.0, 40.0, 0.0), (30.0, 40.0, 0.0))
    base = mg.small_model(cells=12, n_dec=2, steps_per_dec=6, n_receivers=4)
    rec = base.receivers_b[0]
    both = mg.small_model(cells=12, n_dec=2, steps_per_dec=6, n_receivers=4)
    both.sources = [w1, w2]
    both.receivers_b = [rec, rec]
    both.receivers_e = [rec, rec]
    d = str(tmp_path / "both")
    mg.write_model(d, both)
    mg.write_analytic_initial_field(d, both)
    with pkg.Solver(d, "E", 3) as s:
        s.run()
        eb, mb, _ = s.results()
    nr = len(rec)
    for k, w in enumerate((w1, w2)):
        one = mg.small_model(cells=12, n_dec=2, steps_per_dec=6, n_receivers=4)
        one.sources = [w]
        dd = str(tmp_path / ("one%d" % k))
        mg.write_model(dd, one)
        mg.write_analytic_initial_field(dd, one)
        with pkg.Solver(dd, "E", 3) as s:
            s.run()
            e1, m1, _ = s.results()
        assert np.abs(eb[:, :, k * nr:(k + 1) * nr] - e1).max() <= 1e-9 * np.abs(e1).max()
        assert np.abs(mb[:, :, k * nr:(k + 1) * nr] - m1).max() <= 1e-9 * np.abs(m1).max()
