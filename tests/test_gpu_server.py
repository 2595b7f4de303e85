"""GPU tests of the serving loop (tdem_server_*): requests of different sizes,
formulations and schemes run concurrently under an HBM budget, and every result
is bitwise the same as the same model solved alone."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX = [  # (cells, formulation, scheme, n_sources)
    (8, "A", 2, 1),
    (12, "E", 3, 1),
    (10, "A", 3, 2),
    (14, "E", 2, 1),
    (9, "A", 2, 1),
    (11, "E", 3, 2),
]


@pytest.fixture(scope="module")
def mix_models(mg, tmp_path_factory):
    dirs = []
    for i, (cells, form, scheme, ns) in enumerate(MIX):
        d = str(tmp_path_factory.mktemp("req%d" % i))
        spec = mg.small_model(cells=cells, n_dec=2, steps_per_dec=5, n_sources=ns)
        mg.write_model(d, spec)
        mg.write_analytic_initial_field(d, spec)
        dirs.append(d)
    return dirs


def test_results_alone_and_in_the_mix_are_identical(pkg, mix_models):
    alone = []
    for d, (_, form, scheme, _) in zip(mix_models, MIX):
        with pkg.Solver(d, form, scheme) as s:
            s.run()
            alone.append(s.results())
    with pkg.Server(max_active=3, prep_threads=2) as srv:
        ids = [srv.submit(d, form, scheme) for d, (_, form, scheme, _) in zip(mix_models, MIX)]
        got = []
        for rid in ids:
            info = srv.wait(rid)
            got.append(srv.results(rid, info))
            assert info["steps"] > 0 and info["device_bytes"] > 0 and info["admit_s"] >= info["submit_s"]
        st = srv.stats()
    assert st["completed"] == len(MIX) and st["failed"] == 0
    assert st["peak_active"] >= 2
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0
    for a, b in zip(alone, got):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_admission_respects_the_budget(pkg, mix_models):
    """With a budget of one request at a time the requests still all finish, one by one."""
    with pkg.Server(max_active=4, hbm_budget_bytes=1) as srv:
        ids = [srv.submit(d, form, scheme) for d, (_, form, scheme, _) in zip(mix_models[:3], MIX[:3])]
        for rid in ids:
            srv.wait(rid)
        st = srv.stats()
    assert st["completed"] == 3 and st["peak_active"] == 1


def test_failed_request_does_not_stop_the_others(pkg, mix_models, tmp_path):
    bad = str(tmp_path / "empty")
    os.makedirs(bad)
    with pkg.Server(max_active=2) as srv:
        rb = srv.submit(bad, "A", 2)
        rg = srv.submit(mix_models[0], "A", 2)
        with pytest.raises(pkg.TdemError) as ei:
            srv.wait(rb)
        assert ei.value.status == 2
        srv.wait(rg)
        st = srv.stats()
    assert st["completed"] == 1 and st["failed"] == 1
