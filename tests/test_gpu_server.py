"""GPU tests of the serving loop (tdem_server_*): requests of different sizes,
formulations and schemes run concurrently under an HBM budget, and every result
is bitwise the same as the same model solved alone; requests over one earth model
submitted with one batch key run as one multi-source block, each result within the
FP64 tolerance of its solo run."""
import os

import numpy as np
import pytest

from conftest import FP64_TOL

pytestmark = pytest.mark.gpu

MIX = [  # (cells, formulation, scheme, n_sources)
    (8, "A", 2, 1),
    (12, "E", 3, 1),
    (10, "A", 3, 2),
    (14, "E", 2, 1),
    (9, "A", 2, 1),
    (11, "E", 3, 2),
    (40, "A", 3, 1),
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


# transmitter positions of one survey over one earth model: (wires, receivers' y offset)
TX_POSITIONS = [
    ([((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0))], 0.0),
    ([((-30.0, 20.0, 0.0), (30.0, 20.0, 0.0))], 5.0),
    ([((-20.0, -20.0, 0.0), (40.0, -20.0, 0.0)), ((-30.0, 40.0, 0.0), (30.0, 40.0, 0.0))], 10.0),
    ([((0.0, -40.0, 0.0), (0.0, 20.0, 0.0))], 15.0),
]


@pytest.fixture(scope="module")
def survey_models(mg, tmp_path_factory):
    import dataclasses
    base = mg.small_model(cells=10, n_dec=2, steps_per_dec=5)
    dirs = []
    for i, (wires, dy) in enumerate(TX_POSITIONS):
        rec = [(0.0, 10.0 + dy + 25.0 * k, 0.0) for k in range(4 + i)]
        spec = dataclasses.replace(base, sources=wires, receivers_b=[rec] * len(wires),
                                   receivers_e=[rec] * len(wires))
        d = str(tmp_path_factory.mktemp("survey%d" % i))
        mg.write_model(d, spec)
        mg.write_analytic_initial_field(d, spec)
        dirs.append(d)
    return dirs


@pytest.mark.parametrize("form,scheme", [("A", 3), ("E", 2)])
def test_batched_requests_match_their_solo_runs(pkg, survey_models, form, scheme):
    """Four requests over one model (five sources, different receivers) submitted with
    one batch key: those queued together run as one n x k block per step; each gets its
    own receivers' values, equal to its solo run within the FP64 tolerance (the block
    solve adds in another order; measured up to 2.4e-10 of the peak)."""
    alone = []
    for d in survey_models:
        with pkg.Solver(d, form, scheme) as s:
            s.run()
            alone.append(s.results())
    with pkg.Server(max_active=2, prep_threads=1, batch_max=8) as srv:
        ids = [srv.submit(d, form, scheme, batch_key="survey") for d in survey_models]
        infos = [srv.wait(rid) for rid in ids]
        got = [srv.results(rid, info) for rid, info in zip(ids, infos)]
        st = srv.stats()
    assert st["completed"] == len(TX_POSITIONS) and st["failed"] == 0
    # the plan thread takes a request as soon as it is queued, with whatever of the
    # others is queued by then: at least one run solves two or more of them
    assert st["merged_runs"] >= 1 and st["merged_requests"] >= 2
    assert max(i["batch_size"] for i in infos) >= 2
    assert sum(1.0 / i["batch_size"] for i in infos) == pytest.approx(len(TX_POSITIONS) - st["merged_requests"]
                                                                       + st["merged_runs"])
    for info, (wires, _) in zip(infos, TX_POSITIONS):
        assert info["n_sources"] == len(wires)
    for a, b in zip(alone, got):
        for x, y in zip(a, b):  # (the E-form has no B table: zeros both ways)
            assert x.shape == y.shape
            assert np.abs(x - y).max() <= FP64_TOL * np.abs(x).max()


def test_batch_key_over_different_models_runs_them_one_by_one(pkg, mix_models, survey_models):
    """A batch key over models with different meshes: the server finds that they cannot be
    merged and runs them separately, with the results of their solo runs."""
    dirs = [mix_models[0], survey_models[0]]  # 8^3 and 10^3 cells
    alone = []
    for d in dirs:
        with pkg.Solver(d, "A", 2) as s:
            s.run()
            alone.append(s.results())
    with pkg.Server(max_active=2, prep_threads=1, batch_max=4) as srv:
        ids = [srv.submit(d, "A", 2, batch_key="same?") for d in dirs]
        got = [srv.results(rid, srv.wait(rid)) for rid in ids]
        st = srv.stats()
    assert st["completed"] == 2 and st["merged_runs"] == 0
    for a, b in zip(alone, got):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
