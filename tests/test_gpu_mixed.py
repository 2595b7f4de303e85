"""GPU tests of precision 32 (FP32 factorization preconditioning an FP64 conjugate
gradient) on a model whose system FP32 can factor: air of 0.01 S/m instead of 1e-8
keeps the condition number near 1e4.  Both trailing-update engines (CUDA cores and
tcgen05 3xTF32 tensor cores) must converge to the FP64 tolerance and reproduce the
FP64 direct solution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# converged to a 1e-10 relative residual per step: receivers agree with the FP64
# direct solve far below the 1e-5 acceptance level
MIXED_TOL = 1e-7


def peak_rel(a, b):
    worst = 0.0
    for i in range(b.shape[2]):
        sc = np.abs(b[:, :, i]).max()
        if sc > 0:
            worst = max(worst, np.abs(a[:, :, i] - b[:, :, i]).max() / sc)
    return worst


@pytest.fixture(scope="module")
def conductive_air_model(mg, tmp_path_factory):
    d = str(tmp_path_factory.mktemp("mixed"))
    spec = mg.small_model(cells=16, n_dec=3, steps_per_dec=5)
    spec.sigma_air = 0.01
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    return d


@pytest.mark.parametrize("form,scheme", [("A", 3), ("E", 2)])
def test_fp32_factor_engines_match_fp64(pkg, conductive_air_model, form, scheme):
    d = conductive_air_model
    with pkg.Solver(d, form, scheme) as s:
        s.run()
        ref = s.results()
    for engine in ("cuda_cores", "tensor_cores"):
        with pkg.Solver(d, form, scheme, precision=32, fp32_update=engine) as s:
            s.run()
            got = s.results()
            info = s.info()
        assert info["precision"] == 32
        assert info["refine_worst"] <= 1e-10
        assert 0 < info["refine_iters_max"] <= 30, info["refine_iters_max"]
        for k in range(3):
            if np.abs(ref[k]).max() > 0:
                assert peak_rel(got[k], ref[k]) <= MIXED_TOL, (engine, k, peak_rel(got[k], ref[k]))
