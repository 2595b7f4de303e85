"""GPU tests of tdem_residual_norms against numpy FP64 on the host."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def random_system(n, per_row, ncols, seed):
    """Symmetric full-CSR matrix with `per_row` random off-diagonals per row plus
    the diagonal, and random x, b (column-major, ld = n + 3)."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), per_row)
    cols = rng.integers(0, n, size=n * per_row)
    vals = rng.standard_normal(n * per_row)
    import scipy.sparse as sp
    a = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    a = (a + a.T + sp.diags(rng.uniform(1.0, 2.0, n) * per_row)).tocsr()
    a.sort_indices()
    ld = n + 3
    x = rng.standard_normal((ncols, ld))
    b = rng.standard_normal((ncols, ld))
    return a, x, b, ld


def host_norms(a, x, b, n, ncols):
    out = np.empty(2 * ncols)
    for j in range(ncols):
        r = b[j, :n] - a @ x[j, :n]
        out[2 * j] = np.linalg.norm(r)
        out[2 * j + 1] = np.linalg.norm(b[j, :n])
    return out


def device_args(a, x, b):
    dev = torch.device("cuda:0")
    rp = torch.from_numpy(a.indptr.astype(np.int64)).to(dev)
    ci = torch.from_numpy(a.indices.astype(np.int32)).to(dev)
    va = torch.from_numpy(a.data.astype(np.float64)).to(dev)
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    bd = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    return rp, ci, va, xd, bd


@pytest.mark.parametrize("n,per_row,ncols", [(1, 1, 1), (1000, 7, 3), (50_000, 16, 33), (20_000, 31, 64)])
def test_matches_numpy_and_repeats_bitwise(pkg, n, per_row, ncols):
    a, x, b, ld = random_system(n, per_row, ncols, seed=n + ncols)
    rp, ci, va, xd, bd = device_args(a, x, b)
    norms = torch.zeros(2 * ncols, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    pkg.residual_norms(0, n, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), xd.data_ptr(), bd.data_ptr(), ld,
                       ncols, norms.data_ptr(), stream)
    first = norms.cpu().numpy().copy()
    ref = host_norms(a, x, b, n, ncols)
    assert np.allclose(first, ref, rtol=1e-12, atol=0)
    pkg.residual_norms(0, n, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), xd.data_ptr(), bd.data_ptr(), ld,
                       ncols, norms.data_ptr(), stream)
    assert np.array_equal(norms.cpu().numpy(), first)


def test_exact_solution_has_zero_residual(pkg):
    a, x, _, ld = random_system(4096, 9, 5, seed=3)
    b = np.zeros_like(x)
    for j in range(5):
        b[j, :4096] = a @ x[j, :4096]
    rp, ci, va, xd, bd = device_args(a, x, b)
    norms = torch.zeros(10, dtype=torch.float64, device="cuda:0")
    pkg.residual_norms(0, 4096, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), xd.data_ptr(), bd.data_ptr(), ld, 5,
                       norms.data_ptr(), torch.cuda.current_stream().cuda_stream)
    v = norms.cpu().numpy()
    assert np.all(v[0::2] <= 1e-13 * v[1::2])


def test_bad_arguments_are_rejected(pkg):
    lib = pkg.load_library()
    norms = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    rp = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    one = torch.ones(1, dtype=torch.float64, device="cuda:0")
    ci = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    args = dict(rowptr=rp.data_ptr(), col=ci.data_ptr(), val=one.data_ptr(), x=one.data_ptr(), b=one.data_ptr())
    call = lambda n, ld, ncols, **kw: lib.tdem_residual_norms(0, n, kw["rowptr"], kw["col"], kw["val"], kw["x"],
                                                               kw["b"], ld, ncols, norms.data_ptr(), None)
    assert call(1, 1, 0, **args) == 1
    assert call(1, 1, 65, **args) == 1
    assert call(1, 0, 1, **args) == 1
    assert call(-1, 1, 1, **args) == 1
    assert call(1, 1, 1, **dict(args, x=None)) == 1
    assert call(1, 1, 1, **args) == 0
    torch.cuda.synchronize()
