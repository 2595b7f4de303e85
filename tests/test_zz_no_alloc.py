"""GPU test of tdem_residual_norms_noalloc (static device scratch, no allocation),
called through the C-ABI and compared with tdem_residual_norms on the same data,
two calls in a row.  Kept in its own file, collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(n, per_row, ncols, seed):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), per_row)
    a = sp.coo_matrix((rng.standard_normal(n * per_row), (rows, rng.integers(0, n, n * per_row))), shape=(n, n))
    a = (a + a.T + sp.identity(n) * 2.0 * per_row).tocsr()
    a.sort_indices()
    x = rng.standard_normal((ncols, n))
    b = rng.standard_normal((ncols, n))
    return a, x, b


def _bind(lib, name):
    f = getattr(lib, name)
    P = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P, P, P, ctypes.c_int64, ctypes.c_int, P, P]
    f.restype = ctypes.c_int
    return f


def test_noalloc_matches_allocating_entry_point_twice(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    ref_fn, na_fn = _bind(lib, "tdem_residual_norms"), _bind(lib, "tdem_residual_norms_noalloc")
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    # the last case stores its columns with a leading dimension larger than n
    for n, per_row, ncols, seed, pad in ((30_000, 12, 64, 1, 0), (5_000, 5, 7, 2, 0), (4_000, 6, 5, 3, 37)):
        a, x, b = _system(n, per_row, ncols, seed)
        ld = n + pad
        xp = np.zeros((ncols, ld))
        bp = np.full((ncols, ld), 1e300)  # padding rows must not be read
        xp[:, :n], bp[:, :n] = x, b
        rp = torch.from_numpy(a.indptr.astype(np.int64)).to(dev)
        ci = torch.from_numpy(a.indices.astype(np.int32)).to(dev)
        va = torch.from_numpy(a.data).to(dev)
        xd = torch.from_numpy(xp).to(dev)
        bd = torch.from_numpy(bp).to(dev)
        args = (0, n, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), xd.data_ptr(), bd.data_ptr(), ld, ncols)
        ref = torch.zeros(2 * ncols, dtype=torch.float64, device=dev)
        assert ref_fn(*args, ref.data_ptr(), stream) == 0
        for _ in range(2):
            out = torch.full((2 * ncols,), -1.0, dtype=torch.float64, device=dev)
            assert na_fn(*args, out.data_ptr(), stream) == 0
            torch.cuda.synchronize()
            assert np.allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-14, atol=0)


def test_noalloc_rejects_more_columns_than_its_scratch(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    na_fn = _bind(lib, "tdem_residual_norms_noalloc")
    one = torch.ones(4, dtype=torch.float64, device="cuda:0")
    rp = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    ci = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(130, dtype=torch.float64, device="cuda:0")
    assert na_fn(0, 1, rp.data_ptr(), ci.data_ptr(), one.data_ptr(), one.data_ptr(), one.data_ptr(), 1, 65,
                 out.data_ptr(), None) == 1
