"""Synthetic input generator writes the reference's file formats consistently."""
import os

import numpy as np


def test_small_model_files(mg, tmp_path):
    spec = mg.small_model(cells=6)
    info = mg.write_model(str(tmp_path), spec)
    nx, ny, nz = len(spec.x), len(spec.y), len(spec.z)
    assert info["n_nodes"] == nx * ny * nz
    assert os.path.getsize(tmp_path / "xyz.dat") == 24 * info["n_nodes"]
    assert os.path.getsize(tmp_path / "nver.dat") == 56 * info["n_cells"]
    assert os.path.getsize(tmp_path / "edges.dat") == 100 * info["n_cells"]
    assert os.path.getsize(tmp_path / "nodesforedges.dat") == 8 * info["n_edges"]
    tok = open(tmp_path / "tsize3d_.dat").read().split()
    assert int(tok[1]) == info["n_edges"]


def test_edges_lexicographic_and_consistent(mg, tmp_path):
    spec = mg.small_model(cells=6)
    mg.write_model(str(tmp_path), spec)
    nfe = np.fromfile(tmp_path / "nodesforedges.dat", "<i4").reshape(-1, 2)
    # lexicographic order of (lower, upper) node pairs (RegularMeshBuilder BuildEdges)
    key = nfe[:, 0].astype(np.int64) * 10 ** 9 + nfe[:, 1]
    assert np.all(np.diff(key) > 0)
    nver = np.fromfile(tmp_path / "nver.dat", "<i4").reshape(-1, 14)[:, :8]
    ed = np.fromfile(tmp_path / "edges.dat", "<i4").reshape(-1, 25)[:, :12]
    # local edge -> local node pairs (T_Brick edge order)
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 2), (4, 6), (1, 3), (5, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
    for k, (a, b) in enumerate(pairs):
        assert np.all(nfe[ed[:, k] - 1, 0] == nver[:, a])
        assert np.all(nfe[ed[:, k] - 1, 1] == nver[:, b])


def test_time_grid_doubles_per_decade(mg):
    t = mg.decade_time_grid(1e-2, 6, 20)
    h = np.diff(t)
    assert len(t) == 121 and abs(t[-1] - 1e-2) < 1e-15
    for d in range(1, 6):
        assert abs(h[20 * d] / h[20 * d - 1] - 2.0) < 1e-9


def test_workload_sizes(mg):
    assert mg.halfspace_model().n_edges == 201720
    assert mg.layered_block_model().n_edges == 1574640
