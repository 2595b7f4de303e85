"""Reader for the transient output files written by CalcNonstat3DLine
(edsall_anom.N, ball_anom.N, eall_anom.N; format of give_out_vec_loop.cpp:532-609):
per receiver a 6-line header (integer x y; x y z; "1"; "1 1 1 1"; "1"; column
titles) followed by one "t(ms) v1 v2 v3" row per printed time layer."""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def read_transients(path: str) -> List[Tuple[np.ndarray, np.ndarray]]:
    """Returns [(xyz, table)] per receiver; table is (layers, 4): t(ms), 3 components."""
    out = []
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        if lines[i].strip() == "":
            i += 1
            continue
        if i + 5 >= len(lines):
            break
        xyz = np.array([float(v) for v in lines[i + 1].split()])
        i += 6
        rows = []
        while i < len(lines):
            parts = lines[i].split()
            if len(parts) != 4:
                break
            try:
                rows.append([float(v) for v in parts])
            except ValueError:
                break
            i += 1
        out.append((xyz, np.array(rows)))
    return out


def peak_relative_error(a: np.ndarray, b: np.ndarray) -> float:
    """max_t |a - b| / max_t |b| for one transient (b is the reference)."""
    scale = float(np.max(np.abs(b)))
    if scale == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)


def compare_files(path_a: str, path_b: str, vector_scale: bool = True) -> float:
    """Largest per-receiver error between two output files.  With vector_scale
    the error of every component is measured against the peak magnitude of the
    receiver's whole vector transient, so components that vanish by symmetry are
    judged on the field's scale rather than on their own rounding noise."""
    A = read_transients(path_a)
    B = read_transients(path_b)
    if len(A) != len(B):
        raise ValueError("different receiver counts: %d vs %d" % (len(A), len(B)))
    worst = 0.0
    for (xa, ta), (xb, tb) in zip(A, B):
        if ta.shape != tb.shape:
            raise ValueError("different table shapes %s vs %s" % (ta.shape, tb.shape))
        if not np.allclose(ta[:, 0], tb[:, 0], rtol=1e-12, atol=0):
            raise ValueError("time columns differ")
        if vector_scale:
            scale = float(np.max(np.abs(tb[:, 1:])))
            err = float(np.max(np.abs(ta[:, 1:] - tb[:, 1:]))) / scale if scale > 0 else 0.0
        else:
            err = max(peak_relative_error(ta[:, c], tb[:, c]) for c in (1, 2, 3))
        worst = max(worst, err)
    return worst
