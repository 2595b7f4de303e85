"""Golden fixtures of the primary-secondary mode (fdirect = 0 with a normal field):
the reference's own CalcNonstat3DLine_{A2,A3,E2,E3} built from source by
oracle/build_ref.sh, run on the golden case cube8_block turned into a
primary-secondary problem:

* sig3d gives the block a normal conductivity sigma0 equal to the half-space's, so
  the block is the anomaly (sigma - sigma0 = 0.09 S/m);
* mtrsizeforE0 flags the edges of the anomalous elements;
* the normal field of every time layer (itime >= 1) is a seeded smooth field,
  written as the float32 files m<PName>.enor.NNNN that the reference maps as named
  shared memory (the oracle build maps files of those names).

The fixture stores the files that differ from cube8_block's inputs and the
reference's outputs.

    python tests/golden/make_ps_golden.py
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
CASE = "cube8_block_ps"
BASE = "cube8_block"
PNAME = "tdemps"
VARIANTS = ("A2", "A3", "E2", "E3")
OUTPUTS = ("eall_anom", "edsall_anom", "ball_anom")


def _time_count(d: str) -> int:
    with open(os.path.join(d, "infite.0")) as f:
        head = f.read().split("=", 1)[1]
    return int(head.split(";")[0])


def make_primary_secondary(d: str, seed: int = 7, anomaly=None) -> None:
    """Turns the direct-mode model in d into the primary-secondary problem above; with
    `anomaly` the run is one anomaly of several (AnomalType 1, ia = anomaly, files
    suffixed _<ia>)."""
    rows = [line.split() for line in open(os.path.join(d, "sig3d")) if line.strip()]
    sig = np.array([float(r[1]) for r in rows])
    background = 0.01  # the half-space of small_model
    sig0 = np.where(sig > 1e-6, background, sig)
    with open(os.path.join(d, "sig3d"), "w") as f:
        f.write("".join("%s\t%.7e\t%.7e\n" % (r[0], s, s0) for r, s, s0 in zip(rows, sig, sig0)))
    with open(os.path.join(d, "fdirect"), "w") as f:
        f.write("0\n")
    with open(os.path.join(d, "PName"), "w") as f:
        f.write(PNAME + "\n")
    mat = np.fromfile(os.path.join(d, "nvkat.dat"), dtype="<i4")
    ed = np.fromfile(os.path.join(d, "edges.dat"), dtype="<i4").reshape(len(mat), 25)[:, :12] - 1
    ne = int(np.fromfile(os.path.join(d, "nodesforedges.dat"), dtype="<i4").size // 2)
    anom_mat = np.abs(sig - sig0) > 0
    flag = np.zeros(ne, dtype=np.int64)
    flag[np.unique(ed[anom_mat[mat - 1]])] = 1
    with open(os.path.join(d, "mtrsizeforE0"), "w") as f:
        f.write("".join("%d\n" % v for v in flag))
    # normal field per time layer: a smooth pattern over the anomalous edges, decaying in time
    npls = sum(1 for line in open(os.path.join(d, "recvsb")) if line.strip())
    idx = np.nonzero(flag)[0]
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.5, 2.0, (npls, 3))
    t = _infite_times(d)
    suffix = "" if anomaly is None else "_%d" % anomaly
    if anomaly is not None:
        for name, v in (("AnomalType", 1), ("ia", anomaly)):
            with open(os.path.join(d, name), "w") as f:
                f.write("%d\n" % v)
    for it in range(1, len(t)):
        vals = np.stack([np.cos(k[p, 0] * idx / len(idx) * 6.0 + k[p, 1]) * np.exp(-t[it] / (2e-4 * k[p, 2]))
                         for p in range(npls)]) * 1e-3
        vals.astype("<f4").tofile(os.path.join(d, "m%s.enor.%04d%s" % (PNAME, it, suffix)))


def _infite_times(d: str):
    with open(os.path.join(d, "infite.0")) as f:
        txt = f.read()
    n = _time_count(d)
    body = txt.split("T I M E :", 1)[1].replace(";", " ").split()
    return np.array([float(v) for v in body[:n]])


def ps_files(d: str):
    extra = [f for f in ("AnomalType", "ia") if os.path.exists(os.path.join(d, f))]
    return ["sig3d", "fdirect", "PName", "mtrsizeforE0"] + extra + sorted(
        f for f in os.listdir(d) if f.startswith("m" + PNAME))


def write_case_inputs(path: str, case: str = CASE) -> None:
    """cube8_block's inputs with the stored primary-secondary files of `case`."""
    import make_golden
    make_golden.write_case_inputs(BASE, path)
    src = os.path.join(HERE, case)
    for f in os.listdir(src):
        if not f.startswith(VARIANTS):
            shutil.copy2(os.path.join(src, f), os.path.join(path, f))


# the second case: one anomaly of several (file suffix _2), A2 and E3 only
CASE_IA = "cube8_block_ps_ia"
ANOMALY = 2
VARIANTS_IA = ("A2", "E3")


def main() -> None:
    for case, anomaly, variants in ((CASE, None, VARIANTS), (CASE_IA, ANOMALY, VARIANTS_IA)):
        make_case(case, anomaly, variants)


def make_case(case, anomaly, variants) -> None:
    import make_golden
    import run_ref
    out = os.path.join(HERE, case)
    shutil.rmtree(out, ignore_errors=True)
    os.makedirs(out)
    work = tempfile.mkdtemp(prefix="golden_ps_")
    try:
        make_golden.write_case_inputs(BASE, work)
        make_primary_secondary(work, anomaly=anomaly)
        for f in ps_files(work):
            shutil.copy2(os.path.join(work, f), os.path.join(out, f))
        for v in variants:
            d = os.path.join(work, v)
            run_ref.copy_inputs(work, d)
            run_ref.run_transient(d, v)
            for o in OUTPUTS:
                shutil.copy2(os.path.join(d, "%s.1" % o), os.path.join(out, "%s_%s.1" % (v, o)))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    print("wrote", out, sorted(os.listdir(out))[:8], len(os.listdir(out)))


if __name__ == "__main__":
    main()
