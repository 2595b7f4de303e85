"""Golden fixtures of receivers on element boundaries: the reference's own
CalcNonstat3DLine_{A2,A3,E2,E3} built from source by oracle/build_ref.sh, run on the
golden case cube8_block with its receivers replaced by points on mesh nodes, edges and
faces, some on the surface of the conductive block (x, y in [-30, 30] m, z in [-50, -20] m;
nodes at 0, +-20, +-40 m).

Several elements hold each such point; the reference takes the first in element order
(OutputResultant3d.cpp:572-712), and for field values that element's material decides
the smoothing subdomain (one per material).  The fixture stores the receiver files and
the reference's outputs.

    python tests/golden/make_nodes_golden.py
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
CASE = "cube8_receivers_on_nodes"
BASE = "cube8_block"
RECEIVERS = [
    (0.0, 20.0, 0.0),      # node on the surface
    (20.0, 0.0, -20.0),    # node on the block's top face
    (0.0, 30.0, 0.0),      # edge midpoint on the surface
    (10.0, 30.0, -20.0),   # face point on the block's top face
    (-20.0, -20.0, -40.0), # node inside the block
    (40.0, 10.0, -40.0),   # edge point outside the block
]
VARIANTS = ("A2", "A3", "E2", "E3")
OUTPUTS = ("eall_anom", "edsall_anom", "ball_anom")
FILES = ("xyzVectorB", "xyzVectorE", "recvsb", "recvse")


def write_receivers(path: str) -> None:
    for name in ("xyzVectorB", "xyzVectorE"):
        with open(os.path.join(path, name), "w") as f:
            f.write("%d\n" % len(RECEIVERS))
            f.write("".join("%f %f %f\n" % p for p in RECEIVERS))
    for name in ("recvsb", "recvse"):
        with open(os.path.join(path, name), "w") as f:
            f.write("%d\n" % len(RECEIVERS))


def write_case_inputs(path: str) -> None:
    """cube8_block's inputs with the stored receiver files of this case."""
    import make_golden
    make_golden.write_case_inputs(BASE, path)
    for name in FILES:
        shutil.copy2(os.path.join(HERE, CASE, name), os.path.join(path, name))


def main() -> None:
    import make_golden
    import run_ref
    out = os.path.join(HERE, CASE)
    os.makedirs(out, exist_ok=True)
    work = tempfile.mkdtemp(prefix="golden_nodes_")
    try:
        make_golden.write_case_inputs(BASE, work)
        write_receivers(work)
        for name in FILES:
            shutil.copy2(os.path.join(work, name), os.path.join(out, name))
        for v in VARIANTS:
            d = os.path.join(work, v)
            run_ref.copy_inputs(work, d)
            run_ref.run_transient(d, v)
            for o in OUTPUTS:
                shutil.copy2(os.path.join(d, "%s.1" % o), os.path.join(out, "%s_%s.1" % (v, o)))
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
