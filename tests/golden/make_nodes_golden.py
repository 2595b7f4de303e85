"""Golden fixtures of receiver and material edge cases (the first case: receivers on
element boundaries; the others below: ragged per-source lists, no B receivers, a one-level
neighbourhood with a printed window inside the grid, a permeable block): the reference's own
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


# the second case: cube8_two_wires with ragged receiver lists per source (B: 2 and 5,
# E: 3 and 1), the per-source ranges of recvsb / recvse (TaskSP.cpp:467-516)
CASE_RAGGED = "cube8_two_wires_ragged"
BASE_RAGGED = "cube8_two_wires"
RAGGED_B = [[(0.0, 20.0, 0.0), (5.0, 45.0, 0.0)],
            [(0.0, 10.0, 0.0), (0.0, 30.0, 0.0), (-15.0, 60.0, 0.0), (25.0, 85.0, 0.0), (0.0, 110.0, 0.0)]]
RAGGED_E = [[(0.0, 10.0, 0.0), (10.0, 35.0, 0.0), (-5.0, 60.0, 0.0)], [(0.0, 40.0, 0.0)]]


def write_ragged_receivers(path: str) -> None:
    for xyz, cnt, lists in (("xyzVectorB", "recvsb", RAGGED_B), ("xyzVectorE", "recvse", RAGGED_E)):
        pts = [p for lst in lists for p in lst]
        with open(os.path.join(path, xyz), "w") as f:
            f.write("%d\n" % len(pts))
            f.write("".join("%f %f %f\n" % p for p in pts))
        with open(os.path.join(path, cnt), "w") as f:
            f.write("".join("%d\n" % len(lst) for lst in lists))


# the third case: cube6 without B receivers (xyzVectorB and recvsb hold 0); the reference
# then writes empty edsall_anom / ball_anom files
CASE_NO_B = "cube6_no_b_receivers"
BASE_NO_B = "cube6"


def write_no_b_receivers(path: str) -> None:
    for name in ("xyzVectorB", "recvsb"):
        with open(os.path.join(path, name), "w") as f:
            f.write("0\n")


# the fourth case: cube8_block with a one-level receiver neighbourhood (n_neib 1) and a
# printed window inside the grid (timeintervalforprint 2e-4 .. 4.2857e-4 s: from between
# two layers in the second step-size decade to that decade's last layer), so the output
# starts mid-decade and ends before the run does (give_out_vec_loop.cpp:52-73).  A window
# that ends inside a decade is not used: the reference then never projects that decade's
# receivers (OutputResultant3d.cpp:432-474 solves at the decade's last layer, which
# Work2 skips past the window, give_out_vec_loop.cpp:234) and prints zeros there.
CASE_WINDOW = "cube8_neib1_window"
BASE_WINDOW = "cube8_block"


def write_window(path: str) -> None:
    with open(os.path.join(path, "n_neib"), "w") as f:
        f.write("1\n")
    with open(os.path.join(path, "timeintervalforprint"), "w") as f:
        f.write("2.0000000000000e-04 4.2857142857143e-04\n")


# the fifth case: cube8_block with a permeable block (mu3d: relative permeability 20 for
# the block's material 4), so the curl-curl term B/mu varies between elements
# (T_Brick.cpp:142-310 with mu from mu3d, vec_prep_data.cpp:83-257)
CASE_MU = "cube8_permeable_block"
BASE_MU = "cube8_block"


def write_permeable(path: str) -> None:
    rows = [line.split() for line in open(os.path.join(path, "mu3d")) if line.strip()]
    with open(os.path.join(path, "mu3d"), "w") as f:
        for r in rows:
            mu = 20.0 if r[0] == "4" else float(r[1])
            f.write("%s\t%.7e\t%.7e\n" % (r[0], mu, mu))


BASES = {CASE: BASE, CASE_RAGGED: BASE_RAGGED, CASE_NO_B: BASE_NO_B, CASE_WINDOW: BASE_WINDOW, CASE_MU: BASE_MU}
CASE_FILES = {CASE: FILES, CASE_RAGGED: FILES, CASE_NO_B: FILES, CASE_WINDOW: ("n_neib", "timeintervalforprint"),
              CASE_MU: ("mu3d",)}


def write_case_inputs(path: str, case: str = CASE) -> None:
    """The base case's inputs with the stored files of `case`."""
    import make_golden
    make_golden.write_case_inputs(BASES[case], path)
    for name in CASE_FILES[case]:
        shutil.copy2(os.path.join(HERE, case, name), os.path.join(path, name))


def make_case(case: str, base: str, write, npls: int) -> None:
    import make_golden
    import run_ref
    out = os.path.join(HERE, case)
    os.makedirs(out, exist_ok=True)
    work = tempfile.mkdtemp(prefix="golden_nodes_")
    try:
        make_golden.write_case_inputs(base, work)
        write(work)
        for name in CASE_FILES[case]:
            shutil.copy2(os.path.join(work, name), os.path.join(out, name))
        for v in VARIANTS:
            d = os.path.join(work, v)
            run_ref.copy_inputs(work, d)
            run_ref.run_transient(d, v)
            for o in OUTPUTS:
                for p in range(1, npls + 1):
                    shutil.copy2(os.path.join(d, "%s.%d" % (o, p)), os.path.join(out, "%s_%s.%d" % (v, o, p)))
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main() -> None:
    make_case(CASE, BASE, write_receivers, 1)
    make_case(CASE_RAGGED, BASE_RAGGED, write_ragged_receivers, 2)
    make_case(CASE_NO_B, BASE_NO_B, write_no_b_receivers, 1)
    make_case(CASE_WINDOW, BASE_WINDOW, write_window, 1)
    make_case(CASE_MU, BASE_MU, write_permeable, 1)


if __name__ == "__main__":
    main()
