"""Golden fixtures of a grounded wire that runs past the edge of the mesh: the
reference's own CalcNonstat3DLine_{A2,A3,E2,E3} built from source by
oracle/build_ref.sh, run on the golden case cube6 (x, y in [-1000, 1000] m) with
its wire replaced by one from x = 600 m to x = 1400 m at y = z = 0.

No element holds the dipoles beyond x = 1000 m, so the reference places each in the
nearest element (Vec_Prep_Data::GetNearestElement, vec_prep_data.cpp:878-980) with
local coordinates outside [0, 1].  The initial field is cube6's stored stationary
field (the reference's CalcStat3D_3T_A needs its electrodes inside the mesh); the
transient only reads it as the field at the first time layer.

The fixture stores the `sours` file and the reference's outputs.

    python tests/golden/make_beyond_golden.py
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
CASE = "cube6_wire_beyond"
BASE = "cube6"
WIRE = (600.0, 0.0, 0.0, 1400.0, 0.0, 0.0)
VARIANTS = ("A2", "A3", "E2", "E3")
OUTPUTS = ("eall_anom", "edsall_anom", "ball_anom")


def write_sours(path: str) -> None:
    with open(os.path.join(path, "sours"), "w") as f:
        f.write("%f %f %f\n%f %f %f\n" % WIRE)


# the second case: cube6's own wire with a current that ramps down over four layers with
# an undershoot (1, 0.7, 0.3, -0.1, 0.05, then 0) instead of stepping off: the A-form
# source J(t) acts on several layers and the E-form source -dJ/dt is a difference of
# them (time_approx.cpp:1039-1076, E2/time_approx.cpp:1057-1105)
CASE_RAMP = "cube6_ramp_current"
RAMP = (1.0, 0.7, 0.3, -0.1, 0.05)


def write_ramp(path: str) -> None:
    rows = [line.split() for line in open(os.path.join(path, "currentfunction")) if line.strip()]
    with open(os.path.join(path, "currentfunction"), "w") as f:
        for i, r in enumerate(rows):
            f.write("%s\t%.13e\n" % (r[0], RAMP[i] if i < len(RAMP) else 0.0))


CASE_FILES = {CASE: ("sours",), CASE_RAMP: ("currentfunction",)}


def write_case_inputs(path: str, case: str = CASE) -> None:
    """cube6's inputs with the stored files of `case`."""
    import make_golden
    make_golden.write_case_inputs(BASE, path)
    for name in CASE_FILES[case]:
        shutil.copy2(os.path.join(HERE, case, name), os.path.join(path, name))


def main() -> None:
    make_case(CASE, write_sours)
    make_case(CASE_RAMP, write_ramp)


def make_case(case: str, write) -> None:
    import make_golden
    import run_ref
    out = os.path.join(HERE, case)
    os.makedirs(out, exist_ok=True)
    work = tempfile.mkdtemp(prefix="golden_beyond_")
    try:
        make_golden.write_case_inputs(BASE, work)
        write(work)
        for name in CASE_FILES[case]:
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
