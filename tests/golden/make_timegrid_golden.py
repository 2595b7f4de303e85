"""Golden fixtures of the time-grid modules (TimeDirectSolver, CorrectTimeMesh),
made by running the reference's own programs compiled from source by
oracle/build_ref.sh (oracle/_ref/TimeDirectSolver, oracle/_ref/CorrectTimeMesh).

Each case holds the inputs (tcff, infite.0, currentfunction, deltafunction) under
in/, and under out/ every file of the directory after TimeDirectSolver and then
CorrectTimeMesh ran in it, as the pipeline runs them (GeoCalculatorSP.cpp:2111-2126);
the "correct_only" case runs CorrectTimeMesh alone on a grid with a short decade.

    python tests/golden/make_timegrid_golden.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
FIXTURES = os.path.join(HERE, "timegrid")
INPUTS = ("tcff", "infite.0", "currentfunction", "deltafunction")
OUTPUTS = INPUTS[1:] + tuple("!" + f for f in INPUTS[1:]) + tuple("!!" + f for f in INPUTS[1:])


def write_infite(path: str, t, fmt: str = " %.13e;") -> None:
    lines = ["    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n" % (len(t), len(t)),
             "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n",
             "       u0=   0.00000e+000\n", " T I M E :\n"]
    for i in range(0, len(t), 5):
        lines.append("".join(fmt % v for v in t[i:i + 5]) + "\n")
    with open(os.path.join(path, "infite.0"), "w") as f:
        f.write("".join(lines))


def grid_case(path: str, times, tcff: float, seed: int) -> None:
    """A time list with the files the modules read: the step-off source function
    and a seeded delta-function table on its own times."""
    rng = np.random.default_rng(seed)
    os.makedirs(path, exist_ok=True)
    t = np.asarray(times, dtype=float)
    write_infite(path, t)
    with open(os.path.join(path, "tcff"), "w") as f:
        f.write("%g\n" % tcff)
    with open(os.path.join(path, "currentfunction"), "w") as f:
        f.write("".join("%.13e\t%.13e\n" % (v, 1.0 if i == 0 else 0.0) for i, v in enumerate(t)))
    td = np.sort(np.concatenate([[t[0]], rng.uniform(t[0], t[-1] * 1.2, 7)]))
    with open(os.path.join(path, "deltafunction"), "w") as f:
        f.write("%.6f\n%d\n" % (rng.uniform(1, 100), len(td)))
        f.write("".join("%.13e %.13e\n" % (a, b) for a, b in zip(td, rng.standard_normal(len(td)))))


def log_times(n, t_end, t_first):
    return np.concatenate([[0.0], np.geomspace(t_first, t_end, n)])


def short_decade_times():
    """Three decades of steps; the third has too few times for its step (it is
    refilled with the second decade's step)."""
    t = [0.0]
    for h, n in ((1e-6, 10), (2e-6, 10), (4e-6, 2), (8e-6, 6)):
        for _ in range(n):
            t.append(t[-1] + h)
    return np.array(t)


# name -> (times, tcff, seed, run TimeDirectSolver first)
CASES = {
    "log60": (log_times(60, 1e-1, 1e-6), 2.0, 1, True),
    "log200_tcff1.5": (log_times(200, 1.0, 1e-7), 1.5, 2, True),
    "jitter": (np.cumsum(np.concatenate([[0.0], np.random.default_rng(3).uniform(0.5, 1.5, 40) *
                                          np.repeat([1e-5, 3e-5, 1e-4, 4e-4], 10)])), 2.0, 3, True),
    "correct_only": (short_decade_times(), 2.0, 4, False),
}


def make_case(name: str, path: str) -> bool:
    times, tcff, seed, direct = CASES[name]
    grid_case(path, times, tcff, seed)
    return direct


def run_reference(path: str, direct: bool) -> None:
    if direct:
        subprocess.run([os.path.join(REF_BIN, "TimeDirectSolver")], cwd=path, check=True, capture_output=True)
    subprocess.run([os.path.join(REF_BIN, "CorrectTimeMesh")], cwd=path, check=True, capture_output=True)
    for f in os.listdir(path):
        if f.startswith("logfile"):
            os.unlink(os.path.join(path, f))


def main() -> None:
    for name in CASES:
        case = os.path.join(FIXTURES, name)
        shutil.rmtree(case, ignore_errors=True)
        os.makedirs(os.path.join(case, "in"))
        os.makedirs(os.path.join(case, "out"))
        with tempfile.TemporaryDirectory() as tmp:
            direct = make_case(name, tmp)
            for f in INPUTS:
                shutil.copy(os.path.join(tmp, f), os.path.join(case, "in", f))
            run_reference(tmp, direct)
            for f in OUTPUTS:
                if os.path.exists(os.path.join(tmp, f)):
                    shutil.copy(os.path.join(tmp, f), os.path.join(case, "out", f))
        print("wrote", case, sorted(os.listdir(os.path.join(case, "out"))))


if __name__ == "__main__":
    main()
