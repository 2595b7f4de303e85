"""Golden fixtures of the post-processing modules (SumNonstat3DOnly, SummatorEDMN),
made by running the reference's own programs compiled from source by
oracle/build_ref.sh (oracle/_ref/SumNonstat3DOnly, oracle/_ref/SummatorEDMN).

Inputs are seeded synthetic result files in the formats CalcNonstat3DLine writes
(ball_anom.N, edsall_anom.N, eall_anom.N) with the configuration files the two
modules read; the "chain" case instead feeds them the reference's own transients of
the golden case cube8_two_wires (three-point A-formulation).  Every case stores its
inputs under in/ and the reference's outputs under out/.

    python tests/golden/make_postprocess_golden.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
FIXTURES = os.path.join(HERE, "postprocess")

SPLIT_OUTPUTS = ("Bxall", "Byall", "Bzall", "Edsxall", "Edsyall", "Edsall", "Exall", "Eyall", "Ezall")
# the legends CalcNonstat3DLine writes (any text: the modules skip it)
LEG = {"ball_anom": "      t (ms)        Bx_anom (mTl)     By_anom (mTl)     Bz_anom (mTl)",
       "edsall_anom": "      t (ms)         Emfx_anom (mV)     Emfy_anom (mV)     Emfz_anom (mV)",
       "eall_anom": "      t (ms)         Ex_anom n (mV)     Ey_anom a (mV)     Ez_anom s (mV)"}

# the files the two modules read
MODULE_INPUTS = {"group", "timeintervalforprint", "infite.0", "xyzVectorB", "recvsb", "xyzVectorE", "recvse", "xyzmn"}
MODULE_INPUT_STEMS = ("ball_anom.", "edsall_anom.", "eall_anom.", "xyzmn", "xyzVectorElin")

# name -> synthetic case parameters (None: the chain case)
CASES = {
    # 2 transmitters; no B receivers for the second; 9 line points over 2 lines
    # (4 per line, one point left over); rows with exact and negative zeros
    "mixed": dict(seed=11, nb=(3, 0), ne=(8, 9), lines=(2, 2), nt=12, window=(3, 9), with_zeros=True,
                  cut_last_newline=False),
    # odd points per line (the ddV split point is 3 // 2 = 1); the x file of the
    # second transmitter ends without its final newline (its last row is not read)
    "odd_lines": dict(seed=12, nb=(2, 2), ne=(6, 9), lines=(2, 3), nt=10, window=(0, 10), with_zeros=False,
                      cut_last_newline=True),
    "chain": None,
}


def _fmt(v: float) -> str:
    return "%.16e" % v


def write_infite(path: str, t) -> None:
    lines = ["    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n" % (len(t), len(t)),
             "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n",
             "       u0=   0.00000e+000\n", " T I M E :\n"]
    for i in range(0, len(t), 5):
        lines.append("".join(" %.13e;" % v for v in t[i:i + 5]) + "\n")
    with open(os.path.join(path, "infite.0"), "w") as f:
        f.write("".join(lines))


def write_results(path: str, stem: str, p: int, pts, t_ms, vals) -> None:
    """One result file of transmitter p (1-based) in CalcNonstat3DLine's layout."""
    out = []
    for i, pt in enumerate(pts):
        out.append("%d %d\n%s %s %s\n1\n1 1 1 1\n1\n%s\n" % (int(pt[0]), int(pt[1]), _fmt(pt[0]), _fmt(pt[1]),
                                                             _fmt(pt[2]), LEG[stem]))
        for k, tk in enumerate(t_ms):
            out.append("%s\t%s\t%s\t%s\n" % (_fmt(tk), _fmt(vals[i, k, 0]), _fmt(vals[i, k, 1]), _fmt(vals[i, k, 2])))
    if not pts:
        out.append(" \n")
    with open(os.path.join(path, "%s.%d" % (stem, p)), "w") as f:
        f.write("".join(out))


def synth_case(path: str, seed: int, nb, ne, lines, nt, window, with_zeros, cut_last_newline) -> dict:
    """Writes the modules' inputs for len(nb) transmitters of one profile (number 1,
    places 0..); returns the summator calls [(with_ddv, profile, place), ...]."""
    rng = np.random.default_rng(seed)
    os.makedirs(path, exist_ok=True)
    npls = len(nb)
    t = np.concatenate([[0.0], np.cumsum(np.repeat([1e-6, 2e-6, 4e-6], (nt + 2) // 3)[:nt - 1])])
    write_infite(path, t)
    lo, hi = window
    with open(os.path.join(path, "timeintervalforprint"), "w") as f:
        f.write("%.13e %.13e\n" % (t[lo], t[hi - 1]))
    t_ms = [v * 1000.0 for v in t[lo:hi]]
    with open(os.path.join(path, "group"), "w") as f:
        f.write("1\n1 0 %d\n" % (npls - 1))

    def points(n):
        return [tuple(rng.uniform(-1500, 1500, 2)) + (float(rng.uniform(-20, 0)),) for _ in range(n)]

    def values(n):
        v = rng.standard_normal((n, len(t_ms), 3)) * 10.0 ** rng.integers(-9, 3, (n, len(t_ms), 3))
        if with_zeros and n:
            v[0, 0, :] = 0.0
            v[-1, -1, 1] = -0.0
        return v

    rb = [points(n) for n in nb]
    re = [points(n) for n in ne]
    with open(os.path.join(path, "xyzVectorB"), "w") as f:
        f.write("%d\n" % sum(nb) + "".join("%.6f %.6f %.6f\n" % p for lst in rb for p in lst))
    with open(os.path.join(path, "xyzVectorE"), "w") as f:
        f.write("%d\n" % sum(ne) + "".join("%.6f %.6f %.6f\n" % p for lst in re for p in lst))
    with open(os.path.join(path, "recvsb"), "w") as f:
        f.write("".join("%d\n" % n for n in nb))
    with open(os.path.join(path, "recvse"), "w") as f:
        f.write("".join("%d\n" % n for n in ne))
    for p in range(npls):
        write_results(path, "ball_anom", p + 1, rb[p], t_ms, values(nb[p]))
        write_results(path, "edsall_anom", p + 1, rb[p], t_ms, values(nb[p]))
        write_results(path, "eall_anom", p + 1, re[p], t_ms, values(ne[p]))
    calls = []
    with open(os.path.join(path, "xyzmn"), "w") as f:
        f.write("%d\n" % sum(lines))
    for p in range(npls):
        nl = lines[p]
        with open(os.path.join(path, "xyzmn%d_%d" % (p + 1, 1)), "w") as f:
            f.write("%d\n" % nl)
            for _ in range(nl):
                a = rng.uniform(-1000, 1000, 3)
                b = a + rng.uniform(-100, 100, 3)
                f.write(" ".join(_fmt(v) for v in list(a) + list(b)) + "\n")
        with open(os.path.join(path, "xyzVectorElin%d_%d" % (p + 1, 1)), "w") as f:
            f.write("%d\n" % ne[p] + "".join("%s %s %s\n" % tuple(_fmt(v) for v in q) for q in re[p]))
        calls += [(0, 1, p), (1, 1, p)]
    return {"calls": calls, "npls": npls, "cut_last_newline": cut_last_newline}


def chain_case(path: str) -> dict:
    """Inputs from the golden case cube8_two_wires and the reference's own A3
    transients; two-point lines over each transmitter's E receivers."""
    sys.path.insert(0, HERE)
    import make_golden
    make_golden.write_case_inputs("cube8_two_wires", path)
    src = os.path.join(HERE, "cube8_two_wires")
    for f in os.listdir(src):
        if f.startswith("A3_"):
            shutil.copy(os.path.join(src, f), os.path.join(path, f[3:]))
    with open(os.path.join(path, "recvse")) as f:
        ne = [int(v) for v in f.read().split()]
    with open(os.path.join(path, "xyzVectorE")) as f:
        tok = f.read().split()
    pts = np.array([float(v) for v in tok[1:]]).reshape(-1, 3)
    rng = np.random.default_rng(5)
    calls, k = [], 0
    with open(os.path.join(path, "xyzmn"), "w") as f:
        f.write("%d\n" % sum(n // 2 for n in ne))
    for p, n in enumerate(ne):
        own = pts[k:k + n]
        k += n
        nl = n // 2
        with open(os.path.join(path, "xyzmn%d_%d" % (p + 1, 1)), "w") as f:
            f.write("%d\n" % nl)
            for i in range(nl):
                a = own[2 * i] - rng.uniform(1, 10, 3)
                b = own[2 * i + 1] + rng.uniform(1, 10, 3)
                f.write(" ".join(_fmt(v) for v in list(a) + list(b)) + "\n")
        with open(os.path.join(path, "xyzVectorElin%d_%d" % (p + 1, 1)), "w") as f:
            f.write("%d\n" % (2 * nl) + "".join("%s %s %s\n" % tuple(_fmt(v) for v in q) for q in own[:2 * nl]))
        calls += [(0, 1, p), (1, 1, p)]
    return {"calls": calls, "npls": len(ne), "cut_last_newline": False}


def prepare_summator(path: str, npls: int, cut_last_newline: bool) -> None:
    """What the pipeline does between the two modules (GeoCalculatorSP.cpp:388 and
    2289-2310): the per-component E files of transmitter p become exall1_<p>.."""
    for p in range(npls):
        for c in ("x", "y", "z"):
            shutil.copy(os.path.join(path, "E%sall.%d" % (c, p + 1)), os.path.join(path, "e%sall1_%d" % (c, p)))
    if cut_last_newline and npls > 1:
        fn = os.path.join(path, "exall1_1")
        with open(fn, "rb") as f:
            data = f.read()
        with open(fn, "wb") as f:
            f.write(data.rstrip(b"\n"))


def summator_outputs(calls):
    names = []
    for ddv, prof, place in calls:
        names.append("edmnall%d_%d" % (prof, place))
        if ddv:
            names.append("edmoonall%d_%d" % (prof, place))
    return sorted(set(names))


def run_reference(path: str, meta: dict) -> None:
    """Runs the reference's SumNonstat3DOnly and SummatorEDMN in path.  SummatorEDMN
    joins its directory "." and file names with a backslash, which on Linux is part
    of the file name: its files are staged under those names and renamed back."""
    subprocess.run([os.path.join(REF_BIN, "SumNonstat3DOnly")], cwd=path, check=True, capture_output=True)
    prepare_summator(path, meta["npls"], meta["cut_last_newline"])
    for f in os.listdir(path):
        if f[:5] in ("exall", "eyall", "ezall"):
            shutil.copy(os.path.join(path, f), os.path.join(path, ".\\" + f))
    for ddv, prof, place in meta["calls"]:
        subprocess.run([os.path.join(REF_BIN, "SummatorEDMN"), str(ddv), str(prof), str(place)], cwd=path,
                       check=True, capture_output=True)
    for f in os.listdir(path):
        if f.startswith(".\\"):
            if f[2:].startswith(("edmnall", "edmoonall")):
                os.replace(os.path.join(path, f), os.path.join(path, f[2:]))
            else:
                os.unlink(os.path.join(path, f))


def make_case(name: str, path: str) -> dict:
    params = CASES[name]
    return chain_case(path) if params is None else synth_case(path, **params)


def main() -> None:
    for name in CASES:
        case = os.path.join(FIXTURES, name)
        shutil.rmtree(case, ignore_errors=True)
        os.makedirs(os.path.join(case, "in"))
        os.makedirs(os.path.join(case, "out"))
        with tempfile.TemporaryDirectory() as tmp:
            meta = make_case(name, tmp)
            inputs = {f for f in os.listdir(tmp) if f in MODULE_INPUTS or f.startswith(MODULE_INPUT_STEMS)}
            run_reference(tmp, meta)
            for f in sorted(inputs):
                shutil.copy(os.path.join(tmp, f), os.path.join(case, "in", f))
            outs = ["%s.%d" % (s, p + 1) for s in SPLIT_OUTPUTS for p in range(meta["npls"])]
            outs += summator_outputs(meta["calls"])
            for f in outs:
                shutil.copy(os.path.join(tmp, f), os.path.join(case, "out", f))
        print("wrote", case)


if __name__ == "__main__":
    main()
