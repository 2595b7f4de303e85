"""Runs the reference's own executables built from source by oracle/build_ref.sh.

TEST INFRASTRUCTURE ONLY: used by tests/ (as the checker) and by bench.py's
reference / cpu_baseline arm (as the timed CPU implementation), never by the
product path.

  * CalcStat3D_3T_A (CODE/programs to folder Modules/CalcStat3D_3T_A): the
    grounded-wire stationary problem, writing v3a.dat / v3n.dat and a0.dat.  It
    opens its mesh files as "<path>\\name" (TaskSP.h:768-821) and writes
    "<path>\\a0.dat" (TaskSP.cpp:2166), so on Linux the run directory gets
    links named ".\\inftry.dat" etc. and the output is renamed afterwards.
  * CalcNonstat3DLine_{A2,A3,E2,E3}: the 3D transient for the four variants.

The pardiso_64 the binaries link is the oracle's CPU Cholesky
(oracle/pardiso_shim.cpp); TDEM_ORACLE_COORDS lets it order by the mesh
geometry and TDEM_ORACLE_BLAS points it at numpy's bundled OpenBLAS.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import time
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
VARIANTS = ("A2", "A3", "E2", "E3")


def binary(name: str) -> str:
    return os.path.join(REF_DIR, name)


def available(name: str = "CalcNonstat3DLine_A2") -> bool:
    return os.path.exists(binary(name))


def find_openblas() -> Optional[str]:
    try:
        import numpy
        base = os.path.dirname(os.path.dirname(numpy.__file__))
        for pat in ("numpy.libs/libscipy_openblas64_*.so", "scipy_openblas64/lib/libscipy_openblas64_*.so"):
            hits = sorted(glob.glob(os.path.join(base, pat)))
            if hits:
                return hits[0]
    except Exception:
        pass
    return None


def ref_env(threads: Optional[int] = None, coords: bool = True) -> dict:
    env = dict(os.environ)
    if coords:
        env["TDEM_ORACLE_COORDS"] = "1"
    blas = find_openblas()
    if blas:
        env["TDEM_ORACLE_BLAS"] = blas
    if threads:
        env["TDEM_ORACLE_THREADS"] = str(threads)
        env["OPENBLAS_NUM_THREADS"] = str(threads)
    return env


STAT_INPUTS = ("inftry.dat", "xyz.dat", "nver.dat", "nvkat.dat", "l13d.dat", "sig3d")


def run_stationary(workdir: str, threads: Optional[int] = None, timeout: float = 3600) -> float:
    """Writes v3a.dat, v3n.dat and a0.dat into workdir with the reference's
    CalcStat3D_3T_A.  Returns the wall time in seconds."""
    exe = binary("CalcStat3D_3T_A")
    if not os.path.exists(exe):
        raise RuntimeError("oracle/_ref/CalcStat3D_3T_A missing: run oracle/build_ref.sh")
    for name in STAT_INPUTS:
        link = os.path.join(workdir, ".\\" + name)
        if not os.path.lexists(link):
            os.symlink(name, link)
    open(os.path.join(workdir, "forA0"), "w").close()
    t0 = time.time()
    with open(os.path.join(workdir, "stat.log"), "w") as log:
        subprocess.run([exe], cwd=workdir, env=ref_env(threads), stdout=log, stderr=subprocess.STDOUT,
                       check=True, timeout=timeout)
    dt = time.time() - t0
    src = os.path.join(workdir, ".\\a0.dat")
    if os.path.exists(src):
        os.replace(src, os.path.join(workdir, "a0.dat"))
    for name in STAT_INPUTS:
        link = os.path.join(workdir, ".\\" + name)
        if os.path.islink(link):
            os.unlink(link)
    os.unlink(os.path.join(workdir, "forA0"))
    for needed in ("a0.dat", "v3a.dat"):
        if not os.path.exists(os.path.join(workdir, needed)):
            raise RuntimeError("CalcStat3D_3T_A did not write " + needed)
    return dt


def run_transient(workdir: str, variant: str, threads: Optional[int] = None, timeout: float = 3600) -> float:
    """Runs CalcNonstat3DLine_<variant> in workdir; returns the wall time in seconds."""
    if variant not in VARIANTS:
        raise ValueError(variant)
    exe = binary("CalcNonstat3DLine_" + variant)
    if not os.path.exists(exe):
        raise RuntimeError(exe + " missing: run oracle/build_ref.sh")
    t0 = time.time()
    with open(os.path.join(workdir, "ref_%s.log" % variant), "w") as log:
        subprocess.run([exe], cwd=workdir, env=ref_env(threads), stdout=log, stderr=subprocess.STDOUT,
                       check=True, timeout=timeout)
    return time.time() - t0


def copy_inputs(src: str, dst: str) -> None:
    """Copies a model directory without previous outputs."""
    os.makedirs(dst, exist_ok=True)
    for name in os.listdir(src):
        if name.startswith(("edsall_anom.", "ball_anom.", "eall_anom.", "v3.")) or name.endswith(".log"):
            continue
        p = os.path.join(src, name)
        if os.path.isfile(p) and not os.path.islink(p):
            shutil.copy2(p, os.path.join(dst, name))
