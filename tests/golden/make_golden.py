"""Generates the golden fixtures under tests/golden/ by running the reference's
own programs, compiled from source by oracle/build_ref.sh (oracle/_ref):
CalcStat3D_3T_A for the grounded-wire initial field (a0.dat, v3a.dat) and
CalcNonstat3DLine_{A2,A3,E2,E3} for the transients.

Each case directory holds the stationary outputs and, per variant, the three
output files; the remaining inputs are regenerated deterministically from
CASES by the package's model generator.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib
import json
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
PKG = "a-e_formulations_3d_timedomain_em_horizontalgroundedwiresource_b200"

# name -> keyword arguments of modelgen.small_model
CASES = {
    "cube6": dict(cells=6, n_dec=2, steps_per_dec=5, block=False, n_receivers=3),
    "cube8_block": dict(cells=8, n_dec=3, steps_per_dec=6, block=True, n_receivers=5),
    "cube8_two_wires": dict(cells=8, n_dec=2, steps_per_dec=6, block=True, n_sources=2, n_receivers=4),
}
VARIANTS = ("A2", "A3", "E2", "E3")
OUTPUTS = ("eall_anom", "edsall_anom", "ball_anom")


def write_case_inputs(name: str, path: str) -> None:
    """Model inputs of a golden case plus its stored stationary field."""
    mg = importlib.import_module(PKG + ".modelgen")
    spec = mg.small_model(**CASES[name])
    mg.write_model(path, spec)
    for f in ("a0.dat", "v3a.dat", "v3n.dat"):
        shutil.copy2(os.path.join(HERE, name, f), os.path.join(path, f))


def main() -> None:
    import run_ref
    mg = importlib.import_module(PKG + ".modelgen")
    manifest = {}
    for name, kw in CASES.items():
        out = os.path.join(HERE, name)
        os.makedirs(out, exist_ok=True)
        work = tempfile.mkdtemp(prefix="golden_")
        try:
            spec = mg.small_model(**kw)
            mg.write_model(work, spec)
            run_ref.run_stationary(work)
            for f in ("a0.dat", "v3a.dat", "v3n.dat"):
                shutil.copy2(os.path.join(work, f), os.path.join(out, f))
            npls = len(spec.sources)
            for v in VARIANTS:
                d = os.path.join(work, v)
                run_ref.copy_inputs(work, d)
                run_ref.run_transient(d, v)
                for o in OUTPUTS:
                    for p in range(npls):
                        shutil.copy2(os.path.join(d, "%s.%d" % (o, p + 1)), os.path.join(out, "%s_%s.%d" % (v, o, p + 1)))
            manifest[name] = dict(kw, n_sources=npls)
        finally:
            shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"cases": manifest, "variants": VARIANTS, "outputs": OUTPUTS,
                   "generator": "reference CalcStat3D_3T_A + CalcNonstat3DLine_{A2,A3,E2,E3} built "
                                "from source by oracle/build_ref.sh"}, f, indent=1)


if __name__ == "__main__":
    main()
