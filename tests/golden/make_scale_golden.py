"""Generates the golden fixtures of the larger cases under tests/golden/scale/ by
running the reference's own CalcNonstat3DLine, compiled
from source by oracle/build_ref.sh (oracle/_ref):

  * c1_A2: the 40^3 half-space of the plain-method configuration (0.01 S/m under
    air of 1e-8 S/m, 100 m wire, 21 receivers on the y axis), A-formulation,
    two-point scheme, the full 120-step grid (6 doubling decades of 20 steps); the
    analytic initial field of modelgen.write_analytic_initial_field.
  * wires32_{A3,E3}: a 12^3 block model with 32 wires (centres on a 4 x 8 grid, 20 m
    apart), solved by the reference as one npls = 32 right-hand-side block per step
    (time_approx.cpp:1087 solve_nrhs); the analytic initial field of each wire.

Only the outputs are stored; the inputs are regenerated deterministically by the
package's model generator (write_case_inputs).

    python tests/golden/make_scale_golden.py
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
OUT = os.path.join(HERE, "scale")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
PKG = "a-e_formulations_3d_timedomain_em_horizontalgroundedwiresource_b200"
OUTPUTS = ("eall_anom", "edsall_anom", "ball_anom")
CASES = {"c1": ("A2",), "wires32": ("A3", "E3")}


def wire_grid(nx=4, ny=8, spacing=20.0, half=15.0):
    out = []
    for j in range(ny):
        for i in range(nx):
            cx = (i - (nx - 1) / 2.0) * spacing
            cy = (j - (ny - 1) / 2.0) * spacing
            out.append(((cx - half, cy, 0.0), (cx + half, cy, 0.0)))
    return out


def case_spec(name: str):
    mg = importlib.import_module(PKG + ".modelgen")
    if name == "c1":
        return mg.halfspace_model()
    if name == "wires32":
        spec = mg.small_model(cells=12, n_dec=2, steps_per_dec=6, block=True, n_receivers=4)
        srcs = wire_grid()
        rec = spec.receivers_b[0]
        spec.sources = srcs
        spec.receivers_b = [rec] * len(srcs)
        spec.receivers_e = [rec] * len(srcs)
        return spec
    raise ValueError(name)


def write_case_inputs(name: str, path: str) -> None:
    """Model inputs of a case, initial field included."""
    mg = importlib.import_module(PKG + ".modelgen")
    spec = case_spec(name)
    mg.write_model(path, spec)
    mg.write_analytic_initial_field(path, spec)


def main() -> None:
    import run_ref
    mg = importlib.import_module(PKG + ".modelgen")
    manifest = {}
    for name, variants in CASES.items():
        out = os.path.join(OUT, name)
        os.makedirs(out, exist_ok=True)
        work = tempfile.mkdtemp(prefix="golden_scale_")
        try:
            spec = case_spec(name)
            mg.write_model(work, spec)
            mg.write_analytic_initial_field(work, spec)
            npls = len(spec.sources)
            walls = {}
            for v in variants:
                d = os.path.join(work, v)
                run_ref.copy_inputs(work, d)
                walls[v] = run_ref.run_transient(d, v)
                for o in OUTPUTS:
                    for p in range(npls):
                        shutil.copy2(os.path.join(d, "%s.%d" % (o, p + 1)),
                                     os.path.join(out, "%s_%s.%d" % (v, o, p + 1)))
            manifest[name] = {"variants": list(variants), "n_sources": npls, "n_edges": spec.n_edges,
                              "steps": len(spec.times) - 1, "reference_wall_s": walls}
        finally:
            shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump({"cases": manifest, "outputs": OUTPUTS,
                   "generator": "reference CalcNonstat3DLine built from source by "
                                "oracle/build_ref.sh; tests/golden/make_scale_golden.py"}, f, indent=1)


if __name__ == "__main__":
    main()
