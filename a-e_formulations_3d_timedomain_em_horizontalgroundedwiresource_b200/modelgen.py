"""Synthetic direct-mode input generator for the 3D transient edge-FEM solve.

Writes a working directory in exactly the file formats the reference's
``CalcNonstat3DLine`` reads (direct mode, ``fdirect = 1``), so the same directory
feeds the reference built from source, the CPU oracle and this package:

* mesh files as written by RegularMeshBuilder
  (``RegularMeshBuilder/ReadWrite.cpp:241-1057``): ``inftry.dat``, ``xyz.dat``,
  ``nver.dat``, ``nvkat.dat``, ``l13d.dat``, ``tsize3d_.dat``,
  ``nodesforedges.dat`` and ``edges.dat``; edges are numbered in lexicographic
  order of their (lower, upper) 1-based node pair
  (``RegularMeshBuilder/Mesh3D.cpp:130-239``);
* material tables ``sig3d`` / ``mu3d`` (``vec_prep_data.cpp:95-180``), material 1
  is air with sigma = 1e-8 S/m (``RegularMeshBuilder/Model.cpp:22-27``);
* the time grid ``infite.0`` (``ReadWrite.cpp`` ``WriteInfite0``) and the 1 A
  step-off ``currentfunction`` (``ReadWrite.cpp:1338-1360``);
* sources ``sours``, receivers ``xyzVectorB`` / ``xyzVectorE``, the per-source
  receiver counts ``group`` / ``recvsb`` / ``recvse`` (``TaskSP.cpp:467-516``) and
  the single-value config files ``timeintervalforprint``, ``fdirect``,
  ``nSrsRazb``, ``n_neib`` and ``nthreads.txt``
  (``CODE/CalcStarter/main.cpp:302-391``).

The grounded-wire stationary initial field (``a0.dat`` / ``v3a.dat``) is not
written here; it comes from the stationary solve.

All draws are seeded; the same arguments always give byte-identical files.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

MU_REL_DEFAULT = 1.0
SIGMA_AIR = 1e-8


# ----------------------------------------------------------------------------
# 1D axes
# ----------------------------------------------------------------------------
def growth_factor(h0: float, n: int, length: float) -> float:
    """Ratio q with h0 * (q**n - 1) / (q - 1) == length (bisection)."""
    if n <= 0:
        raise ValueError("n must be positive")
    if abs(h0 * n - length) < 1e-12 * length:
        return 1.0
    lo, hi = (1.0 + 1e-12, 10.0) if h0 * n < length else (1e-6, 1.0 - 1e-12)
    f = lambda q: h0 * (q ** n - 1.0) / (q - 1.0) - length
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if (f(mid) > 0) == (f(hi) > 0):
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def graded_run(h0: float, n: int, length: float) -> np.ndarray:
    """Cell sizes of an n-cell geometric run starting at h0 and summing to length."""
    q = growth_factor(h0, n, length)
    sizes = h0 * q ** np.arange(n)
    sizes *= length / sizes.sum()
    return sizes


def symmetric_axis(core_half: float, core_h: float, n_side: int, extent: float) -> np.ndarray:
    """Node coordinates: uniform core [-core_half, core_half] with step core_h,
    then n_side geometrically graded cells on each side out to +-extent."""
    n_core = int(round(2 * core_half / core_h))
    core = -core_half + core_h * np.arange(n_core + 1)
    if n_side > 0:
        g = np.cumsum(graded_run(core_h * 1.0, n_side, extent - core_half))
        # first graded cell equals the core step times the growth ratio
        right = core_half + g
        left = -right[::-1]
        core = np.concatenate([left, core, right])
    core[np.abs(core) < 1e-9] = 0.0
    return core


def vertical_axis(earth_core_depth: float, core_h: float, n_earth_graded: int,
                  depth: float, n_air: int, height: float) -> np.ndarray:
    """Node z coordinates (z up, earth below 0): a uniform run of core_h cells from 0
    down to -earth_core_depth, n_earth_graded graded cells to -depth, and n_air
    graded air cells from 0 up to +height."""
    n_core = int(round(earth_core_depth / core_h))
    earth = -core_h * np.arange(n_core + 1)[::-1]
    if n_earth_graded > 0:
        g = np.cumsum(graded_run(core_h, n_earth_graded, depth - earth_core_depth))
        earth = np.concatenate([-(earth_core_depth + g)[::-1], earth])
    air = np.cumsum(graded_run(core_h, n_air, height)) if n_air > 0 else np.zeros(0)
    z = np.concatenate([earth, air])
    z[np.abs(z) < 1e-9] = 0.0
    return z


# ----------------------------------------------------------------------------
# time grid
# ----------------------------------------------------------------------------
def decade_time_grid(t_end: float, n_dec: int, steps_per_dec: int, ratio: float = 2.0,
                     t0: float = 0.0) -> np.ndarray:
    """Piecewise-constant steps: n_dec runs of steps_per_dec steps, each run's step
    ratio times the previous one (the tcff = 2 rule of TimeDirectSolver), ending at
    t_end.  Returns n_dec*steps_per_dec + 1 times starting at t0."""
    geo = sum(ratio ** d for d in range(n_dec))
    h0 = (t_end - t0) / (steps_per_dec * geo)
    t = [t0]
    for d in range(n_dec):
        h = h0 * ratio ** d
        for _ in range(steps_per_dec):
            t.append(t[-1] + h)
    out = np.array(t)
    out[-1] = t_end
    return out


# ----------------------------------------------------------------------------
# model description
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class Box:
    """Axis-aligned conductive block [x0,x1]x[y0,y1]x[z0,z1] with conductivity sigma."""
    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    z1: float
    sigma: float


@dataclasses.dataclass
class ModelSpec:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    # layered earth: list of (z_top, sigma) from the surface down; z_top of the first
    # layer is 0; a layer extends down to the next layer's top
    layers: List[Tuple[float, float]]
    boxes: List[Box]
    sources: List[Tuple[Tuple[float, float, float], Tuple[float, float, float]]]
    receivers_b: List[List[Tuple[float, float, float]]]   # per source
    receivers_e: List[List[Tuple[float, float, float]]]   # per source
    times: np.ndarray
    print_interval: Optional[Tuple[float, float]] = None
    n_srs_razb: int = 500
    n_neib: int = 3
    nthreads: int = 1
    sigma_air: float = SIGMA_AIR   # conductivity of material 1 (cells above z = 0)

    @property
    def n_nodes(self) -> int:
        return len(self.x) * len(self.y) * len(self.z)

    @property
    def n_cells(self) -> int:
        return (len(self.x) - 1) * (len(self.y) - 1) * (len(self.z) - 1)

    @property
    def n_edges(self) -> int:
        nx, ny, nz = len(self.x), len(self.y), len(self.z)
        return (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)


def cell_materials(spec: ModelSpec) -> Tuple[np.ndarray, List[float]]:
    """Material id per cell (1-based, cell order ix fastest then iy then iz) and
    the conductivity table (index 0 = material 1 = air)."""
    xc = 0.5 * (spec.x[1:] + spec.x[:-1])
    yc = 0.5 * (spec.y[1:] + spec.y[:-1])
    zc = 0.5 * (spec.z[1:] + spec.z[:-1])
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    sig_table = [spec.sigma_air]
    mat = np.ones(X.shape, dtype=np.int32)
    for li, (ztop, sig) in enumerate(spec.layers):
        zbot = spec.layers[li + 1][0] if li + 1 < len(spec.layers) else -np.inf
        sig_table.append(sig)
        mat[(Z < ztop) & (Z >= zbot)] = len(sig_table)
    for b in spec.boxes:
        sig_table.append(b.sigma)
        sel = (X > b.x0) & (X < b.x1) & (Y > b.y0) & (Y < b.y1) & (Z > b.z0) & (Z < b.z1)
        mat[sel & (Z < 0)] = len(sig_table)
    return mat.reshape(-1), sig_table


def edge_numbering(nx: int, ny: int, nz: int):
    """Edge ids (0-based) of the x/y/z edge starting at each node, -1 if none.

    Edges are sorted lexicographically by (lower node, upper node) with 1-based
    node numbers n = 1 + ix + nx*iy + nx*ny*iz; for one lower node the x edge
    (n, n+1) comes before the y edge (n, n+nx) before the z edge (n, n+nx*ny)."""
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hasx = (ix < nx - 1).reshape(-1)
    hasy = (iy < ny - 1).reshape(-1)
    hasz = (iz < nz - 1).reshape(-1)
    cnt = hasx.astype(np.int64) + hasy + hasz
    base = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    ex = np.where(hasx, base, -1)
    ey = np.where(hasy, base + hasx, -1)
    ez = np.where(hasz, base + hasx + hasy, -1)
    return ex, ey, ez, int(cnt.sum())


def write_model(path: str, spec: ModelSpec) -> dict:
    """Write every direct-mode input file for spec into directory path."""
    os.makedirs(path, exist_ok=True)
    nx, ny, nz = len(spec.x), len(spec.y), len(spec.z)
    nxy = nx * ny
    n_nodes = nx * ny * nz
    n_cells = (nx - 1) * (ny - 1) * (nz - 1)

    def w(name, text):
        with open(os.path.join(path, name), "w") as f:
            f.write(text)

    # --- inftry.dat (same field layout as WriteInftry) -----------------------
    kt1 = (nx * ny + nx * (nz - 2) + (ny - 2) * (nz - 2)) * 2
    w("inftry.dat",
      " ISLAU= 0 INDKU1= 0 INDFPO= 0\nKUZLOV= %d   KPAR= %d    KT1= %d   KTR2= 0   KTR3= 0\n"
      "   KT8= 0   KT9= 0\nKISRS1= 0 KISRS2= 0 KISRS3= 0   KBRS= 0\n   KT7= 0   KT10= 0  KTR4= 0  KTSIM= 0\n"
      "   KT6= 0" % (n_nodes, n_cells, kt1))

    # --- xyz.dat --------------------------------------------------------------
    Z, Y, X = np.meshgrid(spec.z, spec.y, spec.x, indexing="ij")
    xyz = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1).astype("<f8")
    xyz.tofile(os.path.join(path, "xyz.dat"))

    # --- nver.dat: 14 int32 per cell, 1-based ---------------------------------
    cz, cy, cx = np.meshgrid(np.arange(nz - 1), np.arange(ny - 1), np.arange(nx - 1), indexing="ij")
    n0 = (cx + nx * cy + nxy * cz).reshape(-1)
    nver = np.zeros((n_cells, 14), dtype="<i4")
    offs = [0, 1, nx, nx + 1, nxy, nxy + 1, nxy + nx, nxy + nx + 1]
    for k, o in enumerate(offs):
        nver[:, k] = n0 + o + 1
    nver.tofile(os.path.join(path, "nver.dat"))

    # --- materials ------------------------------------------------------------
    mat, sig_table = cell_materials(spec)
    mat.astype("<i4").tofile(os.path.join(path, "nvkat.dat"))
    w("sig3d", "".join("%d\t%.7e\t%.7e\n" % (i + 1, s, s) for i, s in enumerate(sig_table)))
    w("mu3d", "".join("%d\t%.7e\t%.7e\n" % (i + 1, MU_REL_DEFAULT, MU_REL_DEFAULT)
                      for i in range(len(sig_table))))

    # --- boundary nodes l13d.dat ---------------------------------------------
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    bnd = ((ix == 0) | (ix == nx - 1) | (iy == 0) | (iy == ny - 1) | (iz == 0) | (iz == nz - 1)).reshape(-1)
    (np.nonzero(bnd)[0] + 1).astype("<i4").tofile(os.path.join(path, "l13d.dat"))

    # --- edges -----------------------------------------------------------------
    ex, ey, ez, n_edges = edge_numbering(nx, ny, nz)
    nfe = np.zeros((n_edges, 2), dtype="<i4")
    node = np.arange(n_nodes)
    for eid, step in ((ex, 1), (ey, nx), (ez, nxy)):
        sel = eid >= 0
        nfe[eid[sel], 0] = node[sel] + 1
        nfe[eid[sel], 1] = node[sel] + step + 1
    nfe.tofile(os.path.join(path, "nodesforedges.dat"))
    w("tsize3d_.dat", "0\n%d\n" % n_edges)
    w("tsize3d.dat", "0\n")

    ed = np.zeros((n_cells, 25), dtype="<i4")
    loc = [(ex, 0), (ex, nx), (ex, nxy), (ex, nxy + nx),
           (ey, 0), (ey, nxy), (ey, 1), (ey, nxy + 1),
           (ez, 0), (ez, 1), (ez, nx), (ez, nx + 1)]
    for k, (arr, o) in enumerate(loc):
        ed[:, k] = arr[n0 + o] + 1
    ed[:, 24] = 1
    ed.tofile(os.path.join(path, "edges.dat"))

    # --- time grid -------------------------------------------------------------
    t = np.asarray(spec.times, dtype=float)
    lines = ["    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n" % (len(t), len(t)),
             "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n",
             "       u0=   0.00000e+000\n",
             " T I M E :\n"]
    for i in range(0, len(t), 5):
        lines.append("".join(" %.13e;" % v for v in t[i:i + 5]) + "\n")
    w("infite.0", "".join(lines))
    w("currentfunction", "".join("%.13e\t%.13e\n" % (v, 1.0 if i == 0 else 0.0) for i, v in enumerate(t)))
    pl, pr = spec.print_interval if spec.print_interval else (5 * (t[1] - t[0]), 1.5 * t[-1])
    w("timeintervalforprint", "%.13e %.13e\n" % (pl, pr))

    # --- sources / receivers / config -------------------------------------------
    npls = len(spec.sources)
    w("group", "1\n1 1 %d\n" % npls)
    w("sours", "".join("%.6f %.6f %.6f\n%.6f %.6f %.6f\n" % (a + b) for a, b in spec.sources))
    rb = [p for lst in spec.receivers_b for p in lst]
    re = [p for lst in spec.receivers_e for p in lst]
    w("xyzVectorB", "%d\n" % len(rb) + "".join("%.6f %.6f %.6f\n" % p for p in rb))
    w("xyzVectorE", "%d\n" % len(re) + "".join("%.6f %.6f %.6f\n" % p for p in re))
    w("recvsb", "".join("%d\n" % len(l) for l in spec.receivers_b))
    w("recvse", "".join("%d\n" % len(l) for l in spec.receivers_e))
    w("fdirect", "1\n")
    w("nSrsRazb", "%d\n" % spec.n_srs_razb)
    w("n_neib", "%d\n" % spec.n_neib)
    w("nthreads.txt", "%d\n" % spec.nthreads)
    return {"n_nodes": n_nodes, "n_cells": n_cells, "n_edges": n_edges, "npls": npls,
            "ntime": len(t), "n_materials": len(sig_table)}


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
def receivers_on_y_axis(n: int = 21, y0: float = 50.0, dy: float = 50.0, x: float = 0.0):
    return [(x, y0 + dy * k, 0.0) for k in range(n)]


def halfspace_model(cells: int = 40, core_h: float = 10.0, core_half: float = 100.0,
                    extent: float = 5000.0, n_air: int = 15, sigma: float = 0.01,
                    n_dec: int = 6, steps_per_dec: int = 20, t_end: float = 1e-2,
                    n_receivers: int = 21, wire_half: float = 50.0, n_srs_razb: int = 500) -> ModelSpec:
    """Homogeneous half-space under air (the 40^3 backward-Euler workload when called
    with the defaults).  Horizontal axes: a uniform core of core_h cells over
    [-core_half, core_half] and equal graded runs to +-extent; the vertical axis
    has n_air graded air cells up to +extent and the remaining cells in the earth
    (10 uniform core_h cells, then graded down to -extent)."""
    n_core = int(round(2 * core_half / core_h))
    n_side = (cells - n_core) // 2
    if n_side < 1:
        raise ValueError("cells too small for the core")
    x = symmetric_axis(core_half, core_h, n_side, extent)
    y = x.copy()
    n_earth = cells - n_air
    n_earth_core = min(10, n_earth - 1)
    z = vertical_axis(n_earth_core * core_h, core_h, n_earth - n_earth_core, extent, n_air, extent)
    t = decade_time_grid(t_end, n_dec, steps_per_dec)
    rec = receivers_on_y_axis(n_receivers)
    return ModelSpec(x=x, y=y, z=z, layers=[(0.0, sigma)], boxes=[],
                     sources=[((-wire_half, 0.0, 0.0), (wire_half, 0.0, 0.0))],
                     receivers_b=[rec], receivers_e=[rec], times=t, n_srs_razb=n_srs_razb)


def layered_block_model(cells: int = 80, core_h: float = 10.0, core_half: float = 200.0,
                        extent: float = 5000.0, n_air: int = 20, n_dec: int = 8,
                        steps_per_dec: int = 20, t_end: float = 1e-1,
                        sources: Optional[Sequence] = None, n_receivers: int = 21,
                        n_srs_razb: int = 500, cells_z: Optional[int] = None,
                        boxes: Optional[Sequence["Box"]] = None) -> ModelSpec:
    """Three-layer earth (100 Ohm.m 0-50 m, 10 Ohm.m 50-300 m, 1000 Ohm.m below) with a
    0.1 S/m 200x200x100 m block whose top is at 150 m depth (or the given boxes);
    cells per horizontal side, cells_z vertically (default: cells)."""
    n_core = int(round(2 * core_half / core_h))
    n_side = (cells - n_core) // 2
    x = symmetric_axis(core_half, core_h, n_side, extent)
    y = x.copy()
    n_earth = (cells if cells_z is None else cells_z) - n_air
    n_earth_core = min(30, n_earth - 1)
    z = vertical_axis(n_earth_core * core_h, core_h, n_earth - n_earth_core, extent, n_air, extent)
    t = decade_time_grid(t_end, n_dec, steps_per_dec)
    if sources is None:
        sources = [((-50.0, 0.0, 0.0), (50.0, 0.0, 0.0))]
    rec = receivers_on_y_axis(n_receivers)
    return ModelSpec(x=x, y=y, z=z,
                     layers=[(0.0, 1.0 / 100.0), (-50.0, 1.0 / 10.0), (-300.0, 1.0 / 1000.0)],
                     boxes=(list(boxes) if boxes is not None
                            else [Box(-100.0, 100.0, -100.0, 100.0, -250.0, -150.0, 0.1)]),
                     sources=list(sources), receivers_b=[rec] * len(sources),
                     receivers_e=[rec] * len(sources), times=t, n_srs_razb=n_srs_razb)


def random_blocks(seed: int, count: int = 5, sigma_lo: float = 0.05, sigma_hi: float = 1.0,
                  edge_lo: float = 50.0, edge_hi: float = 200.0, half_width: float = 180.0,
                  depth_lo: float = 20.0, depth_hi: float = 300.0) -> List["Box"]:
    """count axis-aligned blocks drawn from PCG64(seed): edges uniform in
    [edge_lo, edge_hi] m, centres uniform in the core (|x|, |y| <= half_width minus
    half an edge) with tops between depth_lo and depth_hi, conductivity log-uniform
    in [sigma_lo, sigma_hi] S/m."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        e = rng.uniform(edge_lo, edge_hi, 3)
        cx = rng.uniform(-half_width + e[0] / 2, half_width - e[0] / 2)
        cy = rng.uniform(-half_width + e[1] / 2, half_width - e[1] / 2)
        top = -rng.uniform(depth_lo, depth_hi)
        sig = float(10 ** rng.uniform(np.log10(sigma_lo), np.log10(sigma_hi)))
        out.append(Box(cx - e[0] / 2, cx + e[0] / 2, cy - e[1] / 2, cy + e[1] / 2, top - e[2], top, sig))
    return out


def largest_model(seed: int = 20261203) -> ModelSpec:
    """The largest single model: 120 x 120 x 100 cells, the three-layer earth with five
    random conductive blocks of 0.05-1 S/m (random_blocks(seed)), a 200 m grounded
    wire along x centred at the origin, 200 steps (10 doubling decades of 20) to 1 s."""
    return layered_block_model(cells=120, cells_z=100, n_dec=10, t_end=1.0,
                               sources=[((-100.0, 0.0, 0.0), (100.0, 0.0, 0.0))],
                               boxes=random_blocks(seed))


def random_request_model(seed: int, cells_lo: int = 30, cells_hi: int = 100):
    """One request of the served stream: mesh of U{cells_lo..cells_hi} cells per side,
    1-3 layers with conductivity log-uniform in [1e-4, 1] S/m, 1-3 boxes of 50-400 m
    edge with conductivity log-uniform in [1e-3, 1] S/m, A/E formulation and two- or
    three-point scheme at random, 60-200 steps in doubling decades; every draw comes
    from PCG64(seed).  Returns (spec, formulation, scheme)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cells = int(rng.integers(cells_lo, cells_hi + 1))
    form = "A" if rng.integers(0, 2) == 0 else "E"
    scheme = int(rng.integers(2, 4))
    n_core = max(8, cells // 2)
    core_half = 200.0
    core_h = 2 * core_half / n_core
    n_side = (cells - n_core) // 2
    x = symmetric_axis(core_half, core_h, n_side, 5000.0)
    y = x.copy()
    n_air = max(4, cells // 4)
    n_earth = cells - n_air
    n_earth_core = max(2, min(n_earth // 2, int(300.0 / core_h)))
    z = vertical_axis(n_earth_core * core_h, core_h, n_earth - n_earth_core, 5000.0, n_air, 5000.0)
    n_layers = int(rng.integers(1, 4))
    tops = [0.0] + sorted((-rng.uniform(20.0, 400.0, n_layers - 1)).tolist(), reverse=True)
    layers = [(t, float(10 ** rng.uniform(-4, 0))) for t in tops]
    boxes = []
    for _ in range(int(rng.integers(1, 4))):
        e = rng.uniform(50.0, 400.0, 3)
        c = (rng.uniform(-150, 150), rng.uniform(-150, 150), -rng.uniform(e[2] / 2 + 10, 400))
        boxes.append(Box(c[0] - e[0] / 2, c[0] + e[0] / 2, c[1] - e[1] / 2, c[1] + e[1] / 2,
                         c[2] - e[2] / 2, c[2] + e[2] / 2, float(10 ** rng.uniform(-3, 0))))
    n_steps = int(rng.integers(60, 201))
    n_dec = int(rng.integers(3, 9))
    t = decade_time_grid(10 ** rng.uniform(-3, -1), n_dec, max(8, n_steps // n_dec))
    src = [((-50.0, 0.0, 0.0), (50.0, 0.0, 0.0))]
    rec = receivers_on_y_axis(11)
    spec = ModelSpec(x=x, y=y, z=z, layers=layers, boxes=boxes, sources=src, receivers_b=[rec],
                     receivers_e=[rec], times=t, n_srs_razb=100)
    return spec, form, scheme


def wire_grid_sources(nx: int = 4, ny: int = 8, spacing: float = 100.0, half: float = 50.0):
    """nx*ny 100 m x-directed wires with centres on a surface grid."""
    out = []
    for j in range(ny):
        for i in range(nx):
            cx = (i - (nx - 1) / 2.0) * spacing
            cy = (j - (ny - 1) / 2.0) * spacing
            out.append(((cx - half, cy, 0.0), (cx + half, cy, 0.0)))
    return out


def small_model(cells: int = 10, n_dec: int = 3, steps_per_dec: int = 6, sigma: float = 0.01,
                block: bool = True, n_sources: int = 1, n_receivers: int = 5,
                t_end: float = 1e-3) -> ModelSpec:
    """A small test case (cells^3) that runs in seconds on the CPU: half-space, optional
    conductive block, wire(s) at the surface, receivers on the y axis."""
    core_h = 20.0
    core_half = 40.0
    n_side = (cells - int(round(2 * core_half / core_h))) // 2
    x = symmetric_axis(core_half, core_h, n_side, 1000.0)
    y = x.copy()
    n_air = max(2, cells // 3)
    n_earth = cells - n_air
    z = vertical_axis(min(3, n_earth - 1) * core_h, core_h, n_earth - min(3, n_earth - 1), 1000.0, n_air, 1000.0)
    t = decade_time_grid(t_end, n_dec, steps_per_dec)
    srcs = [((-30.0, 0.0, 0.0), (30.0, 0.0, 0.0))]
    if n_sources > 1:
        srcs = [((-30.0, 20.0 * k, 0.0), (30.0, 20.0 * k, 0.0)) for k in range(n_sources)]
    rec = [(0.0, 10.0 + 25.0 * k, 0.0) for k in range(n_receivers)]
    boxes = [Box(-30.0, 30.0, -30.0, 30.0, -50.0, -20.0, 0.2)] if block else []
    return ModelSpec(x=x, y=y, z=z, layers=[(0.0, sigma), (-60.0, sigma * 0.1)], boxes=boxes,
                     sources=srcs, receivers_b=[rec] * len(srcs), receivers_e=[rec] * len(srcs),
                     times=t, n_srs_razb=100)


# ----------------------------------------------------------------------------
# analytic initial fields (synthetic stand-in for the stationary solve)
# ----------------------------------------------------------------------------
MU0 = 1.25663706143591729e-6


def write_analytic_initial_field(path: str, spec: ModelSpec, current: float = 1.0, reg: float = 1.0) -> None:
    """Writes a0.dat (nodal A0 of each straight wire in free space,
    mu0 I / (4 pi) * integral dl / r) and v3a.dat / v3n.dat (nodal DC potential of
    the wire's electrode pair on a half-space of the top layer's conductivity).
    Distances below `reg` metres are clamped to keep the fields finite.  These are
    smooth synthetic initial conditions with the right shape and scale; the
    transient's cost does not depend on their values."""
    Z, Y, X = np.meshgrid(spec.z, spec.y, spec.x, indexing="ij")
    P = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1)
    sigma = spec.layers[0][1] if spec.layers else 0.01
    a0 = np.zeros((len(spec.sources), P.shape[0], 3))
    v = np.zeros((len(spec.sources), P.shape[0]))
    for k, (A, B) in enumerate(spec.sources):
        A = np.asarray(A, float)
        B = np.asarray(B, float)
        L = np.linalg.norm(B - A)
        t = (B - A) / L
        s = (P - A) @ t                      # along-wire coordinate
        rho2 = np.maximum(np.sum((P - A) ** 2, 1) - s ** 2, reg * reg)
        ra = np.sqrt(s ** 2 + rho2)
        rb = np.sqrt((s - L) ** 2 + rho2)
        pot = MU0 * current / (4 * np.pi) * np.log((ra + s) / (rb + s - L))
        a0[k] = pot[:, None] * t[None, :]
        rA = np.maximum(np.linalg.norm(P - A, axis=1), reg)
        rB = np.maximum(np.linalg.norm(P - B, axis=1), reg)
        v[k] = current / (2 * np.pi * sigma) * (1.0 / rB - 1.0 / rA)
    a0.astype("<f8").tofile(os.path.join(path, "a0.dat"))
    v.astype("<f8").tofile(os.path.join(path, "v3a.dat"))
    np.zeros_like(v).astype("<f8").tofile(os.path.join(path, "v3n.dat"))
