"""CPU restatement of the reference's 3D transient edge-FEM solve -- TEST INFRASTRUCTURE ONLY.

numpy / scipy, FP64.  It follows CalcNonstat3DLine step by step for small meshes
(seconds for up to ~12^3 cells) and writes the same output files, so tests can
compare the GPU product with an independent implementation as well as with the
reference binaries built from source (oracle/_ref).  Never imported by the
product.

Independence from the product: element matrices come from 2-point Gauss
quadrature of the edge basis (the product evaluates closed forms), the linear
systems are solved with SuperLU (the product uses its own GPU Cholesky), and the
receivers are evaluated layer by layer with the nodal L2 projection exactly as
the reference does (the product precomputes one linear functional per receiver).

Reference (paths inside CODE/programs to folder Modules/!programs for
{2,3}-point implicit scheme/!programs for {A,E}-formulation/CalcNonstat3DLine/):
  reading             vec_prep_data.cpp:83-257, 834-853; time_approx.cpp:243-287
  element matrices    T_Brick.cpp:142-540 (basis T_Brick.cpp:741-836)
  assembly            T_Global_SLAE.cpp:76-215; time_approx.cpp:441-470
  boundary            T_Bound_Cond.cpp:58-138
  time stepping       TaskSP.cpp:351-398, 628-702; time_approx.cpp:576-1152
                      (3-point: Two_Layers_Schema for steps 1-2, BDF2 after)
  source              time_approx.cpp:1039-1076 (A), E-form 1057-1105 (-dJ/dt)
  initial field       time_approx.cpp:816-889 (a0.dat), E-form 856-901 (v3a.dat)
  receivers           OutputResultant3d.cpp:343-515, Subdomain.cpp:142-441,
                      time_approx.cpp:1481-1518
  differencing/output give_out_vec_loop.cpp:240-615 (3-point variant: central
                      differences in the interior)
"""
from __future__ import annotations

import os
from typing import Dict, List, Tuple

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

MU0 = 1.25663706143591729e-6
_GP = np.array([-1.0, 1.0]) / np.sqrt(3.0)   # 2-point Gauss on [-1, 1], weights 1


# ---------------------------------------------------------------------------
# input
# ---------------------------------------------------------------------------
def read_model(d: str) -> Dict:
    m: Dict = {}
    rows = []
    with open(os.path.join(d, "sig3d")) as f:
        for line in f:
            p = line.split()
            if len(p) >= 3:
                rows.append((int(p[0]), float(p[1]), float(p[2])))
    nmat = max(r[0] for r in rows)
    m["sigma"] = np.zeros(nmat)
    m["sigma0"] = np.zeros(nmat)
    for r in rows[:nmat]:
        m["sigma"][r[0] - 1] = r[1]
        m["sigma0"][r[0] - 1] = r[2]
    m["mu"] = np.full(nmat, MU0)
    with open(os.path.join(d, "mu3d")) as f:
        vals = f.read().split()
    for i in range(nmat):
        m["mu"][int(vals[3 * i]) - 1] = float(vals[3 * i + 1]) * MU0
    tok = open(os.path.join(d, "inftry.dat")).read().split()
    for key, name in (("KUZLOV=", "kuzlov"), ("KPAR=", "kpar"), ("KT1=", "kt1")):
        m[name] = int(tok[tok.index(key) + 1])
    m["xyz"] = np.fromfile(os.path.join(d, "xyz.dat"), "<f8").reshape(-1, 3)
    m["nver"] = np.fromfile(os.path.join(d, "nver.dat"), "<i4").reshape(-1, 14)[:, :8] - 1
    m["nvkat"] = np.fromfile(os.path.join(d, "nvkat.dat"), "<i4") - 1
    m["l13d"] = np.fromfile(os.path.join(d, "l13d.dat"), "<i4") - 1
    m["edges"] = np.fromfile(os.path.join(d, "nodesforedges.dat"), "<i4").reshape(-1, 2) - 1
    m["ed"] = np.fromfile(os.path.join(d, "edges.dat"), "<i4").reshape(-1, 25)[:, :12] - 1
    m["n"] = m["edges"].shape[0]
    txt = open(os.path.join(d, "infite.0")).read()
    nt = int(txt.split("=", 1)[1].split(";")[0])
    body = txt.split("\n", 4)[4]
    m["time"] = np.array([float(v) for v in body.replace("\n", " ").split(";") if v.strip()][:nt])
    m["print"] = [float(v) for v in open(os.path.join(d, "timeintervalforprint")).read().split()[:2]]

    def recv(name):
        v = open(os.path.join(d, name)).read().split()
        k = int(v[0])
        return np.array([float(x) for x in v[1:1 + 3 * k]]).reshape(k, 3)

    m["rec_b"], m["rec_e"] = recv("xyzVectorB"), recv("xyzVectorE")
    g = open(os.path.join(d, "group")).read().split()
    npls = sum(int(g[3 + 3 * i]) - int(g[2 + 3 * i]) + 1 for i in range(int(g[0])))
    m["npls"] = npls

    def ig(name):
        v = [int(x) for x in open(os.path.join(d, name)).read().split()[:npls]]
        return np.concatenate([[0], np.cumsum(v)]).astype(int)

    m["ig_b"], m["ig_e"] = ig("recvsb"), ig("recvse")
    m["fdirect"] = os.path.exists(os.path.join(d, "fdirect")) and int(open(os.path.join(d, "fdirect")).read().split()[0]) != 0
    m["n_neib"] = int(open(os.path.join(d, "n_neib")).read().split()[0]) if os.path.exists(os.path.join(d, "n_neib")) else 5
    if m["fdirect"]:
        cf = np.loadtxt(os.path.join(d, "currentfunction"))
        m["cf"] = cf[: len(m["time"]), 1]
        nsr = os.path.join(d, "nSrsRazb")
        m["nsrs"] = int(open(nsr).read().split()[0]) if os.path.exists(nsr) else 500
        m["wires"] = np.array([float(v) for v in open(os.path.join(d, "sours")).read().split()]).reshape(-1, 6)[:npls]
    # primary-secondary mode: anomalous edges and the normal-field file name
    # (time_approx.cpp:351-368, 1263-1348)
    mf = os.path.join(d, "mtrsizeforE0")
    m["anom"] = np.zeros(m["n"], bool)
    if os.path.exists(mf):
        m["anom"] = np.array([int(v) for v in open(mf).read().split()[:m["n"]]]) != 0
    pn = os.path.join(d, "PName")
    m["pname"] = open(pn).read().split()[0] if os.path.exists(pn) else ""
    # one anomaly of several: its index ia suffixes the files (TaskSP.cpp:539-596, time_approx.cpp:1280-1287)
    at = os.path.join(d, "AnomalType")
    m["anomaly"] = None
    if os.path.exists(at) and int(open(at).read().split()[0]) != 0:
        m["anomaly"] = int(open(os.path.join(d, "ia")).read().split()[0])
    m["dir"] = d
    return m


# ---------------------------------------------------------------------------
# element matrices by quadrature of the edge basis (T_Brick.cpp:741-836)
# ---------------------------------------------------------------------------
def _l(i, t):
    return (1.0 - t) * 0.5 if i == 0 else (t + 1.0) * 0.5


def _dl(i):
    return -0.5 if i == 0 else 0.5


def basis(j, x, y, z):
    """Reference basis of local edge j at (x, y, z) in [-1,1]^3 (unscaled), and its
    derivatives d/dx, d/dy, d/dz of the non-zero component."""
    c = [x, y, z]
    dirn, a, b = j // 4, j & 1, (j >> 1) & 1
    u, v = (dirn + 1) % 3, (dirn + 2) % 3
    val = _l(a, c[u]) * _l(b, c[v])
    grad = [0.0, 0.0, 0.0]
    grad[u] = _dl(a) * _l(b, c[v])
    grad[v] = _l(a, c[u]) * _dl(b)
    return dirn, val, grad


def local_matrices(h: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Curl-curl B and mass C of a brick with edge lengths h (T_Brick.cpp:142-474)."""
    B = np.zeros((12, 12))
    C = np.zeros((12, 12))
    jac = h[0] * h[1] * h[2] / 8.0
    for x in _GP:
        for y in _GP:
            for z in _GP:
                vals = np.zeros((12, 3))
                curls = np.zeros((12, 3))
                for j in range(12):
                    dirn, val, g = basis(j, x, y, z)
                    s = 2.0 / h[dirn]
                    vals[j, dirn] = val * s
                    dg = [g[k] * 2.0 / h[k] * s for k in range(3)]  # physical gradient
                    # curl of f e_dirn: components
                    if dirn == 0:
                        curls[j] = [0.0, dg[2], -dg[1]]
                    elif dirn == 1:
                        curls[j] = [-dg[2], 0.0, dg[0]]
                    else:
                        curls[j] = [dg[1], -dg[0], 0.0]
                C += jac * vals @ vals.T
                B += jac * curls @ curls.T
    return B, C


def assemble(m: Dict):
    """Global sigma*C and B/mu over all edges (T_Global_SLAE.cpp:76-215)."""
    rows, cols, cv, bv, dv = [], [], [], [], []
    cache = {}
    for e in range(m["nver"].shape[0]):
        p0, p7 = m["xyz"][m["nver"][e, 0]], m["xyz"][m["nver"][e, 7]]
        h = p7 - p0
        key = tuple(np.round(h, 12))
        if key not in cache:
            cache[key] = local_matrices(h)
        Bl, Cl = cache[key]
        idx = m["ed"][e]
        rr, cc = np.meshgrid(idx, idx, indexing="ij")
        rows.append(rr.ravel())
        cols.append(cc.ravel())
        cv.append((Cl * m["sigma"][m["nvkat"][e]]).ravel())
        bv.append((Bl / m["mu"][m["nvkat"][e]]).ravel())
        dv.append((Cl * (m["sigma"][m["nvkat"][e]] - m["sigma0"][m["nvkat"][e]])).ravel())
    n = m["n"]
    r, c = np.concatenate(rows), np.concatenate(cols)
    Cg = sp.csr_matrix((np.concatenate(cv), (r, c)), shape=(n, n))
    Bg = sp.csr_matrix((np.concatenate(bv), (r, c)), shape=(n, n))
    m["Cds"] = sp.csr_matrix((np.concatenate(dv), (r, c)), shape=(n, n))  # (sigma - sigma0) C
    return Cg, Bg


def normal_field(m: Dict, it: int) -> np.ndarray:
    """Normal field of layer it as edge values (time_approx.cpp:1263-1348): float32 per
    anomalous edge and source from m<PName>.enor.NNNN, times half the edge length."""
    idx = np.nonzero(m["anom"])[0]
    name = "m%s.enor.%04d" % (m["pname"], it)
    if m["anomaly"] is not None:
        name += "_%d" % m["anomaly"]
    f = np.fromfile(os.path.join(m["dir"], name), "<f4")
    f = f[: len(idx) * m["npls"]].reshape(m["npls"], len(idx)).astype(np.float64)
    ax = m["xyz"][m["edges"][idx, 1]] - m["xyz"][m["edges"][idx, 0]]
    ln = np.sqrt(ax[:, 0] * ax[:, 0] + ax[:, 1] * ax[:, 1] + ax[:, 2] * ax[:, 2])
    En = np.zeros((m["n"], m["npls"]))
    En[idx] = (f * ln * 0.5).T
    return En


def normal_field_layer(m: Dict, it: int) -> np.ndarray:
    """Layer it of the normal field on the edges for the E-formulation; layer 0 is
    -grad of the normal potential v3n.dat on every edge (E2/time_approx.cpp:1384-1412)."""
    if it > 0:
        return normal_field(m, it)
    npls = m["npls"]
    V = np.fromfile(os.path.join(m["dir"], "v3n.dat"), "<f8")[: m["kuzlov"] * npls].reshape(npls, m["kuzlov"])
    v1, v2 = m["edges"][:, 0], m["edges"][:, 1]
    ax = m["xyz"][v2] - m["xyz"][v1]
    ln = np.sqrt(ax[:, 0] * ax[:, 0] + ax[:, 1] * ax[:, 1] + ax[:, 2] * ax[:, 2])
    etan = -(V[:, v2] - V[:, v1]) / ln
    return (etan * ln * 0.5).T


def normal_field_rate(m: Dict, it: int, t1: int, t2: int, three_point: bool) -> np.ndarray:
    """Minus the time derivative of the normal field at layer it: two-point over
    (it, t1), or three-point over (it, t1, t2) (E2/time_approx.cpp:1419-1431,
    E3/time_approx.cpp:1400-1460)."""
    t = m["time"]
    e0, e1 = normal_field_layer(m, it), normal_field_layer(m, t1)
    if not three_point:
        return -(e0 - e1) / (t[it] - t[t1])
    e2 = normal_field_layer(m, t2)
    tj, tj1, tj2 = t[it], t[t1], t[t2]
    dt, dt0, dt1 = tj - tj2, tj - tj1, tj1 - tj2
    tt = tj
    return -(e2 * (2.0 * tt - tj - tj1) / (dt1 * dt) - e1 * (2.0 * tt - tj - tj2) / (dt1 * dt0)
             + e0 * (2.0 * tt - tj1 - tj2) / (dt * dt0))


# ---------------------------------------------------------------------------
# initial field and source
# ---------------------------------------------------------------------------
def initial_field(m: Dict, eform: bool) -> np.ndarray:
    n, npls, nn = m["n"], m["npls"], m["kuzlov"]
    d = m["dir"]
    ef = os.path.join(d, "e0.edge" if eform else "a0.edge")
    if os.path.exists(ef):
        return np.fromfile(ef, "<f8")[: n * npls].reshape(npls, n).T.copy()
    v1, v2 = m["edges"][:, 0], m["edges"][:, 1]
    axis = m["xyz"][v2] - m["xyz"][v1]
    ln = np.linalg.norm(axis, axis=1)
    u = np.zeros((n, npls))
    if not eform:
        a0 = np.fromfile(os.path.join(d, "a0.dat"), "<f8")[: nn * 3 * npls].reshape(npls, nn, 3)
        for p in range(npls):
            mid = 0.5 * (a0[p, v1] + a0[p, v2])
            u[:, p] = np.sum(mid * axis, 1) / ln * ln * 0.5
    else:
        va = np.fromfile(os.path.join(d, "v3a.dat"), "<f8")[: nn * npls].reshape(npls, nn)
        for p in range(npls):
            u[:, p] = -(va[p, v2] - va[p, v1]) / ln * ln * 0.5
    return u


def _nearest_element(x: np.ndarray, mn: np.ndarray, mx: np.ndarray, p0: np.ndarray, p7: np.ndarray):
    """Element of a dipole that no element holds (vec_prep_data.cpp:878-980, called at
    :1186-1250): the 8 elements of least L1 distance from the point to their node box
    (ties in element order), and of those the first with the least L1 distance of the
    point's local coordinates from [0, 1]."""
    d = np.where(x < mn, mn - x, np.where(x > mx, x - mx, 0.0))
    s = (d[:, 0] + d[:, 1]) + d[:, 2]
    best, e = 1e30, None
    for c in np.lexsort((np.arange(len(s)), s))[:8]:
        loc = (x - p0[c]) / (p7[c] - p0[c])
        o = np.where(loc < 0.0, -loc, np.where(loc > 1.0, loc - 1.0, 0.0))
        so = (o[0] + o[1]) + o[2]
        if so < best:
            best, e = so, int(c)
    return e


def source_vectors(m: Dict) -> np.ndarray:
    """Wire split into nSrsRazb dipoles located in the first element (file order)
    holding them (vec_prep_data.cpp:1050-1183), or the nearest one when none does;
    RHS weights per edge."""
    n, npls = m["n"], m["npls"]
    S = np.zeros((n, npls))
    ns = m["nsrs"]
    mn = m["xyz"][m["nver"]].min(1)
    mx = m["xyz"][m["nver"]].max(1)
    p0 = m["xyz"][m["nver"][:, 0]]
    p7 = m["xyz"][m["nver"][:, 7]]
    for p in range(npls):
        A, B = m["wires"][p, :3], m["wires"][p, 3:]
        dvec = (B - A) / ns
        for j in range(ns):
            x = A + (j + 0.5) * dvec
            inbox = np.all((x >= mn - 1e-3) & (x <= mx + 1e-3), 1)
            e = None
            for cand in np.nonzero(inbox)[0]:
                loc = (x - p0[cand]) / (p7[cand] - p0[cand])
                if np.all((loc > -1e-2) & (loc < 1 + 1e-2)):
                    e = cand
                    break
            if e is None:
                e = _nearest_element(x, mn, mx, p0, p7)
            if e is None:
                raise RuntimeError("dipole outside the mesh")
            loc = (x - p0[e]) / (p7[e] - p0[e])
            c = 2.0 * loc - 1.0
            for k in range(12):
                ii = m["ed"][e, k]
                dirn, val, _ = basis(k, *c)
                ln = np.linalg.norm(m["xyz"][m["edges"][ii, 1]] - m["xyz"][m["edges"][ii, 0]])
                S[ii, p] += val * dvec[dirn] * 2.0 / ln
    return S


# ---------------------------------------------------------------------------
# receivers (OutputResultant3d / Subdomain)
# ---------------------------------------------------------------------------
def _centre_value(m: Dict, u: np.ndarray, elems: np.ndarray, curl: bool, comp: int) -> np.ndarray:
    h = m["xyz"][m["nver"][elems, 7]] - m["xyz"][m["nver"][elems, 0]]
    f = u[m["ed"][elems]]
    out = np.zeros(len(elems))
    for k in range(12):
        dirn, val, g = basis(k, 0.0, 0.0, 0.0)
        s = 2.0 / h[:, dirn]
        if not curl:
            if dirn == comp:
                out += f[:, k] * val * s
            continue
        dg = [g[q] * 2.0 / h[:, q] * s for q in range(3)]
        cvec = ([0.0, dg[2], -dg[1]], [-dg[2], 0.0, dg[0]], [dg[1], -dg[0], 0.0])[dirn]
        out += f[:, k] * cvec[comp]
    return out


class ReceiverSet:
    def __init__(self, m: Dict, pts: np.ndarray, curl: bool):
        self.m, self.pts, self.curl = m, pts, curl
        nver, xyz = m["nver"], m["xyz"]
        lo = xyz[nver[:, 0]] - 1e-6
        hi = xyz[nver[:, 7]] + 1e-6
        self.elem = np.array([int(np.nonzero(np.all((p >= lo) & (p <= hi), 1))[0][0]) for p in pts], int)
        self.cfa = np.zeros((len(pts), 8))
        for i, p in enumerate(pts):
            e = self.elem[i]
            a, b = xyz[nver[e, 0]], xyz[nver[e, 7]]
            loc = (2 * p - a - b) / (b - a)
            for k in range(8):
                self.cfa[i, k] = _l(k & 1, loc[0]) * _l((k >> 1) & 1, loc[1]) * _l((k >> 2) & 1, loc[2])
        mats = [-1] if curl else sorted(set(m["nvkat"][self.elem]))
        self.subs = []
        for mat in mats:
            in_e = np.zeros(len(nver), bool)
            seed = np.zeros(len(nver), bool)
            seed[self.elem] = True
            okm = np.ones(len(nver), bool) if mat == -1 else (m["nvkat"] == mat)
            in_e = seed & okm
            in_n = np.zeros(len(xyz), bool)
            in_n[nver[in_e].ravel()] = True
            for _ in range(m["n_neib"]):
                add = (~in_e) & okm & in_n[nver].any(1)
                in_e |= add
                in_n[nver[add].ravel()] = True
            elems = np.nonzero(in_e)[0]
            nodes = np.nonzero(in_n)[0]
            ren = -np.ones(len(xyz), int)
            ren[nodes] = np.arange(len(nodes))
            h = xyz[nver[elems, 7]] - xyz[nver[elems, 0]]
            V = h.prod(1)
            pop = np.array([[bin(i ^ j).count("1") for j in range(8)] for i in range(8)])
            w = np.array([1 / 27, 1 / 54, 1 / 108, 1 / 216])[pop]
            ln = ren[nver[elems]]
            rr = np.repeat(ln, 8, 1).ravel()
            cc = np.tile(ln, (1, 8)).ravel()
            vv = (V[:, None, None] * w[None]).ravel()
            M = sp.csc_matrix((vv, (rr, cc)), shape=(len(nodes),) * 2)
            g = V[:, None] * w.sum(1)[None, :]  # row sums of the local mass matrix
            recs = [i for i in range(len(pts)) if mat == -1 or m["nvkat"][self.elem[i]] == mat]
            self.subs.append(dict(elems=elems, ln=ln, g=g, lu=spl.splu(M), nn=len(nodes), recs=recs, ren=ren))

    def evaluate(self, u: np.ndarray, owner: np.ndarray) -> np.ndarray:
        """(3, nrec) values for the solution u (n x npls); receiver i samples column owner[i]."""
        out = np.zeros((3, len(self.pts)))
        nver = self.m["nver"]
        for s in self.subs:
            for comp in range(3):
                for p in sorted(set(owner[s["recs"]])):
                    val = _centre_value(self.m, u[:, p], s["elems"], self.curl, comp)
                    pr = np.zeros(s["nn"])
                    np.add.at(pr, s["ln"].ravel(), (s["g"] * val[:, None]).ravel())
                    x = s["lu"].solve(pr)
                    for i in s["recs"]:
                        if owner[i] != p:
                            continue
                        out[comp, i] = x[s["ren"][nver[self.elem[i]]]] @ self.cfa[i]
        return out


# ---------------------------------------------------------------------------
# time stepping
# ---------------------------------------------------------------------------
def decade_starts(t: np.ndarray) -> List[int]:
    ig = [0]
    hpre = t[1] - t[0]
    for i in range(2, len(t)):
        hcur = t[i] - t[i - 1]
        if abs(1.0 - hpre / hcur) > 1e-3:
            ig.append(i)
            hpre = hcur
    return ig + [len(t)]


def find_layer(t: np.ndarray, val: float) -> int:
    if abs(val) < 1e-14 and abs(t[0]) < 1e-14:
        return 0
    for i in range(1, len(t)):
        if abs(1.0 - t[i] / val) < 1e-6:
            return i
    return -1


def _dA_dt(t, uj, uj1, uj2, dt, dt0, dt1, tj, tj1, tj2):
    t = min(max(t, tj2), tj)
    return (uj2 * (2 * t - tj - tj1) / (dt1 * dt) - uj1 * (2 * t - tj - tj2) / (dt1 * dt0)
            + uj * (2 * t - tj1 - tj2) / (dt * dt0))


def run(d: str, formulation: str, scheme: int) -> Dict:
    """Full transient for the model in d; writes the three output files and
    returns the tables."""
    eform = formulation == "E"
    m = read_model(d)
    t = m["time"]
    nt = len(t)
    n, npls = m["n"], m["npls"]
    Cg, Bg = assemble(m)
    bn = np.zeros(m["kuzlov"], bool)
    bn[m["l13d"]] = True
    bound = bn[m["edges"][:, 0]] & bn[m["edges"][:, 1]]
    inner = np.nonzero(~bound)[0]
    anys = m["fdirect"] and np.any(m["cf"][1:] != 0)
    have_src = m["fdirect"] and (eform or anys) and m["nsrs"] > 0
    S = source_vectors(m) if have_src else np.zeros((n, npls))
    u0 = initial_field(m, eform)

    tlf = tll = 2
    for i in range(nt):
        if t[i] >= m["print"][0]:
            tlf = i
            break
    tlf = min(tlf, nt - 1)
    for i in range(nt):
        if t[i] >= m["print"][1] - 1e-6:
            tll = i
            break
    if m["print"][1] > t[-1] - 1e-6:
        tll = nt - 1
    own_b = np.zeros(len(m["rec_b"]), int)
    own_e = np.zeros(len(m["rec_e"]), int)
    for p in range(npls):
        own_b[m["ig_b"][p]:m["ig_b"][p + 1]] = p
        own_e[m["ig_e"][p]:m["ig_e"][p + 1]] = p
    recb = ReceiverSet(m, m["rec_b"], True) if len(m["rec_b"]) else None
    rece = ReceiverSet(m, m["rec_e"], False) if len(m["rec_e"]) else None
    nl = tll - tlf + 1
    VB = np.zeros((nl, 3, len(m["rec_b"])))
    VE = np.zeros((nl, 3, len(m["rec_e"])))
    U: Dict[int, np.ndarray] = {0: u0}

    def record(layer):
        if tlf <= layer <= tll:
            if recb is not None:
                VB[layer - tlf] = recb.evaluate(U[layer], own_b)
            if rece is not None:
                VE[layer - tlf] = rece.evaluate(U[layer], own_e)

    lu = None

    def factor(mult):
        A = (Cg * mult + Bg)[inner][:, inner].tocsc()
        A = A + sp.diags(A.diagonal() * 1e-12)
        return spl.splu(A)

    def coef(it, two, dt):
        if not have_src:
            return 0.0
        cf = m["cf"]
        if not eform:
            return cf[it] if cf[it] != 0 else 0.0
        if it + 1 < nt:
            if cf[it] == 0:
                djdt = (cf[it] - cf[it - 1]) / (dt if two else (t[it] - t[it - 1]))
            else:
                djdt = _dA_dt(t[it], cf[it - 1], cf[it], cf[it + 1], t[it + 1] - t[it - 1], t[it + 1] - t[it],
                              t[it] - t[it - 1], t[it], t[it - 1], t[max(0, it - 2)])
        else:
            djdt = (cf[it] - cf[it - 1]) / (dt if two else (t[it] - t[it - 1]))
        return -djdt

    ps = (not m["fdirect"]) and bool(m["anom"].any())

    def ps_source(it, t1, t2):
        """C_dsigma times the normal field (A) or minus its time derivative (E)."""
        if not eform:
            return m["Cds"] @ normal_field(m, it)
        return m["Cds"] @ normal_field_rate(m, it, t1, t2, scheme == 3 and it > 2)

    def step(it, t1, t2, m1, m2, c):
        hist = U[t1] * m1 + (U[t2] * m2 if m2 != 0 else 0.0)
        rhs = Cg @ hist + c * S
        if ps:
            rhs = rhs + ps_source(it, t1, t2)
        rhs[bound] = 0.0
        x = np.zeros((n, npls))
        x[inner] = lu.solve(rhs[inner])
        U[it] = x

    vpre1 = -np.ones(nt, int)
    vpre2 = -np.ones(nt, int)
    dec = decade_starts(t)
    tn = tn1 = tn2 = 0
    if scheme == 2:
        record(0)
    for di in range(len(dec) - 1):
        tbeg, tend = dec[di], dec[di + 1]
        npre1 = npre2 = -1
        if di > 0:
            hh = t[tbeg + 1] - t[tbeg]
            npre1, npre2 = find_layer(t, t[tbeg] - hh), find_layer(t, t[tbeg] - 2 * hh)
        if scheme == 3 and 1 >= tbeg and 1 < tend:
            dt = t[1] - t[0]
            lu = factor(1.0 / dt)
            for it in (1, 2):
                vpre1[it], vpre2[it] = it - 1, it - 2
                step(it, it - 1, it - 1, 1.0 / dt, 0.0, coef(it, True, dt))
                if it == 2:
                    record(2)
            tn2, tn1, tn = 0, 1, 2
        first = True
        start = max(tbeg, 1 if scheme == 2 else 3)
        for it in range(start, tend):
            fsdiff = first and (it > 1 if scheme == 2 else it != 3)
            if fsdiff:
                tn2, tn1, tn = npre2, npre1, it
            else:
                tn2, tn1, tn = tn1, tn, it
            vpre1[it], vpre2[it] = tn1, tn2
            if first:
                if scheme == 2:
                    mult = m1 = 1.0 / (t[it] - t[tn1])
                    m2 = 0.0
                else:
                    dt, dt0, dt1 = t[it] - t[tn2], t[it] - t[tn1], t[tn1] - t[tn2]
                    mult = (dt + dt0) / (dt * dt0)
                    m1 = dt / (dt1 * dt0)
                    m2 = -dt0 / (dt * dt1)
                lu = factor(mult)
                first = False
            step(it, tn1, tn2, m1, m2, coef(it, False, 0.0))
            record(it)

    def diff(F, sign):
        out = np.zeros_like(F)
        j, j1, j2 = tlf, tlf + 1, tlf + 2
        f = lambda L: F[L - tlf]
        dt, dt1, dt0 = t[j2] - t[j], t[j1] - t[j], t[j2] - t[j1]
        out[0] = sign * (f(j) * (-(dt + dt1) / (dt1 * dt)) + f(j1) * (dt / (dt1 * dt0)) + f(j2) * (-dt1 / (dt * dt0)))
        while True:
            if scheme == 2:
                mt = (-1.0 / (t[j1] - t[j]), 1.0 / (t[j1] - t[j]), 0.0)
            else:
                mt = ((-dt0) / (dt1 * dt), -(dt1 - dt0) / (dt1 * dt0), dt1 / (dt * dt0))
            out[j1 - tlf] = sign * (f(j) * mt[0] + f(j1) * mt[1] + f(j2) * mt[2])
            if j2 == tll:
                break
            j2 += 1
            if scheme == 2:
                j, j1 = vpre2[j2], vpre1[j2]
            else:
                j, j1 = j1, vpre1[j2]
            dt, dt1, dt0 = t[j2] - t[j], t[j1] - t[j], t[j2] - t[j1]
        if scheme == 2:
            mt = (0.0, -1.0 / (t[j2] - t[j1]), 1.0 / (t[j2] - t[j1]))
        else:
            mt = (dt0 / (dt1 * dt), -dt / (dt1 * dt0), (dt + dt0) / (dt * dt0))
        out[j2 - tlf] = sign * (f(j) * mt[0] + f(j1) * mt[1] + f(j2) * mt[2])
        return out

    if eform:
        E, EMF, BB = VE, -VB, np.zeros_like(VB)
    else:
        E, EMF, BB = diff(VE, -1.0), diff(VB, 1.0), VB
    times = t[tlf:tll + 1]
    _write(d, "edsall_anom", m["rec_b"], m["ig_b"], npls, times, EMF * (-1000),
           "      t (ms)         Emfx_anom (mV)     Emfy_anom (mV)     Emfz_anom (mV)")
    _write(d, "ball_anom", m["rec_b"], m["ig_b"], npls, times, BB * 1000,
           "      t (ms)        Bx_anom (mTl)     By_anom (mTl)     Bz_anom (mTl)")
    _write(d, "eall_anom", m["rec_e"], m["ig_e"], npls, times, E * 1000,
           "      t (ms)         Ex_anom n (mV)     Ey_anom a (mV)     Ez_anom s (mV)")
    return {"eall": E * 1000, "emf": EMF * (-1000), "ball": BB * 1000, "first": tlf, "last": tll}


def _write(d, name, pts, ig, npls, times, vals, title):
    for p in range(npls):
        with open(os.path.join(d, "%s.%d" % (name, p + 1)), "w") as f:
            for i in range(len(pts)):
                if i < ig[p] or i >= ig[p + 1]:
                    continue
                x = pts[i]
                f.write("%d %d\n%.16e %.16e %.16e\n1\n1 1 1 1\n1\n%s\n" % (int(x[0]), int(x[1]), x[0], x[1], x[2], title))
                for L in range(len(times)):
                    f.write("%.16e\t%.16e\t%.16e\t%.16e\n" % (times[L] * 1000, vals[L, 0, i], vals[L, 1, i], vals[L, 2, i]))
            if len(pts) == 0:
                f.write(" \n")
