// Grounded-wire stationary initial field (see stationary.h).  Host code builds
// the nodal systems and right-hand sides; both factorizations and all solves run
// on the GPU through the multifrontal Cholesky.
#include "stationary.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <vector>

#include "boxgrid.h"
#include "gpu_cholesky.h"
#include "parallel.h"
#include "symbolic.h"

namespace tdem {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMu0Stat = 4e-7 * kPi;  // MU0 of CalcStat3D_3T_A/TaskSP.h:57-58
constexpr double kPenalty = 1e30;        // boundary-node diagonal (TaskSP.cpp:1191-1221)

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool read_binary(const std::string& fn, void* dst, size_t bytes) {
  FILE* f = fopen(fn.c_str(), "rb");
  if (!f) return false;
  const size_t got = fread(dst, 1, bytes, f);
  fclose(f);
  return got == bytes;
}

struct StatModel {
  int kpnt = 0, krect = 0, kt1 = 0;
  std::vector<std::array<double, 3>> xyz;
  std::vector<std::array<int, 8>> nodes;  // 0-based
  std::vector<int> mtr;                   // material number as in nvkat.dat (1 = air)
  std::vector<int> l1;                    // boundary nodes, 0-based
  std::vector<double> sig;                // by material number
  int npls = 0;
  std::vector<std::array<double, 6>> wires;
  int nsrs = 500;
  double cur = 1.0;
};

// Mesh3DForVP::Read (TaskSP.h:750-830), GetNumberOfPlaces (TaskSP.cpp:1318-1342),
// the sours / nSrsRazb / ImpStatCur reads of SolveStationarProblem3d (:1647-1711).
std::string read_model(const std::string& dir, StatModel& m) {
  auto path = [&](const char* n) { return dir + "/" + n; };
  {
    std::ifstream in(path("inftry.dat"));
    if (!in) return "cannot open inftry.dat";
    in.ignore(1000, '\n');
    in.ignore(1000, '=');
    in >> m.kpnt;
    in.ignore(1000, '=');
    in >> m.krect;
    in.ignore(1000, '=');
    in >> m.kt1;
    if (!in || m.kpnt <= 0 || m.krect <= 0 || m.kt1 < 0) return "inftry.dat: bad sizes";
  }
  {
    std::vector<double> b((size_t)m.kpnt * 3);
    if (!read_binary(path("xyz.dat"), b.data(), b.size() * 8)) return "cannot read xyz.dat";
    m.xyz.resize(m.kpnt);
    for (int i = 0; i < m.kpnt; ++i) m.xyz[i] = {b[3 * i], b[3 * i + 1], b[3 * i + 2]};
  }
  {
    std::vector<int32_t> b((size_t)m.krect * 14);
    if (!read_binary(path("nver.dat"), b.data(), b.size() * 4)) return "cannot read nver.dat";
    m.nodes.resize(m.krect);
    for (int e = 0; e < m.krect; ++e)
      for (int j = 0; j < 8; ++j) {
        const int v = b[(size_t)e * 14 + j] - 1;
        if (v < 0 || v >= m.kpnt) return "nver.dat: node index out of range";
        m.nodes[e][j] = v;
      }
    m.mtr.resize(m.krect);
    if (!read_binary(path("nvkat.dat"), m.mtr.data(), m.mtr.size() * 4)) return "cannot read nvkat.dat";
    std::vector<int32_t> l(m.kt1);
    if (m.kt1 && !read_binary(path("l13d.dat"), l.data(), l.size() * 4)) return "cannot read l13d.dat";
    for (int v : l)
      if (v >= 1 && v <= m.kpnt) m.l1.push_back(v - 1);
  }
  {
    std::ifstream in(path("sig3d"));
    if (!in) return "cannot open sig3d";
    int i;
    double v, v0;
    while (in >> i >> v >> v0) {
      if (i < 0 || i > 100000) return "sig3d: bad material index";
      if ((int)m.sig.size() <= i) m.sig.resize(i + 1, 0.0);
      m.sig[i] = v;
    }
    for (int e = 0; e < m.krect; ++e)
      if (m.mtr[e] < 0 || m.mtr[e] >= (int)m.sig.size()) return "nvkat.dat: material missing from sig3d";
  }
  {
    std::ifstream in(path("group"));
    if (!in) return "cannot open group";
    int nprof = 0;
    in >> nprof;
    for (int i = 0; i < nprof; ++i) {
      int k, p1, p2;
      if (!(in >> k >> p1 >> p2)) return "group: truncated";
      m.npls += p2 - p1 + 1;
    }
    if (m.npls <= 0) return "group: no sources";
  }
  {
    std::ifstream in(path("sours"));
    if (!in) return "cannot open sours";
    m.wires.resize(m.npls);
    for (auto& w : m.wires)
      for (double& c : w)
        if (!(in >> c)) return "sours: truncated";
  }
  {
    std::ifstream in(path("nSrsRazb"));
    if (in) in >> m.nsrs;
    if (m.nsrs <= 0) return "nSrsRazb must be positive";
    std::ifstream ic(path("ImpStatCur"));
    if (ic) ic >> m.cur;
  }
  return "";
}

struct PointSource {
  int elem = -1;
  double x = 0, y = 0, z = 0;     // position
  double dx = 0, dy = 0, dz = 0;  // dipole vector (zero for electrodes)
  double l[3] = {0, 0, 0};        // local coordinates in elem
};

// Local coordinates of p in the axis-aligned brick spanned by nodes 0 and 7
// (the trilinear map CheckInHex inverts, CheckInHex.cpp:195).
void local_coords(const StatModel& m, int e, const PointSource& p, double l[3]) {
  const auto& a = m.xyz[m.nodes[e][0]];
  const auto& b = m.xyz[m.nodes[e][7]];
  l[0] = (p.x - a[0]) / (b[0] - a[0]);
  l[1] = (p.y - a[1]) / (b[1] - a[1]);
  l[2] = (p.z - a[2]) / (b[2] - a[2]);
}

void bbox(const StatModel& m, int e, double mn[3], double mx[3]) {
  for (int c = 0; c < 3; ++c) {
    mn[c] = 1e300;
    mx[c] = -1e300;
  }
  for (int k = 0; k < 8; ++k)
    for (int c = 0; c < 3; ++c) {
      mn[c] = std::min(mn[c], m.xyz[m.nodes[e][k]][c]);
      mx[c] = std::max(mx[c], m.xyz[m.nodes[e][k]][c]);
    }
}

// First earth element (file order) whose box (+-1e-3) holds the point with local
// coordinates in (-0.01, 1.01) (TaskSP.cpp:1745-1942, CheckAndGet :1361-1377);
// otherwise the nearest earth element (GetNearestElement, :1379-1474).  The first
// search looks only at the earth elements listed in the point's cell of a grid of the
// boxes (BoxGrid: every box holding the point is listed there, in element order), the
// points on host threads.
std::string locate(const StatModel& m, std::vector<PointSource*>& pts) {
  const double lo = -1e-2, hi = 1.0 + 1e-2;
  std::vector<double> bmn(3 * (size_t)m.krect), bmx(3 * (size_t)m.krect);
  parallel_ranges(m.krect, [&](int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; ++e) {
      double mn[3], mx[3];
      bbox(m, (int)e, mn, mx);
      for (int c = 0; c < 3; ++c) {
        // air elements are never candidates: an empty box is not listed
        bmn[3 * e + c] = m.mtr[e] == 1 ? 1.0 : mn[c] - 1e-3;
        bmx[3 * e + c] = m.mtr[e] == 1 ? 0.0 : mx[c] + 1e-3;
      }
    }
  });
  double qlo[3] = {INFINITY, INFINITY, INFINITY}, qhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const PointSource* p : pts) {
    const double q[3] = {p->x, p->y, p->z};
    for (int c = 0; c < 3; ++c)
      if (!std::isnan(q[c])) {
        qlo[c] = std::min(qlo[c], q[c]);
        qhi[c] = std::max(qhi[c], q[c]);
      }
  }
  BoxGrid grid;
  grid.build(bmn, bmx, qlo, qhi);
  parallel_ranges((int64_t)pts.size(), [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
      PointSource* p = pts[k];
      if (p->elem != -1) continue;
      const double q[3] = {p->x, p->y, p->z};
      const auto cand = grid.candidates(q);
      for (const int* c = cand.first; c != cand.second; ++c) {
        const int e = *c;
        const double* mn = &bmn[3 * (size_t)e];
        const double* mx = &bmx[3 * (size_t)e];
        if (p->x < mn[0] || p->x > mx[0] || p->y < mn[1] || p->y > mx[1] || p->z < mn[2] || p->z > mx[2]) continue;
        double l[3];
        local_coords(m, e, *p, l);
        if (l[0] > lo && l[0] < hi && l[1] > lo && l[1] < hi && l[2] > lo && l[2] < hi) {
          p->elem = e;
          std::copy(l, l + 3, p->l);
          break;
        }
      }
    }
  }, 256);
  for (PointSource* p : pts) {
    if (p->elem != -1) continue;
    // 8 nearest earth elements by L1 distance to their boxes, then the one whose
    // local coordinates leave [0, 1] least
    std::vector<std::pair<double, int>> best;
    for (int e = 0; e < m.krect; ++e) {
      if (m.mtr[e] == 1) continue;
      double mn[3], mx[3];
      bbox(m, e, mn, mx);
      const double q[3] = {p->x, p->y, p->z};
      double d = 0;
      for (int c = 0; c < 3; ++c) d += (q[c] < mn[c]) ? mn[c] - q[c] : (q[c] > mx[c]) ? q[c] - mx[c] : 0.0;
      best.push_back({d, e});
    }
    const size_t nb = std::min<size_t>(8, best.size());
    std::stable_sort(best.begin(), best.end(),
                     [](const std::pair<double, int>& a, const std::pair<double, int>& b) { return a.first < b.first; });
    double sb = 1e30;
    for (size_t i = 0; i < nb; ++i) {
      double l[3];
      local_coords(m, best[i].second, *p, l);
      double s = 0;
      for (int c = 0; c < 3; ++c) s += (l[c] < 0.0) ? -l[c] : (l[c] > 1.0) ? l[c] - 1.0 : 0.0;
      if (s < sb) {
        sb = s;
        p->elem = best[i].second;
        std::copy(l, l + 3, p->l);
      }
    }
    if (p->elem == -1) return "no element found for a source point";
  }
  return "";
}

// Trilinear basis, node i = ix + 2 iy + 4 iz (CheckInHex.cpp:64-79).
double phi(int i, const double l[3]) {
  const double fx = (i & 1) ? l[0] : 1.0 - l[0];
  const double fy = (i & 2) ? l[1] : 1.0 - l[1];
  const double fz = (i & 4) ? l[2] : 1.0 - l[2];
  return fx * fy * fz;
}

// Element stiffness: integral of grad phi_i . grad phi_j over an hx x hy x hz brick
// (GetStiffnessMatrixForRect3D, localcontributionsrect3d.cpp:49-81).
void stiffness(double hx, double hy, double hz, double K[8][8]) {
  const double G[2][2] = {{1, -1}, {-1, 1}}, M[2][2] = {{2, 1}, {1, 2}};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      const int ix = i & 1, iy = (i >> 1) & 1, iz = i >> 2, jx = j & 1, jy = (j >> 1) & 1, jz = j >> 2;
      K[i][j] = (G[ix][jx] * M[iy][jy] * M[iz][jz] * hy * hz / hx + M[ix][jx] * G[iy][jy] * M[iz][jz] * hx * hz / hy +
                 M[ix][jx] * M[iy][jy] * G[iz][jz] * hx * hy / hz) /
                36.0;
    }
}

// D_c[i][j] = integral of (d phi_i / dc) phi_j (GradMatrix_X/Y/Z,
// localcontributionsrect3d.cpp:300-386): the 1D factors are +-1/2 along c and
// h/3, h/6 across.
void grad_matrix(int c, double hx, double hy, double hz, double D[8][8]) {
  const double h[3] = {hx, hy, hz};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      double v = 1.0;
      for (int a = 0; a < 3; ++a) {
        const int bi = (i >> a) & 1, bj = (j >> a) & 1;
        if (a == c) v *= bi ? 0.5 : -0.5;
        else v *= (bi == bj ? h[a] / 3.0 : h[a] / 6.0);
      }
      D[i][j] = v;
    }
}

struct NodalPattern {
  std::vector<int64_t> rowptr;  // full symmetric CSR
  std::vector<int> col;
  std::vector<int64_t> lrowptr;  // lower triangle (col <= row)
  std::vector<int> lcol;
  std::vector<int64_t> lsrc;     // full-CSR index of each lower entry
};

void build_pattern(const StatModel& m, NodalPattern& p) {
  const int n = m.kpnt;
  std::vector<std::vector<int>> nb(n);
  for (const auto& el : m.nodes)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) nb[el[a]].push_back(el[b]);
  p.rowptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    auto& r = nb[i];
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    p.rowptr[i + 1] = p.rowptr[i] + (int64_t)r.size();
  }
  p.col.resize(p.rowptr[n]);
  p.lrowptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    std::copy(nb[i].begin(), nb[i].end(), p.col.begin() + p.rowptr[i]);
    for (int64_t q = p.rowptr[i]; q < p.rowptr[i + 1]; ++q)
      if (p.col[q] <= i) {
        p.lcol.push_back(p.col[q]);
        p.lsrc.push_back(q);
      }
    p.lrowptr[i + 1] = (int64_t)p.lcol.size();
    std::vector<int>().swap(nb[i]);
  }
}

inline int64_t slot(const NodalPattern& p, int i, int j) {
  const int* b = p.col.data() + p.rowptr[i];
  const int* e = p.col.data() + p.rowptr[i + 1];
  return p.rowptr[i] + (std::lower_bound(b, e, j) - b);
}

#define STAT_CUDA(x)                                                              \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) return std::string("CUDA: " #x ": ") + cudaGetErrorString(e_); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

bool write_file(const std::string& fn, const double* v, size_t count, bool append) {
  FILE* f = fopen(fn.c_str(), append ? "ab" : "wb");
  if (!f) return false;
  const bool ok = fwrite(v, sizeof(double), count, f) == count;
  return fclose(f) == 0 && ok;
}

// per wire its nSrsRazb dipoles, then electrodes A and B (pts in that order)
void source_points(const StatModel& m, std::vector<std::vector<PointSource>>& dip, std::vector<PointSource>& elA,
                   std::vector<PointSource>& elB, std::vector<PointSource*>& pts) {
  const int npls = m.npls;
  dip.assign(npls, std::vector<PointSource>(m.nsrs));
  elA.assign(npls, PointSource());
  elB.assign(npls, PointSource());
  pts.clear();
  for (int i = 0; i < npls; ++i) {
    const auto& w = m.wires[i];
    const double d[3] = {(w[3] - w[0]) / m.nsrs, (w[4] - w[1]) / m.nsrs, (w[5] - w[2]) / m.nsrs};
    for (int j = 0; j < m.nsrs; ++j) {
      PointSource& s = dip[i][j];
      s.x = w[0] + (j + 0.5) * d[0];
      s.y = w[1] + (j + 0.5) * d[1];
      s.z = w[2] + (j + 0.5) * d[2];
      s.dx = d[0];
      s.dy = d[1];
      s.dz = d[2];
      pts.push_back(&s);
    }
    elA[i].x = w[0], elA[i].y = w[1], elA[i].z = w[2];
    elB[i].x = w[3], elB[i].y = w[4], elB[i].z = w[5];
    pts.push_back(&elA[i]);
    pts.push_back(&elB[i]);
  }
}

}  // namespace

std::string stationary_source_points(const std::string& dir, std::vector<std::array<double, 4>>& out) {
  StatModel m;
  std::string e = read_model(dir, m);
  if (!e.empty()) return e;
  std::vector<std::vector<PointSource>> dip;
  std::vector<PointSource> elA, elB;
  std::vector<PointSource*> pts;
  source_points(m, dip, elA, elB, pts);
  if (!(e = locate(m, pts)).empty()) return e;
  out.clear();
  for (const PointSource* p : pts) out.push_back({(double)p->elem, p->l[0], p->l[1], p->l[2]});
  return "";
}

std::string solve_stationary(const std::string& dir, int device, StationaryTimes* times) {
  const double t0 = now_s();
  StatModel m;
  std::string e = read_model(dir, m);
  if (!e.empty()) return e;
  const int n = m.kpnt, npls = m.npls;

  // sources: nSrsRazb dipoles per wire and the two electrodes
  std::vector<std::vector<PointSource>> dip;
  std::vector<PointSource> elA, elB;
  std::vector<PointSource*> pts;
  source_points(m, dip, elA, elB, pts);
  if (!(e = locate(m, pts)).empty()) return e;

  NodalPattern pat;
  build_pattern(m, pat);
  const int64_t nnz = (int64_t)pat.col.size();

  // V system: sigma * stiffness, electrodes -I at A, +I at B
  std::vector<double> K(nnz, 0.0), F((size_t)n * npls, 0.0);
  std::vector<std::array<double, 3>> hs(m.krect);
  for (int el = 0; el < m.krect; ++el) {
    const auto& a = m.xyz[m.nodes[el][0]];
    const auto& b = m.xyz[m.nodes[el][7]];
    hs[el] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double S[8][8];
    stiffness(hs[el][0], hs[el][1], hs[el][2], S);
    const double sg = m.sig[m.mtr[el]];
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) K[slot(pat, m.nodes[el][i], m.nodes[el][j])] += sg * S[i][j];
  }
  for (int p = 0; p < npls; ++p) {
    for (int s = 0; s < 2; ++s) {
      const PointSource& q = s ? elB[p] : elA[p];
      const double c = (s ? 1.0 : -1.0) * m.cur;
      for (int i = 0; i < 8; ++i) F[(size_t)p * n + m.nodes[q.elem][i]] += phi(i, q.l) * c;
    }
  }
  std::vector<int64_t> diag(n);
  for (int i = 0; i < n; ++i) diag[i] = slot(pat, i, i);
  std::vector<double> Kv = K;
  for (int i = 0; i < n; ++i)
    if (std::fabs(Kv[diag[i]]) < 1e-30) {
      Kv[diag[i]] = kPenalty;
      for (int p = 0; p < npls; ++p) F[(size_t)p * n + i] = 0.0;
    }
  for (int v : m.l1) {
    Kv[diag[v]] = kPenalty;
    for (int p = 0; p < npls; ++p) F[(size_t)p * n + v] = 0.0;
  }

  // GPU factorization of the nodal pattern (node positions drive the dissection)
  std::vector<double> xyz((size_t)n * 3);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) xyz[3 * (size_t)i + c] = m.xyz[i][c];
  Symbolic sy;
  e = analyse(n, pat.lrowptr.data(), pat.lcol.data(), xyz.data(), sy);
  if (!e.empty()) return "stationary analysis: " + e;
  const long long nnz_l = sy.nnz_l;
  std::vector<int> p2v(n);
  for (int q = 0; q < n; ++q) p2v[q] = sy.iperm[q];
  STAT_CUDA(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  STAT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> st_guard(st, [](cudaStream_t s) { cudaStreamDestroy(s); });
  const int nrhs_max = std::min(kMaxRhs, 3 * npls);
  GpuCholesky chol;
  if (!(e = chol.setup(std::move(sy), p2v, nrhs_max, st, 8)).empty()) return e;
  const int64_t nl = (int64_t)pat.lcol.size();
  DevBuf dv, db, dx;
  STAT_CUDA(cudaMalloc(&dv.p, sizeof(double) * nl));
  STAT_CUDA(cudaMalloc(&db.p, sizeof(double) * (size_t)n * 3 * npls));
  STAT_CUDA(cudaMalloc(&dx.p, sizeof(double) * (size_t)n * 3 * npls));
  cudaEvent_t ev[4];
  for (auto& x : ev) STAT_CUDA(cudaEventCreate(&x));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]);
    }
  } evg{ev};
  std::vector<double> lv(nl);
  auto factor = [&](const std::vector<double>& full) -> std::string {
    for (int64_t q = 0; q < nl; ++q) lv[q] = full[pat.lsrc[q]];
    STAT_CUDA(cudaMemcpyAsync(dv.p, lv.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, st));
    chol.factor((const double*)dv.p, st);
    STAT_CUDA(cudaGetLastError());
    return "";
  };
  auto solve = [&](const std::vector<double>& rhs, int ncol, std::vector<double>& out) -> std::string {
    STAT_CUDA(cudaMemcpyAsync(db.p, rhs.data(), sizeof(double) * (size_t)n * ncol, cudaMemcpyHostToDevice, st));
    for (int c0 = 0; c0 < ncol; c0 += nrhs_max) {
      const int nc = std::min(nrhs_max, ncol - c0);
      chol.solve((const double*)db.p + (size_t)c0 * n, (double*)dx.p + (size_t)c0 * n, n, nc, st);
    }
    STAT_CUDA(cudaGetLastError());
    out.resize((size_t)n * ncol);
    STAT_CUDA(cudaMemcpyAsync(out.data(), dx.p, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, st));
    return "";
  };
  const double t_setup = now_s() - t0;

  std::vector<double> V;
  STAT_CUDA(cudaEventRecord(ev[0], st));
  if (!(e = factor(Kv)).empty()) return e;
  STAT_CUDA(cudaEventRecord(ev[1], st));
  if (!(e = solve(F, npls, V)).empty()) return e;
  STAT_CUDA(cudaEventRecord(ev[2], st));
  STAT_CUDA(cudaStreamSynchronize(st));
  if (const int bad = chol.status(st)) return "stationary V system: non-positive pivot at column " + std::to_string(bad);

  // A0 system: stiffness / mu0; right-hand sides -sigma grad V and the dipoles
  std::vector<double> Ka(nnz, 0.0);
  for (int el = 0; el < m.krect; ++el) {
    double S[8][8];
    stiffness(hs[el][0], hs[el][1], hs[el][2], S);
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) Ka[slot(pat, m.nodes[el][i], m.nodes[el][j])] += S[i][j] / kMu0Stat;
  }
  for (int v : m.l1) Ka[diag[v]] = kPenalty;
  std::vector<double> F3((size_t)n * 3 * npls, 0.0);
  for (int c = 0; c < 3; ++c)
    for (int p = 0; p < npls; ++p) {
      double* f = F3.data() + ((size_t)c * npls + p) * n;
      const double* vp = V.data() + (size_t)p * n;
      for (int el = 0; el < m.krect; ++el) {
        double D[8][8];
        grad_matrix(c, hs[el][0], hs[el][1], hs[el][2], D);
        const double sg = m.sig[m.mtr[el]];
        for (int i = 0; i < 8; ++i) {
          double s = 0.0;
          for (int j = 0; j < 8; ++j) s += sg * D[j][i] * vp[m.nodes[el][j]];
          f[m.nodes[el][i]] -= s;
        }
      }
      for (const PointSource& q : dip[p]) {
        const double val = (c == 0 ? q.dx : c == 1 ? q.dy : q.dz) * m.cur;
        for (int i = 0; i < 8; ++i) f[m.nodes[q.elem][i]] += phi(i, q.l) * val;
      }
      for (int v : m.l1) f[v] = 0.0;
    }
  std::vector<double> U;
  STAT_CUDA(cudaEventRecord(ev[0], st));
  if (!(e = factor(Ka)).empty()) return e;
  STAT_CUDA(cudaEventRecord(ev[3], st));
  if (!(e = solve(F3, 3 * npls, U)).empty()) return e;
  STAT_CUDA(cudaEventRecord(ev[2], st));
  STAT_CUDA(cudaStreamSynchronize(st));
  if (const int bad = chol.status(st)) return "stationary A0 system: non-positive pivot at column " + std::to_string(bad);
  if (chol.solve_status(st)) return "CUDA: a wait of the level triangular solves gave up";

  // outputs (TaskSP.cpp:1990-2012, 2148-2175)
  std::vector<double> zeros(n, 0.0), a0((size_t)n * 3);
  for (int p = 0; p < npls; ++p) {
    if (!write_file(dir + "/v3n.dat", zeros.data(), n, p > 0)) return "cannot write v3n.dat";
    if (!write_file(dir + "/v3a.dat", V.data() + (size_t)p * n, n, p > 0)) return "cannot write v3a.dat";
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) a0[3 * (size_t)i + c] = U[((size_t)c * npls + p) * n + i];
    if (!write_file(dir + "/a0.dat", a0.data(), a0.size(), p > 0)) return "cannot write a0.dat";
  }
  if (times) {
    float ms = 0.f;
    times->setup_s = t_setup;
    cudaEventElapsedTime(&ms, ev[0], ev[3]);
    times->factor_gpu_ms = ms;
    cudaEventElapsedTime(&ms, ev[3], ev[2]);
    times->solve_gpu_ms = ms;
    times->total_s = now_s() - t0;
    times->n_nodes = n;
    times->n_sources = npls;
    times->nnz_factor = nnz_l;
  }
  return "";
}

}  // namespace tdem
