// Readers for the reference's direct-mode input files (see model.h).
#include "model.h"
#include "boxgrid.h"
#include "parallel.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace tdem {
namespace {

constexpr double kMu0Ref = 1.25663706143591729e-6;  // MU_0, CalcNonstat3DLine/vfem_const.h

std::string path(const Model& m, const char* name) { return m.dir + "/" + name; }

bool read_binary(const std::string& fn, void* dst, size_t bytes) {
  FILE* f = fopen(fn.c_str(), "rb");
  if (!f) return false;
  size_t got = fread(dst, 1, bytes, f);
  fclose(f);
  return got == bytes;
}

template <class T>
bool read_one(const std::string& fn, T& v) {
  std::ifstream in(fn);
  if (!in) return false;
  in >> v;
  return (bool)in;
}

}  // namespace

std::string load_model(const std::string& dir, Model& m) {
  m = Model();
  m.dir = dir;

  // --- materials: sig3d (index, sigma, sigma0), mu3d (index, mu, mu0) -----------
  {
    std::ifstream in(path(m, "sig3d"));
    if (!in) return "cannot open sig3d";
    int idx;
    double a, b;
    int nmat = 0;
    std::vector<std::array<double, 3>> rows;
    while (in >> idx >> a >> b) {
      nmat = std::max(nmat, idx);
      rows.push_back({(double)idx, a, b});
    }
    if (nmat <= 0) return "sig3d holds no materials";
    m.sigma.assign(nmat, 0.0);
    m.sigma0.assign(nmat, 0.0);
    // the reference reads exactly n_materials records in file order
    for (int i = 0; i < nmat && i < (int)rows.size(); ++i) {
      const int k = (int)rows[i][0] - 1;
      if (k < 0 || k >= nmat) return "sig3d: bad material index";
      m.sigma[k] = rows[i][1];
      m.sigma0[k] = rows[i][2];
    }
    std::ifstream mu(path(m, "mu3d"));
    if (!mu) return "cannot open mu3d";
    m.mu.assign(nmat, kMu0Ref);
    for (int i = 0; i < nmat; ++i) {
      double v0, v1;
      if (!(mu >> idx >> v0 >> v1)) return "mu3d: too few records";
      if (idx < 1 || idx > nmat) return "mu3d: bad material index";
      m.mu[idx - 1] = v0 * kMu0Ref;
    }
  }

  // --- receivers ---------------------------------------------------------------
  auto read_recv = [&](const char* name, std::vector<std::array<double, 3>>& out) -> std::string {
    std::ifstream in(path(m, name));
    if (!in) return std::string("cannot open ") + name;
    int n = 0;
    in >> n;
    if (!in || n < 0) return std::string("bad receiver count in ") + name;
    out.resize(n);
    for (int i = 0; i < n; ++i)
      if (!(in >> out[i][0] >> out[i][1] >> out[i][2])) return std::string("truncated ") + name;
    return "";
  };
  if (auto e = read_recv("xyzVectorB", m.rec_b); !e.empty()) return e;
  if (auto e = read_recv("xyzVectorE", m.rec_e); !e.empty()) return e;

  // --- inftry.dat ---------------------------------------------------------------
  {
    std::ifstream in(path(m, "inftry.dat"));
    if (!in) return "cannot open inftry.dat";
    std::string tok;
    while (in >> tok) {
      if (tok == "KUZLOV=") in >> m.n_nodes;
      else if (tok == "KPAR=") in >> m.n_elem;
      else if (tok == "KT1=") in >> m.n_bound_nodes;
    }
    if (m.n_nodes <= 0 || m.n_elem <= 0) return "inftry.dat: bad sizes";
  }
  {
    std::vector<int32_t> buf((size_t)m.n_elem * 14);
    if (!read_binary(path(m, "nver.dat"), buf.data(), buf.size() * 4)) return "cannot read nver.dat";
    m.nver.resize(m.n_elem);
    for (int e = 0; e < m.n_elem; ++e)
      for (int j = 0; j < 8; ++j) {
        const int v = buf[(size_t)e * 14 + j] - 1;
        if (v < 0 || v >= m.n_nodes) return "nver.dat: node index out of range";
        m.nver[e][j] = v;
      }
    std::vector<int32_t> mat(m.n_elem);
    if (!read_binary(path(m, "nvkat.dat"), mat.data(), mat.size() * 4)) return "cannot read nvkat.dat";
    m.nvkat.resize(m.n_elem);
    for (int e = 0; e < m.n_elem; ++e) {
      m.nvkat[e] = mat[e] - 1;
      if (m.nvkat[e] < 0 || m.nvkat[e] >= (int)m.sigma.size()) return "nvkat.dat: material out of range";
    }
    std::vector<double> xyz((size_t)m.n_nodes * 3);
    if (!read_binary(path(m, "xyz.dat"), xyz.data(), xyz.size() * 8)) return "cannot read xyz.dat";
    m.xyz.resize(m.n_nodes);
    for (int i = 0; i < m.n_nodes; ++i) m.xyz[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    std::vector<int32_t> l1(m.n_bound_nodes);
    if (!read_binary(path(m, "l13d.dat"), l1.data(), l1.size() * 4)) return "cannot read l13d.dat";
    m.l13d.resize(m.n_bound_nodes);
    for (int i = 0; i < m.n_bound_nodes; ++i) {
      m.l13d[i] = l1[i] - 1;
      if (m.l13d[i] < 0 || m.l13d[i] >= m.n_nodes) return "l13d.dat: node out of range";
    }
  }
  {
    int fd = 0;
    if (read_one(path(m, "fdirect"), fd)) m.fdirect = fd != 0;
  }

  // --- edges (time_approx.cpp:243-287) ---------------------------------------------
  {
    std::ifstream in(path(m, "tsize3d_.dat"));
    int j = 0;
    if (!(in >> j >> m.n_edges) || m.n_edges <= 0) return "tsize3d_.dat: bad edge count";
    std::vector<int32_t> nfe((size_t)m.n_edges * 2);
    if (!read_binary(path(m, "nodesforedges.dat"), nfe.data(), nfe.size() * 4))
      return "cannot read nodesforedges.dat";
    m.edge_nodes.resize(m.n_edges);
    for (int e = 0; e < m.n_edges; ++e) {
      m.edge_nodes[e] = {nfe[2 * e] - 1, nfe[2 * e + 1] - 1};
      if (m.edge_nodes[e][0] < 0 || m.edge_nodes[e][1] < 0 || m.edge_nodes[e][0] >= m.n_nodes ||
          m.edge_nodes[e][1] >= m.n_nodes)
        return "nodesforedges.dat: node out of range";
    }
    std::vector<int32_t> ed((size_t)m.n_elem * 25);
    if (!read_binary(path(m, "edges.dat"), ed.data(), ed.size() * 4)) return "cannot read edges.dat";
    m.ed.resize(m.n_elem);
    for (int e = 0; e < m.n_elem; ++e)
      for (int j = 0; j < 12; ++j) {
        const int v = ed[(size_t)e * 25 + j] - 1;
        if (v < 0 || v >= m.n_edges) return "edges.dat: edge index out of range";
        m.ed[e][j] = v;
      }
  }
  // Dirichlet edges: both end nodes on the boundary (T_Bound_Cond.cpp:58-89)
  {
    std::vector<char> bn(m.n_nodes, 0);
    for (int v : m.l13d) bn[v] = 1;
    m.edge_bound.assign(m.n_edges, 0);
    for (int e = 0; e < m.n_edges; ++e)
      m.edge_bound[e] = bn[m.edge_nodes[e][0]] && bn[m.edge_nodes[e][1]];
  }

  // --- anomalous edges of the primary-secondary mode (time_approx.cpp:351-368) -------
  {
    std::ifstream in(path(m, "mtrsizeforE0"));
    m.edge_anom.assign(m.n_edges, 0);
    m.n_anom = 0;
    if (in) {
      for (int e = 0; e < m.n_edges; ++e) {
        int k = 0;
        if (!(in >> k)) return "mtrsizeforE0: fewer flags than edges";
        m.edge_anom[e] = k != 0;
        m.n_anom += k != 0;
      }
    }
    std::ifstream pn(path(m, "PName"));
    if (pn) pn >> m.pname;
    // one anomaly of several (TaskSP.cpp:539-596): its index names the normal-field files
    int at = 0;
    m.anomal_type = read_one(path(m, "AnomalType"), at) ? at : 0;
    m.anomaly = -1;
    if (m.anomal_type) {
      std::ifstream ia(path(m, "ia"));
      if (!ia) return "cannot open ia (AnomalType is set)";
      ia >> m.anomaly;
    }
  }

  // --- time grid infite.0 (vec_prep_data.cpp:834-853) -----------------------------
  {
    std::ifstream in(path(m, "infite.0"));
    if (!in) return "cannot open infite.0";
    in.ignore(1000, '=');
    int nt = 0;
    in >> nt;
    if (!in || nt < 3) return "infite.0: bad time count";
    for (int k = 0; k < 4; ++k) in.ignore(1000, '\n');
    m.time.resize(nt);
    for (int i = 0; i < nt; ++i) {
      if (!in.good()) return "infite.0: truncated";
      in >> m.time[i];
      in.ignore(1000, ';');
    }
  }
  {
    std::ifstream in(path(m, "timeintervalforprint"));
    if (!(in >> m.print_left >> m.print_right)) return "cannot read timeintervalforprint";
  }

  // --- sources / receivers per source (TaskSP.cpp:467-535) --------------------------
  {
    std::ifstream in(path(m, "group"));
    if (!in) return "cannot open group";
    int ngrp = 0;
    in >> ngrp;
    m.npls = 0;
    for (int i = 0; i < ngrp; ++i) {
      int j, p1, p2;
      if (!(in >> j >> p1 >> p2)) return "group: truncated";
      m.npls += p2 - p1 + 1;
    }
    if (m.npls <= 0) return "group: no sources";
    auto read_ig = [&](const char* name, std::vector<int>& ig, int total) -> std::string {
      std::ifstream f(path(m, name));
      if (!f) return std::string("cannot open ") + name;
      ig.assign(m.npls + 1, 0);
      for (int i = 0; i < m.npls; ++i) {
        if (!(f >> ig[i + 1])) return std::string("truncated ") + name;
        ig[i + 1] += ig[i];
      }
      if (ig[m.npls] > total) return std::string(name) + " lists more receivers than the receiver file";
      return "";
    };
    if (auto e = read_ig("recvsb", m.rec_b_ig, (int)m.rec_b.size()); !e.empty()) return e;
    if (auto e = read_ig("recvse", m.rec_e_ig, (int)m.rec_e.size()); !e.empty()) return e;
  }
  {
    int nn = 0;
    if (read_one(path(m, "n_neib"), nn)) m.n_neib = nn;
  }

  // --- direct-mode source (vec_prep_data.cpp:982-1048) ------------------------------
  if (m.fdirect) {
    std::ifstream in(path(m, "currentfunction"));
    if (!in) return "cannot open currentfunction";
    m.currentfunction.assign(m.time.size(), 0.0);
    for (size_t i = 0; i < m.time.size(); ++i) {
      double t;
      in >> t >> m.currentfunction[i];
    }
    int ns = 0;
    if (read_one(path(m, "nSrsRazb"), ns)) m.n_srs_razb = ns;
    std::ifstream s(path(m, "sours"));
    if (!s) return "cannot open sours";
    m.wires.resize(m.npls);
    for (int i = 0; i < m.npls; ++i)
      for (int k = 0; k < 6; ++k)
        if (!(s >> m.wires[i][k])) return "sours: truncated";
  }
  return "";
}

std::string locate_dipoles(Model& m) {
  m.dipoles.assign(m.npls, {});
  if (!m.fdirect || m.n_srs_razb <= 0) return "";
  const int nd = m.n_srs_razb;
  struct P { double x, y, z; };
  std::vector<std::vector<P>> pos(m.npls);
  for (int i = 0; i < m.npls; ++i) {
    const auto& w = m.wires[i];
    const double dx = (w[3] - w[0]) / nd, dy = (w[4] - w[1]) / nd, dz = (w[5] - w[2]) / nd;
    m.dipoles[i].resize(nd);
    pos[i].resize(nd);
    for (int j = 0; j < nd; ++j) {
      pos[i][j] = {w[0] + (j + 0.5) * dx, w[1] + (j + 0.5) * dy, w[2] + (j + 0.5) * dz};
      m.dipoles[i][j].dx = dx;
      m.dipoles[i][j].dy = dy;
      m.dipoles[i][j].dz = dz;
    }
  }
  // every dipole goes to the first element (in element order) that holds it: the
  // elements whose box (+-1e-3) holds the dipole are all in its grid cell's list
  const double lo = -1e-2, hi = 1.0 + 1e-2;
  const int nall = m.npls * nd;
  auto local = [&](int e, const P& p, double l[3]) {
    const auto& p0 = m.xyz[m.nver[e][0]];
    const auto& p7 = m.xyz[m.nver[e][7]];
    // local coordinates on the axis-aligned brick spanned by nodes 0 and 7
    l[0] = (p.x - p0[0]) / (p7[0] - p0[0]);
    l[1] = (p.y - p0[1]) / (p7[1] - p0[1]);
    l[2] = (p.z - p0[2]) / (p7[2] - p0[2]);
  };
  std::vector<double> bmn(3 * (size_t)m.n_elem), bmx(3 * (size_t)m.n_elem);
  parallel_ranges(m.n_elem, [&](int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; ++e) {
      double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
      for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 3; ++a) {
          mn[a] = std::min(mn[a], m.xyz[m.nver[e][k]][a]);
          mx[a] = std::max(mx[a], m.xyz[m.nver[e][k]][a]);
        }
      for (int a = 0; a < 3; ++a) {
        bmn[3 * e + a] = mn[a] - 1e-3;
        bmx[3 * e + a] = mx[a] + 1e-3;
      }
    }
  });
  double qlo[3] = {INFINITY, INFINITY, INFINITY}, qhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const auto& w : pos)
    for (const P& p : w) {
      const double q[3] = {p.x, p.y, p.z};
      for (int a = 0; a < 3; ++a)
        if (!std::isnan(q[a])) {
          qlo[a] = std::min(qlo[a], q[a]);
          qhi[a] = std::max(qhi[a], q[a]);
        }
    }
  BoxGrid grid;
  grid.build(bmn, bmx, qlo, qhi);
  parallel_ranges(nall, [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
      const int i = (int)(k / nd), j = (int)(k % nd);
      const P& p = pos[i][j];
      const double q[3] = {p.x, p.y, p.z};
      const auto cand = grid.candidates(q);
      for (const int* c = cand.first; c != cand.second; ++c) {
        const int e = *c;
        const double* mn = &bmn[3 * (size_t)e];
        const double* mx = &bmx[3 * (size_t)e];
        if (p.x < mn[0] || p.x > mx[0] || p.y < mn[1] || p.y > mx[1] || p.z < mn[2] || p.z > mx[2]) continue;
        double l[3];
        local(e, p, l);
        if (!(l[0] > lo && l[0] < hi && l[1] > lo && l[1] < hi && l[2] > lo && l[2] < hi)) continue;
        Dipole& d = m.dipoles[i][j];
        d.elem = e;
        d.ksi = l[0];
        d.eta = l[1];
        d.zeta = l[2];
        break;
      }
    }
  }, 256);
  // A dipole that no element holds (outside the mesh) goes to the nearest element
  // (Vec_Prep_Data::GetNearestElement, vec_prep_data.cpp:878-980, called from :1186-1250):
  // of the 8 elements with the least L1 distance from the dipole to their node box
  // (ties in element order), the first with the least L1 distance of the dipole's local
  // coordinates from [0, 1]; the dipole keeps those local coordinates (outside [0, 1]).
  std::vector<int64_t> lost;
  for (int64_t k = 0; k < nall; ++k)
    if (m.dipoles[k / nd][k % nd].elem < 0) lost.push_back(k);
  if (!lost.empty() && m.n_elem == 0) return "source dipole outside the mesh";
  parallel_ranges((int64_t)lost.size(), [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
      const int i = (int)(lost[k] / nd), j = (int)(lost[k] % nd);
      const P& p = pos[i][j];
      const double q[3] = {p.x, p.y, p.z};
      const int n_best = std::min(8, m.n_elem);
      double sb[8];
      int eb[8];
      for (int b = 0; b < 8; ++b) {
        sb[b] = 1e30;
        eb[b] = -1;
      }
      double sbest = sb[7];
      for (int e = 0; e < m.n_elem; ++e) {
        double mn[3], mx[3];
        for (int a = 0; a < 3; ++a) mn[a] = mx[a] = m.xyz[m.nver[e][0]][a];
        for (int v = 1; v < 8; ++v)
          for (int a = 0; a < 3; ++a) {
            const double c = m.xyz[m.nver[e][v]][a];
            if (c < mn[a]) mn[a] = c;
            if (c > mx[a]) mx[a] = c;
          }
        double sc = 0.0;
        for (int a = 0; a < 3; ++a) sc += (q[a] < mn[a]) ? (mn[a] - q[a]) : (q[a] > mx[a]) ? (q[a] - mx[a]) : 0.0;
        if (!(sc < sbest)) continue;
        int b = 0;
        while (b < n_best && eb[b] != -1 && !(sc < sb[b])) ++b;
        for (int c = n_best - 1; c > b; --c) {
          eb[c] = eb[c - 1];
          sb[c] = sb[c - 1];
        }
        eb[b] = e;
        sb[b] = sc;
        sbest = sb[n_best - 1];
      }
      double lbest = 1e30;
      for (int b = 0; b < n_best && eb[b] != -1; ++b) {
        double l[3];
        local(eb[b], p, l);
        double sc = 0.0;
        for (int a = 0; a < 3; ++a) sc += (l[a] < 0.0) ? -l[a] : (l[a] > 1.0) ? (l[a] - 1.0) : 0.0;
        if (sc < lbest) {
          lbest = sc;
          Dipole& d = m.dipoles[i][j];
          d.elem = eb[b];
          d.ksi = l[0];
          d.eta = l[1];
          d.zeta = l[2];
        }
      }
    }
  }, 1);
  for (int i = 0; i < m.npls; ++i)
    for (int j = 0; j < nd; ++j)
      if (m.dipoles[i][j].elem < 0) return "source dipole outside the mesh";
  return "";
}

std::string load_initial_field(const Model& m, bool eform, std::vector<double>& u0) {
  return load_initial_field(m, m.dir, m.npls, eform, u0);
}

std::string load_initial_field(const Model& m, const std::string& dir, int npls, bool eform,
                               std::vector<double>& u0) {
  const size_t n = (size_t)m.n_edges, np = (size_t)npls;
  auto path = [&dir](const Model&, const char* name) { return dir + "/" + name; };
  u0.assign(n * np, 0.0);
  const std::string edge_file = path(m, eform ? "e0.edge" : "a0.edge");
  {
    FILE* f = fopen(edge_file.c_str(), "rb");
    if (f) {
      size_t got = fread(u0.data(), 8, u0.size(), f);
      fclose(f);
      if (got != u0.size()) return "truncated initial edge field";
      return "";
    }
  }
  const size_t nn = (size_t)m.n_nodes;
  if (!eform) {
    std::vector<double> a0(nn * 3 * np);
    if (!read_binary(path(m, "a0.dat"), a0.data(), a0.size() * 8)) return "cannot read a0.dat";
    // every (source, edge) value on its own: ranges of edges on host threads
    parallel_ranges((int64_t)n, [&](int64_t e0, int64_t e1) {
    for (size_t p = 0; p < np; ++p)
      for (size_t e = (size_t)e0; e < (size_t)e1; ++e) {
        const int v1 = m.edge_nodes[e][0], v2 = m.edge_nodes[e][1];
        double axis[3], mid[3], len2 = 0.0, dot = 0.0;
        for (int j = 0; j < 3; ++j) {
          axis[j] = m.xyz[v2][j] - m.xyz[v1][j];
          mid[j] = 0.5 * (a0[v1 * 3 + j + p * nn * 3] + a0[v2 * 3 + j + p * nn * 3]);
          len2 += axis[j] * axis[j];
          dot += mid[j] * axis[j];
        }
        const double len = std::sqrt(len2);
        u0[e + p * n] = dot / std::sqrt(len2) * len * 0.5;
      }
    });
  } else {
    std::vector<double> va(nn * np);
    if (!read_binary(path(m, "v3a.dat"), va.data(), va.size() * 8)) return "cannot read v3a.dat";
    parallel_ranges((int64_t)n, [&](int64_t e0, int64_t e1) {
    for (size_t p = 0; p < np; ++p)
      for (size_t e = (size_t)e0; e < (size_t)e1; ++e) {
        const int v1 = m.edge_nodes[e][0], v2 = m.edge_nodes[e][1];
        double len2 = 0.0;
        for (int j = 0; j < 3; ++j) {
          const double a = m.xyz[v2][j] - m.xyz[v1][j];
          len2 += a * a;
        }
        const double len = std::sqrt(len2);
        const double etan = -(va[v2 + p * nn] - va[v1 + p * nn]) / len;
        u0[e + p * n] = etan * len * 0.5;
      }
    });
  }
  return "";
}

std::string merge_models(const std::vector<Model>& parts, Model& out) {
  if (parts.empty()) return "no models to merge";
  const Model& a = parts[0];
  for (size_t i = 1; i < parts.size(); ++i) {
    const Model& b = parts[i];
    if (!a.fdirect || !b.fdirect) return "only direct-mode models are merged";
    if (b.n_nodes != a.n_nodes || b.n_elem != a.n_elem || b.n_edges != a.n_edges ||
        b.n_bound_nodes != a.n_bound_nodes || b.xyz != a.xyz || b.nver != a.nver || b.nvkat != a.nvkat ||
        b.l13d != a.l13d || b.ed != a.ed || b.edge_nodes != a.edge_nodes || b.edge_bound != a.edge_bound)
      return "the meshes differ";
    if (b.sigma != a.sigma || b.sigma0 != a.sigma0 || b.mu != a.mu) return "the materials differ";
    if (b.time != a.time || b.currentfunction != a.currentfunction || b.print_left != a.print_left ||
        b.print_right != a.print_right)
      return "the time grids differ";
    if (b.n_srs_razb != a.n_srs_razb || b.n_neib != a.n_neib || b.eps_reg != a.eps_reg)
      return "the source or receiver settings differ";
  }
  out = a;
  out.npls = 0;
  out.wires.clear();
  out.dipoles.clear();
  out.rec_b.clear();
  out.rec_e.clear();
  out.rec_b_ig.assign(1, 0);
  out.rec_e_ig.assign(1, 0);
  for (const Model& p : parts) {
    if ((int)p.rec_b_ig.size() != p.npls + 1 || (int)p.rec_e_ig.size() != p.npls + 1)
      return "receiver ranges missing";
    const int ob = (int)out.rec_b.size(), oe = (int)out.rec_e.size();
    out.wires.insert(out.wires.end(), p.wires.begin(), p.wires.end());
    out.rec_b.insert(out.rec_b.end(), p.rec_b.begin(), p.rec_b.end());
    out.rec_e.insert(out.rec_e.end(), p.rec_e.begin(), p.rec_e.end());
    for (int s = 1; s <= p.npls; ++s) {
      out.rec_b_ig.push_back(ob + p.rec_b_ig[s]);
      out.rec_e_ig.push_back(oe + p.rec_e_ig[s]);
    }
    out.npls += p.npls;
  }
  return "";
}

void edge_pattern(const Model& m, std::vector<int64_t>& rowptr, std::vector<int>& col) {
  const int n = m.n_edges;
  // elements of every edge (ascending), then each row gathers the 12 edges of each
  // of its elements (at most 4 x 12), sorts and deduplicates them
  std::vector<int64_t> eptr(n + 1, 0);
  for (int e = 0; e < m.n_elem; ++e)
    for (int i = 0; i < 12; ++i) ++eptr[m.ed[e][i] + 1];
  for (int i = 0; i < n; ++i) eptr[i + 1] += eptr[i];
  std::vector<int> elems(eptr[n]);
  {
    std::vector<int64_t> fill(eptr.begin(), eptr.end() - 1);
    for (int e = 0; e < m.n_elem; ++e)
      for (int i = 0; i < 12; ++i) elems[fill[m.ed[e][i]]++] = e;
  }
  // two passes over the rows, each range on its own thread with its own marks: the
  // distinct edges of each row are counted, then written in place and sorted (a row
  // holds at most 33 of its at most 48 gathered edges)
  const int nt = chunk_count(n, 4096);
  rowptr.assign(n + 1, 0);
  parallel_chunks(n, nt, [&](int, int64_t r0, int64_t r1) {
    std::vector<int> seen(n, -1);  // row that last listed each edge
    for (int64_t i = r0; i < r1; ++i) {
      int64_t c = 0;
      for (int64_t q = eptr[i]; q < eptr[i + 1]; ++q)
        for (int j = 0; j < 12; ++j) {
          const int e = m.ed[elems[q]][j];
          if (seen[e] != (int)i) {
            seen[e] = (int)i;
            ++c;
          }
        }
      rowptr[i + 1] = c;
    }
  });
  for (int i = 0; i < n; ++i) rowptr[i + 1] += rowptr[i];
  col.resize(rowptr[n]);
  parallel_chunks(n, nt, [&](int, int64_t r0, int64_t r1) {
    std::vector<int> seen(n, -1);
    for (int64_t i = r0; i < r1; ++i) {
      int* out = col.data() + rowptr[i];
      int c = 0;
      for (int64_t q = eptr[i]; q < eptr[i + 1]; ++q)
        for (int j = 0; j < 12; ++j) {
          const int e = m.ed[elems[q]][j];
          if (seen[e] != (int)i) {
            seen[e] = (int)i;
            int y = c++;
            for (; y > 0 && out[y - 1] > e; --y) out[y] = out[y - 1];
            out[y] = e;
          }
        }
    }
  });
}

std::string init_normal_field(const Model& m, bool eform, NormalField& nf) {
  nf = NormalField();
  auto length = [&](int i) {
    const auto& a = m.xyz[m.edge_nodes[i][0]];
    const auto& b = m.xyz[m.edge_nodes[i][1]];
    const double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
    return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  };
  for (int i = 0; i < m.n_edges; ++i)
    if (m.edge_anom[i]) {
      nf.idx.push_back(i);
      nf.len.push_back(length(i));
    }
  if (!eform) return "";
  const size_t nv = (size_t)m.n_nodes * m.npls;
  std::vector<double> V(nv);
  if (!read_binary(path(m, "v3n.dat"), V.data(), nv * sizeof(double)))
    return "cannot read v3n.dat (the normal potential, layer 0 of the normal field)";
  nf.e0.assign((size_t)m.n_edges * m.npls, 0.0);
  for (int p = 0; p < m.npls; ++p)
    for (int i = 0; i < m.n_edges; ++i) {
      const int v1 = m.edge_nodes[i][0], v2 = m.edge_nodes[i][1];
      const double len = length(i);
      const double etan = -(V[v2 + (size_t)p * m.n_nodes] - V[v1 + (size_t)p * m.n_nodes]) / len;
      nf.e0[i + (size_t)p * m.n_edges] = etan * len * 0.5;
    }
  return "";
}

std::string normal_field_file(const Model& m, int layer) {
  char num[48];
  if (m.anomal_type)
    std::snprintf(num, sizeof num, "%04d_%d", layer, m.anomaly);
  else
    std::snprintf(num, sizeof num, "%04d", layer);
  return m.dir + "/m" + m.pname + ".enor." + num;
}

std::string normal_field_layer(const Model& m, const NormalField& nf, int layer, std::vector<double>& out) {
  const size_t n = (size_t)m.n_edges;
  if (layer == 0 && !nf.e0.empty()) {
    out = nf.e0;
    return "";
  }
  out.assign(n * m.npls, 0.0);
  const std::string name = normal_field_file(m, layer);
  FILE* f = std::fopen(name.c_str(), "rb");
  if (!f) return std::string("cannot open the normal field ") + name;
  std::vector<float> v(nf.idx.size() * (size_t)m.npls);
  const size_t got = std::fread(v.data(), sizeof(float), v.size(), f);
  std::fclose(f);
  if (got != v.size()) return std::string("normal field too short: ") + name;
  for (int p = 0; p < m.npls; ++p)
    for (size_t k = 0; k < nf.idx.size(); ++k)
      out[nf.idx[k] + (size_t)p * n] = v[k + (size_t)p * nf.idx.size()] * nf.len[k] * 0.5;
  return "";
}

std::string normal_field_rate(const Model& m, const NormalField& nf, int it, int t1, int t2, bool three_point,
                              std::vector<double>& out) {
  std::vector<double> e1, e2;
  std::string e = normal_field_layer(m, nf, it, out);
  if (e.empty()) e = normal_field_layer(m, nf, t1, e1);
  if (!e.empty()) return e;
  const std::vector<double>& t = m.time;
  if (!three_point) {
    for (size_t j = 0; j < out.size(); ++j) out[j] = -(out[j] - e1[j]) / (t[it] - t[t1]);
    return "";
  }
  if (!(e = normal_field_layer(m, nf, t2, e2)).empty()) return e;
  const double tj = t[it], tj1 = t[t1], tj2 = t[t2], tt = t[it];
  const double dt = tj - tj2, dt0 = tj - tj1, dt1 = tj1 - tj2;
  for (size_t j = 0; j < out.size(); ++j)
    out[j] = -(e2[j] * (2.0 * tt - tj - tj1) / (dt1 * dt) - e1[j] * (2.0 * tt - tj - tj2) / (dt1 * dt0) +
               out[j] * (2.0 * tt - tj1 - tj2) / (dt * dt0));
  return "";
}

std::string element_colouring(const Model& m, std::vector<int>& order, std::vector<int>& cstart) {
  const int ne = m.n_elem, n = m.n_edges;
  // elements of every edge, ascending (CSR)
  std::vector<int64_t> ptr(n + 1, 0);
  for (int el = 0; el < ne; ++el)
    for (int j = 0; j < 12; ++j) ++ptr[m.ed[el][j] + 1];
  for (int i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
  std::vector<int> elems(ptr[n]);
  {
    std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
    for (int el = 0; el < ne; ++el)
      for (int j = 0; j < 12; ++j) elems[fill[m.ed[el][j]]++] = el;
  }
  std::vector<int> color(ne, -1);
  int ncol = 0;
  for (int el = 0; el < ne; ++el) {
    uint64_t used = 0;
    for (int j = 0; j < 12; ++j) {
      const int ed = m.ed[el][j];
      for (int64_t q = ptr[ed]; q < ptr[ed + 1]; ++q) {
        const int c = color[elems[q]];
        if (c >= 0 && c < 64) used |= (1ull << c);
      }
    }
    int c = 0;
    while (c < 64 && (used >> c & 1)) ++c;
    if (c >= 64) return "element colouring needs more than 64 colours";
    color[el] = c;
    ncol = std::max(ncol, c + 1);
  }
  // counting sort by colour keeps the elements ascending inside a colour
  cstart.assign(ncol + 1, 0);
  for (int el = 0; el < ne; ++el) ++cstart[color[el] + 1];
  for (int c = 0; c < ncol; ++c) cstart[c + 1] += cstart[c];
  order.assign(ne, 0);
  std::vector<int> at(cstart.begin(), cstart.end() - 1);
  for (int el = 0; el < ne; ++el) order[at[color[el]]++] = el;
  return "";
}

}  // namespace tdem
