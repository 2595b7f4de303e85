// Receiver operator precomputation (see receivers.h).
#include "receivers.h"

#include <algorithm>
#include <atomic>
#include <cmath>

#include "boxgrid.h"
#include "parallel.h"

namespace tdem {
namespace {

// Nodal trilinear mass matrix of a brick: V * {1/27, 1/54, 1/108, 1/216} by the
// number of coordinate bits in which the two local nodes differ
// (Hex_Local_Matrix.cpp:87-165).
void nodal_mass(double hx, double hy, double hz, double b[8][8]) {
  const double t2 = hx * hy * hz;
  const double v[4] = {t2 / 27.0, t2 / 54.0, t2 / 108.0, t2 / 216.0};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) b[i][j] = v[__builtin_popcount(i ^ j)];
}

// Centre-value coefficients of local edge l for component comp.
double centre_coef(bool curl, int comp, int l, double hx, double hy, double hz) {
  const int dir = l >> 2, a = l & 1, bb = (l >> 1) & 1;
  const double sa = a ? 1.0 : -1.0, sb = bb ? 1.0 : -1.0;
  if (!curl) {
    if (dir != comp) return 0.0;
    const double h = (dir == 0) ? hx : (dir == 1) ? hy : hz;
    return 0.25 * 2.0 / h;
  }
  // curl of the edge basis at the element centre
  if (dir == 0) {  // x-edge, sides (y: a, z: b)
    if (comp == 1) return sb / (hx * hz);
    if (comp == 2) return -sa / (hx * hy);
    return 0.0;
  }
  if (dir == 1) {  // y-edge, sides (z: a, x: b)
    if (comp == 0) return -sa / (hy * hz);
    if (comp == 2) return sb / (hx * hy);
    return 0.0;
  }
  // z-edge, sides (x: a, y: b)
  if (comp == 0) return sb / (hy * hz);
  if (comp == 1) return -sa / (hx * hz);
  return 0.0;
}

struct Sub {
  std::vector<int> elems;     // global element ids (increasing)
  std::vector<int> nodes;     // global node ids (increasing)
  std::vector<std::array<int, 8>> lnode;  // local node numbers per subdomain element
  std::vector<std::array<double, 8>> g;   // mass row sums per element
  std::vector<std::array<double, 3>> h;
  std::vector<std::array<double, 4>> mv;  // the element's nodal_mass values by popcount
  std::vector<double> diag;
};

void matvec(const Sub& s, const std::vector<double>& x, std::vector<double>& y) {
  std::fill(y.begin(), y.end(), 0.0);
  for (size_t e = 0; e < s.elems.size(); ++e) {
    const std::array<int, 8>& ln = s.lnode[e];
    const std::array<double, 4>& v = s.mv[e];
    double xl[8];
    for (int j = 0; j < 8; ++j) xl[j] = x[ln[j]];
    for (int i = 0; i < 8; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 8; ++j) acc += v[__builtin_popcount(i ^ j)] * xl[j];
      y[ln[i]] += acc;
    }
  }
}

// Jacobi-preconditioned CG to machine precision (the mass matrix is well conditioned).
std::string pcg(const Sub& s, const std::vector<double>& rhs, std::vector<double>& x) {
  const size_t n = s.nodes.size();
  x.assign(n, 0.0);
  std::vector<double> r = rhs, z(n), p(n), q(n);
  double bn = 0.0;
  for (double v : rhs) bn += v * v;
  bn = std::sqrt(bn);
  if (bn == 0.0) return "";
  for (size_t i = 0; i < n; ++i) z[i] = r[i] / s.diag[i];
  p = z;
  double rz = 0.0;
  for (size_t i = 0; i < n; ++i) rz += r[i] * z[i];
  for (int it = 0; it < 5000; ++it) {
    matvec(s, p, q);
    double pq = 0.0;
    for (size_t i = 0; i < n; ++i) pq += p[i] * q[i];
    const double alpha = rz / pq;
    double rn = 0.0;
    for (size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      rn += r[i] * r[i];
    }
    if (std::sqrt(rn) <= 1e-15 * bn) return "";
    for (size_t i = 0; i < n; ++i) z[i] = r[i] / s.diag[i];
    double rz2 = 0.0;
    for (size_t i = 0; i < n; ++i) rz2 += r[i] * z[i];
    const double beta = rz2 / rz;
    rz = rz2;
    for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    if (it > 200 && std::sqrt(rn) <= 1e-13 * bn) return "";
  }
  return "receiver projection: CG did not converge";
}

}  // namespace

std::string build_receiver_operator(const Model& m, const std::vector<std::array<double, 3>>& pts,
                                    const std::vector<int>& owner, bool curl, ReceiverOperator& out) {
  out = ReceiverOperator();
  const int nrec = (int)pts.size();
  out.nrec = nrec;
  out.ncomp = 3;
  out.elem.assign(nrec, -1);
  if (nrec == 0) {
    out.rowptr.assign(1, 0);
    return "";
  }
  // receiver -> first element (file order) whose node0/node7 box (+-1e-6) holds it
  // (OutputResultant3d.cpp:572-712)
  std::vector<double> mn(3 * (size_t)m.n_elem), mx(3 * (size_t)m.n_elem);
  for (int e = 0; e < m.n_elem; ++e)
    for (int a = 0; a < 3; ++a) {
      mn[3 * e + a] = m.xyz[m.nver[e][0]][a] - 1e-6;
      mx[3 * e + a] = m.xyz[m.nver[e][7]][a] + 1e-6;
    }
  double qlo[3] = {INFINITY, INFINITY, INFINITY}, qhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const auto& p : pts)
    for (int a = 0; a < 3; ++a)
      if (!std::isnan(p[a])) {
        qlo[a] = std::min(qlo[a], p[a]);
        qhi[a] = std::max(qhi[a], p[a]);
      }
  BoxGrid grid;
  grid.build(mn, mx, qlo, qhi);
  for (int i = 0; i < nrec; ++i) {
    const auto cand = grid.candidates(pts[i].data());
    for (const int* c = cand.first; c != cand.second; ++c) {
      const int e = *c;
      bool in = true;
      for (int a = 0; a < 3 && in; ++a) in = pts[i][a] >= mn[3 * e + a] && pts[i][a] <= mx[3 * e + a];
      if (in) {
        out.elem[i] = e;
        break;
      }
    }
    if (out.elem[i] < 0) return "receiver outside the mesh";
  }
  // trilinear coefficients (T_Brick::ScalarFieldOnParCff, T_Brick.cpp:1792-1805)
  std::vector<std::array<double, 8>> cfa(nrec);
  for (int i = 0; i < nrec; ++i) {
    const auto& n0 = m.xyz[m.nver[out.elem[i]][0]];
    const auto& n7 = m.xyz[m.nver[out.elem[i]][7]];
    double loc[3];
    for (int a = 0; a < 3; ++a) loc[a] = (2.0 * pts[i][a] - n0[a] - n7[a]) / (n7[a] - n0[a]);
    auto l0 = [](double t) { return (1.0 - t) * 0.5; };
    auto l1 = [](double t) { return (t + 1.0) * 0.5; };
    for (int k = 0; k < 8; ++k)
      cfa[i][k] = ((k & 1) ? l1(loc[0]) : l0(loc[0])) * ((k & 2) ? l1(loc[1]) : l0(loc[1])) *
                  ((k & 4) ? l1(loc[2]) : l0(loc[2]));
  }
  // subdomain materials
  std::vector<int> mats;
  if (curl) {
    mats.push_back(-1);
  } else {
    for (int i = 0; i < nrec; ++i) mats.push_back(m.nvkat[out.elem[i]]);
    std::sort(mats.begin(), mats.end());
    mats.erase(std::unique(mats.begin(), mats.end()), mats.end());
  }
  std::vector<char> has_rec(m.n_elem, 0);
  for (int i = 0; i < nrec; ++i) has_rec[out.elem[i]] = 1;

  // row comp*nrec+i: edge ids (increasing) and weights
  std::vector<std::vector<int>> row_col((size_t)3 * nrec);
  std::vector<std::vector<double>> row_val((size_t)3 * nrec);
  std::vector<int> edge_local(m.n_edges, -1);
  for (int mat : mats) {
    // --- subdomain growth (Subdomain.cpp:165-242) -------------------------------
    std::vector<char> in_e(m.n_elem, 0), in_n(m.n_nodes, 0);
    for (int e = 0; e < m.n_elem; ++e)
      if (has_rec[e] && (mat == -1 || m.nvkat[e] == mat)) {
        in_e[e] = 1;
        for (int k = 0; k < 8; ++k) in_n[m.nver[e][k]] = 1;
      }
    for (int lev = 0; lev < m.n_neib; ++lev) {
      std::vector<int> add;
      for (int e = 0; e < m.n_elem; ++e) {
        if (in_e[e]) continue;
        if (mat != -1 && m.nvkat[e] != mat) continue;
        bool touch = false;
        for (int k = 0; k < 8 && !touch; ++k) touch = in_n[m.nver[e][k]];
        if (touch) add.push_back(e);
      }
      for (int e : add) {
        in_e[e] = 1;
        for (int k = 0; k < 8; ++k) in_n[m.nver[e][k]] = 1;
      }
    }
    Sub s;
    std::vector<int> renum(m.n_nodes, -1);
    for (int v = 0; v < m.n_nodes; ++v)
      if (in_n[v]) {
        renum[v] = (int)s.nodes.size();
        s.nodes.push_back(v);
      }
    for (int e = 0; e < m.n_elem; ++e)
      if (in_e[e]) s.elems.push_back(e);
    const size_t ne = s.elems.size(), nn = s.nodes.size();
    s.lnode.resize(ne);
    s.g.resize(ne);
    s.h.resize(ne);
    s.mv.resize(ne);
    s.diag.assign(nn, 0.0);
    for (size_t t = 0; t < ne; ++t) {
      const int e = s.elems[t];
      for (int k = 0; k < 8; ++k) s.lnode[t][k] = renum[m.nver[e][k]];
      for (int a = 0; a < 3; ++a) s.h[t][a] = m.xyz[m.nver[e][7]][a] - m.xyz[m.nver[e][0]][a];
      double b[8][8];
      nodal_mass(s.h[t][0], s.h[t][1], s.h[t][2], b);
      for (int d = 0; d < 4; ++d) s.mv[t][d] = b[0][(1 << d) - 1];
      for (int j = 0; j < 8; ++j) {
        double gsum = 0.0;
        for (int k = 0; k < 8; ++k) gsum += b[j][k];
        s.g[t][j] = gsum;
        s.diag[s.lnode[t][j]] += b[j][j];
      }
    }
    // the subdomain's edges in increasing id order, and each element's edges by that order
    std::vector<int> sub_edges;
    for (size_t t = 0; t < ne; ++t)
      for (int l = 0; l < 12; ++l) sub_edges.push_back(m.ed[s.elems[t]][l]);
    std::sort(sub_edges.begin(), sub_edges.end());
    sub_edges.erase(std::unique(sub_edges.begin(), sub_edges.end()), sub_edges.end());
    const size_t nse = sub_edges.size();
    for (size_t k = 0; k < nse; ++k) edge_local[sub_edges[k]] = (int)k;
    std::vector<std::array<int, 12>> ledge(ne);
    std::vector<std::array<double, 36>> cfe(ne);  // centre coefficients [comp][l]
    for (size_t t = 0; t < ne; ++t)
      for (int l = 0; l < 12; ++l) {
        ledge[t][l] = edge_local[m.ed[s.elems[t]][l]];
        for (int comp = 0; comp < 3; ++comp)
          cfe[t][comp * 12 + l] = centre_coef(curl, comp, l, s.h[t][0], s.h[t][1], s.h[t][2]);
      }
    for (int ge : sub_edges) edge_local[ge] = -1;
    // --- one mass-matrix solve per receiver of this subdomain; the receivers are
    // taken by host threads one at a time, and receiver i writes rows comp*nrec+i only,
    // so the rows do not depend on the thread count -------------------------------
    std::vector<int> todo;
    for (int i = 0; i < nrec; ++i)
      if (mat == -1 || m.nvkat[out.elem[i]] == mat) todo.push_back(i);
    const int nt = std::max(1, std::min(host_threads(), (int)todo.size()));
    std::atomic<int64_t> next(0);
    std::vector<std::string> errs(nt);
    parallel_chunks(nt, nt, [&](int th, int64_t, int64_t) {
      std::vector<double> c(nn), y, acc(3 * nse);
      std::vector<char> hit(3 * nse);
      for (int64_t k; (k = next++) < (int64_t)todo.size();) {
        const int i = todo[k], e = out.elem[i];
        std::fill(c.begin(), c.end(), 0.0);
        for (int q = 0; q < 8; ++q) c[renum[m.nver[e][q]]] += cfa[i][q];
        std::string err = pcg(s, c, y);
        if (!err.empty()) {
          errs[th] = err;
          return;
        }
        // weights summed per edge in element order (dense over the subdomain's edges)
        std::fill(acc.begin(), acc.end(), 0.0);
        std::fill(hit.begin(), hit.end(), 0);
        for (size_t t = 0; t < ne; ++t) {
          double wt = 0.0;
          for (int j = 0; j < 8; ++j) wt += s.g[t][j] * y[s.lnode[t][j]];
          if (wt == 0.0) continue;
          for (int comp = 0; comp < 3; ++comp)
            for (int l = 0; l < 12; ++l) {
              const double cf = cfe[t][comp * 12 + l];
              if (cf == 0.0) continue;
              const size_t q = comp * nse + ledge[t][l];
              acc[q] += wt * cf;
              hit[q] = 1;
            }
        }
        for (int comp = 0; comp < 3; ++comp) {
          std::vector<int>& rc = row_col[(size_t)comp * nrec + i];
          std::vector<double>& rv = row_val[(size_t)comp * nrec + i];
          for (size_t q = 0; q < nse; ++q)
            if (hit[comp * nse + q]) {
              rc.push_back(sub_edges[q]);
              rv.push_back(acc[comp * nse + q]);
            }
        }
      }
    });
    for (const std::string& err : errs)
      if (!err.empty()) return err;
  }
  out.rowptr.assign(1, 0);
  out.src.resize((size_t)3 * nrec);
  for (int comp = 0; comp < 3; ++comp)
    for (int i = 0; i < nrec; ++i) {
      const size_t r = (size_t)comp * nrec + i;
      out.col.insert(out.col.end(), row_col[r].begin(), row_col[r].end());
      out.val.insert(out.val.end(), row_val[r].begin(), row_val[r].end());
      out.rowptr.push_back((int64_t)out.col.size());
      out.src[(size_t)comp * nrec + i] = owner[i];
    }
  return "";
}

}  // namespace tdem
