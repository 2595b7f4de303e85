// Test driver (CPU): point location and receiver smoothing on host threads.
//  1. BoxGrid against a linear scan (first box, in box order, whose closed extent holds
//     the point) on a graded tensor-product mesh (nodes, face centres, interior and
//     outside points) and on random overlapping boxes (thinned cuts, empty and NaN
//     boxes).
//  2. argv[1], a model directory: the dipoles' elements and local coordinates against a
//     linear scan over the elements (with the nearest-element rule for dipoles outside
//     the mesh), and the receiver operators built on 1 and on 3 host threads, which must
//     be byte-identical.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "boxgrid.h"
#include "model.h"
#include "receivers.h"
using namespace tdem;

static int first_scan(const std::vector<double>& lo, const std::vector<double>& hi, const double p[3]) {
  const int n = (int)lo.size() / 3;
  for (int b = 0; b < n; ++b) {
    bool in = true;
    for (int a = 0; a < 3 && in; ++a) in = p[a] >= lo[3 * b + a] && p[a] <= hi[3 * b + a];
    if (in) return b;
  }
  return -1;
}

static int first_grid(const BoxGrid& g, const std::vector<double>& lo, const std::vector<double>& hi,
                      const double p[3]) {
  const auto c = g.candidates(p);
  for (const int* q = c.first; q != c.second; ++q) {
    const int b = *q;
    bool in = true;
    for (int a = 0; a < 3 && in; ++a) in = p[a] >= lo[3 * b + a] && p[a] <= hi[3 * b + a];
    if (in) return b;
  }
  return -1;
}

static int check(const BoxGrid& g, const std::vector<double>& lo, const std::vector<double>& hi,
                 const std::vector<std::array<double, 3>>& pts, const char* what) {
  int found = 0;
  for (const auto& p : pts) {
    const int a = first_scan(lo, hi, p.data()), b = first_grid(g, lo, hi, p.data());
    if (a != b) {
      printf("%s: point (%.17g, %.17g, %.17g): scan %d, grid %d\n", what, p[0], p[1], p[2], a, b);
      return -1;
    }
    found += a >= 0;
  }
  return found;
}

int main(int argc, char** argv) {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  int npts = 0;
  // --- graded tensor mesh: element boxes +-1e-6 --------------------------------------
  {
    std::vector<double> ax[3];
    const int nc[3] = {17, 12, 9};
    for (int a = 0; a < 3; ++a) {
      double x = -100.0, h = 0.5;
      for (int i = 0; i <= nc[a]; ++i) {
        ax[a].push_back(x);
        x += h;
        h *= 1.7;
      }
    }
    std::vector<double> lo, hi;
    for (int k = 0; k < nc[2]; ++k)
      for (int j = 0; j < nc[1]; ++j)
        for (int i = 0; i < nc[0]; ++i) {
          const int id[3] = {i, j, k};
          for (int a = 0; a < 3; ++a) {
            lo.push_back(ax[a][id[a]] - 1e-6);
            hi.push_back(ax[a][id[a] + 1] + 1e-6);
          }
        }
    BoxGrid g;
    g.build(lo, hi);
    std::vector<std::array<double, 3>> pts;
    for (double x : ax[0])
      for (double y : ax[1])
        for (double z : ax[2]) pts.push_back({x, y, z});  // nodes: shared by up to 8 boxes
    for (int i = 0; i < nc[0]; ++i)
      for (int j = 0; j < nc[1]; ++j)
        for (int k = 0; k <= nc[2]; ++k)  // face centres
          pts.push_back({0.5 * (ax[0][i] + ax[0][i + 1]), 0.5 * (ax[1][j] + ax[1][j + 1]), ax[2][k]});
    for (int t = 0; t < 20000; ++t) {  // inside and a margin outside
      std::array<double, 3> p;
      for (int a = 0; a < 3; ++a) p[a] = ax[a].front() - 5.0 + u(rng) * (ax[a].back() - ax[a].front() + 10.0);
      pts.push_back(p);
    }
    pts.push_back({ax[0].back() + 2e-6, ax[1][3], ax[2][2]});  // just outside the tolerance
    pts.push_back({ax[0].back() + 5e-7, ax[1][3], ax[2][2]});  // just inside it
    const int f = check(g, lo, hi, pts, "tensor mesh");
    if (f < 0) return 1;
    if (f == (int)pts.size() || f < 1000) {
      printf("tensor mesh: %d of %zu points found\n", f, pts.size());
      return 1;
    }
    npts += (int)pts.size();
  }
  // --- random overlapping boxes, a few empty or NaN ------------------------------------
  {
    std::vector<double> lo, hi;
    const int n = 3000;
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < 3; ++a) {
        const double c = u(rng) * 100.0, w = std::pow(10.0, -2.0 + 3.0 * u(rng));
        lo.push_back(c - w);
        hi.push_back(c + w);
      }
    lo[3 * 10] = hi[3 * 10] + 1.0;  // empty
    lo[3 * 20 + 1] = std::nan("");  // NaN
    BoxGrid g;
    g.build(lo, hi);
    std::vector<std::array<double, 3>> pts;
    for (int t = 0; t < 20000; ++t) pts.push_back({u(rng) * 110.0 - 5.0, u(rng) * 110.0 - 5.0, u(rng) * 110.0 - 5.0});
    for (int b = 0; b < n; b += 7) pts.push_back({lo[3 * b], hi[3 * b + 1], lo[3 * b + 2]});  // corners
    if (check(g, lo, hi, pts, "random boxes") < 0) return 1;
    npts += (int)pts.size();
  }
  // --- a model: dipoles and receiver operators ------------------------------------------
  if (argc > 1) {
    Model m;
    std::string e = load_model(argv[1], m);
    if (e.empty()) e = locate_dipoles(m);
    if (!e.empty()) {
      printf("model: %s\n", e.c_str());
      return 1;
    }
    // the dipole search: first element whose node box (+-1e-3) holds the dipole and whose
    // local coordinates on nodes 0/7 lie in (-1e-2, 1 + 1e-2)
    int beyond = 0;
    for (int i = 0; i < m.npls; ++i)
      for (size_t j = 0; j < m.dipoles[i].size(); ++j) {
        const auto& w = m.wires[i];
        const int nd = (int)m.dipoles[i].size();
        double p[3];
        for (int a = 0; a < 3; ++a) p[a] = w[a] + (j + 0.5) * ((w[3 + a] - w[a]) / nd);
        int want = -1;
        for (int el = 0; el < m.n_elem && want < 0; ++el) {
          bool in = true;
          for (int a = 0; a < 3 && in; ++a) {
            double mn = 1e300, mx = -1e300;
            for (int k = 0; k < 8; ++k) {
              mn = std::min(mn, m.xyz[m.nver[el][k]][a]);
              mx = std::max(mx, m.xyz[m.nver[el][k]][a]);
            }
            const double x0 = m.xyz[m.nver[el][0]][a], x7 = m.xyz[m.nver[el][7]][a];
            const double l = (p[a] - x0) / (x7 - x0);
            in = !(p[a] < mn - 1e-3 || p[a] > mx + 1e-3) && l > -1e-2 && l < 1.0 + 1e-2;
          }
          if (in) want = el;
        }
        double lw[3] = {0, 0, 0};
        if (want < 0) {
          // none holds it: of the 8 nearest boxes (L1, ties in element order) the first
          // whose local coordinates lie least far (L1) outside [0, 1]
          std::vector<std::pair<double, int>> dist;
          for (int el = 0; el < m.n_elem; ++el) {
            double s = 0.0;
            for (int a = 0; a < 3; ++a) {
              double mn = 1e300, mx = -1e300;
              for (int k = 0; k < 8; ++k) {
                mn = std::min(mn, m.xyz[m.nver[el][k]][a]);
                mx = std::max(mx, m.xyz[m.nver[el][k]][a]);
              }
              s += p[a] < mn ? mn - p[a] : p[a] > mx ? p[a] - mx : 0.0;
            }
            dist.push_back({s, el});
          }
          std::sort(dist.begin(), dist.end());
          double best = 1e30;
          for (size_t b = 0; b < 8 && b < dist.size(); ++b) {
            const int el = dist[b].second;
            double l[3], o = 0.0;
            for (int a = 0; a < 3; ++a) {
              const double x0 = m.xyz[m.nver[el][0]][a], x7 = m.xyz[m.nver[el][7]][a];
              l[a] = (p[a] - x0) / (x7 - x0);
              o += l[a] < 0.0 ? -l[a] : l[a] > 1.0 ? l[a] - 1.0 : 0.0;
            }
            if (o < best) {
              best = o;
              want = el;
              std::copy(l, l + 3, lw);
            }
          }
          ++beyond;
        } else {
          for (int a = 0; a < 3; ++a) {
            const double x0 = m.xyz[m.nver[want][0]][a], x7 = m.xyz[m.nver[want][7]][a];
            lw[a] = (p[a] - x0) / (x7 - x0);
          }
        }
        const Dipole& dp = m.dipoles[i][j];
        if (want != dp.elem || lw[0] != dp.ksi || lw[1] != dp.eta || lw[2] != dp.zeta) {
          printf("dipole %d/%zu: scan %d (%g %g %g), located %d (%g %g %g)\n", i, j, want, lw[0], lw[1], lw[2],
                 dp.elem, dp.ksi, dp.eta, dp.zeta);
          return 1;
        }
      }
    ReceiverOperator op[2][2];
    const char* threads[2] = {"1", "3"};
    for (int t = 0; t < 2; ++t) {
      setenv("TDEM_HOST_THREADS", threads[t], 1);
      std::vector<int> ob(m.rec_b.size(), 0), oe(m.rec_e.size(), 0);
      if (!(e = build_receiver_operator(m, m.rec_b, ob, true, op[t][0])).empty() ||
          !(e = build_receiver_operator(m, m.rec_e, oe, false, op[t][1])).empty()) {
        printf("receivers: %s\n", e.c_str());
        return 1;
      }
    }
    for (int k = 0; k < 2; ++k) {
      const ReceiverOperator &a = op[0][k], &b = op[1][k];
      if (a.rowptr != b.rowptr || a.col != b.col || a.elem != b.elem || a.src != b.src ||
          a.val.size() != b.val.size() || std::memcmp(a.val.data(), b.val.data(), 8 * a.val.size()) != 0 ||
          a.col.empty()) {
        printf("receiver operator %d differs between 1 and 3 threads\n", k);
        return 1;
      }
    }
    printf("ok %d points, %d dipoles (%d outside the mesh), %zu + %zu receiver weights\n", npts,
           m.npls * m.n_srs_razb, beyond, op[0][0].val.size(), op[0][1].val.size());
    return 0;
  }
  printf("ok %d points\n", npts);
  return 0;
}
