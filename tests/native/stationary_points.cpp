// Test driver (CPU): the source points of the stationary module (stationary_source_points,
// no device) against a scan over all elements, restated here: for each point (per wire
// its nSrsRazb dipoles, then electrodes A and B) the first earth element (material 1 is
// air) whose node box +-1e-3 holds it with local coordinates in (-0.01, 1.01); otherwise,
// of the 8 earth elements nearest by L1 box distance (ties in element order), the first
// whose local coordinates lie least far (L1) outside [0, 1].  Prints "ok <points>
// (<outside> outside)".
#include <algorithm>
#include <array>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "model.h"
#include "stationary.h"
using namespace tdem;

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  Model m;
  std::string e = load_model(argv[1], m);
  std::vector<std::array<double, 4>> got;
  if (e.empty()) e = stationary_source_points(argv[1], got);
  if (!e.empty()) {
    printf("%s\n", e.c_str());
    return 1;
  }
  std::vector<std::array<double, 3>> pts;
  for (int i = 0; i < m.npls; ++i) {
    const auto& w = m.wires[i];
    const int nd = m.n_srs_razb;
    const double d[3] = {(w[3] - w[0]) / nd, (w[4] - w[1]) / nd, (w[5] - w[2]) / nd};
    for (int j = 0; j < nd; ++j) pts.push_back({w[0] + (j + 0.5) * d[0], w[1] + (j + 0.5) * d[1], w[2] + (j + 0.5) * d[2]});
    pts.push_back({w[0], w[1], w[2]});
    pts.push_back({w[3], w[4], w[5]});
  }
  if (pts.size() != got.size()) {
    printf("point count %zu vs %zu\n", got.size(), pts.size());
    return 1;
  }
  auto box = [&](int el, int a, double& mn, double& mx) {
    mn = 1e300;
    mx = -1e300;
    for (int k = 0; k < 8; ++k) {
      mn = std::min(mn, m.xyz[m.nver[el][k]][a]);
      mx = std::max(mx, m.xyz[m.nver[el][k]][a]);
    }
  };
  auto local = [&](int el, const std::array<double, 3>& p, double l[3]) {
    for (int a = 0; a < 3; ++a) {
      const double x0 = m.xyz[m.nver[el][0]][a], x7 = m.xyz[m.nver[el][7]][a];
      l[a] = (p[a] - x0) / (x7 - x0);
    }
  };
  int outside = 0;
  for (size_t k = 0; k < pts.size(); ++k) {
    const auto& p = pts[k];
    int want = -1;
    double lw[3] = {0, 0, 0};
    for (int el = 0; el < m.n_elem && want < 0; ++el) {
      if (m.nvkat[el] == 0) continue;  // air
      bool in = true;
      for (int a = 0; a < 3 && in; ++a) {
        double mn, mx;
        box(el, a, mn, mx);
        in = !(p[a] < mn - 1e-3 || p[a] > mx + 1e-3);
      }
      double l[3];
      local(el, p, l);
      for (int a = 0; a < 3 && in; ++a) in = l[a] > -1e-2 && l[a] < 1.0 + 1e-2;
      if (in) {
        want = el;
        std::copy(l, l + 3, lw);
      }
    }
    if (want < 0) {
      ++outside;
      std::vector<std::pair<double, int>> dist;
      for (int el = 0; el < m.n_elem; ++el) {
        if (m.nvkat[el] == 0) continue;
        double s = 0.0;
        for (int a = 0; a < 3; ++a) {
          double mn, mx;
          box(el, a, mn, mx);
          s += p[a] < mn ? mn - p[a] : p[a] > mx ? p[a] - mx : 0.0;
        }
        dist.push_back({s, el});
      }
      std::sort(dist.begin(), dist.end());
      double best = 1e30;
      for (size_t b = 0; b < 8 && b < dist.size(); ++b) {
        double l[3], o = 0.0;
        local(dist[b].second, p, l);
        for (int a = 0; a < 3; ++a) o += l[a] < 0.0 ? -l[a] : l[a] > 1.0 ? l[a] - 1.0 : 0.0;
        if (o < best) {
          best = o;
          want = dist[b].second;
          std::copy(l, l + 3, lw);
        }
      }
    }
    if ((double)want != got[k][0] || lw[0] != got[k][1] || lw[1] != got[k][2] || lw[2] != got[k][3]) {
      printf("point %zu: scan %d (%g %g %g), located %g (%g %g %g)\n", k, want, lw[0], lw[1], lw[2], got[k][0],
             got[k][1], got[k][2], got[k][3]);
      return 1;
    }
  }
  printf("ok %zu (%d outside)\n", pts.size(), outside);
  return 0;
}
