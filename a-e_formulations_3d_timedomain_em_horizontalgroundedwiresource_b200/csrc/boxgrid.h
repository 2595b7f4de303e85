// Point location over the elements' axis-aligned boxes.  The reference walks all
// elements for every point and takes the first (in element order) whose box holds
// it (CalcNonstat3DLine/OutputResultant3d.cpp:572-712 for receivers,
// Vec_Prep_Data::LoadAndInitCurrent, vec_prep_data.cpp:1080-1180, for the wire's
// dipoles); BoxGrid returns, for a point, a short list that holds every box
// containing it, in increasing box order, so scanning that list with the same test
// gives the same element.
//
// Cells are cut per axis at the sorted distinct box centres (thinned so that the
// cell count stays near the box count): on a tensor-product mesh every element is
// listed in 2 cells per axis, 8 in all.  A box is listed in every cell between the
// cells of its low and high corners; the cell of a value v on an axis is the number
// of cuts <= v, which is monotone in v, so a point inside a box falls in one of the
// box's cells whatever the rounding of the cut values.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

namespace tdem {

class BoxGrid {
 public:
  // lo, hi: 3 per box (x, y, z); a box with !(lo <= hi) on some axis (empty or NaN)
  // is never listed.  With qlo/qhi (the bounding box of the points that will be
  // looked up), boxes that do not reach it are not listed either: none of them can
  // hold such a point.
  void build(const std::vector<double>& lo, const std::vector<double>& hi, const double* qlo = nullptr,
             const double* qhi = nullptr) {
    const int64_t n = (int64_t)lo.size() / 3;
    std::vector<char> ok(n, 1);
    for (int64_t b = 0; b < n; ++b)
      for (int a = 0; a < 3; ++a) {
        if (!(lo[3 * b + a] <= hi[3 * b + a])) ok[b] = 0;
        if (qlo && (hi[3 * b + a] < qlo[a] || lo[3 * b + a] > qhi[a])) ok[b] = 0;
      }
    int64_t listed = 0;
    for (int64_t b = 0; b < n; ++b) listed += ok[b];
    int64_t cells = 1;
    for (int a = 0; a < 3; ++a) {
      std::vector<double>& c = cut_[a];
      c.clear();
      for (int64_t b = 0; b < n; ++b)
        if (ok[b]) {
          const double m = 0.5 * (lo[3 * b + a] + hi[3 * b + a]);
          if (std::isfinite(m)) c.push_back(m);
        }
      std::sort(c.begin(), c.end());
      c.erase(std::unique(c.begin(), c.end()), c.end());
    }
    // thin the cuts while the cell count is above twice the listed box count
    const double target = 2.0 * (double)std::max<int64_t>(listed, 32);
    double prod = 1.0;
    for (int a = 0; a < 3; ++a) prod *= (double)(cut_[a].size() + 1);
    if (prod > target) {
      const double f = std::cbrt(target / prod);
      for (int a = 0; a < 3; ++a) {
        std::vector<double>& c = cut_[a];
        const size_t keep = std::max<size_t>(1, (size_t)((double)c.size() * f));
        if (keep >= c.size()) continue;
        std::vector<double> t(keep);
        for (size_t i = 0; i < keep; ++i) t[i] = c[(i * c.size()) / keep];
        c.swap(t);
      }
    }
    for (int a = 0; a < 3; ++a) {
      dim_[a] = (int)cut_[a].size() + 1;
      cells *= dim_[a];
    }
    start_.assign(cells + 1, 0);
    // two passes: count per cell, then list the boxes in increasing order
    auto each_cell = [&](int64_t b, auto&& f) {
      int l[3], h[3];
      for (int a = 0; a < 3; ++a) {
        l[a] = index(a, lo[3 * b + a]);
        h[a] = index(a, hi[3 * b + a]);
      }
      for (int x = l[0]; x <= h[0]; ++x)
        for (int y = l[1]; y <= h[1]; ++y)
          for (int z = l[2]; z <= h[2]; ++z) f(((int64_t)x * dim_[1] + y) * dim_[2] + z);
    };
    for (int64_t b = 0; b < n; ++b)
      if (ok[b]) each_cell(b, [&](int64_t c) { ++start_[c + 1]; });
    for (int64_t c = 0; c < cells; ++c) start_[c + 1] += start_[c];
    box_.assign(start_[cells], 0);
    std::vector<int64_t> fill(start_.begin(), start_.end() - 1);
    for (int64_t b = 0; b < n; ++b)
      if (ok[b]) each_cell(b, [&](int64_t c) { box_[fill[c]++] = (int)b; });
  }

  // the boxes listed in the cell that holds p, in increasing order
  std::pair<const int*, const int*> candidates(const double p[3]) const {
    int64_t c = 0;
    for (int a = 0; a < 3; ++a) c = c * dim_[a] + index(a, p[a]);
    return {box_.data() + start_[c], box_.data() + start_[c + 1]};
  }

 private:
  // cell of v on axis a: the number of cuts <= v (NaN: cell 0, which no test passes)
  int index(int a, double v) const {
    const std::vector<double>& c = cut_[a];
    if (std::isnan(v)) return 0;
    return (int)(std::upper_bound(c.begin(), c.end(), v) - c.begin());
  }

  std::array<std::vector<double>, 3> cut_;
  int dim_[3] = {1, 1, 1};
  std::vector<int64_t> start_;
  std::vector<int> box_;
};

}  // namespace tdem
