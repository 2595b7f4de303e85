// Host preparation of the time grid (see timegrid.h).  Small text files; the
// arithmetic follows the reference's order step by step so that the rewritten
// grids and tables are byte-identical, and the files are read with the same C
// library routines the reference uses (fscanf tokens for TimeDirectSolver's grid
// reader, stream extraction elsewhere).
#include "timegrid.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

namespace tdem {
namespace {

std::string join(const std::string& dir, const std::string& name) { return dir + "/" + name; }

// Linear interpolation in a table sorted by time, constant beyond its ends; the
// interval is found by bisection (TimeDirectSolver/main.cpp:43-97,
// CorrectTimeMesh/main.cpp:32-86).  A one-point table gives its value everywhere.
double table_value(double t, const std::vector<double>& vt, const std::vector<double>& vv) {
  const int last = (int)vt.size() - 1;
  if (t < vt[0]) return vv[0];
  if (t > vt[last]) return vv[last];
  if (last == 0) return vv[0];
  int lo = 0, hi = last, mid = (lo + hi) / 2;
  do {
    if (t > vt[mid])
      lo = mid;
    else
      hi = mid;
    mid = (lo + hi) / 2;
  } while (mid != lo);
  const double t1 = vt[lo], t2 = vt[lo + 1];
  return ((t2 - t) * vv[lo] + (t - t1) * vv[lo + 1]) / (t2 - t1);
}

// infite.0 with five times per line, "%.7e" (TimeDirectSolver/TimeStep.cpp:144-168)
std::string write_grid(const std::string& fn, const std::vector<double>& t) {
  FILE* f = std::fopen(fn.c_str(), "w");
  if (!f) return "cannot write " + fn;
  const int n = (int)t.size();
  std::fprintf(f, "    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n", n, n);
  std::fprintf(f, "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n");
  std::fprintf(f, "       u0=   0.00000e+000\n T I M E :\n");
  for (int i = 0; i < n; i += 5) {
    for (int j = i; j < i + 5 && j < n; ++j) std::fprintf(f, " %.7e;", t[j]);
    std::fprintf(f, "\n");
  }
  return std::fclose(f) == 0 ? "" : "cannot write " + fn;
}

// a function table on the new times, "%.14e %.14e" per line, optionally preceded by
// the receiver radius and the count (deltafunction's layout)
std::string write_table(const std::string& fn, const std::vector<double>& t, const std::vector<double>& v,
                        const double* recrad) {
  FILE* f = std::fopen(fn.c_str(), "w");
  if (!f) return "cannot write " + fn;
  if (recrad) std::fprintf(f, "%.14e\n%d\n", *recrad, (int)t.size());
  for (size_t i = 0; i < t.size(); ++i) std::fprintf(f, "%.14e %.14e\n", t[i], v[i]);
  return std::fclose(f) == 0 ? "" : "cannot write " + fn;
}

std::string read_growth(const std::string& dir, double& tcff) {
  std::ifstream in(join(dir, "tcff"));
  if (!in) return "cannot open tcff";
  in >> tcff;
  return "";
}

// deltafunction: receiver radius, count, then (time, value) pairs
std::string read_delta(const std::string& dir, double& recrad, std::vector<double>& t, std::vector<double>& v) {
  std::ifstream in(join(dir, "deltafunction"));
  int n = 0;
  in >> recrad >> n;
  if (!in) return "cannot read deltafunction";
  if (n <= 0) return "deltafunction: empty table";
  t.assign(n, 0.0);
  v.assign(n, 0.0);
  for (int i = 0; i < n; ++i) in >> t[i] >> v[i];
  return "";
}

std::vector<double> on_grid(const std::vector<double>& grid, const std::vector<double>& t, const std::vector<double>& v) {
  std::vector<double> out(grid.size());
  for (size_t i = 0; i < grid.size(); ++i) out[i] = table_value(grid[i], t, v);
  return out;
}

}  // namespace

std::string time_direct_solver(const std::string& dir) {
  double growth = 0;
  std::string e = read_growth(dir, growth);
  if (!e.empty()) return e;

  // the given times: the count after the token "ktime=", the list after "T I M E :"
  // (TimeStep.cpp:37-75)
  std::vector<double> t0;
  {
    const std::string fn = join(dir, "infite.0");
    FILE* f = std::fopen(fn.c_str(), "r");
    if (!f) return "cannot open infite.0";
    char tok[256];
    int nt = -1;
    bool listed = false;
    while (!std::feof(f)) {
      if (std::fscanf(f, "%255s", tok) != 1) break;
      if (!std::strcmp(tok, "ktime=")) {
        if (std::fscanf(f, "%d", &nt) != 1) break;
        t0.assign(nt > 0 ? nt : 0, 0.0);
        continue;
      }
      if (!std::strcmp(tok, "T") && nt >= 0) {
        for (int i = 0; i < 4; ++i) (void)!std::fscanf(f, "%255s", tok);  // "I M E :"
        for (int i = 0; i < nt; ++i) {
          (void)!std::fscanf(f, "%lf", &t0[i]);
          (void)!std::fscanf(f, "%255s", tok);  // ";"
        }
        listed = true;
        break;
      }
    }
    std::fclose(f);
    if (!listed) return "infite.0: no time list";
    if (t0.size() < 3) return "infite.0: fewer than three times";
  }

  // piecewise-uniform grid (TimeStep.cpp:76-143): an interval ends at the first
  // given time whose step exceeds growth x the current step (or at the last time);
  // it holds whole steps of the current size up to that time, and the next
  // interval's step is growth times larger.  Steps past the last given time are
  // dropped until only the final one reaches beyond it.
  std::vector<double> grid;
  {
    std::vector<double> start{t0[0]}, width;
    std::vector<int> count;
    double h = t0[1] - t0[0];
    width.push_back(h);
    for (size_t k = 2; k < t0.size(); ++k) {
      const double step = t0[k] - t0[k - 1];
      if (step > growth * h || k + 1 == t0.size()) {
        count.push_back((int)((t0[k] - start.back()) / h + 1));
        start.push_back(start.back() + count.back() * h);
        h *= growth;
        width.push_back(h);
      }
    }
    grid.push_back(t0[0]);
    for (size_t i = 0; i + 1 < start.size(); ++i)
      for (int j = 0; j < count[i]; ++j) grid.push_back(start[i] + (j + 1) * width[i]);
    while (grid.size() >= 2 && grid[grid.size() - 2] > t0.back()) {
      if (count.empty()) return "time grid: no interval left";
      if (count.back() == 1)
        count.pop_back();
      else
        --count.back();
      grid.pop_back();
    }
    if (grid.size() < 2) return "time grid: fewer than two times";
  }
  std::rename(join(dir, "infite.0").c_str(), join(dir, "!infite.0").c_str());
  if (!(e = write_grid(join(dir, "infite.0"), grid)).empty()) return e;

  // currentfunction: (time, value) pairs up to the end of the file (main.cpp:139-175)
  {
    std::ifstream in(join(dir, "currentfunction"));
    if (!in) return "cannot open currentfunction";
    std::vector<double> t, v;
    while (!in.eof()) {
      double x = 0;
      in >> x;
      if (in.eof() || !in.good()) break;
      t.push_back(x);
      in >> x;
      v.push_back(x);
    }
    in.close();
    if (t.empty()) return "currentfunction: empty table";
    std::rename(join(dir, "currentfunction").c_str(), join(dir, "!currentfunction").c_str());
    if (!(e = write_table(join(dir, "currentfunction"), grid, on_grid(grid, t, v), nullptr)).empty()) return e;
  }
  // deltafunction (main.cpp:184-215)
  {
    double recrad = 0;
    std::vector<double> t, v;
    if (!(e = read_delta(dir, recrad, t, v)).empty()) return e;
    std::rename(join(dir, "deltafunction").c_str(), join(dir, "!deltafunction").c_str());
    if (!(e = write_table(join(dir, "deltafunction"), grid, on_grid(grid, t, v), &recrad)).empty()) return e;
  }
  return "";
}

std::string correct_time_mesh(const std::string& dir) {
  double growth = 0;
  std::string e = read_growth(dir, growth);
  if (!e.empty()) return e;
  // times of infite.0 (CorrectTimeMesh/main.cpp:196-220)
  std::vector<double> t;
  {
    std::ifstream in(join(dir, "infite.0"));
    if (!in) return "cannot open infite.0";
    in.ignore(1000, '=');
    int n = 0;
    in >> n;
    if (n < 2) return "infite.0: fewer than two times";
    t.assign(n, 0.0);
    for (int k = 0; k < 4; ++k) in.ignore(1000, '\n');
    for (int i = 0; i < n; ++i) {
      if (!in.good()) return "infite.0: truncated";
      in >> t[i];
      in.ignore(1000, ';');
    }
  }
  const int n = (int)t.size();
  // decades: runs of steps equal to 1e-3 relative (main.cpp:87-105)
  std::vector<int> dec{0};
  {
    double h = t[1] - t[0];
    for (int i = 2; i < n; ++i) {
      const double hc = t[i] - t[i - 1];
      if (std::fabs(1.0 - h / hc) > 1e-3) {
        dec.push_back(i);
        h = hc;
      }
    }
    dec.push_back(n);
  }
  // a decade is kept when it has more than one time and, after the first, more than
  // 1 / growth of the previous decade's count; otherwise its span is refilled with
  // the previous decade's step (main.cpp:222-257)
  std::vector<double> out;
  for (size_t d = 0; d + 1 < dec.size(); ++d) {
    const int len = dec[d + 1] - dec[d];
    if (len > 1 && (d == 0 || len * growth > dec[d] - dec[d - 1])) {
      for (int i = dec[d]; i < dec[d + 1]; ++i) out.push_back(t[i]);
    } else {
      if (d == 0) return "time grid: the first decade has a single time";
      const double h = (t[dec[d] - 1] - t[dec[d - 1]]) / (dec[d] - dec[d - 1] - 1);
      const double base = t[dec[d] - 1];
      int i = 1;
      double tc = base + h;
      while (tc - 0.5 * h < t[dec[d + 1] - 1]) {
        out.push_back(tc);
        ++i;
        tc = base + i * h;
      }
    }
  }
  // tables on the corrected times: deltafunction's values go to both function files
  // (main.cpp:106-177)
  double recrad = 0;
  std::vector<double> dt, dv;
  if (!(e = read_delta(dir, recrad, dt, dv)).empty()) return e;
  for (const char* f : {"currentfunction", "infite.0", "deltafunction"})
    std::rename(join(dir, f).c_str(), join(dir, std::string("!!") + f).c_str());
  const std::vector<double> val = on_grid(out, dt, dv);
  if (!(e = write_table(join(dir, "deltafunction"), out, val, &recrad)).empty()) return e;
  if (!(e = write_table(join(dir, "currentfunction"), out, val, nullptr)).empty()) return e;
  return write_grid(join(dir, "infite.0"), out);
}

}  // namespace tdem
