// CPU FP64 supernodal multifrontal Cholesky -- oracle / test infrastructure only.
// See cpu_cholesky.h for what it is used for and why.
#include "cpu_cholesky.h"

#include <dlfcn.h>
#include <atomic>
#include <thread>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>

namespace oracle {

// ---------------------------------------------------------------------------
// optional dense kernels (OpenBLAS from numpy, 64-bit integer interface)
// ---------------------------------------------------------------------------
namespace {
typedef void (*dgemm_t)(int, int, int, int64_t, int64_t, int64_t, double, const double*, int64_t,
                        const double*, int64_t, double, double*, int64_t);
typedef void (*dsyrk_t)(int, int, int, int64_t, int64_t, double, const double*, int64_t, double,
                        double*, int64_t);
typedef void (*dtrsm_t)(int, int, int, int, int, int64_t, int64_t, double, const double*, int64_t,
                        double*, int64_t);
typedef int64_t (*dpotrf_t)(int, char, int64_t, double*, int64_t);
typedef void (*setnt_t)(int64_t);
enum { ColMajor = 102, NoTrans = 111, Trans = 112, Upper = 121, Lower = 122, NonUnit = 131,
       Left = 141, Right = 142 };

struct Blas {
  bool tried = false, ok = false;
  dgemm_t gemm = nullptr;
  dsyrk_t syrk = nullptr;
  dtrsm_t trsm = nullptr;
  dpotrf_t potrf = nullptr;
  setnt_t setnt = nullptr;
} g_blas;

void load_blas() {
  if (g_blas.tried) return;
  g_blas.tried = true;
  const char* p = getenv("TDEM_ORACLE_BLAS");
  if (!p || !*p) return;
  void* h = dlopen(p, RTLD_NOW | RTLD_LOCAL);
  if (!h) return;
  g_blas.gemm = (dgemm_t)dlsym(h, "scipy_cblas_dgemm64_");
  g_blas.syrk = (dsyrk_t)dlsym(h, "scipy_cblas_dsyrk64_");
  g_blas.trsm = (dtrsm_t)dlsym(h, "scipy_cblas_dtrsm64_");
  g_blas.potrf = (dpotrf_t)dlsym(h, "scipy_LAPACKE_dpotrf64_");
  g_blas.setnt = (setnt_t)dlsym(h, "scipy_openblas_set_num_threads64_");
  g_blas.ok = g_blas.gemm && g_blas.syrk && g_blas.trsm && g_blas.potrf;
}

// Right-looking partial Cholesky of the leading k columns of the m x m lower
// front F (column-major, leading dimension m), blocked by nb columns so the
// trailing update streams each target column once per panel.
int partial_chol_loops(double* F, int m, int k) {
  const int nb = 32;
  for (int j0 = 0; j0 < k; j0 += nb) {
    const int j1 = std::min(k, j0 + nb);
    // factor the panel columns j0..j1 (updates restricted to the panel)
    for (int j = j0; j < j1; ++j) {
      double* cj = F + (int64_t)j * m;
      double d = cj[j];
      if (!(d > 0.0)) return j + 1;
      d = std::sqrt(d);
      cj[j] = d;
      const double inv = 1.0 / d;
      for (int i = j + 1; i < m; ++i) cj[i] *= inv;
      for (int c = j + 1; c < j1; ++c) {
        const double f = cj[c];
        if (f == 0.0) continue;
        double* cc = F + (int64_t)c * m;
        for (int i = c; i < m; ++i) cc[i] -= cj[i] * f;
      }
    }
    // trailing update with the finished panel
    for (int c = j1; c < m; ++c) {
      double* cc = F + (int64_t)c * m;
      for (int j = j0; j < j1; ++j) {
        const double* cj = F + (int64_t)j * m;
        const double f = cj[c];
        if (f == 0.0) continue;
        for (int i = c; i < m; ++i) cc[i] -= cj[i] * f;
      }
    }
  }
  return 0;
}

int partial_chol_blas(double* F, int m, int k) {
  int64_t info = g_blas.potrf(ColMajor, 'L', k, F, m);
  if (info != 0) return (int)info;
  const int r = m - k;
  if (r > 0) {
    // L21 = F21 * L11^-T
    g_blas.trsm(ColMajor, Right, Lower, Trans, NonUnit, r, k, 1.0, F, m, F + k, m);
    // F22 -= L21 L21^T
    g_blas.syrk(ColMajor, Lower, NoTrans, r, k, -1.0, F + k, m, 1.0, F + k + (int64_t)k * m, m);
  }
  return 0;
}


// Dynamic-schedule parallel loop over [0, count) on nthreads std::threads.
template <class Fn>
void parallel_for(int nthreads, int count, Fn fn) {
  if (nthreads <= 1 || count <= 1) {
    for (int i = 0; i < count; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  const int nt = std::min(nthreads, count);
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&]() {
      for (int i = next++; i < count; i = next++) fn(i);
    });
  for (auto& th : pool) th.join();
}


// ---------------------------------------------------------------------------
// nested dissection
// ---------------------------------------------------------------------------
struct Graph {
  int n = 0;
  std::vector<int64_t> xadj;
  std::vector<int> adj;
};

struct NDBuilder {
  const Graph& g;
  const double* xyz;  // may be null
  std::vector<int> order;           // new -> old
  std::vector<int> mark, side;
  int stamp = 0;
  struct Node { int c0, c1; std::vector<int> kids; };
  std::vector<Node> nodes;
  static const int kLeaf = 64;

  NDBuilder(const Graph& gg, const double* c) : g(gg), xyz(c), mark(gg.n, 0), side(gg.n, 0) {}

  int emit(const std::vector<int>& verts, std::vector<int> kids) {
    Node nd;
    nd.c0 = (int)order.size();
    for (int v : verts) order.push_back(v);
    nd.c1 = (int)order.size();
    nd.kids = std::move(kids);
    nodes.push_back(std::move(nd));
    return (int)nodes.size() - 1;
  }

  // Splits verts into left / sep / right.  Returns false if no split was found.
  bool split_coords(const std::vector<int>& verts, std::vector<int>& L, std::vector<int>& S,
                    std::vector<int>& R) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : verts)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], xyz[3 * (int64_t)v + a]);
        hi[a] = std::max(hi[a], xyz[3 * (int64_t)v + a]);
      }
    // try axes in order of decreasing number of distinct coordinate values
    int axes[3] = {0, 1, 2};
    int ndist[3];
    std::vector<double> vals(verts.size());
    for (int a = 0; a < 3; ++a) {
      for (size_t i = 0; i < verts.size(); ++i) vals[i] = xyz[3 * (int64_t)verts[i] + a];
      std::sort(vals.begin(), vals.end());
      ndist[a] = (int)(std::unique(vals.begin(), vals.end()) - vals.begin());
    }
    std::sort(axes, axes + 3, [&](int a, int b) { return ndist[a] > ndist[b]; });
    for (int ai = 0; ai < 3; ++ai) {
      const int a = axes[ai];
      if (ndist[a] < 3) continue;
      for (size_t i = 0; i < verts.size(); ++i) vals[i] = xyz[3 * (int64_t)verts[i] + a];
      std::sort(vals.begin(), vals.end());
      const size_t nv = vals.size();
      const size_t q0 = nv * 35 / 100, q1 = std::max(q0 + 1, nv * 65 / 100);
      // most frequent value inside the central window (node planes win), ties
      // broken towards the median
      double best = vals[nv / 2];
      size_t bestcnt = 0;
      double bestdist = 1e300;
      size_t i = q0;
      while (i < q1) {
        size_t j = i;
        while (j < nv && vals[j] == vals[i]) ++j;
        size_t cnt = j - i;
        double dist = std::fabs((double)((i + j) / 2) - (double)(nv / 2));
        if (cnt > bestcnt || (cnt == bestcnt && dist < bestdist)) {
          best = vals[i];
          bestcnt = cnt;
          bestdist = dist;
        }
        i = j;
      }
      if (best <= vals.front()) continue;
      ++stamp;
      for (int v : verts) mark[v] = stamp;
      L.clear(); S.clear(); R.clear();
      for (int v : verts) {
        const double c = xyz[3 * (int64_t)v + a];
        if (c < best) { L.push_back(v); continue; }
        bool touches = false;
        for (int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
          const int u = g.adj[p];
          if (mark[u] == stamp && xyz[3 * (int64_t)u + a] < best) { touches = true; break; }
        }
        (touches ? S : R).push_back(v);
      }
      if (!L.empty() && !S.empty()) return true;
    }
    return false;
  }

  // Breadth-first level-set bisection.  Returns 0 = no split, 1 = split with a
  // separator level, 2 = verts is disconnected (L = one component, R = rest).
  int split_bfs(const std::vector<int>& verts, std::vector<int>& L, std::vector<int>& S,
                std::vector<int>& R) {
    ++stamp;
    const int mystamp = stamp;
    for (int v : verts) mark[v] = mystamp;
    auto bfs = [&](int s, std::vector<int>& lev, std::vector<int>& seen) {
      ++stamp;  // visited marker uses side[] with the new stamp
      const int vs = stamp;
      seen.clear();
      lev.clear();
      seen.push_back(s);
      side[s] = vs;
      std::vector<int> depth_start{0};
      size_t head = 0;
      int depth = 0;
      size_t level_end = 1;
      while (head < seen.size()) {
        const int v = seen[head++];
        lev.push_back(depth);
        for (int64_t p = g.xadj[v]; p < g.xadj[v + 1]; ++p) {
          const int u = g.adj[p];
          if (mark[u] == mystamp && side[u] != vs) {
            side[u] = vs;
            seen.push_back(u);
          }
        }
        if (head == level_end) {
          ++depth;
          level_end = seen.size();
        }
      }
    };
    std::vector<int> lev, seen;
    int s = verts[0];
    for (int it = 0; it < 3; ++it) {
      bfs(s, lev, seen);
      s = seen.back();
    }
    bfs(s, lev, seen);
    if (seen.size() < verts.size()) {
      L = seen;
      ++stamp;
      for (int v : seen) side[v] = stamp;
      R.clear();
      for (int v : verts)
        if (side[v] != stamp) R.push_back(v);
      S.clear();
      return 2;
    }
    const int maxd = lev.back();
    if (maxd < 2) return 0;
    // cut level: first level where the running count passes half
    size_t half = seen.size() / 2, run = 0;
    int cut = 1;
    for (size_t i = 0; i < seen.size(); ++i) {
      ++run;
      if (run >= half) { cut = std::max(1, std::min(maxd - 1, lev[i])); break; }
    }
    L.clear(); S.clear(); R.clear();
    for (size_t i = 0; i < seen.size(); ++i) {
      if (lev[i] < cut) L.push_back(seen[i]);
      else if (lev[i] == cut) S.push_back(seen[i]);
      else R.push_back(seen[i]);
    }
    return 1;
  }

  int build(std::vector<int> verts) {
    if ((int)verts.size() <= kLeaf) return emit(verts, {});
    std::vector<int> L, S, R;
    int kind = 0;
    if (xyz && split_coords(verts, L, S, R)) kind = 1;
    if (!kind) kind = split_bfs(verts, L, S, R);
    if (!kind) return emit(verts, {});
    verts.clear();
    verts.shrink_to_fit();
    std::vector<int> kids;
    if (!L.empty()) kids.push_back(build(std::move(L)));
    if (!R.empty()) kids.push_back(build(std::move(R)));
    return emit(S, kids);
  }
};

}  // namespace

bool blas_available() {
  load_blas();
  return g_blas.ok;
}

// ---------------------------------------------------------------------------
// analysis
// ---------------------------------------------------------------------------
int SparseCholesky::analyze(int n_, const int64_t* ptr, const int64_t* ind, const double* coords,
                            int nthreads_) {
  load_blas();
  n = n_;
  nthreads = std::max(1, nthreads_);
  nnz_a = ptr[n];
  // pattern hash (lets callers skip re-analysis of an unchanged pattern)
  uint64_t h = 1469598103934665603ull ^ (uint64_t)n;
  for (int i = 0; i <= n; ++i) h = (h ^ (uint64_t)ptr[i]) * 1099511628211ull;
  for (int64_t q = 0; q < nnz_a; ++q) h = (h ^ (uint64_t)ind[q]) * 1099511628211ull;
  pattern_hash = (int64_t)h;

  // symmetric adjacency without the diagonal
  Graph g;
  g.n = n;
  std::vector<int64_t> deg(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int64_t j = ind[q];
      if (j == i) continue;
      if (j < 0 || j >= n) return -1;
      ++deg[i];
      ++deg[j];
    }
  g.xadj.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) g.xadj[i + 1] = g.xadj[i] + deg[i];
  g.adj.resize(g.xadj[n]);
  std::vector<int64_t> fill(g.xadj.begin(), g.xadj.end() - 1);
  for (int i = 0; i < n; ++i)
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int j = (int)ind[q];
      if (j == i) continue;
      g.adj[fill[i]++] = j;
      g.adj[fill[j]++] = i;
    }

  NDBuilder nd(g, coords);
  std::vector<int> all(n);
  std::iota(all.begin(), all.end(), 0);
  nd.build(std::move(all));
  iperm = nd.order;
  perm.assign(n, -1);
  for (int i = 0; i < n; ++i) perm[iperm[i]] = i;

  // fronts in dissection-tree postorder (nodes were emitted children-first)
  const int nf = (int)nd.nodes.size();
  fronts.assign(nf, Front());
  for (int s = 0; s < nf; ++s) {
    fronts[s].c0 = nd.nodes[s].c0;
    fronts[s].c1 = nd.nodes[s].c1;
    fronts[s].children = nd.nodes[s].kids;
    for (int c : nd.nodes[s].kids) fronts[c].parent = s;
  }
  std::vector<int> colfront(n);
  for (int s = 0; s < nf; ++s)
    for (int c = fronts[s].c0; c < fronts[s].c1; ++c) colfront[c] = s;

  // row structures
  std::vector<int> stampv(n, -1), pos(n, -1);
  std::vector<int> tmp;
  for (int s = 0; s < nf; ++s) {
    Front& f = fronts[s];
    tmp.clear();
    for (int c = f.c0; c < f.c1; ++c) {
      const int i = iperm[c];
      for (int64_t p = g.xadj[i]; p < g.xadj[i + 1]; ++p) {
        const int r = perm[g.adj[p]];
        if (r >= f.c1 && stampv[r] != s) { stampv[r] = s; tmp.push_back(r); }
      }
    }
    for (int ch : f.children)
      for (int r : fronts[ch].rows)
        if (r >= f.c1 && stampv[r] != s) { stampv[r] = s; tmp.push_back(r); }
    std::sort(tmp.begin(), tmp.end());
    f.rows = tmp;
  }
  // relative indices of each child's rows inside its parent front
  for (int s = 0; s < nf; ++s) {
    Front& f = fronts[s];
    for (int c = f.c0; c < f.c1; ++c) pos[c] = c - f.c0;
    for (size_t t = 0; t < f.rows.size(); ++t) pos[f.rows[t]] = f.k() + (int)t;
    for (int ch : f.children) {
      Front& fc = fronts[ch];
      fc.rel.resize(fc.rows.size());
      for (size_t t = 0; t < fc.rows.size(); ++t) fc.rel[t] = pos[fc.rows[t]];
    }
  }
  // original entries -> (front, local row, local col)
  std::vector<int64_t> cnt(nf + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int a = perm[i], b = perm[(int)ind[q]];
      ++cnt[colfront[std::min(a, b)]];
    }
  for (int s = 0; s < nf; ++s) {
    fronts[s].a_idx.reserve(cnt[s]);
    fronts[s].a_r.reserve(cnt[s]);
    fronts[s].a_c.reserve(cnt[s]);
  }
  for (int i = 0; i < n; ++i)
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int a = perm[i], b = perm[(int)ind[q]];
      const int col = std::min(a, b), row = std::max(a, b);
      Front& f = fronts[colfront[col]];
      f.a_idx.push_back(q);
      f.a_r.push_back(row);  // global for now
      f.a_c.push_back(col - f.c0);
    }
  for (int s = 0; s < nf; ++s) {
    Front& f = fronts[s];
    for (int c = f.c0; c < f.c1; ++c) pos[c] = c - f.c0;
    for (size_t t = 0; t < f.rows.size(); ++t) pos[f.rows[t]] = f.k() + (int)t;
    for (auto& r : f.a_r) r = pos[r];
  }
  // storage and flop count
  int64_t off = 0;
  flops = 0.0;
  for (int s = 0; s < nf; ++s) {
    Front& f = fronts[s];
    f.lofs = off;
    const double m = f.m(), k = f.k();
    off += (int64_t)f.m() * f.k();
    flops += 2.0 * (k * k * k / 3.0 + (m - k) * k * k + (m - k) * (m - k) * k);
  }
  nnz_l = off;
  L.assign(off, 0.0);
  build_schedule();
  return 0;
}

void SparseCholesky::build_schedule() {
  const int nf = (int)fronts.size();
  std::vector<double> cost(nf, 0.0);
  for (int s = 0; s < nf; ++s) {
    const double m = fronts[s].m(), k = fronts[s].k();
    cost[s] += k * k * k / 3.0 + (m - k) * k * k + (m - k) * (m - k) * k + m * m;
    if (fronts[s].parent >= 0) cost[fronts[s].parent] += cost[s];
  }
  double total = 0.0;
  std::vector<int> roots;
  for (int s = 0; s < nf; ++s)
    if (fronts[s].parent < 0) { roots.push_back(s); total += cost[s]; }
  auto cmp = [&](int a, int b) { return cost[a] < cost[b]; };
  std::priority_queue<int, std::vector<int>, decltype(cmp)> pq(cmp);
  for (int r : roots) pq.push(r);
  top_.clear();
  const size_t want = (size_t)4 * nthreads;
  while (!pq.empty() && nthreads > 1) {
    const int s = pq.top();
    if (pq.size() >= want || cost[s] < total / (double)(4 * nthreads) || fronts[s].children.empty())
      break;
    pq.pop();
    top_.push_back(s);
    for (int c : fronts[s].children) pq.push(c);
  }
  std::vector<int> sub_roots;
  while (!pq.empty()) { sub_roots.push_back(pq.top()); pq.pop(); }
  std::sort(top_.begin(), top_.end());
  subtrees_.assign(sub_roots.size(), {});
  for (size_t t = 0; t < sub_roots.size(); ++t) {
    // postorder list of the subtree: fronts are stored in postorder, and a
    // subtree occupies a contiguous index range ending at its root
    int r = sub_roots[t];
    int lo = r;
    std::vector<int> st{r};
    while (!st.empty()) {
      int v = st.back();
      st.pop_back();
      lo = std::min(lo, v);
      for (int c : fronts[v].children) st.push_back(c);
    }
    for (int v = lo; v <= r; ++v) subtrees_[t].push_back(v);
  }
}

// ---------------------------------------------------------------------------
// numeric factorization
// ---------------------------------------------------------------------------
int SparseCholesky::factor(const double* val) {
  const int nf = (int)fronts.size();
  std::vector<std::vector<double>> upd(nf);
  int err = 0;

  auto do_front = [&](int s, bool use_blas) -> int {
    Front& f = fronts[s];
    const int m = f.m(), k = f.k(), r = m - k;
    std::vector<double> F((size_t)m * m, 0.0);
    for (size_t e = 0; e < f.a_idx.size(); ++e) F[f.a_r[e] + (int64_t)f.a_c[e] * m] += val[f.a_idx[e]];
    for (int ch : f.children) {
      const Front& fc = fronts[ch];
      const int rc = (int)fc.rows.size();
      const double* U = upd[ch].data();
      for (int b = 0; b < rc; ++b) {
        double* col = F.data() + (int64_t)fc.rel[b] * m;
        const double* ub = U + (int64_t)b * rc;
        for (int a = b; a < rc; ++a) col[fc.rel[a]] += ub[a];
      }
      std::vector<double>().swap(upd[ch]);
    }
    int e = 0;
    if (k > 0)
      e = (use_blas && g_blas.ok && m >= 64) ? partial_chol_blas(F.data(), m, k)
                                             : partial_chol_loops(F.data(), m, k);
    if (e) return f.c0 + e;
    double* Ls = L.data() + f.lofs;
    for (int c = 0; c < k; ++c) std::memcpy(Ls + (int64_t)c * m, F.data() + (int64_t)c * m, sizeof(double) * m);
    if (r > 0) {
      upd[s].resize((size_t)r * r);
      for (int c = 0; c < r; ++c)
        std::memcpy(upd[s].data() + (int64_t)c * r, F.data() + k + (int64_t)(k + c) * m, sizeof(double) * r);
    }
    return 0;
  };

  if (nthreads > 1 && !subtrees_.empty()) {
    // independent subtrees on separate threads, each calling single-threaded BLAS
    if (g_blas.setnt) g_blas.setnt(1);
    std::atomic<int> aerr{0};
    parallel_for(nthreads, (int)subtrees_.size(), [&](int t) {
      for (int s : subtrees_[t]) {
        int e = do_front(s, g_blas.setnt != nullptr);
        if (e) {
          int zero = 0;
          aerr.compare_exchange_strong(zero, e);
          break;
        }
      }
    });
    err = aerr.load();
    if (err) return err;
    if (g_blas.setnt) g_blas.setnt(nthreads);
    for (int s : top_) {
      int e = do_front(s, true);
      if (e) return e;
    }
  } else {
    if (g_blas.setnt) g_blas.setnt(nthreads);
    for (int s = 0; s < nf; ++s) {
      int e = do_front(s, true);
      if (e) return e;
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// solve
// ---------------------------------------------------------------------------
void SparseCholesky::solve(int nrhs, const double* b, double* x) const {
  std::vector<double> y((size_t)n * nrhs);
  for (int r = 0; r < nrhs; ++r)
    for (int i = 0; i < n; ++i) y[(int64_t)r * n + perm[i]] = b[(int64_t)r * n + i];

  // contributions of independent subtrees to rows above them are deferred and
  // applied in a fixed order, so the result does not depend on thread timing
  std::vector<std::vector<std::pair<int64_t, double>>> deferred(subtrees_.size());
  auto fwd = [&](int s, std::vector<std::pair<int64_t, double>>* defer, int top_c0) {
    const Front& f = fronts[s];
    const int m = f.m(), k = f.k(), r = m - k;
    const double* Ls = L.data() + f.lofs;
    std::vector<double> tmp(r);
    for (int rr = 0; rr < nrhs; ++rr) {
      double* yr = y.data() + (int64_t)rr * n;
      double* xs = yr + f.c0;
      // diagonal block: column-oriented forward substitution
      for (int j = 0; j < k; ++j) {
        const double* lj = Ls + (int64_t)j * m;
        const double v = xs[j] / lj[j];
        xs[j] = v;
        for (int i = j + 1; i < k; ++i) xs[i] -= lj[i] * v;
      }
      // rows below: tmp = L21 * xs, streamed column by column
      std::fill(tmp.begin(), tmp.end(), 0.0);
      for (int j = 0; j < k; ++j) {
        const double* lj = Ls + (int64_t)j * m + k;
        const double v = xs[j];
        if (v == 0.0) continue;
        for (int t = 0; t < r; ++t) tmp[t] += lj[t] * v;
      }
      for (int t = 0; t < r; ++t) {
        if (defer && f.rows[t] >= top_c0) {
          defer->push_back({(int64_t)rr * n + f.rows[t], tmp[t]});
        } else {
          yr[f.rows[t]] -= tmp[t];
        }
      }
    }
  };
  auto bwd = [&](int s) {
    const Front& f = fronts[s];
    const int m = f.m(), k = f.k();
    const double* Ls = L.data() + f.lofs;
    std::vector<double> tmp(f.rows.size());
    for (int r = 0; r < nrhs; ++r) {
      double* yr = y.data() + (int64_t)r * n;
      double* xs = yr + f.c0;
      for (size_t t = 0; t < f.rows.size(); ++t) tmp[t] = yr[f.rows[t]];
      for (int j = 0; j < k; ++j) {
        const double* lj = Ls + (int64_t)j * m + k;
        double acc = 0.0;
        for (size_t t = 0; t < tmp.size(); ++t) acc += lj[t] * tmp[t];
        xs[j] -= acc;
      }
      for (int j = k - 1; j >= 0; --j) {
        const double* lj = Ls + (int64_t)j * m;
        double v = xs[j];
        for (int i = j + 1; i < k; ++i) v -= lj[i] * xs[i];
        xs[j] = v / lj[j];
      }
    }
  };

  if (nthreads > 1 && !subtrees_.empty()) {
    parallel_for(nthreads, (int)subtrees_.size(), [&](int t) {
      const int root = subtrees_[t].back();
      for (int s : subtrees_[t]) fwd(s, &deferred[t], fronts[root].c1);
    });
    for (auto& d : deferred)
      for (auto& pr : d) y[pr.first] -= pr.second;
    for (int s : top_) fwd(s, nullptr, 0);
    for (auto it = top_.rbegin(); it != top_.rend(); ++it) bwd(*it);
    parallel_for(nthreads, (int)subtrees_.size(), [&](int t) {
      for (auto it = subtrees_[t].rbegin(); it != subtrees_[t].rend(); ++it) bwd(*it);
    });
  } else {
    for (size_t s = 0; s < fronts.size(); ++s) fwd((int)s, nullptr, 0);
    for (int s = (int)fronts.size() - 1; s >= 0; --s) bwd(s);
  }
  for (int r = 0; r < nrhs; ++r)
    for (int i = 0; i < n; ++i) x[(int64_t)r * n + i] = y[(int64_t)r * n + perm[i]];
}

}  // namespace oracle
