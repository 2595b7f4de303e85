// Host symbolic analysis: nested-dissection ordering, assembly tree, and the
// flattened maps / task lists consumed by the GPU factorization and solves.
#include "symbolic.h"

#include <cstdlib>
#include "parallel.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <climits>
#include <numeric>
#include <exception>
#include <thread>

namespace tdem {
namespace {

// symmetric adjacency without the diagonal: the caller's arrays or its own storage
struct Graph {
  int n = 0;
  const int64_t* xadj = nullptr;  // n + 1 row starts
  const int* adj = nullptr;
  std::vector<int64_t> xadj_store;
  std::vector<int> adj_store;
};

// Recursive dissection producing fronts in postorder.
// The two halves of a split near the top of the tree are dissected on separate
// threads, each by its own Dissector (own marks and stamps); the right half's
// nodes are then appended after the left half's, which is the serial postorder,
// so the ordering does not depend on the threading.
class Dissector {
 public:
  Dissector(const Graph& g, const double* xyz, int leaf)
      : g_(g), xyz_(xyz), leaf_(leaf), mark_(g.n, 0), vis_(g.n, 0) {
    // rank of every coordinate among the distinct values of its axis: the splits
    // then count values instead of sorting them (same order, same cuts)
    if (xyz_) {
      own_rank_.resize(3 * (size_t)g.n);
      // distinct values per axis: each range of vertices sorts and deduplicates its
      // own, then the (short, on a tensor-product mesh) lists are merged
      const int nt = chunk_count(g.n, 65536);
      std::vector<double> vals[3];
      std::vector<std::vector<double>> part((size_t)3 * nt);
      parallel_chunks(g.n, nt, [&](int t, int64_t v0, int64_t v1) {
        for (int a = 0; a < 3; ++a) {
          std::vector<double>& p = part[(size_t)a * nt + t];
          p.reserve((size_t)(v1 - v0));
          for (int64_t v = v0; v < v1; ++v) p.push_back(c((int)v, a));
          std::sort(p.begin(), p.end());
          p.erase(std::unique(p.begin(), p.end()), p.end());
        }
      });
      for (int a = 0; a < 3; ++a) {
        for (int t = 0; t < nt; ++t) {
          const std::vector<double>& p = part[(size_t)a * nt + t];
          vals[a].insert(vals[a].end(), p.begin(), p.end());
        }
        std::sort(vals[a].begin(), vals[a].end());
        vals[a].erase(std::unique(vals[a].begin(), vals[a].end()), vals[a].end());
      }
      parallel_ranges(g.n, [&](int64_t v0, int64_t v1) {
        for (int64_t v = v0; v < v1; ++v)
          for (int a = 0; a < 3; ++a)
            own_rank_[3 * (size_t)v + a] =
                (int)(std::lower_bound(vals[a].begin(), vals[a].end(), c((int)v, a)) - vals[a].begin());
      });
      grank_ = own_rank_.data();
    }
  }

  std::vector<int> order;  // new -> old
  struct Node { int c0, c1; std::vector<int> kids; };
  std::vector<Node> nodes;

  // levels of splits that fork their second half onto a thread: enough for one
  // subtree per host thread (the forked halves are appended in serial order, so the
  // result does not depend on it)
  static int fork_depth() {
    int d = 0;
    while ((1 << d) < host_threads() && d < 5) ++d;
    return d;
  }

  // depth: splits still allowed to fork a thread below this call (fork_depth() at the top)
  int build(std::vector<int>& verts, int depth) {
    if ((int)verts.size() <= leaf_) return emit(verts, {});
    std::vector<int> L, S, R;
    int kind = 0;
    // threads for the passes of one large split: all at the top, fewer where the
    // recursion already runs on several threads
    const int split_threads =
        (int)verts.size() >= kParSplitMin ? std::max(1, host_threads() >> std::max(0, fork_depth() - depth)) : 1;
    if (xyz_ && split_coords(verts, L, S, R, split_threads)) kind = 1;
    if (!kind) kind = split_levels(verts, L, S, R);
    if (!kind) return emit(verts, {});
    std::vector<int>().swap(verts);
    std::vector<int> kids;
    if (depth > 0 && L.size() >= kForkMin && R.size() >= kForkMin) {
      Dissector right(*this);
      int rroot = -1;
      std::exception_ptr err;
      std::thread t([&] {
        try {
          rroot = right.build(R, depth - 1);
        } catch (...) {
          err = std::current_exception();
        }
      });
      try {
        kids.push_back(build(L, depth - 1));
      } catch (...) {
        t.join();
        throw;
      }
      t.join();
      if (err) std::rethrow_exception(err);
      kids.push_back(append(right, rroot));
    } else {
      if (!L.empty()) kids.push_back(build(L, depth - 1));
      if (!R.empty()) kids.push_back(build(R, depth - 1));
    }
    return emit(S, std::move(kids));
  }

 private:
  static constexpr size_t kForkMin = 20000;
  static constexpr int kParSplitMin = 100000;
  const Graph& g_;
  const double* xyz_;
  int leaf_;
  std::vector<int> mark_, vis_;
  std::vector<int> own_rank_;
  const int* grank_ = nullptr;  // per vertex and axis: rank of the coordinate
  std::vector<int> cnt_[3];
  int stamp_ = 0;

  // a dissector for a disjoint part of the same graph, sharing the coordinate ranks
  Dissector(const Dissector& o)
      : g_(o.g_), xyz_(o.xyz_), leaf_(o.leaf_), mark_(o.g_.n, 0), vis_(o.g_.n, 0), grank_(o.grank_) {}

  // appends another dissector's nodes (postorder, renumbered); returns its root's index
  int append(const Dissector& o, int root) {
    const int nb = (int)nodes.size(), cb = (int)order.size();
    order.insert(order.end(), o.order.begin(), o.order.end());
    for (const Node& x : o.nodes) {
      Node nd{x.c0 + cb, x.c1 + cb, x.kids};
      for (int& k : nd.kids) k += nb;
      nodes.push_back(std::move(nd));
    }
    return root + nb;
  }

  int emit(const std::vector<int>& verts, std::vector<int> kids) {
    Node nd;
    nd.c0 = (int)order.size();
    order.insert(order.end(), verts.begin(), verts.end());
    nd.c1 = (int)order.size();
    nd.kids = std::move(kids);
    nodes.push_back(std::move(nd));
    return (int)nodes.size() - 1;
  }

  double c(int v, int a) const { return xyz_[3 * (int64_t)v + a]; }
  int rank(int v, int a) const { return grank_[3 * (size_t)v + a]; }

  // Cut perpendicular to the axis with the most distinct positions, at the most
  // populated coordinate value inside the central 30 % (a node plane on a
  // tensor-product mesh).  The separator is the set of vertices at or above the
  // cut that touch a vertex below it.
  // nt > 1: the histograms and the partition run on nt ranges of verts, each with its
  // own counts and lists, summed and concatenated in range order (the same result)
  bool split_coords(const std::vector<int>& verts, std::vector<int>& L, std::vector<int>& S,
                    std::vector<int>& R, int nt = 1) {
    const size_t nv = verts.size();
    // per axis: histogram of the coordinate ranks over [lo, hi]
    int ndist[3], lo[3];
    {
      std::vector<std::array<int, 6>> ext(nt);  // per range: min and max rank per axis
      parallel_chunks((int64_t)nv, nt, [&](int t, int64_t b, int64_t e) {
        std::array<int, 6>& x = ext[t];
        for (int a = 0; a < 3; ++a) {
          x[a] = INT_MAX;
          x[3 + a] = -1;
        }
        for (int64_t i = b; i < e; ++i)
          for (int a = 0; a < 3; ++a) {
            const int r = rank(verts[i], a);
            x[a] = std::min(x[a], r);
            x[3 + a] = std::max(x[3 + a], r);
          }
      });
      int hi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = INT_MAX;
        hi[a] = -1;
        for (const std::array<int, 6>& x : ext) {
          lo[a] = std::min(lo[a], x[a]);
          hi[a] = std::max(hi[a], x[3 + a]);
        }
      }
      size_t span = 0;
      for (int a = 0; a < 3; ++a) span += (size_t)(hi[a] - lo[a] + 1);
      const int ht = span <= ((size_t)1 << 20) ? nt : 1;  // per-range histograms only when short
      std::vector<std::vector<int>> part(ht);
      parallel_chunks((int64_t)nv, ht, [&](int t, int64_t b, int64_t e) {
        std::vector<int>& h = part[t];
        h.assign(span, 0);
        for (int64_t i = b; i < e; ++i) {
          size_t off = 0;
          for (int a = 0; a < 3; ++a) {
            ++h[off + (size_t)(rank(verts[i], a) - lo[a])];
            off += (size_t)(hi[a] - lo[a] + 1);
          }
        }
      });
      size_t off = 0;
      for (int a = 0; a < 3; ++a) {
        std::vector<int>& cnt = cnt_[a];
        cnt.assign((size_t)(hi[a] - lo[a] + 1), 0);
        for (const std::vector<int>& h : part)
          for (size_t k = 0; k < cnt.size(); ++k) cnt[k] += h[off + k];
        off += cnt.size();
        ndist[a] = (int)(cnt.size() - std::count(cnt.begin(), cnt.end(), 0));
      }
    }
    int axes[3] = {0, 1, 2};
    std::sort(axes, axes + 3, [&](int a, int b) { return ndist[a] > ndist[b]; });
    for (int ai = 0; ai < 3; ++ai) {
      const int a = axes[ai];
      if (ndist[a] < 3) continue;
      // runs of equal values in sorted order: rank lo + idx occupies positions
      // [s0, s0 + cnt[idx]); the window starts at q0 (possibly inside a run)
      const size_t q0 = nv * 35 / 100, q1 = std::max(q0 + 1, nv * 65 / 100);
      const std::vector<int>& cnt = cnt_[a];
      int cut = -1;
      size_t best = 0, pos = 0;
      double bestd = 1e300;
      for (size_t idx = 0; idx < cnt.size(); ++idx) {
        if (!cnt[idx]) continue;
        const size_t s0 = pos, e0 = pos + (size_t)cnt[idx];
        pos = e0;
        if (e0 <= q0) continue;
        const size_t i = std::max(s0, q0), j = e0;
        if (i >= q1) break;
        const double d = std::fabs(0.5 * (double)(i + j) - 0.5 * (double)nv);
        if (j - i > best || (j - i == best && d < bestd)) {
          best = j - i;
          bestd = d;
          cut = lo[a] + (int)idx;
        }
      }
      if (cut <= lo[a]) continue;
      const int st = ++stamp_;
      parallel_chunks((int64_t)nv, nt, [&](int, int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) mark_[verts[i]] = st;
      });
      // 0: below the cut, 1: at or above it and touching a vertex below (separator), 2: the rest
      auto side = [&](int v) {
        if (rank(v, a) < cut) return 0;
        for (int64_t p = g_.xadj[v]; p < g_.xadj[v + 1]; ++p) {
          const int u = g_.adj[p];
          if (mark_[u] == st && rank(u, a) < cut) return 1;
        }
        return 2;
      };
      L.clear();
      S.clear();
      R.clear();
      std::vector<int>* out[3] = {&L, &S, &R};
      if (nt == 1) {
        for (int v : verts) out[side(v)]->push_back(v);
      } else {
        std::vector<std::array<std::vector<int>, 3>> piece(nt);
        parallel_chunks((int64_t)nv, nt, [&](int t, int64_t b, int64_t e) {
          for (int64_t i = b; i < e; ++i) piece[t][side(verts[i])].push_back(verts[i]);
        });
        for (int k = 0; k < 3; ++k)
          for (int t = 0; t < nt; ++t) out[k]->insert(out[k]->end(), piece[t][k].begin(), piece[t][k].end());
      }
      if (!L.empty() && !S.empty()) return true;
    }
    return false;
  }

  // Level-set bisection from a pseudo-peripheral vertex.  Returns 1 (split with a
  // separator level), 2 (disconnected: L = one component, R = the rest), 0 (none).
  int split_levels(const std::vector<int>& verts, std::vector<int>& L, std::vector<int>& S,
                   std::vector<int>& R) {
    const int in = ++stamp_;
    for (int v : verts) mark_[v] = in;
    std::vector<int> seen, lev;
    auto bfs = [&](int s) {
      const int vs = ++stamp_;
      seen.assign(1, s);
      lev.clear();
      vis_[s] = vs;
      size_t head = 0, level_end = 1;
      int depth = 0;
      while (head < seen.size()) {
        const int v = seen[head++];
        lev.push_back(depth);
        for (int64_t p = g_.xadj[v]; p < g_.xadj[v + 1]; ++p) {
          const int u = g_.adj[p];
          if (mark_[u] == in && vis_[u] != vs) {
            vis_[u] = vs;
            seen.push_back(u);
          }
        }
        if (head == level_end) {
          ++depth;
          level_end = seen.size();
        }
      }
    };
    int s = verts[0];
    for (int it = 0; it < 2; ++it) {
      bfs(s);
      s = seen.back();
    }
    bfs(s);
    if (seen.size() < verts.size()) {
      const int vs = stamp_;  // the last bfs stamp marks the component
      L = seen;
      R.clear();
      for (int v : verts)
        if (vis_[v] != vs) R.push_back(v);
      S.clear();
      return 2;
    }
    const int maxd = lev.back();
    if (maxd < 2) return 0;
    int cut = 1;
    for (size_t i = 0; i < seen.size(); ++i)
      if (2 * (i + 1) >= seen.size()) {
        cut = std::max(1, std::min(maxd - 1, lev[i]));
        break;
      }
    L.clear();
    S.clear();
    R.clear();
    for (size_t i = 0; i < seen.size(); ++i)
      (lev[i] < cut ? L : lev[i] == cut ? S : R).push_back(seen[i]);
    return 1;
  }
};

void add_tasks(Symbolic& sy, TaskList& tl, const std::vector<int>& fr,
               const std::vector<int64_t>& ctas) {
  tl.off = (int64_t)sy.tasks.size();
  tl.pre = (int64_t)sy.task_prefix.size();
  tl.count = (int)fr.size();
  int64_t acc = 0;
  sy.task_prefix.push_back(0);
  for (size_t i = 0; i < fr.size(); ++i) {
    sy.tasks.push_back(fr[i]);
    sy.task_aux.push_back(0);
    acc += ctas[i];
    sy.task_prefix.push_back(acc);
  }
  tl.ctas = acc;
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

std::string analyse(int n, const int64_t* rowptr, const int* colind, const double* coords,
                    Symbolic& sy, int leaf_size, const int64_t* adj_ptr, const int* adj) {
  sy = Symbolic();
  sy.n = n;
  sy.nnz_lower = rowptr[n];
  if (n <= 0) return "empty matrix";

  // symmetric adjacency without the diagonal
  Graph g;
  g.n = n;
  if (adj_ptr && adj) {
    // the caller's (each row ascending, the order built below); the lower triangle is
    // only checked
    std::vector<char> bad(host_threads() + 1, 0);
    parallel_ranges(n, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i)
        for (int64_t q = rowptr[i]; q < rowptr[i + 1]; ++q)
          if (colind[q] < 0 || colind[q] > i) bad[0] = 1;
    });
    if (bad[0]) return "lower-triangle pattern expected (column index out of range)";
    g.xadj = adj_ptr;
    g.adj = adj;
  } else {
    // Row v lists its own lower entries (CSR order) and then the rows i > v that hold
    // an entry in column v, ascending.  The transposed part is placed per range of
    // rows after the entries of the lower ranges, which keeps that order.
    std::vector<int64_t>& xadj = g.xadj_store;
    std::vector<int>& adjv = g.adj_store;
    const int nt = chunk_count(n, 16384);
    std::vector<int64_t> own(n, 0);
    std::vector<int> upper((size_t)nt * n, 0);  // per range: entries of each column
    std::vector<char> bad(nt, 0);
    parallel_chunks(n, nt, [&](int t, int64_t i0, int64_t i1) {
      int* up = upper.data() + (size_t)t * n;
      for (int64_t i = i0; i < i1; ++i)
        for (int64_t q = rowptr[i]; q < rowptr[i + 1]; ++q) {
          const int j = colind[q];
          if (j < 0 || j > i) {
            bad[t] = 1;
            return;
          }
          if (j == i) continue;
          ++own[i];
          ++up[j];
        }
    });
    for (char b : bad)
      if (b) return "lower-triangle pattern expected (column index out of range)";
    xadj.assign(n + 1, 0);
    for (int v = 0; v < n; ++v) {
      int64_t d = own[v];
      for (int t = 0; t < nt; ++t) d += upper[(size_t)t * n + v];
      xadj[v + 1] = xadj[v] + d;
    }
    // turn the per-range counts into the first slot of each range in each column
    parallel_ranges(n, [&](int64_t v0, int64_t v1) {
      for (int64_t v = v0; v < v1; ++v) {
        int64_t at = xadj[v] + own[v];
        for (int t = 0; t < nt; ++t) {
          int& c = upper[(size_t)t * n + v];
          const int k = c;
          c = (int)(at - xadj[v]);
          at += k;
        }
      }
    });
    adjv.resize(xadj[n]);
    parallel_chunks(n, nt, [&](int t, int64_t i0, int64_t i1) {
      int* up = upper.data() + (size_t)t * n;
      for (int64_t i = i0; i < i1; ++i) {
        int64_t o = xadj[i];
        for (int64_t q = rowptr[i]; q < rowptr[i + 1]; ++q) {
          const int j = colind[q];
          if (j == i) continue;
          adjv[o++] = j;
          adjv[xadj[j] + up[j]++] = (int)i;
        }
      }
    });
    g.xadj = xadj.data();
    g.adj = adjv.data();
  }

  // ordering + tree
  Dissector d(g, coords, std::max(8, leaf_size));
  {
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    d.build(all, Dissector::fork_depth());
  }
  sy.iperm = d.order;
  if ((int)sy.iperm.size() != n) return "ordering lost vertices";
  sy.perm.assign(n, -1);
  for (int i = 0; i < n; ++i) sy.perm[sy.iperm[i]] = i;

  const int nf = (int)d.nodes.size();
  sy.fronts.assign(nf, FrontInfo());
  for (int s = 0; s < nf; ++s) {
    sy.fronts[s].c0 = d.nodes[s].c0;
    sy.fronts[s].c1 = d.nodes[s].c1;
    sy.fronts[s].children = d.nodes[s].kids;
    for (int ch : d.nodes[s].kids) sy.fronts[ch].parent = s;
  }
  std::vector<int> colfront(n);
  for (int s = 0; s < nf; ++s)
    for (int cc = sy.fronts[s].c0; cc < sy.fronts[s].c1; ++cc) colfront[cc] = s;

  // row structures: a front's rows are its columns' neighbours and its children's
  // rows beyond its columns.  Tree levels first (postorder: children first), then
  // the fronts of one level in parallel, each thread with its own marks.
  {
    for (int s = 0; s < nf; ++s) {
      int lev = 0;
      for (int ch : sy.fronts[s].children) lev = std::max(lev, sy.fronts[ch].level + 1);
      sy.fronts[s].level = lev;
    }
    int nlev_rs = 0;
    for (const FrontInfo& f : sy.fronts) nlev_rs = std::max(nlev_rs, f.level + 1);
    std::vector<std::vector<int>> by_level(nlev_rs);
    for (int s = 0; s < nf; ++s) by_level[sy.fronts[s].level].push_back(s);
    const int nth = host_threads();
    std::vector<std::vector<int>> marks(nth);
    for (const std::vector<int>& lvl : by_level) {
      const int nt = std::min(nth, chunk_count((int64_t)lvl.size(), 8));
      parallel_chunks((int64_t)lvl.size(), nt, [&](int t, int64_t a, int64_t b) {
        std::vector<int>& st = marks[t];
        if (st.empty()) st.assign(n, -1);
        std::vector<int> tmp;
        for (int64_t x = a; x < b; ++x) {
          const int s = lvl[x];
          FrontInfo& f = sy.fronts[s];
          tmp.clear();
          for (int cc = f.c0; cc < f.c1; ++cc) {
            const int i = sy.iperm[cc];
            for (int64_t p = g.xadj[i]; p < g.xadj[i + 1]; ++p) {
              const int r = sy.perm[g.adj[p]];
              if (r >= f.c1 && st[r] != s) {
                st[r] = s;
                tmp.push_back(r);
              }
            }
          }
          for (int ch : f.children)
            for (int r : sy.fronts[ch].rows)
              if (r >= f.c1 && st[r] != s) {
                st[r] = s;
                tmp.push_back(r);
              }
          std::sort(tmp.begin(), tmp.end());
          f.rows = tmp;
        }
      });
    }
  }

  // offsets, sizes, stats
  sy.l_off.resize(nf);
  sy.u_off.assign(nf, 0);
  sy.front_m.resize(nf);
  sy.front_k.resize(nf);
  sy.front_c0.resize(nf);
  sy.front_parent.resize(nf);
  sy.rows_off.resize(nf + 1);
  sy.wvec_off.resize(nf);
  int64_t off = 0, woff = 0, roff = 0;
  for (int s = 0; s < nf; ++s) {
    const FrontInfo& f = sy.fronts[s];
    const int64_t m = f.m(), k = f.k();
    sy.l_off[s] = off;
    sy.front_m[s] = (int)m;
    sy.front_k[s] = (int)k;
    sy.front_c0[s] = f.c0;
    sy.front_parent[s] = f.parent;
    sy.wvec_off[s] = woff;
    sy.rows_off[s] = roff;
    off += m * k;
    sy.u_sum += (m - k) * (m - k);
    woff += m;
    roff += m;
    sy.nnz_l += m * k;
    const double dm = (double)m, dk = (double)k;
    // k^3/3 (pivot block) + r k^2 (panel solve) + r^2 k (lower-triangle Schur update),
    // r = m - k, a multiply-add counted as two flops
    sy.flops += dk * dk * dk / 3.0 + (dm - dk) * dk * dk + (dm - dk) * (dm - dk) * dk;
    sy.max_m = std::max(sy.max_m, (int)m);
    sy.max_k = std::max(sy.max_k, (int)k);
  }
  sy.rows_off[nf] = roff;
  sy.wvec_elems = woff;
  sy.rows_all.resize(roff);
  for (int s = 0; s < nf; ++s) {
    const FrontInfo& f = sy.fronts[s];
    int64_t o = sy.rows_off[s];
    for (int cc = f.c0; cc < f.c1; ++cc) sy.rows_all[o++] = cc;
    for (int r : f.rows) sy.rows_all[o++] = r;
  }

  // relative maps child rows -> parent front slots (parents in parallel, each thread
  // with its own slot map and the parent that set each slot)
  {
    sy.rel_off.assign(nf + 1, 0);
    for (int s = 0; s < nf; ++s) sy.rel_off[s + 1] = sy.rel_off[s] + (int64_t)sy.fronts[s].rows.size();
    sy.rel.assign(sy.rel_off[nf], -1);
    const int nt = chunk_count(nf, 64);
    std::vector<char> missing(nt, 0);
    parallel_chunks(nf, nt, [&](int t, int64_t p0, int64_t p1) {
      std::vector<int> pos(n, -1), owner(n, -1);
      for (int64_t p = p0; p < p1; ++p) {
        const FrontInfo& fp = sy.fronts[p];
        for (int cc = fp.c0; cc < fp.c1; ++cc) {
          pos[cc] = cc - fp.c0;
          owner[cc] = (int)p;
        }
        for (size_t x = 0; x < fp.rows.size(); ++x) {
          pos[fp.rows[x]] = fp.k() + (int)x;
          owner[fp.rows[x]] = (int)p;
        }
        for (int ch : fp.children) {
          const FrontInfo& fc = sy.fronts[ch];
          for (size_t x = 0; x < fc.rows.size(); ++x) {
            const int r = fc.rows[x];
            if (owner[r] != p) {
              missing[t] = 1;
              return;
            }
            sy.rel[sy.rel_off[ch] + x] = pos[r];
          }
        }
      }
    });
    for (char b : missing)
      if (b) return "internal error: child row missing from parent front";
    for (int s = 0; s < nf; ++s)
      if (sy.fronts[s].parent < 0 && !sy.fronts[s].rows.empty())
        return "internal error: root front with off-diagonal rows";
  }

  // entry map: lower-CSR entry -> front element.  An entry (i, j) lands in the front
  // of column min(perm i, perm j), at the local row of max(perm i, perm j): one of the
  // front's own columns, or found by binary search in its sorted row list (rows_all).
  // Every entry is placed on its own, so rows of the CSR run in parallel.
  {
    sy.entry_dst.assign(sy.nnz_lower, -1);
    const int nt = chunk_count(n, 16384);
    std::vector<char> bad(nt, 0);
    parallel_chunks(n, nt, [&](int t, int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) {
        const int a = sy.perm[i];
        for (int64_t q = rowptr[i]; q < rowptr[i + 1]; ++q) {
          const int b = sy.perm[colind[q]];
          const int col = std::min(a, b), row = std::max(a, b);
          const int f = colfront[col];
          const int c0 = sy.front_c0[f], k = sy.front_k[f];
          const int64_t m = sy.front_m[f];
          const int lc = col - c0;
          int64_t lr;
          if (row < c0 + k) {
            lr = row - c0;
          } else {
            const int* r0 = sy.rows_all.data() + sy.rows_off[f] + k;
            const int* r1 = sy.rows_all.data() + sy.rows_off[f] + m;
            const int* p = std::lower_bound(r0, r1, row);
            if (p == r1 || *p != row) {
              bad[t] = 1;
              return;
            }
            lr = k + (p - r0);
          }
          if (lc < 0 || lc >= k || lr < lc) {
            bad[t] = 1;
            return;
          }
          sy.entry_dst[q] = sy.l_off[f] + lr + (int64_t)lc * m;
        }
      }
    });
    for (char x : bad)
      if (x) return "internal error: entry outside its front";
  }

  // level plans
  int nlev = 0;
  for (auto& f : sy.fronts) nlev = std::max(nlev, f.level + 1);
  sy.levels.assign(nlev, LevelPlan());
  for (int s = 0; s < nf; ++s) sy.levels[sy.fronts[s].level].fronts.push_back(s);
  int64_t max_partials = 0;
  for (int l = 0; l < nlev; ++l) {
    LevelPlan& lp = sy.levels[l];
    // extend-add slots: slot j = j-th child of each front at this level; one CTA
    // per child column block of 8 columns
    int max_kids = 0;
    for (int s : lp.fronts) max_kids = std::max(max_kids, (int)sy.fronts[s].children.size());
    for (int j = 0; j < max_kids; ++j) {
      std::vector<int> fr;
      std::vector<int64_t> ct, cv;
      for (int s : lp.fronts)
        if ((int)sy.fronts[s].children.size() > j) {
          const int ch = sy.fronts[s].children[j];
          const int64_t r = (int64_t)sy.fronts[ch].rows.size();
          if (r == 0) continue;
          fr.push_back(ch);
          ct.push_back(cdiv(r, 8));
          cv.push_back(cdiv(r, kSolveRows));
        }
      TaskList tl, tv;
      add_tasks(sy, tl, fr, ct);
      add_tasks(sy, tv, fr, cv);
      lp.extend_slots.push_back(tl);
      lp.extend_vec.push_back(tv);
    }
    {
      std::vector<int64_t> ct;
      for (int s : lp.fronts) ct.push_back(cdiv(sy.front_m[s], kSolveRows));
      add_tasks(sy, lp.assemble, lp.fronts, ct);
    }
    int kmax = 0;
    for (int s : lp.fronts) kmax = std::max(kmax, sy.front_k[s]);
    // TDEM_OZAKI_ALL=1 plans every trailing update that fits the digit buffer on the
    // integer tensor pipe (tests of small models)
    const char* oz_all = std::getenv("TDEM_OZAKI_ALL");
    const double oz_min_flops = (oz_all && oz_all[0] == '1') ? 0.0 : kOzMinFlops;
    for (int j0 = 0; j0 < kmax; j0 += kPanel) {
      PanelStep ps;
      ps.j0 = j0;
      std::vector<int> fr, fin, fbig, frest;
      std::vector<int64_t> c1, c2, c3, c4, c5, c6, c6a, c6b;
      const int J0 = (j0 / kOuter) * kOuter;
      for (int s : lp.fronts) {
        const int k = sy.front_k[s], m = sy.front_m[s];
        if (k <= j0) continue;
        const int j1 = std::min(k, j0 + kPanel);
        const int J1 = std::min(k, J0 + kOuter);
        const int64_t below = m - j1;
        fr.push_back(s);
        c1.push_back(1);
        c2.push_back(cdiv(below, kTrsmRows));
        c4.push_back(cdiv(below, kSolveRows));
        if (j1 < J1) {
          // rows [j1, m) x columns [j1, J1) of the outer panel, lower-triangle tiles
          const int64_t nr = cdiv(below, kTileSyrk), nc = cdiv(J1 - j1, kTileSyrk);
          fin.push_back(s);
          c3.push_back(nc * nr - nc * (nc - 1) / 2);
          // 128 x 64 tiles: column tile bj with row tiles bj / 2 .. nr128 - 1
          const int64_t nr128 = cdiv(below, kTileBig), nc64 = cdiv(J1 - j1, 64);
          int64_t w6 = 0;
          for (int64_t bj = 0; bj < nc64; ++bj) w6 += nr128 - bj / 2;
          c6.push_back(w6);
          c6a.push_back(nr128);
          if (w6 > nr128) {
            frest.push_back(s);
            c6b.push_back(w6 - nr128);
          }
        } else if (m > J1) {
          const int64_t nt = cdiv(m - J1, kTileBig);
          fbig.push_back(s);
          c5.push_back(nt * (nt + 1) / 2);
        }
      }
      add_tasks(sy, ps.potrf, fr, c1);
      add_tasks(sy, ps.trsm, fr, c2);
      add_tasks(sy, ps.syrk, fin, c3);
      add_tasks(sy, ps.syrk_wide, fin, c6);
      add_tasks(sy, ps.syrk_next, fin, c6a);
      add_tasks(sy, ps.syrk_rest, frest, c6b);
      add_tasks(sy, ps.syrk_big, fbig, c5);
      {
        // the Ozaki path: slice-buffer rows of the fronts, in task order
        int64_t rows = 0;
        double fl = 0.0;
        std::vector<int64_t> c7;
        for (size_t q = 0; q < fbig.size(); ++q) {
          const int s = fbig[q], k = sy.front_k[s], m = sy.front_m[s];
          const int J1 = std::min(k, J0 + kOuter);
          sy.task_aux[ps.syrk_big.off + q] = rows;
          rows += m - J1;
          fl += (double)(m - J1) * (m - J1) * (J1 - J0);
          c7.push_back(cdiv(m - J1, 64));
        }
        if (!fbig.empty() && rows <= kOzRowsCap && fl >= oz_min_flops) {
          ps.ozaki = true;
          ps.oz_rows = rows;
          // 128 x 64 output tiles (the right half of a last 128-column tile past the
          // front is skipped) x K blocks of 64 digits x the kept digit pairs
          for (int s : fbig) {
            const int k = sy.front_k[s], m = sy.front_m[s];
            const int J1 = std::min(k, J0 + kOuter);
            const int64_t r = m - J1, nt = cdiv(r, 128);
            const int64_t ctas = nt * (nt + 1) - ((r - (nt - 1) * 128) <= 64 ? 1 : 0);
            const int64_t kpad = cdiv(J1 - J0, 64) * 64;
            sy.oz_macs += (double)ctas * 128.0 * 64.0 * (double)kpad * (kOzSlices * (kOzSlices + 1) / 2);
          }
          sy.oz_rows_max = std::max(sy.oz_rows_max, rows);
          sy.oz_flops += fl;
          add_tasks(sy, ps.oz_slice, fbig, c7);
          for (size_t q = 0; q < fbig.size(); ++q) sy.task_aux[ps.oz_slice.off + q] = sy.task_aux[ps.syrk_big.off + q];
        }
      }
      add_tasks(sy, ps.solve_upd, fr, c4);
      max_partials = std::max(max_partials, ps.solve_upd.ctas);
      lp.panels.push_back(ps);
    }
  }
  sy.solve_partials = max_partials * kPanel;

  // fused-solve items, flags and inverted diagonal blocks
  {
    sy.flag_off.assign(nf, 0);
    sy.dinv_off.assign(nf, 0);
    for (int s = 0; s < nf; ++s) {
      const int k = sy.front_k[s];
      const int pb = (int)cdiv(k, kPanel);
      sy.flag_off[s] = sy.n_flags;
      sy.n_flags += pb;
      sy.dinv_off[s] = sy.dinv_elems;
      sy.dinv_elems += (int64_t)(pb - 1) * kPanel * kPanel + (int64_t)(k - (pb - 1) * kPanel) * (k - (pb - 1) * kPanel);
    }
    auto push = [&](int s, int b) {
      sy.solve_items.push_back(s);
      sy.solve_items.push_back(b);
    };
    // A unit of a level solve: row block (forward) or column block (backward) R of
    // one front, the block range [lo, hi) it accumulates, its partial-sum slot, the
    // counter of its row and, for the final unit of a row, the number of partials
    // to add.  The final unit of a row takes the newest blocks (the ones next to
    // the diagonal), the older ones are split into chunks of kSolveChunk blocks
    // whose partial sums it adds; the dependency chain then advances by one block
    // per link.  The record also carries the front's sizes and offsets, so a CTA
    // needs one load per unit.
    struct Cand {
      int key, cls;
      int rec[kUnitInts];
    };
    auto make = [&](std::vector<Cand>& out, int key, int cls, int s, int row, int lo, int hi, int slot, int cnt,
                    int nparts, int fin) {
      Cand c;
      c.key = key;
      c.cls = cls;
      int* r = c.rec;
      r[0] = row; r[1] = lo; r[2] = hi; r[3] = slot; r[4] = cnt; r[5] = nparts; r[6] = fin;
      r[7] = sy.front_m[s]; r[8] = sy.front_k[s]; r[9] = (int)sy.flag_off[s];
      const int64_t o64[3] = {sy.l_off[s], sy.wvec_off[s], sy.dinv_off[s]};
      for (int j = 0; j < 3; ++j) {
        r[10 + 2 * j] = (int)(uint32_t)(o64[j] & 0xffffffffu);
        r[11 + 2 * j] = (int)(uint32_t)((uint64_t)o64[j] >> 32);
      }
      out.push_back(c);
    };
    // Ticket order: by key (when the unit's inputs start to appear along the
    // dependency chain), final units before the others of the same key, then by
    // row (forward) or last column first (backward).  Every unit a unit waits for
    // must hold a smaller ticket; the replay below checks this for every launch.
    auto emit = [&](std::vector<Cand>& v) {
      std::stable_sort(v.begin(), v.end(), [](const Cand& a, const Cand& b) {
        return a.key != b.key ? a.key < b.key : a.cls < b.cls;
      });
      for (const Cand& c : v) sy.solve_units.insert(sy.solve_units.end(), c.rec, c.rec + kUnitInts);
    };
    int64_t max_slots = 0;
    if ((int64_t)sy.n_flags >= (int64_t)INT32_MAX) return "too many pivot blocks";
    for (int l = 0; l < nlev; ++l) {
      LevelPlan& lp = sy.levels[l];
      std::vector<Cand> cand;
      // forward: row block R < pb (pivot rows, needs q < R) or R >= pb (update rows,
      // needs q < pb).  A pivot row is a link of the dependency chain: its final
      // unit takes the newest kSolveLookahead + 1 blocks and is queued by the first
      // of them, so it is running (streaming its blocks as their flags appear) well
      // before the chain reaches it.  Chunks and update rows are queued by the last
      // block they need.
      int rmax = 0;
      for (int s : lp.fronts)
        rmax = std::max(rmax, (int)(cdiv(sy.front_k[s], kPanel) + cdiv(sy.front_m[s] - sy.front_k[s], kPanel)));
      lp.fwd_off = (int64_t)sy.solve_units.size() / kUnitInts;
      int64_t slots = 0;
      for (int R = 0; R < rmax; ++R)
        for (int s : lp.fronts) {
          const int pb = (int)cdiv(sy.front_k[s], kPanel), ub = (int)cdiv(sy.front_m[s] - sy.front_k[s], kPanel);
          if (R >= pb + ub) continue;
          const int cnt = (int)sy.n_counters++;
          if (R < pb) {
            const int lo = std::max(0, R - 1 - kSolveLookahead);
            const int nch = (int)cdiv(lo, kSolveChunk);
            for (int c = 0; c < nch; ++c) {
              const int hi = std::min(lo, (c + 1) * kSolveChunk);
              make(cand, hi - 1, 1, s, R, c * kSolveChunk, hi, (int)(slots + c), cnt, 0, 0);
            }
            make(cand, R == 0 ? -1 : lo, 0, s, R, lo, R, (int)slots, cnt, nch, 1);
            slots += nch;
          } else {
            // short rows stay in one unit; long ones leave only the newest block to the final unit
            const int nch = pb - 1 > kSolveChunk ? (int)cdiv(pb - 1, kSolveChunk) : 0;
            for (int c = 0; c < nch; ++c) {
              const int hi = std::min(pb - 1, (c + 1) * kSolveChunk);
              make(cand, hi - 1, 1, s, R, c * kSolveChunk, hi, (int)(slots + c), cnt, 0, 0);
            }
            make(cand, pb - 1, 1, s, R, nch > 0 ? pb - 1 : 0, pb, (int)slots, cnt, nch, 1);
            slots += nch;
          }
        }
      emit(cand);
      lp.fwd_count = (int64_t)sy.solve_units.size() / kUnitInts - lp.fwd_off;
      max_slots = std::max(max_slots, slots);
      // backward: column block p (last first) needs the row blocks R in (p, pb + ub).
      // Flag R is set at step pb - 1 - R of the chain.  The final unit of column p
      // takes rows [p + 1, p + 2 + kSolveLookahead) and is queued by the earliest
      // flag among them; chunks (the rows beyond) are queued by their latest flag.
      // Units that wait for no flag come first: an empty final unit at -2, chunks
      // over update rows only at -1, a final unit over update rows only at 0 (after
      // its chunks).
      cand.clear();
      int pmax = 0;
      for (int s : lp.fronts) pmax = std::max(pmax, (int)cdiv(sy.front_k[s], kPanel));
      lp.bwd_off = (int64_t)sy.solve_units.size() / kUnitInts;
      slots = 0;
      for (int d = 0; d < pmax; ++d)
        for (int s : lp.fronts) {
          const int pb = (int)cdiv(sy.front_k[s], kPanel), ub = (int)cdiv(sy.front_m[s] - sy.front_k[s], kPanel);
          if (d >= pb) continue;
          const int p = pb - 1 - d, rend = pb + ub;
          const int cnt = (int)sy.n_counters++;
          const int lo = std::min(p + 1, rend), first = std::min(rend, p + 2 + kSolveLookahead);
          const int nch = (int)cdiv(rend - first, kSolveChunk);
          for (int c = 0; c < nch; ++c) {
            const int clo = first + c * kSolveChunk, chi = std::min(rend, first + (c + 1) * kSolveChunk);
            make(cand, clo < pb ? pb - 1 - clo : -1, 1, s, p, clo, chi, (int)(slots + c), cnt, 0, 0);
          }
          const int fkey = lo == first ? -2 : (lo < pb ? pb - std::min(first, pb) : 0);
          make(cand, fkey, 0, s, p, lo, first, (int)slots, cnt, nch, 1);
          slots += nch;
        }
      emit(cand);
      lp.bwd_count = (int64_t)sy.solve_units.size() / kUnitInts - lp.bwd_off;
      max_slots = std::max(max_slots, slots);
    }
    sy.solve_slots = max_slots;
    // Replay every launch's units in ticket order: each pivot-block flag and
    // chunk counter a unit waits for must come from an earlier unit, otherwise
    // CTAs holding early tickets could wait for units that never start.
    {
      std::vector<char> flag(sy.n_flags);
      std::vector<int> done(sy.n_counters);
      for (int dir = 0; dir < 2; ++dir)
        for (const LevelPlan& lp : sy.levels) {
          const int64_t off = dir ? lp.bwd_off : lp.fwd_off, cnt = dir ? lp.bwd_count : lp.fwd_count;
          for (int64_t x = off; x < off + cnt; ++x) {
            const int* u = &sy.solve_units[kUnitInts * x];
            const int R = u[0], lo = u[1], hi = u[2], c = u[4], nparts = u[5], fin = u[6], f0 = u[9];
            const int pb = (int)cdiv(u[8], kPanel);
            if (hi - lo > kUnitBlocks) return "internal error: level-solve unit longer than kUnitBlocks";
            for (int q = lo; q < std::min(hi, pb); ++q)
              if (!flag[f0 + q]) return "internal error: level-solve unit waits for a later unit";
            if (fin && done[c] != nparts) return "internal error: level-solve row finishes before its chunks";
            if (!fin) ++done[c];
            else if (dir == 1 || R < pb) flag[f0 + R] = 1;
          }
          if (dir == 0 && &lp == &sy.levels.back()) std::fill(flag.begin(), flag.end(), 0);
        }
    }
    sy.inv_off = (int64_t)sy.solve_items.size() / 2;
    for (int s = 0; s < nf; ++s)
      for (int b = 0; b < cdiv(sy.front_k[s], kPanel); ++b) push(s, b);
    sy.inv_count = (int64_t)sy.solve_items.size() / 2 - sy.inv_off;
  }

  // Update-block workspace: first-fit plan over the level sequence.  A block is
  // allocated when its front's level starts and released once the parent's level
  // has assembled it (children are consumed at the start of the parent's level).
  {
    struct Blk { int64_t off, len; };
    std::vector<Blk> free_list{{0, INT64_MAX / 4}};
    auto alloc = [&](int64_t len) -> int64_t {
      len = (len + 31) / 32 * 32;  // 256-byte alignment in FP64
      for (size_t i = 0; i < free_list.size(); ++i)
        if (free_list[i].len >= len) {
          const int64_t o = free_list[i].off;
          free_list[i].off += len;
          free_list[i].len -= len;
          if (free_list[i].len == 0) free_list.erase(free_list.begin() + i);
          return o;
        }
      return -1;
    };
    auto release = [&](int64_t o, int64_t len) {
      len = (len + 31) / 32 * 32;
      auto it = std::lower_bound(free_list.begin(), free_list.end(), o,
                                 [](const Blk& b, int64_t v) { return b.off < v; });
      it = free_list.insert(it, {o, len});
      // merge with neighbours
      size_t i = it - free_list.begin();
      if (i + 1 < free_list.size() && free_list[i].off + free_list[i].len == free_list[i + 1].off) {
        free_list[i].len += free_list[i + 1].len;
        free_list.erase(free_list.begin() + i + 1);
      }
      if (i > 0 && free_list[i - 1].off + free_list[i - 1].len == free_list[i].off) {
        free_list[i - 1].len += free_list[i].len;
        free_list.erase(free_list.begin() + i);
      }
    };
    int64_t peak = 0;
    for (int l = 0; l < nlev; ++l) {
      for (int s : sy.levels[l].fronts) {
        const int64_t r = sy.front_m[s] - sy.front_k[s];
        if (r == 0) continue;
        const int64_t o = alloc(r * r);
        if (o < 0) return "internal error: workspace plan failed";
        sy.u_off[s] = o;
        peak = std::max(peak, o + (r * r + 31) / 32 * 32);
      }
      for (int s : sy.levels[l].fronts)
        for (int ch : sy.fronts[s].children) {
          const int64_t r = sy.front_m[ch] - sy.front_k[ch];
          if (r > 0) release(sy.u_off[ch], r * r);
        }
    }
    sy.u_elems = peak;
  }
  return "";
}

uint64_t plan_digest(const Symbolic& sy) {
  uint64_t h = 1469598103934665603ull;
  auto word = [&](uint64_t u) {
    for (int b = 0; b < 8; ++b) h = (h ^ ((u >> (8 * b)) & 0xff)) * 1099511628211ull;
  };
  auto ints = [&](const auto& v) {
    word(v.size());
    for (auto x : v) word((uint64_t)(int64_t)x);
  };
  ints(sy.perm);
  for (const FrontInfo& f : sy.fronts) {
    word((uint64_t)f.c0);
    word((uint64_t)f.c1);
    ints(f.rows);
  }
  ints(sy.entry_dst);
  ints(sy.solve_units);
  return h;
}

}  // namespace tdem
