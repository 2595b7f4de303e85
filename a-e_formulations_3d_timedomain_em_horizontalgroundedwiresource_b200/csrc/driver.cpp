// Transient driver (see driver.h).
#include "driver.h"
#include "parallel.h"

#include <algorithm>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <ctime>
#include <sys/stat.h>
#include <nvtx3/nvToolsExt.h>

#include "fem_kernels.h"
#include "symbolic.h"

namespace tdem {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Wall time at library load: phase marks count clock ticks from here, as clock()
// counts from process start on the reference's platform.
const double g_process_origin_s = now_s();

bool file_exists(const std::string& path) {
  struct stat st;
  return !path.empty() && ::stat(path.c_str(), &st) == 0;
}

#define TRY_CUDA(x)                                                              \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_); \
  } while (0)

// Reference-cube edge basis at `in` (each coordinate in [-1, 1]) dotted with d
// (T_Brick::Basis_func_on_reference_vec_par, T_Brick.cpp:741-811).
double basis_dot(int j, const double in[3], const double d[3]) {
  auto l0 = [](double t) { return (1.0 - t) * 0.5; };
  auto l1 = [](double t) { return (t + 1.0) * 0.5; };
  const int dir = j >> 2, a = j & 1, b = (j >> 1) & 1;
  const int u = (dir + 1) % 3, v = (dir + 2) % 3;
  const double fa = a ? l1(in[u]) : l0(in[u]);
  const double fb = b ? l1(in[v]) : l0(in[v]);
  return fa * fb * d[dir];
}

// dA_dt of the reference with its argument order (time_approx.cpp:1361-1374).
double ref_dA_dt(double t, double u_j, double u_j1, double u_j2, double dt, double dt0, double dt1,
                 double t_j, double t_j1, double t_j2) {
  if (t < t_j2) t = t_j2;
  if (t > t_j) t = t_j;
  return u_j2 * (2.0 * t - t_j - t_j1) / (dt1 * dt) - u_j1 * (2.0 * t - t_j - t_j2) / (dt1 * dt0) +
         u_j * (2.0 * t - t_j1 - t_j2) / (dt * dt0);
}

}  // namespace

std::vector<int> decade_starts(const std::vector<double>& time) {
  std::vector<int> ig{0};
  const int nt = (int)time.size();
  double hpre = time[1] - time[0];
  for (int i = 2; i < nt; ++i) {
    const double hcur = time[i] - time[i - 1];
    if (std::fabs(1.0 - hpre / hcur) > 1e-3) {
      ig.push_back(i);
      hpre = hcur;
    }
  }
  ig.push_back(nt);
  return ig;
}

int find_time_layer(const std::vector<double>& time, double val) {
  const int nt = (int)time.size();
  if (nt < 1) return -1;
  if (std::fabs(val) < 1e-14 && std::fabs(time[0]) < 1e-14) return 0;
  for (int it = 1; it < nt; ++it)
    if (std::fabs(1.0 - time[it] / val) < 1e-6) return it;
  return -1;
}

void TransientSolve::mark_host(const std::string& label) {
  if (opt_.time_watcher.empty()) return;
  nvtxMarkA(label.c_str());
  PhaseMark m;
  m.label = label;
  m.wall_s = now_s();
  marks_.push_back(std::move(m));
}

std::string TransientSolve::mark_device(const std::string& label, cudaStream_t s) {
  if (opt_.time_watcher.empty()) return "";
  nvtxMarkA(label.c_str());
  PhaseMark m;
  m.label = label;
  TRY_CUDA(cudaEventCreate(&m.ev));
  marks_.push_back(m);
  TRY_CUDA(cudaEventRecord(m.ev, s));
  return "";
}

std::string TransientSolve::flush_marks() {
  if (opt_.time_watcher.empty() || marks_.empty()) return "";
  std::vector<std::pair<double, std::string>> lines;
  std::string err;
  for (PhaseMark& m : marks_) {
    double w = m.wall_s;
    if (m.ev) {
      float ms = 0.f;
      if (mark_origin_ && cudaEventElapsedTime(&ms, mark_origin_, m.ev) == cudaSuccess)
        w = mark_origin_s_ + 1e-3 * ms;
      else
        err = "CUDA: a phase mark did not complete";
      cudaEventDestroy(m.ev);
    }
    lines.emplace_back(w, m.label);
  }
  marks_.clear();
  std::stable_sort(lines.begin(), lines.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  FILE* f = std::fopen(opt_.time_watcher.c_str(), "a");
  if (!f) return "cannot append to " + opt_.time_watcher;
  for (const auto& l : lines)
    std::fprintf(f, "%lld\t%s\n", (long long)((l.first - g_process_origin_s) * CLOCKS_PER_SEC), l.second.c_str());
  std::fclose(f);
  return err;
}

TransientSolve::TransientSolve() = default;
TransientSolve::~TransientSolve() {
  for (PhaseMark& m : marks_)
    if (m.ev) cudaEventDestroy(m.ev);
  if (mark_origin_) cudaEventDestroy(mark_origin_);
  chol_.reset();
  if (hs_) cudaStreamDestroy(hs_);
  if (fs_) cudaStreamDestroy(fs_);
  for (cudaEvent_t& ev : ev_)
    if (ev) cudaEventDestroy(ev);
  for (void* p : allocs_) cudaFree(p);
}

std::string TransientSolve::alloc(void** p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) return std::string("cudaMalloc: ") + cudaGetErrorString(e);
  allocs_.push_back(*p);
  return "";
}

template <class T>
std::string TransientSolve::upload(T** d, const std::vector<T>& h) {
  std::string e = alloc((void**)d, h.size() * sizeof(T));
  if (!e.empty()) return e;
  if (!h.empty()) TRY_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s_));
  pt_.h2d_bytes += (int64_t)(h.size() * sizeof(T));
  return "";
}

double TransientSolve::source_coef(int itime, bool two_layer, double dt) const {
  if (!have_source_) return 0.0;
  const auto& cf = m_.currentfunction;
  const auto& t = m_.time;
  if (opt_.formulation == 0) return cf[itime] != 0.0 ? cf[itime] : 0.0;
  // E-form: -dJ/dt (time_approx.cpp E-form 1085-1102; Two_Layers_Schema 756-773)
  double djdt;
  if (itime + 1 < ntime_) {
    if (cf[itime] == 0.0) {
      const double den = two_layer ? dt : (t[itime] - t[itime - 1]);
      djdt = ((cf[itime] - cf[itime - 1]) / den) * 1.0;
    } else {
      const double tm2 = t[std::max(0, itime - 2)];
      djdt = ref_dA_dt(t[itime], cf[itime - 1], cf[itime], cf[itime + 1], t[itime + 1] - t[itime - 1],
                       t[itime + 1] - t[itime], t[itime] - t[itime - 1], t[itime], t[itime - 1], tm2);
    }
  } else {
    const double den = two_layer ? dt : (t[itime] - t[itime - 1]);
    djdt = (cf[itime] - cf[itime - 1]) / den;
  }
  return -djdt;
}

std::string TransientSolve::prepare(const std::string& dir, const RunOptions& opt, cudaStream_t stream) {
  opt_.time_watcher = opt.time_watcher;  // the marks below precede plan()'s copy of the options
  mark_host("Start CalcSP");
  if (file_exists(opt.stop_file)) return "cancelled";  // TaskSP.cpp:462
  mark_host("Start Prepare_To_Schema");
  std::string e = plan(dir, opt);
  if (!e.empty()) return e;
  if (!(e = setup_device(stream)).empty()) return e;
  mark_host("Finish Prepare_To_Schema");
  return flush_marks();
}

std::string TransientSolve::build_sources_and_receivers() {
  std::string e;
  // source vectors S[e, p] = sum over dipoles of basis . dl * 2 / edge length
  {
    std::vector<double>& S = S_;
    S.assign((size_t)n_ * npls_, 0.0);
    if (have_source_) {
      for (int p = 0; p < npls_; ++p)
        for (const Dipole& d : m_.dipoles[p]) {
          const double in[3] = {2.0 * d.ksi - 1.0, 2.0 * d.eta - 1.0, 2.0 * d.zeta - 1.0};
          const double dl[3] = {d.dx, d.dy, d.dz};
          for (int j = 0; j < 12; ++j) {
            const int ii = m_.ed[d.elem][j];
            const auto& a = m_.xyz[m_.edge_nodes[ii][0]];
            const auto& b = m_.xyz[m_.edge_nodes[ii][1]];
            const double len = std::sqrt((b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) +
                                         (b[2] - a[2]) * (b[2] - a[2]));
            S[ii + (size_t)p * n_] += basis_dot(j, in, dl) * 2.0 / len;
          }
        }
    }
  }
  // receivers
  {
    auto owners = [&](const std::vector<int>& ig, int nrec) {
      std::vector<int> o(nrec, 0);
      for (int p = 0; p < npls_; ++p)
        for (int i = ig[p]; i < ig[p + 1] && i < nrec; ++i) o[i] = p;
      return o;
    };
    // A merged plan evaluates each directory's receivers on their own neighbourhood,
    // as its solo run does: the reference smooths the field over the elements around
    // all receivers of a run, so pooling the receivers would change every value (by
    // up to 1e-2 relative for E-type values at 10^3 cells).
    auto build = [&](const std::vector<std::array<double, 3>>& pts, const std::vector<int>& ig, bool curl,
                     bool b_set, ReceiverOperator& out) -> std::string {
      const std::vector<int> own = owners(ig, (int)pts.size());
      if (parts_.empty()) return build_receiver_operator(m_, pts, own, curl, out);
      std::vector<ReceiverOperator> ops(parts_.size());
      int r0 = 0;
      for (size_t k = 0; k < parts_.size(); ++k) {
        const int nr = b_set ? parts_[k].nrec_b : parts_[k].nrec_e;
        if (r0 + nr > (int)pts.size()) return "merged receivers out of range";
        std::vector<std::array<double, 3>> p(pts.begin() + r0, pts.begin() + r0 + nr);
        std::vector<int> o(own.begin() + r0, own.begin() + r0 + nr);
        std::string err = build_receiver_operator(m_, p, o, curl, ops[k]);
        if (!err.empty()) return err;
        r0 += nr;
      }
      // rows are component-major over all receivers: component c of part k's
      // receiver i is row c * nrec + (part k's first receiver) + i
      out = ReceiverOperator();
      out.nrec = r0;
      out.ncomp = ops.empty() ? 3 : ops[0].ncomp;
      out.rowptr.assign(1, 0);
      for (int c = 0; c < out.ncomp; ++c)
        for (const ReceiverOperator& op : ops)
          for (int i = 0; i < op.nrec; ++i) {
            const int64_t row = (int64_t)c * op.nrec + i;
            for (int64_t q = op.rowptr[row]; q < op.rowptr[row + 1]; ++q) {
              out.col.push_back(op.col[q]);
              out.val.push_back(op.val[q]);
            }
            out.rowptr.push_back((int64_t)out.col.size());
            out.src.push_back(op.src[row]);
          }
      for (const ReceiverOperator& op : ops) out.elem.insert(out.elem.end(), op.elem.begin(), op.elem.end());
      return "";
    };
    e = build(m_.rec_b, m_.rec_b_ig, true, true, rop_b_);
    if (!e.empty()) return e;
    e = build(m_.rec_e, m_.rec_e_ig, false, false, rop_e_);
    if (!e.empty()) return e;
  }
  return "";
}

std::string TransientSolve::plan(const std::string& dir, const RunOptions& opt) {
  const double t0 = now_s();
  opt_ = opt;
  if (opt.formulation != 0 && opt.formulation != 1) return "formulation must be 0 (A) or 1 (E)";
  if (opt.scheme != 2 && opt.scheme != 3) return "scheme must be 2 or 3";
  parts_.clear();
  std::string e = load_model(dir, m_);
  if (!e.empty()) return e;
  return plan_model(opt, t0);
}

std::string TransientSolve::plan_merged(const std::vector<std::string>& dirs, const RunOptions& opt,
                                        std::vector<std::array<int, 3>>* part_info) {
  const double t0 = now_s();
  opt_ = opt;
  if (opt.formulation != 0 && opt.formulation != 1) return "formulation must be 0 (A) or 1 (E)";
  if (opt.scheme != 2 && opt.scheme != 3) return "scheme must be 2 or 3";
  if (dirs.empty()) return "no model directories";
  // the directories are read side by side; the first failure in order is reported
  std::vector<Model> parts(dirs.size());
  std::vector<std::string> errs(dirs.size());
  parallel_chunks((int64_t)dirs.size(), (int)std::min<size_t>(dirs.size(), (size_t)host_threads()),
                  [&](int, int64_t b, int64_t e) {
                    for (int64_t i = b; i < e; ++i) errs[i] = load_model(dirs[i], parts[i]);
                  });
  for (size_t i = 0; i < dirs.size(); ++i)
    if (!errs[i].empty()) return dirs[i] + ": " + errs[i];
  std::string e = merge_models(parts, m_);
  if (!e.empty()) return e;
  parts_.clear();
  for (size_t i = 0; i < dirs.size(); ++i)
    parts_.push_back({dirs[i], parts[i].npls, (int)parts[i].rec_b.size(), (int)parts[i].rec_e.size()});
  if (part_info) {
    part_info->clear();
    for (const Model& p : parts) part_info->push_back({p.npls, (int)p.rec_b.size(), (int)p.rec_e.size()});
  }
  parts.clear();
  return plan_model(opt, t0);
}

std::string TransientSolve::plan_model(const RunOptions& opt, double t0) {
  std::string e;
  n_ = m_.n_edges;
  npls_ = m_.npls;
  ntime_ = (int)m_.time.size();

  // printed layers (give_out_vec_loop.cpp:52-73)
  tlf_ = tll_ = 2;
  for (int i = 0; i < ntime_; ++i)
    if (m_.time[i] >= m_.print_left) { tlf_ = i; break; }
  if (tlf_ > ntime_ - 1) tlf_ = ntime_ - 1;
  for (int i = 0; i < ntime_; ++i)
    if (m_.time[i] >= m_.print_right - 1e-6) { tll_ = i; break; }
  if (m_.print_right > m_.time[ntime_ - 1] - 1e-6) tll_ = ntime_ - 1;
  if (tll_ - tlf_ < 2) return "fewer than three printed time layers";

  // source
  if (m_.fdirect) {
    bool any = false;
    for (int i = 1; i < ntime_; ++i) any = any || m_.currentfunction[i] != 0.0;
    have_source_ = (opt.formulation == 1 || any) && m_.n_srs_razb > 0;
    if (have_source_) {
      e = locate_dipoles(m_);
      if (!e.empty()) return e;
    }
  }
  // primary-secondary mode: the normal field of the anomalous edges is the source
  // (time_approx.cpp:351-368, 671-683, 1263-1348)
  ps_ = !m_.fdirect && m_.n_anom > 0;
  nf_ = NormalField();
  if (ps_) {
    if (m_.pname.empty()) return "cannot read PName (it names the normal-field files m<PName>.enor.NNNN)";
    e = init_normal_field(m_, opt.formulation == 1, nf_);
    if (!e.empty()) return e;
  }

  // the initial field, and the source vectors with the receiver operators, read only
  // the model: they are built on two more threads while the patterns and the analysis
  // run (the threads are joined on every way out of this scope)
  std::string e_init, e_rec;
  std::thread side_init, side_rec;
  struct Join {
    std::thread& a;
    std::thread& b;
    void operator()() {
      if (a.joinable()) a.join();
      if (b.joinable()) b.join();
    }
    ~Join() { (*this)(); }
  } join_sides{side_init, side_rec};
  side_init = std::thread([this, &opt, &e_init] {
    try {
      if (parts_.empty()) {
        e_init = load_initial_field(m_, opt.formulation == 1, u0_);
      } else {
        // each directory's sources in turn (columns of the n x npls field)
        u0_.clear();
        for (const MergedPart& pd : parts_) {
          std::vector<double> u;
          e_init = load_initial_field(m_, pd.dir, pd.npls, opt.formulation == 1, u);
          if (!e_init.empty()) break;
          u0_.insert(u0_.end(), u.begin(), u.end());
        }
      }
    } catch (const std::exception& x) {
      e_init = std::string("host error: ") + x.what();
    }
  });
  side_rec = std::thread([this, &e_rec] {
    try {
      e_rec = build_sources_and_receivers();
    } catch (const std::exception& x) {
      e_rec = std::string("host error: ") + x.what();
    }
  });
  auto main_error = [&](const std::string& err) {
    join_sides();
    return e_init.empty() ? err : e_init;
  };

  // patterns: full symmetric CSR over all edges, lower triangle of the interior system
  edge_pattern(m_, rowptr_, col_);
  std::vector<int> int_id(n_, -1), int_edge;
  for (int i = 0; i < n_; ++i)
    if (!m_.edge_bound[i]) {
      int_id[i] = (int)int_edge.size();
      int_edge.push_back(i);
    }
  n_int_ = (int64_t)int_edge.size();
  if (n_int_ == 0) return main_error("no interior edges");
  // lower triangle of the interior system (rows independent: count, then fill)
  std::vector<int64_t> lptr(n_int_ + 1, 0), aptr(n_int_ + 1, 0);
  std::vector<double> xyz((size_t)n_int_ * 3);
  parallel_ranges(n_int_, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; ++r) {
      const int i = int_edge[r];
      int64_t c = 0, a = 0;
      for (int64_t q = rowptr_[i]; q < rowptr_[i + 1]; ++q) {
        const int j = col_[q];
        c += (int_id[j] >= 0 && int_id[j] <= r);
        a += (int_id[j] >= 0 && j != i);
      }
      lptr[r + 1] = c;
      aptr[r + 1] = a;
      for (int a = 0; a < 3; ++a)
        xyz[3 * r + a] = 0.5 * (m_.xyz[m_.edge_nodes[i][0]][a] + m_.xyz[m_.edge_nodes[i][1]][a]);
    }
  });
  for (int64_t r = 0; r < n_int_; ++r) {
    lptr[r + 1] += lptr[r];
    aptr[r + 1] += aptr[r];
  }
  std::vector<int64_t> src(lptr[n_int_]);
  std::vector<int> lcol(lptr[n_int_]), adj(aptr[n_int_]);
  std::vector<uint8_t> diag(lptr[n_int_]);
  parallel_ranges(n_int_, [&](int64_t r0, int64_t r1) {
    for (int64_t r = r0; r < r1; ++r) {
      const int i = int_edge[r];
      int64_t o = lptr[r], oa = aptr[r];
      for (int64_t q = rowptr_[i]; q < rowptr_[i + 1]; ++q) {
        const int j = col_[q];
        if (int_id[j] >= 0 && int_id[j] <= r) {
          lcol[o] = int_id[j];
          src[o] = q;
          diag[o] = int_id[j] == r;
          ++o;
        }
        if (int_id[j] >= 0 && j != i) adj[oa++] = int_id[j];
      }
    }
  });
  if (opt.precision != 64 && opt.precision != 32) return main_error("precision must be 64 or 32");
  sy_.reset(new Symbolic());
  // the interior graph's adjacency comes from the full pattern's rows (ascending, the
  // order the analysis would build from the lower triangle)
  e = analyse((int)n_int_, lptr.data(), lcol.data(), xyz.data(), *sy_, opt.leaf_size, aptr.data(), adj.data());
  if (!e.empty()) return main_error("analysis: " + e);
  p2v_.resize(n_int_);
  for (int64_t p = 0; p < n_int_; ++p) p2v_[p] = int_edge[sy_->iperm[p]];
  src_ = std::move(src);
  diag_ = std::move(diag);
  join_sides();
  if (!e_init.empty()) return e_init;
  if (!e_rec.empty()) return e_rec;
  pt_.setup_s = now_s() - t0;
  planned_ = true;
  return "";
}

int64_t TransientSolve::device_bytes_needed() const {
  if (!planned_ || !sy_) return 0;
  const int64_t nn = n_, np = npls_, nnz = (int64_t)col_.size(), nl = (int64_t)src_.size();
  // two factor slots are counted only when asked for (0 adds one only if free memory allows)
  const int slots = opt_.factor_slots == 2 ? 2 : 1;
  int64_t b = GpuCholesky::bytes_needed(*sy_, npls_, opt_.precision == 32 ? 4 : 8, slots, factor_bytes());
  b += 8 * (nn + 1) + 4 * nnz + 16 * nnz + 8 * nl + nl + 8 * nl + nn;  // pattern, C, B, map, diag, values, bound
  b += 8 * nn * np * (ring_ + 4);                                       // S, history ring, rhs, x, u0
  if (opt_.precision == 32) b += 8 * nnz * slots + 8 * nn * np * 4;     // A per slot and the CG vectors
  b += 8 * (int64_t)(rop_b_.val.size() + rop_e_.val.size()) * 3;        // receiver operators (approx.)
  b += 8 * (int64_t)(tll_ - tlf_ + 1) * 3 * (rop_b_.nrec + rop_e_.nrec) + 8 * ntime_;
  b += (int64_t)m_.n_elem * (12 * 4 + 5 * 8 + 4);                       // assembly inputs
  if (ps_) b += 8 * nnz + 8 * nn * np + (int64_t)nf_.idx.size() * (4 * np + 12);  // C_dsigma, En, staging
  return b;
}

std::string TransientSolve::setup_device(cudaStream_t stream) {
  if (!planned_) return "setup_device before plan";
  const double t0 = now_s();
  s_ = stream;
  std::string e;
  chol_.reset(new GpuCholesky());
  if (opt_.fp32_update != 0) chol_->set_tensor_core_update(opt_.fp32_update == 2);
  if (const char* oz = std::getenv("TDEM_OZAKI")) chol_->set_ozaki(oz[0] != '0');
  chol_->set_ozaki_timing(true);
  int slots = opt_.factor_slots;
  // The integer-pipe trailing update holds 199 KB of shared memory and 168 x 320
  // registers per CTA, so it cannot share an SM with a level-solve CTA; a
  // factorization ahead of use still fills the SMs its panel chain (one front's
  // 64-column steps at a time) leaves idle.  Measured at 80^3 (E-form, BDF2, 160
  // steps): one slot 0.161 forward solves/s; two slots with the level solves kept
  // to one CTA per SM 0.157, with their full two CTAs per SM 0.169.
  const char* oz_env = std::getenv("TDEM_OZAKI");
  const bool oz_planned = sy_->oz_rows_max > 0 && factor_bytes() == 8 && !(oz_env && oz_env[0] == '0');
  if (slots == 0) {
    size_t free_b = 0, total_b = 0;
    TRY_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // one slot counted: a second adds its factor (and the system values of mixed precision)
    const int64_t need = device_bytes_needed() + GpuCholesky::slot_bytes(*sy_, opt_.precision == 32 ? 4 : 8) +
                         (opt_.precision == 32 ? 8 * (int64_t)col_.size() : 0);
    slots = ((int64_t)free_b > need + (int64_t)(total_b / 20) + ((int64_t)2 << 30)) ? 2 : 1;
  }
  if (slots < 1 || slots > kMaxSlots) return "factor_slots must be 0, 1 or 2";
  pt_.factor_slots = slots;
  {
    int least = 0, greatest = 0;
    TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    TRY_CUDA(cudaStreamCreateWithPriority(&hs_, cudaStreamNonBlocking, greatest));
    TRY_CUDA(cudaStreamCreateWithPriority(&fs_, cudaStreamNonBlocking, least));
  }
  e = chol_->setup(std::move(*sy_), p2v_, npls_, s_, opt_.precision == 32 ? 4 : 8, slots, factor_bytes());
  sy_.reset();
  if (!e.empty()) return e;
  if (const char* ps = std::getenv("TDEM_PANEL_SOLVE")) chol_->set_panel_solve(ps[0] == '1');
  if (const char* la = std::getenv("TDEM_LOOKAHEAD")) chol_->set_lookahead(la[0] != '0');
  if (const char* at = std::getenv("TDEM_SOLVE_AUTOTUNE")) chol_->set_autotune(at[0] != '0');
  if (const char* fs = std::getenv("TDEM_SOLVE_SCHEDULE")) {  // "kind,split": a fixed schedule
    SolveSchedule sc;
    if (std::sscanf(fs, "%d,%d", &sc.kind, &sc.split) == 2 && sc.kind >= 0 && sc.kind <= 2 && sc.split >= 1 &&
        sc.split <= kMaxRhs)
      chol_->force_schedule(sc);
    else
      return "TDEM_SOLVE_SCHEDULE must be \"kind,split\" with kind 0, 1 or 2";
  }
  // with a factorization on the FP64 tensor pipe running beside the steps, the level
  // solves keep one CTA per SM so its kernels can share every SM (with the
  // integer-pipe update they keep their two, see above)
  if (slots > 1 && !oz_planned) chol_->set_solve_ctas_per_sm(1);
  const RunOptions& opt = opt_;

  // device buffers
  if (!(e = upload(&d_rowptr_, rowptr_)).empty()) return e;
  if (!(e = upload(&d_col_, col_)).empty()) return e;
  if (!(e = alloc((void**)&d_C_, sizeof(double) * col_.size())).empty()) return e;
  if (!(e = alloc((void**)&d_B_, sizeof(double) * col_.size())).empty()) return e;
  if (!(e = upload(&d_src_, src_)).empty()) return e;
  if (!(e = upload(&d_diag_, diag_)).empty()) return e;
  if (!(e = alloc((void**)&d_avals_, sizeof(double) * src_.size())).empty()) return e;
  {
    std::vector<uint8_t> b(m_.edge_bound.begin(), m_.edge_bound.end());
    if (!(e = upload(&d_bound_, b)).empty()) return e;
  }
  if (!(e = upload(&d_S_, S_)).empty()) return e;
  std::vector<double>().swap(S_);
  if (!(e = alloc((void**)&d_hist_, sizeof(double) * (size_t)ring_ * n_ * npls_)).empty()) return e;
  if (!(e = alloc((void**)&d_rhs_, sizeof(double) * (size_t)n_ * npls_)).empty()) return e;
  if (!(e = alloc((void**)&d_x_, sizeof(double) * (size_t)n_ * npls_)).empty()) return e;
  // Dirichlet entries of the solution are never written by the solve: they stay 0
  TRY_CUDA(cudaMemsetAsync(d_x_, 0, sizeof(double) * (size_t)n_ * npls_, s_));
  if (opt.precision == 32) {
    const size_t vb = sizeof(double) * (size_t)n_ * npls_;
    for (int k = 0; k < slots; ++k)
      if (!(e = alloc((void**)&d_Aslot_[k], sizeof(double) * col_.size())).empty()) return e;
    for (double** v : {&d_r_, &d_z_, &d_p_, &d_q_})
      if (!(e = alloc((void**)v, vb)).empty()) return e;
    TRY_CUDA(cudaMemsetAsync(d_z_, 0, vb, s_));
    if (!(e = alloc((void**)&d_work_, sizeof(double) * kDotBlocks * npls_)).empty()) return e;
    for (double** v : {&d_rz_, &d_rzn_, &d_pq_, &d_rr_, &d_bn_})
      if (!(e = alloc((void**)v, sizeof(double) * npls_)).empty()) return e;
  }
  if (!(e = upload(&d_u0_, u0_)).empty()) return e;
  for (cudaEvent_t& ev : ev_) TRY_CUDA(cudaEventCreate(&ev));

  // assembly of sigma*C and B/mu, one launch per element colour
  {
    const double ta = now_s();
    std::vector<int> ed((size_t)m_.n_elem * 12);
    std::vector<double> h((size_t)m_.n_elem * 3), sig(m_.n_elem), imu(m_.n_elem);
    for (int el = 0; el < m_.n_elem; ++el) {
      for (int j = 0; j < 12; ++j) ed[(size_t)el * 12 + j] = m_.ed[el][j];
      for (int a = 0; a < 3; ++a) h[3 * el + a] = m_.xyz[m_.nver[el][7]][a] - m_.xyz[m_.nver[el][0]][a];
      sig[el] = m_.sigma[m_.nvkat[el]];
      imu[el] = 1.0 / m_.mu[m_.nvkat[el]];
    }
    // greedy colouring: elements sharing an edge get different colours
    std::vector<int> order, cstart;
    if (!(e = element_colouring(m_, order, cstart)).empty()) return e;
    const int ncol = (int)cstart.size() - 1;
    int *d_ed = nullptr, *d_order = nullptr;
    double *d_h = nullptr, *d_sig = nullptr, *d_imu = nullptr;
    if (!(e = upload(&d_ed, ed)).empty()) return e;
    if (!(e = upload(&d_h, h)).empty()) return e;
    if (!(e = upload(&d_sig, sig)).empty()) return e;
    if (!(e = upload(&d_imu, imu)).empty()) return e;
    if (!(e = upload(&d_order, order)).empty()) return e;
    TRY_CUDA(cudaMemsetAsync(d_C_, 0, sizeof(double) * col_.size(), s_));
    TRY_CUDA(cudaMemsetAsync(d_B_, 0, sizeof(double) * col_.size(), s_));
    ElemDev ev{d_ed, d_h, d_sig, d_imu};
    for (int c = 0; c < ncol; ++c) {
      launch_assemble(ev, d_order + cstart[c], cstart[c + 1] - cstart[c], d_rowptr_, d_col_, d_C_, d_B_, s_);
      ++launches_;
    }
    if (ps_) {
      // C_dsigma: the mass matrix weighted by sigma - sigma0 (T_Brick.cpp:518-525)
      std::vector<double> dsig(m_.n_elem);
      for (int el = 0; el < m_.n_elem; ++el) dsig[el] = m_.sigma[m_.nvkat[el]] - m_.sigma0[m_.nvkat[el]];
      double* d_dsig = nullptr;
      if (!(e = upload(&d_dsig, dsig)).empty()) return e;
      if (!(e = alloc((void**)&d_Cds_, sizeof(double) * col_.size())).empty()) return e;
      TRY_CUDA(cudaMemsetAsync(d_Cds_, 0, sizeof(double) * col_.size(), s_));
      ElemDev evd{d_ed, d_h, d_dsig, d_imu};
      for (int c = 0; c < ncol; ++c) {
        launch_assemble(evd, d_order + cstart[c], cstart[c + 1] - cstart[c], d_rowptr_, d_col_, d_Cds_, nullptr, s_);
        ++launches_;
      }
      const size_t ve = sizeof(double) * (size_t)n_ * npls_;
      if (!(e = alloc((void**)&d_En_, ve)).empty()) return e;
      TRY_CUDA(cudaMemsetAsync(d_En_, 0, ve, s_));  // entries of normal edges stay 0
      if (!(e = alloc((void**)&d_Ef_, sizeof(float) * nf_.idx.size() * npls_)).empty()) return e;
      if (!(e = upload(&d_anom_, nf_.idx)).empty()) return e;
      if (!(e = upload(&d_alen_, nf_.len)).empty()) return e;
      ef_host_.assign(nf_.idx.size() * (size_t)npls_, 0.0f);
    }
    TRY_CUDA(cudaStreamSynchronize(s_));
    TRY_CUDA(cudaGetLastError());
    pt_.assemble_s = now_s() - ta;
  }

  // receivers
  {
    if (!(e = upload(&d_rb_ptr_, rop_b_.rowptr)).empty()) return e;
    if (!(e = upload(&d_rb_col_, rop_b_.col)).empty()) return e;
    if (!(e = upload(&d_rb_val_, rop_b_.val)).empty()) return e;
    if (!(e = upload(&d_rb_src_, rop_b_.src)).empty()) return e;
    if (!(e = upload(&d_re_ptr_, rop_e_.rowptr)).empty()) return e;
    if (!(e = upload(&d_re_col_, rop_e_.col)).empty()) return e;
    if (!(e = upload(&d_re_val_, rop_e_.val)).empty()) return e;
    if (!(e = upload(&d_re_src_, rop_e_.src)).empty()) return e;
    const int nl = tll_ - tlf_ + 1;
    const size_t rb = (size_t)3 * rop_b_.nrec, re = (size_t)3 * rop_e_.nrec;
    if (!(e = alloc((void**)&d_vb_, sizeof(double) * nl * std::max<size_t>(rb, 1))).empty()) return e;
    if (!(e = alloc((void**)&d_ve_, sizeof(double) * nl * std::max<size_t>(re, 1))).empty()) return e;
    TRY_CUDA(cudaMemsetAsync(d_vb_, 0, sizeof(double) * nl * std::max<size_t>(rb, 1), s_));
    TRY_CUDA(cudaMemsetAsync(d_ve_, 0, sizeof(double) * nl * std::max<size_t>(re, 1), s_));
    if (!(e = upload(&d_time_, m_.time)).empty()) return e;
  }
  TRY_CUDA(cudaStreamSynchronize(s_));
  pt_.setup_s += now_s() - t0 - pt_.assemble_s;
  return "";
}

std::string TransientSolve::factor_with(double mult, int slot, cudaStream_t s) {
  launch_combine(d_C_, d_B_, d_src_, d_diag_, (int64_t)chol_->symbolic().nnz_lower, mult, d_avals_, s);
  if (opt_.precision == 32) {
    launch_combine_full(d_rowptr_, d_col_, d_C_, d_B_, d_bound_, n_, mult, d_Aslot_[slot], s);
    ++launches_;
  }
  const std::string me = mark_device("Start factorization", s);
  if (!me.empty()) return me;
  chol_->factor(d_avals_, s, slot);
  launches_ += 1 + chol_->kernel_launches_factor();
  ++pt_.factorizations;
  return "";
}

std::string TransientSolve::step(int itime, int t1, int t2, double m1, double m2, double coef) {
  if (itime - t1 >= ring_ || (m2 != 0.0 && itime - t2 >= ring_))
    return "time grid needs a restart layer older than the history ring holds";
  const double* u1 = layer(t1);
  const double* u2 = (t2 >= 0) ? layer(t2) : layer(t1);
  launch_history_rhs(d_rowptr_, d_col_, d_C_, u1, u2, m1, (t2 >= 0) ? m2 : 0.0, d_S_, coef, d_bound_, n_, npls_,
                     d_rhs_, s_);
  if (ps_) {
    const std::string se = anomaly_source(itime, t1, t2);
    if (!se.empty()) return se;
  }
  std::string e = (opt_.precision == 32) ? refine(d_x_) : chol_->solve_graph(d_rhs_, d_x_, n_, npls_, s_, slot_);
  if (!e.empty()) return e;
  TRY_CUDA(cudaMemcpyAsync(layer(itime), d_x_, sizeof(double) * (size_t)n_ * npls_, cudaMemcpyDeviceToDevice, s_));
  launches_ += 1 + chol_->kernel_launches_solve();
  ++pt_.steps;
  return "";
}

// Primary-secondary source of the step to layer itime (history layers t1, t2).
// A-form: the normal field of layer itime, float32 per anomalous edge (ascending)
// and source (source-major), from the file m<PName>.enor.<itime as %04d> in the model
// directory, the Linux stand-in for the named shared memory the reference maps
// (time_approx.cpp:1263-1348); it is scaled onto the edges on the device.  E-form:
// minus its rate over the history layers, formed on the host on every edge (layer 0,
// the normal potential's gradient, is dense) and copied whole.  Either is multiplied
// by C_dsigma and added to the right-hand side.
std::string TransientSolve::anomaly_source(int itime, int t1, int t2) {
  if (opt_.formulation == 1) {
    const bool three = opt_.scheme == 3 && itime > 2 && t2 >= 0;
    const std::string e = normal_field_rate(m_, nf_, itime, t1, t2, three, en_host_);
    if (!e.empty()) return e;
    TRY_CUDA(cudaMemcpyAsync(d_En_, en_host_.data(), sizeof(double) * en_host_.size(), cudaMemcpyHostToDevice, s_));
    pt_.h2d_bytes += (int64_t)(sizeof(double) * en_host_.size());
    launch_anomaly_rhs(d_rowptr_, d_col_, d_Cds_, d_En_, d_bound_, n_, npls_, d_rhs_, s_);
    launches_ += 1;
    return "";
  }
  const std::string name = normal_field_file(m_, itime);
  FILE* f = std::fopen(name.c_str(), "rb");
  if (!f) return std::string("cannot open the normal field ") + name;
  const size_t want = ef_host_.size();
  const size_t got = std::fread(ef_host_.data(), sizeof(float), want, f);
  std::fclose(f);
  if (got != want) return std::string("normal field too short: ") + name;
  TRY_CUDA(cudaMemcpyAsync(d_Ef_, ef_host_.data(), sizeof(float) * want, cudaMemcpyHostToDevice, s_));
  pt_.h2d_bytes += (int64_t)(sizeof(float) * want);
  launch_normal_field(d_Ef_, d_anom_, d_alen_, (int)nf_.idx.size(), n_, npls_, d_En_, s_);
  launch_anomaly_rhs(d_rowptr_, d_col_, d_Cds_, d_En_, d_bound_, n_, npls_, d_rhs_, s_);
  launches_ += 2;
  return "";
}

// FP64 conjugate gradients on the interior system preconditioned by the FP32
// factor: x = A^-1 rhs to a relative residual of refine_tol in every column.
std::string TransientSolve::refine(double* x) {
  const size_t vb = sizeof(double) * (size_t)n_ * npls_;
  std::vector<double> rr(npls_), bn(npls_);
  TRY_CUDA(cudaMemsetAsync(x, 0, vb, s_));
  TRY_CUDA(cudaMemcpyAsync(d_r_, d_rhs_, vb, cudaMemcpyDeviceToDevice, s_));
  launch_dots(d_rhs_, d_rhs_, n_, npls_, d_work_, d_bn_, s_);
  std::string e = chol_->solve_graph(d_r_, d_z_, n_, npls_, s_, slot_);
  if (!e.empty()) return e;
  TRY_CUDA(cudaMemcpyAsync(d_p_, d_z_, vb, cudaMemcpyDeviceToDevice, s_));
  launch_dots(d_r_, d_z_, n_, npls_, d_work_, d_rz_, s_);
  TRY_CUDA(cudaMemcpyAsync(bn.data(), d_bn_, sizeof(double) * npls_, cudaMemcpyDeviceToHost, s_));
  launches_ += 4 + chol_->kernel_launches_solve();
  int it = 0;
  double worst = 0.0;
  for (it = 1; it <= opt_.refine_maxit; ++it) {
    launch_spmv(d_rowptr_, d_col_, d_Aslot_[slot_], d_p_, n_, npls_, d_q_, s_);
    launch_dots(d_p_, d_q_, n_, npls_, d_work_, d_pq_, s_);
    launch_pcg_step(d_rz_, d_pq_, x, d_r_, d_p_, d_q_, n_, npls_, d_work_, d_rr_, s_);
    TRY_CUDA(cudaMemcpyAsync(rr.data(), d_rr_, sizeof(double) * npls_, cudaMemcpyDeviceToHost, s_));
    TRY_CUDA(cudaStreamSynchronize(s_));
    launches_ += 5;
    bool done = true;
    worst = 0.0;
    for (int p = 0; p < npls_; ++p) {
      const double rel = bn[p] > 0 ? std::sqrt(rr[p] / bn[p]) : 0.0;
      worst = std::max(worst, rel);
      done = done && rel <= opt_.refine_tol;
    }
    if (done) break;
    e = chol_->solve_graph(d_r_, d_z_, n_, npls_, s_, slot_);
    if (!e.empty()) return e;
    launch_dots(d_r_, d_z_, n_, npls_, d_work_, d_rzn_, s_);
    launch_pcg_dir(d_rz_, d_rzn_, d_z_, d_p_, n_, npls_, s_);
    launches_ += 4 + chol_->kernel_launches_solve();
  }
  if (it > opt_.refine_maxit) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "mixed-precision refinement did not reach the tolerance: relative residual %.3e after %d "
                  "iterations (step %d)",
                  worst, opt_.refine_maxit, pt_.steps + 1);
    return buf;
  }
  pt_.refine_iters += it;
  pt_.refine_iters_max = std::max(pt_.refine_iters_max, it);
  pt_.refine_worst = std::max(pt_.refine_worst, worst);
  return "";
}

void TransientSolve::eval_receivers(int t) {
  if (t < tlf_ || t > tll_) return;
  const int li = t - tlf_;
  if (rop_b_.nrec) {
    launch_receivers(d_rb_ptr_, d_rb_col_, d_rb_val_, d_rb_src_, 3 * rop_b_.nrec, layer(t), n_,
                     d_vb_ + (size_t)li * 3 * rop_b_.nrec, s_);
    ++launches_;
  }
  if (rop_e_.nrec) {
    launch_receivers(d_re_ptr_, d_re_col_, d_re_val_, d_re_src_, 3 * rop_e_.nrec, layer(t), n_,
                     d_ve_ + (size_t)li * 3 * rop_e_.nrec, s_);
    ++launches_;
  }
}

std::string TransientSolve::run() {
  const double tstart = now_s();
  const std::vector<double>& t = m_.time;
  pt_.factorizations = 0;
  pt_.steps = 0;
  pt_.refine_iters = pt_.refine_iters_max = 0;
  pt_.refine_worst = 0.0;
  pt_.factor_gpu_ms = pt_.solve_gpu_ms = pt_.run_gpu_ms = 0;
  pt_.ozaki_ms = 0;
  chol_->take_ozaki_ms();  // events of an earlier run that ended early
  launches_ = 0;
  for (PhaseMark& m : marks_)  // marks of a run that ended early are dropped
    if (m.ev) cudaEventDestroy(m.ev);
  marks_.clear();
  // Everything runs on the high-priority stream hs_ (factorizations ahead of use
  // on fs_), ordered after the caller's stream and joined back into it at the end.
  cudaStream_t caller = s_;
  TRY_CUDA(cudaEventRecord(ev_[2], caller));
  TRY_CUDA(cudaStreamWaitEvent(hs_, ev_[2], 0));
  TRY_CUDA(cudaStreamWaitEvent(fs_, ev_[2], 0));
  s_ = hs_;
  struct Restore {
    TransientSolve* ts;
    cudaStream_t caller;
    ~Restore() {
      cudaEventRecord(ts->ev_[3], ts->hs_);
      cudaEventRecord(ts->ev_[4], ts->fs_);
      cudaStreamWaitEvent(caller, ts->ev_[3], 0);
      cudaStreamWaitEvent(caller, ts->ev_[4], 0);
      ts->s_ = caller;
    }
  } restore{this, caller};
  TRY_CUDA(cudaEventRecord(ev_[0], s_));
  if (!opt_.time_watcher.empty()) {
    if (!mark_origin_) TRY_CUDA(cudaEventCreate(&mark_origin_));
    TRY_CUDA(cudaEventRecord(mark_origin_, s_));
    mark_origin_s_ = now_s();
  }
  TRY_CUDA(cudaMemcpyAsync(layer(0), d_u0_, sizeof(double) * u0_.size(), cudaMemcpyDeviceToDevice, s_));
  dec_ig_ = decade_starts(t);
  const int ndec = (int)dec_ig_.size() - 1;
  vpre1_.assign(ntime_, -1);
  vpre2_.assign(ntime_, -1);
  std::string e;
  auto check = [&]() -> std::string {
    if (opt_.cancel && *opt_.cancel) return "cancelled";
    if (file_exists(opt_.stop_file)) return "cancelled";
    return "";
  };

  // The decades: `use(mult)` is called where a factorization with multiplier
  // mult starts to be needed, `stepf(...)` for every time step, `recv(it)` for
  // every stored layer.  A dry walk (no steps) lists the multipliers first, so
  // every factorization is known before the first step runs.
  auto walk = [&](auto&& use, auto&& stepf, auto&& recv) -> std::string {
    int tn = 0, tn1 = 0, tn2 = 0;
    if (opt_.scheme == 2) {
      recv(0);
      for (int d = 0; d < ndec; ++d) {
        const int tbeg = dec_ig_[d], tend = dec_ig_[d + 1];
        int npre1 = -1, npre2 = -1;
        if (d > 0) {
          if (tbeg + 1 >= ntime_) return "last decade has a single step";
          const double h = t[tbeg + 1] - t[tbeg];
          npre1 = find_time_layer(t, t[tbeg] - h);
          npre2 = find_time_layer(t, t[tbeg] - 2 * h);
          if (npre1 < 0 || npre2 < 0) return "restart layers of a decade not on the time grid";
        }
        bool first = true;
        double mult = 0.0;
        for (int it = std::max(tbeg, 1); it < tend; ++it) {
          if (first && it > 1) {
            tn2 = npre2;
            tn1 = npre1;
            tn = it;
          } else {
            tn2 = tn1;
            tn1 = tn;
            tn = it;
          }
          vpre1_[it] = tn1;
          vpre2_[it] = tn2;
          if (first) {
            mult = 1.0 / (t[it] - t[tn1]);
            std::string ue = use(mult);
            if (!ue.empty()) return ue;
            first = false;
          }
          std::string se = stepf(it, tn1, tn2, mult, 0.0, source_coef(it, false, 0.0));
          if (!se.empty()) return se;
          recv(it);
        }
      }
    } else {
      for (int d = 0; d < ndec; ++d) {
        const int tbeg = dec_ig_[d], tend = dec_ig_[d + 1];
        int npre1 = -1, npre2 = -1;
        if (d > 0) {
          if (tbeg + 1 >= ntime_) return "last decade has a single step";
          const double h = t[tbeg + 1] - t[tbeg];
          npre1 = find_time_layer(t, t[tbeg] - h);
          npre2 = find_time_layer(t, t[tbeg] - 2 * h);
          if (npre1 < 0 || npre2 < 0) return "restart layers of a decade not on the time grid";
        }
        if (1 >= tbeg && 1 < tend) {
          // two backward-Euler steps with the first step length (Two_Layers_Schema)
          if (tend < 3) return "first decade shorter than the two start-up steps";
          const double dt = t[1] - t[0];
          std::string ue = use(1.0 / dt);
          if (!ue.empty()) return ue;
          for (int it = 1; it < 3; ++it) {
            vpre1_[it] = it - 1;
            vpre2_[it] = it - 2;
            std::string se = stepf(it, it - 1, -1, 1.0 / dt, 0.0, source_coef(it, true, dt));
            if (!se.empty()) return se;
            if (it == 2) recv(2);
          }
          tn2 = 0;
          tn1 = 1;
          tn = 2;
        }
        bool first = true;
        double mult = 0, m1 = 0, m2 = 0;
        for (int it = std::max(tbeg, 3); it < tend; ++it) {
          if (first && it != 3) {
            tn2 = npre2;
            tn1 = npre1;
            tn = it;
          } else {
            tn2 = tn1;
            tn1 = tn;
            tn = it;
          }
          vpre1_[it] = tn1;
          vpre2_[it] = tn2;
          if (first) {
            const double dt = t[it] - t[tn2], dt0 = t[it] - t[tn1], dt1 = t[tn1] - t[tn2];
            mult = (dt + dt0) / (dt * dt0);
            m1 = dt / (dt1 * dt0);
            m2 = -dt0 / (dt * dt1);
            std::string ue = use(mult);
            if (!ue.empty()) return ue;
            first = false;
          }
          std::string se = stepf(it, tn1, tn2, m1, m2, source_coef(it, false, 0.0));
          if (!se.empty()) return se;
          recv(it);
        }
      }
    }
    return "";
  };

  std::vector<double> mults;
  auto no_step = [&](int, int, int, double, double, double) { return std::string(); };
  e = walk([&](double mult) { mults.push_back(mult); return std::string(); }, no_step, [](int) {});
  if (!e.empty()) return e;

  const int nslots = chol_->slots();
  const int nf = (int)mults.size();
  // factorization f goes to slot f % nslots; its device time is bracketed by events
  std::vector<cudaEvent_t> fev(2 * (size_t)nf, nullptr), dev_span;
  struct EventPool {
    std::vector<cudaEvent_t>* a;
    std::vector<cudaEvent_t>* b;
    ~EventPool() {
      for (auto* v : {a, b})
        for (cudaEvent_t ev : *v)
          if (ev) cudaEventDestroy(ev);
    }
  } pool{&fev, &dev_span};
  for (cudaEvent_t& ev : fev) TRY_CUDA(cudaEventCreate(&ev));
  // with one slot a factorization runs on hs_ between the decades; with two it
  // runs on fs_ as soon as the steps that used its slot have been issued
  auto enqueue_factor = [&](int f) -> std::string {
    cudaStream_t fst = nslots > 1 ? fs_ : s_;
    if (nslots > 1 && f >= nslots) {
      // the slot was last used by the steps issued so far on hs_
      TRY_CUDA(cudaEventRecord(ev_[5], s_));
      TRY_CUDA(cudaStreamWaitEvent(fst, ev_[5], 0));
    }
    TRY_CUDA(cudaEventRecord(fev[2 * f], fst));
    std::string me;
    if (!(me = mark_device("Start prepare matrix for new decade", fst)).empty()) return me;
    nvtxRangePushA("factorization");
    me = factor_with(mults[f], f % nslots, fst);
    nvtxRangePop();
    if (!me.empty()) return me;
    TRY_CUDA(cudaEventRecord(fev[2 * f + 1], fst));
    return mark_device("Finish factorization", fst);
  };
  int nextf = 0;   // next factorization to be used by the steps
  int queued = 0;  // factorizations enqueued so far
  if (nslots > 1)
    while (queued < std::min(nf, nslots - 1)) {
      if (!(e = enqueue_factor(queued)).empty()) return e;
      ++queued;
    }
  auto span_mark = [&]() -> std::string {
    cudaEvent_t ev;
    TRY_CUDA(cudaEventCreate(&ev));
    dev_span.push_back(ev);
    TRY_CUDA(cudaEventRecord(ev, s_));
    return "";
  };
  int decade = 0;  // decade whose steps are being issued (the reference's iDec)
  auto decade_end = [&]() -> std::string {
    std::string me;
    if (!(me = mark_device("Processing decade results iDec= " + std::to_string(decade), s_)).empty()) return me;
    if (!(me = mark_device("Finish decade iDec= " + std::to_string(decade), s_)).empty()) return me;
    nvtxRangePop();
    ++decade;
    return "";
  };
  auto use = [&](double) -> std::string {
    std::string ue;
    if (!dev_span.empty() && dev_span.size() % 2 == 1) {  // decade end
      if (!(ue = span_mark()).empty()) return ue;
      if (!(ue = decade_end()).empty()) return ue;
    }
    nvtxRangePushA(("decade " + std::to_string(decade)).c_str());
    if (!(ue = mark_device("Start decade iDec= " + std::to_string(decade), s_)).empty()) return ue;
    if (!(ue = mark_device("Start schema iDec= " + std::to_string(decade), s_)).empty()) return ue;
    const int f = nextf++;
    if (nslots == 1) {
      if (!(ue = enqueue_factor(f)).empty()) return ue;
      ++queued;
    } else {
      // keep nslots - 1 factorizations ahead: the one after f reuses the slot of f - 1
      while (queued < std::min(nf, f + nslots)) {
        if (!(ue = enqueue_factor(queued)).empty()) return ue;
        ++queued;
      }
      TRY_CUDA(cudaStreamWaitEvent(s_, fev[2 * f + 1], 0));
    }
    slot_ = f % nslots;
    return span_mark();  // decade start
  };
  auto stepf = [&](int it, int t1, int t2, double m1, double m2, double coef) -> std::string {
    std::string ce = check();
    if (!ce.empty()) return ce;
    if (!(ce = mark_device("Start Direct-Inverse", s_)).empty()) return ce;
    nvtxRangePushA("time step");
    ce = step(it, t1, t2, m1, m2, coef);
    nvtxRangePop();
    if (!ce.empty()) return ce;
    return mark_device("Finish Direct-Inverse", s_);
  };
  auto recvf = [&](int it) {
    mark_device("Start Resultant", s_);
    eval_receivers(it);
    mark_device("Finish Resultant", s_);
  };
  e = walk(use, stepf, recvf);
  if (!e.empty()) return e;
  if (dev_span.size() % 2 == 1) {
    if (!(e = span_mark()).empty()) return e;
    if (!(e = decade_end()).empty()) return e;
  }
  // join the factor stream (nothing is left on it once every factor was used)
  TRY_CUDA(cudaEventRecord(ev_[5], fs_));
  TRY_CUDA(cudaStreamWaitEvent(s_, ev_[5], 0));
  TRY_CUDA(cudaEventRecord(ev_[1], s_));
  TRY_CUDA(cudaStreamSynchronize(s_));
  TRY_CUDA(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
  pt_.run_gpu_ms = ms;
  for (int f = 0; f < nf; ++f) {
    cudaEventElapsedTime(&ms, fev[2 * f], fev[2 * f + 1]);
    pt_.factor_gpu_ms += ms;
  }
  for (size_t k = 0; k + 1 < dev_span.size(); k += 2) {
    cudaEventElapsedTime(&ms, dev_span[k], dev_span[k + 1]);
    pt_.solve_gpu_ms += ms;
  }
  const int bad = chol_->status(s_);
  if (bad) return "factorization met a non-positive pivot at column " + std::to_string(bad);
  if (const int ss = chol_->solve_status(s_))
    return ss == 1 ? "CUDA: a wait of the level triangular solves gave up"
                   : "CUDA: a wait of the tensor-core update gave up";
  pt_.ozaki_ms = chol_->take_ozaki_ms();
  pt_.factor_s = pt_.factor_gpu_ms * 1e-3;
  pt_.steps_s = pt_.solve_gpu_ms * 1e-3;
  (void)tstart;
  return flush_marks();
}

std::string TransientSolve::time_step(bool block, int reps, double* ms) {
  if (pt_.steps == 0) return "time_step needs a completed run";
  if (reps < 1) return "time_step: reps must be positive";
  if (opt_.precision != 64) return "time_step: FP64 solves only";
  const int64_t n = n_;
  const double* u = layer(0);  // any finite history: only the time is measured
  auto one = [&]() -> std::string {
    if (block) {
      launch_history_rhs(d_rowptr_, d_col_, d_C_, u, u, 1.0, 0.0, d_S_, 0.0, d_bound_, n_, npls_, d_rhs_, s_);
      return chol_->solve_graph(d_rhs_, d_x_, n_, npls_, s_, slot_);
    }
    for (int j = 0; j < npls_; ++j) {
      launch_history_rhs(d_rowptr_, d_col_, d_C_, u + j * n, u + j * n, 1.0, 0.0, d_S_ + j * n, 0.0, d_bound_, n_,
                         1, d_rhs_ + j * n, s_);
      chol_->solve(d_rhs_ + j * n, d_x_ + j * n, n_, 1, s_, slot_);
    }
    return "";
  };
  std::string e = one();  // warm-up (captures the block graph on first use)
  if (!e.empty()) return e;
  TRY_CUDA(cudaEventRecord(ev_[0], s_));
  for (int r = 0; r < reps; ++r)
    if (!(e = one()).empty()) return e;
  TRY_CUDA(cudaEventRecord(ev_[1], s_));
  TRY_CUDA(cudaStreamSynchronize(s_));
  TRY_CUDA(cudaGetLastError());
  float t = 0.f;
  TRY_CUDA(cudaEventElapsedTime(&t, ev_[0], ev_[1]));
  *ms = t / reps;
  if (chol_->solve_status(s_)) return "CUDA: a wait of the level triangular solves gave up";
  return "";
}

std::string TransientSolve::results(std::vector<double>& eall, std::vector<double>& emf,
                                    std::vector<double>& ball) {
  const int nl = tll_ - tlf_ + 1;
  const size_t rb = (size_t)3 * rop_b_.nrec, re = (size_t)3 * rop_e_.nrec;
  std::vector<double> vb(nl * rb), ve(nl * re);
  if (rb) TRY_CUDA(cudaMemcpyAsync(vb.data(), d_vb_, sizeof(double) * vb.size(), cudaMemcpyDeviceToHost, s_));
  if (re) TRY_CUDA(cudaMemcpyAsync(ve.data(), d_ve_, sizeof(double) * ve.size(), cudaMemcpyDeviceToHost, s_));
  TRY_CUDA(cudaStreamSynchronize(s_));
  pt_.d2h_bytes += (int64_t)((vb.size() + ve.size()) * sizeof(double));
  if (opt_.formulation == 1) {
    // E-form: receivers hold E and curl E; emf = -curl E, no differencing
    eall = ve;
    emf.resize(vb.size());
    for (size_t i = 0; i < vb.size(); ++i) emf[i] = -vb[i];
    ball.assign(vb.size(), 0.0);
    return "";
  }
  // A-form: differencing on the device
  double *d_out_b = nullptr, *d_out_e = nullptr;
  int *d_v1 = nullptr, *d_v2 = nullptr;
  std::string e;
  if (!(e = alloc((void**)&d_out_b, sizeof(double) * std::max<size_t>(vb.size(), 1))).empty()) return e;
  if (!(e = alloc((void**)&d_out_e, sizeof(double) * std::max<size_t>(ve.size(), 1))).empty()) return e;
  if (!(e = upload(&d_v1, vpre1_)).empty()) return e;
  if (!(e = upload(&d_v2, vpre2_)).empty()) return e;
  launch_time_diff(d_vb_, nl, (int)rb, tlf_, d_time_, d_v1, d_v2, opt_.scheme, 1.0, d_out_b, s_);
  launch_time_diff(d_ve_, nl, (int)re, tlf_, d_time_, d_v1, d_v2, opt_.scheme, -1.0, d_out_e, s_);
  launches_ += 2;
  emf.resize(vb.size());
  eall.resize(ve.size());
  if (rb) TRY_CUDA(cudaMemcpyAsync(emf.data(), d_out_b, sizeof(double) * emf.size(), cudaMemcpyDeviceToHost, s_));
  if (re) TRY_CUDA(cudaMemcpyAsync(eall.data(), d_out_e, sizeof(double) * eall.size(), cudaMemcpyDeviceToHost, s_));
  TRY_CUDA(cudaStreamSynchronize(s_));
  TRY_CUDA(cudaGetLastError());
  ball = vb;
  return "";
}

std::string TransientSolve::write_outputs() {
  const double ta = now_s();
  std::vector<double> eall, emf, ball;
  std::string e = results(eall, emf, ball);
  if (!e.empty()) return e;
  const int nl = tll_ - tlf_ + 1;
  const int nb = rop_b_.nrec, ne = rop_e_.nrec;
  auto header = [](FILE* f, const std::array<double, 3>& p, const char* cols) {
    fprintf(f, "%d %d\n", (int)p[0], (int)p[1]);
    fprintf(f, "%.16e %.16e %.16e\n", p[0], p[1], p[2]);
    fprintf(f, "1\n1 1 1 1\n1\n%s\n", cols);
  };
  for (int p = 0; p < npls_; ++p) {
    char fn[512];
    // edsall_anom.N: emf (mV) = Edsx * (-1000)
    snprintf(fn, sizeof fn, "%s/edsall_anom.%d", m_.dir.c_str(), p + 1);
    FILE* f = fopen(fn, "w");
    if (!f) return std::string("cannot write ") + fn;
    for (int i = 0; i < nb; ++i) {
      if (i < m_.rec_b_ig[p] || i >= m_.rec_b_ig[p + 1]) continue;
      header(f, m_.rec_b[i], "      t (ms)         Emfx_anom (mV)     Emfy_anom (mV)     Emfz_anom (mV)");
      for (int l = 0; l < nl; ++l) {
        const double* v = emf.data() + (size_t)l * 3 * nb;
        fprintf(f, "%.16e\t%.16e\t%.16e\t%.16e\n", m_.time[tlf_ + l] * 1000, v[i] * (-1000), v[nb + i] * (-1000),
                v[2 * nb + i] * (-1000));
      }
    }
    if (nb == 0) fprintf(f, " \n");
    fclose(f);
    snprintf(fn, sizeof fn, "%s/ball_anom.%d", m_.dir.c_str(), p + 1);
    f = fopen(fn, "w");
    if (!f) return std::string("cannot write ") + fn;
    for (int i = 0; i < nb; ++i) {
      if (i < m_.rec_b_ig[p] || i >= m_.rec_b_ig[p + 1]) continue;
      header(f, m_.rec_b[i], "      t (ms)        Bx_anom (mTl)     By_anom (mTl)     Bz_anom (mTl)");
      for (int l = 0; l < nl; ++l) {
        const double* v = ball.data() + (size_t)l * 3 * nb;
        if (opt_.formulation == 1)
          fprintf(f, "%.16e\t%.16e\t%.16e\t%.16e\n", m_.time[tlf_ + l] * 1000, 0.0, 0.0, 0.0);
        else
          fprintf(f, "%.16e\t%.16e\t%.16e\t%.16e\n", m_.time[tlf_ + l] * 1000, v[i] * 1000, v[nb + i] * 1000,
                  v[2 * nb + i] * 1000);
      }
    }
    if (nb == 0) fprintf(f, " \n");
    fclose(f);
    snprintf(fn, sizeof fn, "%s/eall_anom.%d", m_.dir.c_str(), p + 1);
    f = fopen(fn, "w");
    if (!f) return std::string("cannot write ") + fn;
    for (int i = 0; i < ne; ++i) {
      if (i < m_.rec_e_ig[p] || i >= m_.rec_e_ig[p + 1]) continue;
      header(f, m_.rec_e[i], "      t (ms)         Ex_anom n (mV)     Ey_anom a (mV)     Ez_anom s (mV)");
      for (int l = 0; l < nl; ++l) {
        const double* v = eall.data() + (size_t)l * 3 * ne;
        fprintf(f, "%.16e\t%.16e\t%.16e\t%.16e\n", m_.time[tlf_ + l] * 1000, v[i] * 1000, v[ne + i] * 1000,
                v[2 * ne + i] * 1000);
      }
    }
    if (ne == 0) fprintf(f, " \n");
    fclose(f);
  }
  pt_.output_s = now_s() - ta;
  return "";
}

}  // namespace tdem
