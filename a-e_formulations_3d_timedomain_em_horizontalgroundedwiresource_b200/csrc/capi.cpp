// C-ABI entry points (include/tdem.h).
#include "../../include/tdem.h"

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "driver.h"
#include "postprocess.h"

#include <exception>
#include <new>
#include "timegrid.h"
#include "gpu_cholesky.h"
#include "server.h"
#include "stationary.h"
#include "symbolic.h"

// Owns the solver's stream; declared before the solve so that it is destroyed
// after it (members are destroyed in reverse order), on every path: a failed
// create as well as tdem_solver_destroy.
struct StreamHolder {
  cudaStream_t stream = nullptr;
  int device = 0;
  ~StreamHolder() {
    if (stream) {
      cudaSetDevice(device);
      cudaStreamDestroy(stream);
    }
  }
};

struct tdem_solver {
  StreamHolder owned;
  tdem::TransientSolve solve;
  cudaStream_t stream = nullptr;
  int device = 0;
  std::string error;
  volatile int cancel = 0;
  int precision = 64;
  bool prepared = false;
  bool ran = false;
};

namespace {

tdem_status classify(const std::string& e) {
  if (e.empty()) return TDEM_OK;
  if (e == "cancelled") return TDEM_ERR_CANCELLED;
  if (e.rfind("host error", 0) == 0 || e.rfind("host memory", 0) == 0) return TDEM_ERR_HOST;
  if (e.find("cuda") != std::string::npos || e.find("CUDA") != std::string::npos) return TDEM_ERR_CUDA;
  if (e.find("non-positive pivot") != std::string::npos) return TDEM_ERR_NUMERIC;
  if (e.find("refinement") != std::string::npos) return TDEM_ERR_NUMERIC;
  return TDEM_ERR_INPUT;
}

void put_err(char* buf, size_t len, const std::string& e) {
  if (!buf || !len) return;
  std::strncpy(buf, e.c_str(), len - 1);
  buf[len - 1] = 0;
}

// Runs one entry point; a C++ exception (host memory exhausted, or any other) becomes
// TDEM_ERR_HOST with its message in errbuf / *msg instead of crossing the C boundary.
template <class F>
tdem_status guard(F&& f, char* errbuf = nullptr, size_t errlen = 0, std::string* msg = nullptr) noexcept {
  std::string what;
  try {
    return f();
  } catch (const std::bad_alloc&) {
    what = "host memory exhausted";
  } catch (const std::exception& x) {
    what = std::string("host error: ") + x.what();
  } catch (...) {
    what = "host error";
  }
  try {
    put_err(errbuf, errlen, what);
    if (msg) *msg = what;
  } catch (...) {
  }
  return TDEM_ERR_HOST;
}

}  // namespace

extern "C" {

const char* tdem_version(void) { return "tdem-b200 0.1 (sm_100a, FP64 multifrontal)"; }

tdem_status tdem_solver_create(const char* workdir, int formulation, int scheme, int device,
                               tdem_solver** out) {
  return guard([&]() -> tdem_status {
    return tdem_solver_create_ex(workdir, formulation, scheme, device, nullptr, out);
  });
}

namespace {
// module_mode: the behaviour of the reference's executable in its Calculations
// directory (a `stop` file ends the run, phase marks go to TimeWatcher.log).
tdem_status create_solver(const char* workdir, int formulation, int scheme, int device, const tdem_options* opts,
                          bool module_mode, tdem_solver** out);
}  // namespace

tdem_status tdem_solver_create_ex(const char* workdir, int formulation, int scheme, int device,
                                  const tdem_options* opts, tdem_solver** out) {
  return create_solver(workdir, formulation, scheme, device, opts, false, out);
}

namespace {
tdem_status create_solver(const char* workdir, int formulation, int scheme, int device, const tdem_options* opts,
                          bool module_mode, tdem_solver** out) {
  return guard([&]() -> tdem_status {
    if (!workdir || !out) return TDEM_ERR_ARGUMENT;
    *out = nullptr;
    if ((formulation != 0 && formulation != 1) || (scheme != 2 && scheme != 3)) return TDEM_ERR_ARGUMENT;
    // options are checked before any device resource exists
    tdem::RunOptions opt;
    opt.formulation = formulation;
    opt.scheme = scheme;
    if (opts) {
      if (opts->precision) opt.precision = opts->precision;
      if (opts->refine_tol > 0) opt.refine_tol = opts->refine_tol;
      if (opts->refine_maxit > 0) opt.refine_maxit = opts->refine_maxit;
      if (opts->leaf_size > 0) opt.leaf_size = opts->leaf_size;
      if (opts->fp32_update < 0 || opts->fp32_update > 2) return TDEM_ERR_ARGUMENT;
      opt.fp32_update = opts->fp32_update;
      if (opts->factor_slots < 0 || opts->factor_slots > 2) return TDEM_ERR_ARGUMENT;
      opt.factor_slots = opts->factor_slots;
    }
    if (opt.precision != 64 && opt.precision != 32) return TDEM_ERR_ARGUMENT;
    if (module_mode) {
      opt.stop_file = std::string(workdir) + "/stop";
      opt.time_watcher = std::string(workdir) + "/TimeWatcher.log";
    }
    auto s = std::make_unique<tdem_solver>();
    s->device = device;
    opt.cancel = &s->cancel;
    if (cudaSetDevice(device) != cudaSuccess) return TDEM_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return TDEM_ERR_CUDA;
    s->owned.stream = s->stream;
    s->owned.device = device;
    s->precision = opt.precision;
    s->error = s->solve.prepare(workdir, opt, s->stream);
    s->prepared = s->error.empty();
    const tdem_status st = classify(s->error);
    *out = s.release();
    return st;
  });
}
}  // namespace

tdem_status tdem_solver_plan(const char* workdir, int formulation, int scheme, const tdem_options* opts,
                             tdem_plan_info* out, char* err, size_t err_len) {
  return guard([&]() -> tdem_status {
    auto fail = [&](tdem_status st, const std::string& msg) {
      if (err && err_len) {
        std::strncpy(err, msg.c_str(), err_len - 1);
        err[err_len - 1] = 0;
      }
      return st;
    };
    if (err && err_len) err[0] = 0;
    if (!workdir || !out) return fail(TDEM_ERR_ARGUMENT, "null argument");
    if ((formulation != 0 && formulation != 1) || (scheme != 2 && scheme != 3))
      return fail(TDEM_ERR_ARGUMENT, "formulation must be 0 or 1 and scheme 2 or 3");
    std::memset(out, 0, sizeof(*out));
    tdem::RunOptions opt;
    opt.formulation = formulation;
    opt.scheme = scheme;
    if (opts) {
      if (opts->precision) opt.precision = opts->precision;
      if (opts->leaf_size > 0) opt.leaf_size = opts->leaf_size;
      if (opts->factor_slots < 0 || opts->factor_slots > 2) return fail(TDEM_ERR_ARGUMENT, "factor_slots out of range");
      opt.factor_slots = opts->factor_slots;
    }
    if (opt.precision != 64 && opt.precision != 32) return fail(TDEM_ERR_ARGUMENT, "precision must be 64 or 32");
    tdem::TransientSolve ts;
    const std::string e = ts.plan(workdir, opt);
    if (!e.empty()) return fail(classify(e), e);
    const tdem::Symbolic* sy = ts.planned_symbolic();
    const tdem::Model& m = ts.model();
    out->n_edges = m.n_edges;
    out->n_interior = ts.n_interior();
    out->nnz_matrix = ts.nnz_full();
    out->nnz_factor = sy->nnz_l;
    out->factor_flops = sy->flops;
    out->device_bytes = ts.device_bytes_needed();
    out->factor_slot_bytes = tdem::GpuCholesky::slot_bytes(*sy, opt.precision == 32 ? 4 : 8);
    out->solve_units = (int64_t)sy->solve_units.size() / tdem::kUnitInts;
    out->n_fronts = (int)sy->fronts.size();
    out->tree_levels = (int)sy->levels.size();
    out->n_sources = m.npls;
    out->n_times = (int)m.time.size();
    out->plan_seconds = ts.times().setup_s;
    out->digest = tdem::plan_digest(*sy);
    out->ozaki_flops = sy->oz_flops;
    out->ozaki_rows = sy->oz_rows_max;
    out->solve_chain = 0;
    for (const tdem::LevelPlan& lp : sy->levels) {
      int64_t mx = 0;
      for (int f : lp.fronts) mx = std::max<int64_t>(mx, (sy->front_k[f] + tdem::kPanel - 1) / tdem::kPanel);
      out->solve_chain += mx;
    }
    return TDEM_OK;
  }, err, err_len);
}

tdem_status tdem_solver_run(tdem_solver* s) {
  return guard([&]() -> tdem_status {
    if (!s) return TDEM_ERR_ARGUMENT;
    if (!s->prepared) return TDEM_ERR_STATE;
    cudaSetDevice(s->device);
    s->error = s->solve.run();
    s->ran = s->error.empty();
    s->cancel = 0;  // a cancellation request applies to one run
    return classify(s->error);
  }, nullptr, 0, s ? &s->error : nullptr);
}

tdem_status tdem_solver_write_outputs(tdem_solver* s) {
  return guard([&]() -> tdem_status {
    if (!s) return TDEM_ERR_ARGUMENT;
    if (!s->ran) return TDEM_ERR_STATE;
    cudaSetDevice(s->device);
    s->error = s->solve.write_outputs();
    return classify(s->error);
  }, nullptr, 0, s ? &s->error : nullptr);
}

tdem_status tdem_solver_results(tdem_solver* s, double* eall, double* emf, double* ball) {
  return guard([&]() -> tdem_status {
    if (!s) return TDEM_ERR_ARGUMENT;
    if (!s->ran) return TDEM_ERR_STATE;
    cudaSetDevice(s->device);
    std::vector<double> e, m, b;
    s->error = s->solve.results(e, m, b);
    if (!s->error.empty()) return classify(s->error);
    // units and signs as written to the files (Gather_edsall)
    if (eall)
      for (size_t i = 0; i < e.size(); ++i) eall[i] = e[i] * 1000;
    if (emf)
      for (size_t i = 0; i < m.size(); ++i) emf[i] = m[i] * (-1000);
    if (ball)
      for (size_t i = 0; i < b.size(); ++i) ball[i] = b[i] * 1000;
    return TDEM_OK;
  }, nullptr, 0, s ? &s->error : nullptr);
}

tdem_status tdem_solver_info(const tdem_solver* s, tdem_info* info) {
  return guard([&]() -> tdem_status {
    if (!s || !info) return TDEM_ERR_ARGUMENT;
    std::memset(info, 0, sizeof(*info));
    const tdem::Model& m = s->solve.model();
    info->n_edges = m.n_edges;
    info->n_sources = m.npls;
    info->n_times = (int)m.time.size();
    info->n_rec_b = (int)m.rec_b.size();
    info->n_rec_e = (int)m.rec_e.size();
    info->first_layer = s->solve.first_layer();
    info->last_layer = s->solve.last_layer();
    info->n_interior = s->solve.n_interior();
    info->nnz_matrix = s->solve.nnz_full();
    const tdem::PhaseTimes& pt = s->solve.times();
    info->factorizations = pt.factorizations;
    info->steps = pt.steps;
    info->t_setup_s = pt.setup_s;
    info->t_assemble_s = pt.assemble_s;
    info->t_factor_s = pt.factor_s;
    info->t_steps_s = pt.steps_s;
    info->t_output_s = pt.output_s;
    info->kernel_launches = s->solve.kernel_launches();
    info->run_gpu_ms = pt.run_gpu_ms;
    info->factor_gpu_ms = pt.factor_gpu_ms;
    info->solve_gpu_ms = pt.solve_gpu_ms;
    info->h2d_bytes = pt.h2d_bytes;
    info->d2h_bytes = pt.d2h_bytes;
    info->precision = s->precision;
    info->refine_iters = pt.refine_iters;
    info->refine_iters_max = pt.refine_iters_max;
    info->refine_worst = pt.refine_worst;
    info->factor_slots = pt.factor_slots;
    if (m.n_edges > 0 && s->solve.n_interior() > 0) {
      const tdem::GpuCholesky& c = s->solve.cholesky();
      info->nnz_factor = c.symbolic().nnz_l;
      info->factor_flops = c.symbolic().flops;
      info->device_bytes = (int64_t)c.device_bytes();
      const tdem::SolveSchedule sc = c.schedule_for(m.npls);
      info->solve_schedule = sc.kind;
      info->solve_split = sc.split;
      info->solve_tuned_ms = sc.ms;
      info->ozaki_ms = pt.ozaki_ms;
      info->ozaki_macs = c.ozaki() ? c.symbolic().oz_macs : 0.0;
      for (const auto& t : c.tune_log())
        if (t.first == m.npls) info->solve_candidates = (int)t.second.size();
    }
    return TDEM_OK;
  });
}

tdem_status tdem_solver_time_step(tdem_solver* s, int block, int reps, double* ms_per_step) {
  return guard([&]() -> tdem_status {
    if (!s || !ms_per_step || reps < 1) return TDEM_ERR_ARGUMENT;
    if (!s->ran) return TDEM_ERR_STATE;
    cudaSetDevice(s->device);
    s->error = s->solve.time_step(block != 0, reps, ms_per_step);
    return classify(s->error);
  }, nullptr, 0, s ? &s->error : nullptr);
}

tdem_status tdem_solver_tune_log(const tdem_solver* s, int* kinds, int* splits, double* ms, int max, int* count) {
  return guard([&]() -> tdem_status {
    if (!s || !count || max < 0) return TDEM_ERR_ARGUMENT;
    *count = 0;
    if (s->solve.model().n_edges <= 0 || s->solve.n_interior() <= 0) return TDEM_OK;
    for (const auto& t : s->solve.cholesky().tune_log()) {
      if (t.first != s->solve.model().npls) continue;
      const int n = (int)t.second.size();
      for (int i = 0; i < n && i < max; ++i) {
        if (kinds) kinds[i] = t.second[i].kind;
        if (splits) splits[i] = t.second[i].split;
        if (ms) ms[i] = t.second[i].ms;
      }
      *count = n;
    }
    return TDEM_OK;
  });
}

tdem_status tdem_solver_cancel(tdem_solver* s) {
  return guard([&]() -> tdem_status {
    if (!s) return TDEM_ERR_ARGUMENT;
    s->cancel = 1;
    return TDEM_OK;
  }, nullptr, 0, s ? &s->error : nullptr);
}

const char* tdem_solver_error(const tdem_solver* s) { return s ? s->error.c_str() : "null solver"; }

void tdem_solver_destroy(tdem_solver* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  delete s;  // the solve's buffers first, then its stream (StreamHolder)
}

tdem_status tdem_run_directory(const char* workdir, int formulation, int scheme, int device, char* errbuf,
                               size_t errlen) {
  return guard([&]() -> tdem_status {
    tdem_solver* s = nullptr;
    tdem_status st = create_solver(workdir, formulation, scheme, device, nullptr, true, &s);
    if (st == TDEM_OK) st = tdem_solver_run(s);
    if (st == TDEM_OK) st = tdem_solver_write_outputs(s);
    put_err(errbuf, errlen, s ? s->error : std::string("invalid arguments"));
    tdem_solver_destroy(s);
    return st;
  }, errbuf, errlen);
}

tdem_status tdem_pipeline_directory(const char* workdir, int formulation, int scheme, int device, int flags,
                                    char* errbuf, size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    if ((formulation != 0 && formulation != 1) || (scheme != 2 && scheme != 3)) return TDEM_ERR_ARGUMENT;
    if (flags & ~(TDEM_PIPE_TIME_GRID | TDEM_PIPE_STATIONARY | TDEM_PIPE_SPLIT)) return TDEM_ERR_ARGUMENT;
    const std::string dir(workdir);
    auto exists = [&](const char* name) {
      FILE* f = std::fopen((dir + "/" + name).c_str(), "rb");
      if (f) std::fclose(f);
      return f != nullptr;
    };
    char err[1024] = {0};
    auto stage = [&](const char* module, tdem_status st) {
      if (st != TDEM_OK) put_err(errbuf, errlen, std::string(module) + ": " + err);
      return st;
    };
    if (exists("stop")) {
      put_err(errbuf, errlen, "stop file present");
      return TDEM_ERR_CANCELLED;
    }
    tdem_status st = TDEM_OK;
    if ((flags & TDEM_PIPE_TIME_GRID) && exists("tcff")) {
      if ((st = stage("TimeDirectSolver", tdem_time_direct_solver(workdir, err, sizeof err))) != TDEM_OK) return st;
      if ((st = stage("CorrectTimeMesh", tdem_correct_time_mesh(workdir, err, sizeof err))) != TDEM_OK) return st;
    }
    if (flags & TDEM_PIPE_STATIONARY)
      if ((st = stage("CalcStat3D_3T_A", tdem_stationary_directory(workdir, device, err, sizeof err))) != TDEM_OK)
        return st;
    if (!exists("xyzVectorE0")) {
      FILE* f = std::fopen((dir + "/xyzVectorE0").c_str(), "w");
      if (!f) {
        put_err(errbuf, errlen, "cannot write xyzVectorE0");
        return TDEM_ERR_INPUT;
      }
      std::fprintf(f, "0\n");
      std::fclose(f);
    }
    if ((st = stage("CalcNonstat3DLine", tdem_run_directory(workdir, formulation, scheme, device, err, sizeof err))) !=
        TDEM_OK)
      return st;
    if (flags & TDEM_PIPE_SPLIT)
      if ((st = stage("SumNonstat3DOnly", tdem_sum_nonstat_3d_only(workdir, err, sizeof err))) != TDEM_OK) return st;
    return TDEM_OK;
  }, errbuf, errlen);
}

struct tdem_server {
  tdem::Server srv;
  std::mutex mu;
  std::map<int64_t, tdem::RequestResult> done;  // results fetched by tdem_server_wait
};

namespace {
tdem::RunOptions run_options(int formulation, int scheme, const tdem_options* opts) {
  tdem::RunOptions o;
  o.formulation = formulation;
  o.scheme = scheme;
  if (opts) {
    if (opts->precision) o.precision = opts->precision;
    if (opts->refine_tol > 0) o.refine_tol = opts->refine_tol;
    if (opts->refine_maxit > 0) o.refine_maxit = opts->refine_maxit;
    if (opts->leaf_size > 0) o.leaf_size = opts->leaf_size;
    o.fp32_update = opts->fp32_update;
  }
  // the admission budget counts one factor slot unless two are asked for
  o.factor_slots = (opts && opts->factor_slots) ? opts->factor_slots : 1;
  return o;
}
}  // namespace

tdem_status tdem_server_create(const tdem_server_options* opts, tdem_server** out) {
  return guard([&]() -> tdem_status {
    if (!out) return TDEM_ERR_ARGUMENT;
    *out = nullptr;
    tdem::ServerOptions o;
    if (opts) {
      o.device = opts->device;
      if (opts->max_active > 0) o.max_active = opts->max_active;
      if (opts->prep_threads > 0) o.prep_threads = opts->prep_threads;
      o.hbm_budget = opts->hbm_budget_bytes;
      o.batch_max = opts->batch_max;
    }
    auto s = std::make_unique<tdem_server>();
    const std::string e = s->srv.start(o);
    if (!e.empty()) return classify(e);
    *out = s.release();
    return TDEM_OK;
  });
}

tdem_status tdem_server_submit_keyed(tdem_server* srv, const char* workdir, int formulation, int scheme,
                                     const tdem_options* opts, int write_outputs, const char* batch_key,
                                     int64_t* request_id) {
  return guard([&]() -> tdem_status {
    if (!srv || !workdir || !request_id) return TDEM_ERR_ARGUMENT;
    if ((formulation != 0 && formulation != 1) || (scheme != 2 && scheme != 3)) return TDEM_ERR_ARGUMENT;
    if (opts && (opts->precision != 0 && opts->precision != 32 && opts->precision != 64)) return TDEM_ERR_ARGUMENT;
    if (opts && (opts->fp32_update < 0 || opts->fp32_update > 2)) return TDEM_ERR_ARGUMENT;
    if (opts && (opts->factor_slots < 0 || opts->factor_slots > 2)) return TDEM_ERR_ARGUMENT;
    *request_id = srv->srv.submit(workdir, run_options(formulation, scheme, opts), write_outputs != 0,
                                  batch_key ? batch_key : "");
    return TDEM_OK;
  });
}

tdem_status tdem_server_submit(tdem_server* srv, const char* workdir, int formulation, int scheme,
                               const tdem_options* opts, int write_outputs, int64_t* request_id) {
  return tdem_server_submit_keyed(srv, workdir, formulation, scheme, opts, write_outputs, nullptr, request_id);
}

tdem_status tdem_server_wait(tdem_server* srv, int64_t request_id, tdem_request_info* info) {
  return guard([&]() -> tdem_status {
    if (!srv) return TDEM_ERR_ARGUMENT;
    tdem::RequestResult r;
    if (!srv->srv.wait(request_id, &r)) return TDEM_ERR_ARGUMENT;
    const tdem_status st = classify(r.error);
    if (info) {
      std::memset(info, 0, sizeof(*info));
      info->status = st;
      info->first_layer = r.first_layer;
      info->last_layer = r.last_layer;
      info->n_rec_b = r.n_rec_b;
      info->n_rec_e = r.n_rec_e;
      info->n_sources = r.n_sources;
      info->steps = r.steps;
      info->factorizations = r.factorizations;
      info->submit_s = r.submit_s;
      info->admit_s = r.admit_s;
      info->done_s = r.done_s;
      info->run_gpu_ms = r.run_gpu_ms;
      info->device_bytes = r.device_bytes;
      info->batch_size = r.batch_size;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->done[request_id] = std::move(r);
    return st;
  });
}

tdem_status tdem_server_results(tdem_server* srv, int64_t request_id, double* eall, double* emf, double* ball) {
  return guard([&]() -> tdem_status {
    if (!srv) return TDEM_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->done.find(request_id);
    if (it == srv->done.end()) return TDEM_ERR_STATE;
    const tdem::RequestResult& r = it->second;
    if (!r.error.empty()) return classify(r.error);
    if (eall) std::copy(r.eall.begin(), r.eall.end(), eall);
    if (emf) std::copy(r.emf.begin(), r.emf.end(), emf);
    if (ball) std::copy(r.ball.begin(), r.ball.end(), ball);
    return TDEM_OK;
  });
}

const char* tdem_server_error(tdem_server* srv, int64_t request_id) {
  if (!srv) return "";
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->done.find(request_id);
  return it == srv->done.end() ? "" : it->second.error.c_str();
}

tdem_status tdem_server_stats_get(tdem_server* srv, tdem_server_stats* st) {
  return guard([&]() -> tdem_status {
    if (!srv || !st) return TDEM_ERR_ARGUMENT;
    const tdem::ServerStats s = srv->srv.stats();
    st->submitted = s.submitted;
    st->completed = s.completed;
    st->failed = s.failed;
    st->latency_p50_s = s.latency_p50_s;
    st->latency_p99_s = s.latency_p99_s;
    st->makespan_s = s.makespan_s;
    st->solves_per_s = s.solves_per_s;
    st->peak_device_bytes = s.peak_device_bytes;
    st->peak_active = s.peak_active;
    st->merged_runs = s.merged_runs;
    st->merged_requests = s.merged_requests;
    return TDEM_OK;
  });
}

void tdem_server_destroy(tdem_server* srv) { delete srv; }

tdem_status tdem_time_direct_solver(const char* workdir, char* errbuf, size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    const std::string e = tdem::time_direct_solver(workdir);
    put_err(errbuf, errlen, e);
    return e.empty() ? TDEM_OK : TDEM_ERR_INPUT;
  }, errbuf, errlen);
}

tdem_status tdem_correct_time_mesh(const char* workdir, char* errbuf, size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    const std::string e = tdem::correct_time_mesh(workdir);
    put_err(errbuf, errlen, e);
    return e.empty() ? TDEM_OK : TDEM_ERR_INPUT;
  }, errbuf, errlen);
}

tdem_status tdem_sum_nonstat_3d_only(const char* workdir, char* errbuf, size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    const std::string e = tdem::split_components(workdir);
    put_err(errbuf, errlen, e);
    return e.empty() ? TDEM_OK : TDEM_ERR_INPUT;
  }, errbuf, errlen);
}

tdem_status tdem_summator_edmn(const char* workdir, int with_ddv, int profile, int place, char* errbuf,
                               size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    const std::string e = tdem::line_voltages(workdir, with_ddv != 0, profile, place);
    put_err(errbuf, errlen, e);
    return e.empty() ? TDEM_OK : TDEM_ERR_INPUT;
  }, errbuf, errlen);
}

tdem_status tdem_stationary_directory(const char* workdir, int device, char* errbuf, size_t errlen) {
  return guard([&]() -> tdem_status {
    if (!workdir) return TDEM_ERR_ARGUMENT;
    const std::string e = tdem::solve_stationary(workdir, device);
    put_err(errbuf, errlen, e);
    return classify(e);
  }, errbuf, errlen);
}

// ---------------------------------------------------------------------------
// pardiso_64 on the GPU
// ---------------------------------------------------------------------------
namespace {
struct PardisoHandle {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::unique_ptr<tdem::GpuCholesky> chol;
  int64_t n = 0, nnz = 0;
  uint64_t hash = 0;
  std::vector<int64_t> upper_to_lower;  // upper-CSR entry -> lower-CSR entry
  double* d_vals = nullptr;
  double* d_x = nullptr;
  int nrhs_cap = 0;    // columns d_x holds
  int solve_cols = 1;  // columns one solve takes (the nrhs given to the analysing phase 12)
};

uint64_t pattern_hash(int64_t n, const long long* ia, const long long* ja) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)n;
  for (int64_t i = 0; i <= n; ++i) h = (h ^ (uint64_t)ia[i]) * 1099511628211ull;
  for (int64_t q = 0; q < ia[n] - 1; ++q) h = (h ^ (uint64_t)ja[q]) * 1099511628211ull;
  return h;
}

// Handles by the address of the caller's pt array.  The reference's
// pardiso_solver::factorize zeroes pt[0..63] before every phase 12 and calls phase
// -1 only at the end of the run (CalcNonstat3DLine/pardiso.cpp:43-58, 76, 104;
// time_approx.cpp:755, 1002, 1149), so a phase 12 that finds pt[0] null looks its
// handle up here: one analysis, one device factor and one stream per pt array for
// the whole run instead of a new set per factorization.  pt is a member of the
// caller's solver object, so its address is stable for the object's life; phase
// -1 forgets it.
std::mutex g_pardiso_mu;
std::map<const void*, PardisoHandle*> g_pardiso_handles;

PardisoHandle* pardiso_lookup(const void* pt) {
  std::lock_guard<std::mutex> lk(g_pardiso_mu);
  auto it = g_pardiso_handles.find(pt);
  return it == g_pardiso_handles.end() ? nullptr : it->second;
}

void pardiso_register(const void* pt, PardisoHandle* h) {
  std::lock_guard<std::mutex> lk(g_pardiso_mu);
  if (h)
    g_pardiso_handles[pt] = h;
  else
    g_pardiso_handles.erase(pt);
}

int pardiso_analyse(PardisoHandle* h, int64_t n, const long long* ia, const long long* ja, int nrhs) {
  // upper 1-based CSR (row i: columns j >= i) -> lower 0-based CSR (row j: columns i <= j)
  const int64_t nnz = ia[n] - 1;
  std::vector<int64_t> cnt(n + 1, 0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t q = ia[i] - 1; q < ia[i + 1] - 1; ++q) {
      const int64_t j = ja[q] - 1;
      if (j < i || j >= n) return -1;
      ++cnt[j + 1];
    }
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::vector<int> col(nnz);
  h->upper_to_lower.assign(nnz, 0);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t q = ia[i] - 1; q < ia[i + 1] - 1; ++q) {
      const int64_t j = ja[q] - 1;
      const int64_t p = fill[j]++;
      col[p] = (int)i;
      h->upper_to_lower[q] = p;
    }
  tdem::Symbolic sy;
  if (!tdem::analyse((int)n, cnt.data(), col.data(), nullptr, sy).empty()) return -1;
  std::vector<int> p2v(n);
  for (int64_t p = 0; p < n; ++p) p2v[p] = sy.iperm[p];
  h->chol.reset(new tdem::GpuCholesky());
  h->solve_cols = std::min(tdem::kMaxRhs, std::max(1, nrhs));
  if (!h->chol->setup(std::move(sy), p2v, h->solve_cols, h->stream).empty()) return -2;
  if (!h->d_vals || h->nnz != nnz) {  // the values stay when only the column count changes
    if (h->d_vals) cudaFree(h->d_vals);
    h->d_vals = nullptr;
    if (cudaMalloc(&h->d_vals, sizeof(double) * std::max<int64_t>(nnz, 1)) != cudaSuccess) return -2;
  }
  h->n = n;
  h->nnz = nnz;
  h->hash = pattern_hash(n, ia, ja);
  return 0;
}
}  // namespace

static void pardiso_impl(void* pt, const long long* mtype, const long long* phase, const long long* n,
                         const void* a, const long long* ia, const long long* ja, const long long* nrhs, void* b,
                         void* x, long long* error) {
  void** ptv = (void**)pt;
  PardisoHandle* h = (PardisoHandle*)ptv[0];
  if (!h) {
    // pt zeroed by the caller since the handle was made (see g_pardiso_handles)
    h = pardiso_lookup(pt);
    ptv[0] = h;
  }
  *error = 0;
  if (*phase == -1) {
    if (h) {
      cudaSetDevice(h->device);
      h->chol.reset();
      if (h->d_vals) cudaFree(h->d_vals);
      if (h->d_x) cudaFree(h->d_x);
      if (h->stream) cudaStreamDestroy(h->stream);
      delete h;
    }
    pardiso_register(pt, nullptr);
    ptv[0] = nullptr;
    return;
  }
  if (*mtype != 2) {
    *error = -1;
    return;
  }
  if (*phase == 12) {
    if (!h) {
      h = new PardisoHandle();
      const char* dv = getenv("TDEM_PARDISO_DEVICE");
      h->device = dv ? atoi(dv) : 0;
      if (cudaSetDevice(h->device) != cudaSuccess ||
          cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        *error = -2;
        return;
      }
      ptv[0] = h;
      pardiso_register(pt, h);
    }
    cudaSetDevice(h->device);
    if (!h->chol || h->n != *n || h->nnz != ia[*n] - 1 || h->hash != pattern_hash(*n, ia, ja)) {
      // the solve workspace takes the nrhs of this call (the reference passes its
      // right-hand-side count to every phase)
      const int r = pardiso_analyse(h, *n, ia, ja, nrhs ? (int)std::min<long long>(*nrhs, tdem::kMaxRhs) : 1);
      if (r) {
        *error = r;
        return;
      }
    }
    // values: upper CSR order -> lower CSR order
    std::vector<double> lv(h->nnz);
    const double* av = (const double*)a;
    for (int64_t q = 0; q < h->nnz; ++q) lv[h->upper_to_lower[q]] = av[q];
    cudaMemcpyAsync(h->d_vals, lv.data(), sizeof(double) * h->nnz, cudaMemcpyHostToDevice, h->stream);
    h->chol->factor(h->d_vals, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
      *error = -2;
      return;
    }
    if (h->chol->status(h->stream)) *error = -4;
    return;
  }
  if (*phase == 33) {
    if (!h || !h->chol) {
      *error = -1;
      return;
    }
    cudaSetDevice(h->device);
    const int nr = (int)*nrhs;
    if (nr < 1) {
      *error = -1;
      return;
    }
    if (nr > h->nrhs_cap) {
      if (h->d_x) cudaFree(h->d_x);
      h->d_x = nullptr;
      if (cudaMalloc(&h->d_x, sizeof(double) * h->n * nr) != cudaSuccess) {
        *error = -2;
        return;
      }
      h->nrhs_cap = nr;
    }
    if (nr > h->solve_cols && h->solve_cols < tdem::kMaxRhs && ia && ja && h->n == *n &&
        h->hash == pattern_hash(*n, ia, ja)) {
      // The reference analyses with nrhs = 1 (pardiso_solver::init) and then solves
      // npls columns per call (pardiso.cpp:113-120): widen the solve to this call's
      // column count once, refactoring from the values already on the device.
      const int r = pardiso_analyse(h, *n, ia, ja, std::min(nr, tdem::kMaxRhs));
      if (r) {
        *error = r;
        return;
      }
      h->chol->factor(h->d_vals, h->stream);
      if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        *error = -2;
        return;
      }
      if (h->chol->status(h->stream)) {
        *error = -4;
        return;
      }
    }
    // all columns in one copy, solved in blocks of the analysed right-hand-side count
    cudaMemcpyAsync(h->d_x, b, sizeof(double) * h->n * nr, cudaMemcpyHostToDevice, h->stream);
    for (int r = 0; r < nr; r += h->solve_cols) {
      const int cols = std::min(h->solve_cols, nr - r);
      h->chol->solve(h->d_x + h->n * r, h->d_x + h->n * r, h->n, cols, h->stream);
    }
    cudaMemcpyAsync(x, h->d_x, sizeof(double) * h->n * nr, cudaMemcpyDeviceToHost, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) *error = -2;
    return;
  }
  *error = -1;
}

// A C++ exception inside the adapter becomes PARDISO's error -2 (not enough memory)
// for exhausted host memory and -1 otherwise, instead of crossing the C boundary.
void tdem_pardiso_64(void* pt, const long long* /*maxfct*/, const long long* /*mnum*/, const long long* mtype,
                     const long long* phase, const long long* n, const void* a, const long long* ia,
                     const long long* ja, long long* /*perm*/, const long long* nrhs, long long* /*iparm*/,
                     const long long* /*msglvl*/, void* b, void* x, long long* error) {
  try {
    pardiso_impl(pt, mtype, phase, n, a, ia, ja, nrhs, b, x, error);
  } catch (const std::bad_alloc&) {
    *error = -2;
  } catch (...) {
    *error = -1;
  }
}

void pardiso_64(void* pt, const long long* maxfct, const long long* mnum, const long long* mtype,
                const long long* phase, const long long* n, const void* a, const long long* ia,
                const long long* ja, long long* perm, const long long* nrhs, long long* iparm,
                const long long* msglvl, void* b, void* x, long long* error) {
  tdem_pardiso_64(pt, maxfct, mnum, mtype, phase, n, a, ia, ja, perm, nrhs, iparm, msglvl, b, x, error);
}

void mkl_set_num_threads(int) {}

int tdem_pardiso_handles(void) {
  std::lock_guard<std::mutex> lk(g_pardiso_mu);
  return (int)g_pardiso_handles.size();
}

}  // extern "C"
