// Serving loop (see server.h).
#include "server.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>

namespace tdem {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (std::thread& t : threads_) t.join();
}

std::string Server::start(const ServerOptions& opt) {
  opt_ = opt;
  if (opt_.max_active < 1) opt_.max_active = 1;
  if (opt_.prep_threads < 1) opt_.prep_threads = 1;
  cudaError_t e = cudaSetDevice(opt_.device);
  if (e != cudaSuccess) return std::string("CUDA: cudaSetDevice: ") + cudaGetErrorString(e);
  if (opt_.hbm_budget <= 0) {
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return std::string("CUDA: cudaMemGetInfo: ") + cudaGetErrorString(e);
    opt_.hbm_budget = (int64_t)(0.85 * (double)free_b);
  }
  for (int i = 0; i < opt_.prep_threads; ++i) threads_.emplace_back(&Server::plan_loop, this);
  for (int i = 0; i < opt_.max_active; ++i) threads_.emplace_back(&Server::run_loop, this);
  return "";
}

bool Server::same_options(const RunOptions& a, const RunOptions& b) {
  return a.formulation == b.formulation && a.scheme == b.scheme && a.precision == b.precision &&
         a.refine_tol == b.refine_tol && a.refine_maxit == b.refine_maxit && a.leaf_size == b.leaf_size &&
         a.fp32_update == b.fp32_update && a.factor_slots == b.factor_slots;
}

int64_t Server::submit(const std::string& dir, const RunOptions& opt, bool write_outputs,
                       const std::string& batch_key) {
  auto r = std::make_unique<Request>();
  r->dir = dir;
  r->opt = opt;
  r->opt.cancel = nullptr;
  r->write_outputs = write_outputs;
  r->key = batch_key;
  r->res.submit_s = now_s();
  int64_t id;
  {
    std::lock_guard<std::mutex> lk(mu_);
    id = next_id_++;
    reqs_[id] = std::move(r);
    to_plan_.push_back(id);
  }
  cv_.notify_all();
  return id;
}

void Server::plan_loop() {
  for (;;) {
    int64_t id;
    Request* r;
    std::vector<int64_t> batch;
    std::vector<std::string> dirs;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || !to_plan_.empty(); });
      if (stop_ && to_plan_.empty()) return;
      id = to_plan_.front();
      to_plan_.pop_front();
      r = reqs_[id].get();
      batch.push_back(id);
      // queued requests with the same key and options join this one
      if (opt_.batch_max > 1 && !r->key.empty() && !r->write_outputs) {
        for (auto it = to_plan_.begin(); it != to_plan_.end() && (int)batch.size() < opt_.batch_max;) {
          const Request* q = reqs_[*it].get();
          if (q->key == r->key && !q->write_outputs && same_options(q->opt, r->opt)) {
            batch.push_back(*it);
            it = to_plan_.erase(it);
          } else {
            ++it;
          }
        }
      }
      for (int64_t b : batch) dirs.push_back(reqs_[b]->dir);
    }
    std::string e;
    try {
      r->solve.reset(new TransientSolve());
      if (batch.size() > 1) {
        e = r->solve->plan_merged(dirs, r->opt, &r->part_info);
        if (e.empty()) {
          r->members = batch;
        } else {
          // not mergeable after all: this request alone, the others back at the head
          // of the queue, never merged again
          {
            std::lock_guard<std::mutex> lk(mu_);
            for (size_t k = batch.size(); k-- > 1;) {
              reqs_[batch[k]]->key.clear();
              to_plan_.push_front(batch[k]);
            }
          }
          cv_.notify_all();
          r->solve.reset(new TransientSolve());
          e = r->solve->plan(r->dir, r->opt);
        }
      } else {
        e = r->solve->plan(r->dir, r->opt);
      }
    } catch (const std::exception& x) {  // host memory exhausted or another host failure
      e = std::string("host error: ") + x.what();
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!e.empty()) {
        r->res.error = e;
        r->res.done_s = now_s();
        r->solve.reset();
        r->done = true;
        for (size_t k = 1; k < r->members.size(); ++k) {
          Request* q = reqs_[r->members[k]].get();
          q->res.error = e;
          q->res.done_s = r->res.done_s;
          q->done = true;
        }
      } else {
        r->bytes = r->solve->device_bytes_needed();
        planned_.push_back(id);
        if (r->members.size() > 1) {
          ++merged_runs_;
          merged_requests_ += (int64_t)r->members.size();
        }
      }
    }
    cv_.notify_all();
  }
}

void Server::split_results(Request& lead) {
  const int nl = lead.res.last_layer - lead.res.first_layer + 1;
  const int NB = lead.res.n_rec_b, NE = lead.res.n_rec_e;
  const RequestResult all = lead.res;
  int ob = 0, oe = 0;
  for (size_t k = 0; k < lead.members.size(); ++k) {
    Request& q = *reqs_[lead.members[k]];
    const int ns = lead.part_info[k][0], nb = lead.part_info[k][1], ne = lead.part_info[k][2];
    RequestResult& rr = q.res;
    const double submit = rr.submit_s;
    rr = all;
    rr.submit_s = submit;
    rr.n_sources = ns;
    rr.n_rec_b = nb;
    rr.n_rec_e = ne;
    rr.batch_size = (int)lead.members.size();
    if (k > 0) rr.device_bytes = 0;  // counted with the first request of the run
    auto slice = [nl](const std::vector<double>& src, int total, int off, int cnt, std::vector<double>& dst) {
      dst.assign((size_t)nl * 3 * cnt, 0.0);
      if (src.size() < (size_t)nl * 3 * total) return;
      for (int l = 0; l < nl; ++l)
        for (int c = 0; c < 3; ++c)
          for (int j = 0; j < cnt; ++j)
            dst[((size_t)l * 3 + c) * cnt + j] = src[((size_t)l * 3 + c) * total + off + j];
    };
    if (all.error.empty()) {
      slice(all.eall, NE, oe, ne, rr.eall);
      slice(all.emf, NB, ob, nb, rr.emf);
      slice(all.ball, NB, ob, nb, rr.ball);
    }
    ob += nb;
    oe += ne;
    q.done = true;
  }
}

void Server::run_loop() {
  cudaSetDevice(opt_.device);
  for (;;) {
    int64_t id;
    Request* r;
    {
      std::unique_lock<std::mutex> lk(mu_);
      // FIFO admission: the head runs when it fits next to the running requests
      // (or when nothing runs, so a request above the budget still gets its turn)
      cv_.wait(lk, [&] {
        if (stop_ && planned_.empty() && to_plan_.empty()) return true;
        if (planned_.empty()) return false;
        const Request* h = reqs_[planned_.front()].get();
        return active_ == 0 || used_ + h->bytes <= opt_.hbm_budget;
      });
      if (planned_.empty()) {
        if (stop_ && to_plan_.empty()) return;
        continue;
      }
      id = planned_.front();
      planned_.pop_front();
      r = reqs_[id].get();
      used_ += r->bytes;
      ++active_;
      peak_used_ = std::max(peak_used_, used_);
      peak_active_ = std::max(peak_active_, active_);
      r->res.admit_s = now_s();
      r->res.device_bytes = r->bytes;
    }
    std::string e;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) e = "CUDA: cudaStreamCreate failed";
    try {
      if (e.empty()) e = r->solve->setup_device(s);
      if (e.empty()) e = r->solve->run();
      if (e.empty() && r->write_outputs) e = r->solve->write_outputs();
      if (e.empty()) {
        std::vector<double> ea, em, eb;
        e = r->solve->results(ea, em, eb);
        for (double& v : ea) v *= 1000;    // units and signs as written to the files
        for (double& v : em) v *= -1000;
        for (double& v : eb) v *= 1000;
        r->res.eall.swap(ea);
        r->res.emf.swap(em);
        r->res.ball.swap(eb);
      }
    } catch (const std::exception& x) {  // host memory exhausted or another host failure
      e = std::string("host error: ") + x.what();
    }
    const Model& m = r->solve->model();
    r->res.first_layer = r->solve->first_layer();
    r->res.last_layer = r->solve->last_layer();
    r->res.n_rec_b = (int)m.rec_b.size();
    r->res.n_rec_e = (int)m.rec_e.size();
    r->res.n_sources = m.npls;
    r->res.steps = r->solve->times().steps;
    r->res.factorizations = r->solve->times().factorizations;
    r->res.run_gpu_ms = r->solve->times().run_gpu_ms;
    r->solve.reset();  // releases the request's device memory
    if (s) cudaStreamDestroy(s);
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->res.error = e;
      r->res.done_s = now_s();
      if (r->members.size() > 1) split_results(*r);
      r->done = true;
      used_ -= r->bytes;
      --active_;
    }
    cv_.notify_all();
  }
}

bool Server::wait(int64_t id, RequestResult* out) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = reqs_.find(id);
  if (it == reqs_.end()) return false;
  Request* r = it->second.get();
  cv_.wait(lk, [&] { return r->done; });
  if (out) *out = r->res;
  return true;
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  ServerStats st;
  std::vector<double> lat;
  double first = 1e300, last = 0;
  for (const auto& kv : reqs_) {
    const Request& r = *kv.second;
    ++st.submitted;
    first = std::min(first, r.res.submit_s);
    if (!r.done) continue;
    if (!r.res.error.empty()) {
      ++st.failed;
      continue;
    }
    ++st.completed;
    lat.push_back(r.res.done_s - r.res.submit_s);
    last = std::max(last, r.res.done_s);
  }
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
      const double pos = q * (lat.size() - 1);
      const size_t i = (size_t)pos;
      const double f = pos - i;
      return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat[i];
    };
    st.latency_p50_s = pct(0.50);
    st.latency_p99_s = pct(0.99);
    st.makespan_s = last - first;
    st.solves_per_s = st.makespan_s > 0 ? st.completed / st.makespan_s : 0.0;
  }
  st.peak_device_bytes = peak_used_;
  st.peak_active = peak_active_;
  st.merged_runs = merged_runs_;
  st.merged_requests = merged_requests_;
  return st;
}

}  // namespace tdem
