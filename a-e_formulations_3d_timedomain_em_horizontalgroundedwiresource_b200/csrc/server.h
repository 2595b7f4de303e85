// Serving loop: a stream of forward-modelling requests (one model directory each)
// on one GPU.
//
//   submit -> plan (host threads: read inputs, analysis, receiver operators) ->
//   admission (FIFO; the head request is admitted when its device footprint, known
//   from its analysis, fits the HBM budget next to the requests already running,
//   or when nothing is running) -> run (worker thread with its own CUDA stream:
//   device set-up, all time steps, outputs) -> device memory released.
//
// Up to max_active requests run at once; their kernels overlap on the device
// through their streams, and factors and field histories stay resident until the
// request finishes.  Every kernel is deterministic, so a request's results do not
// depend on what else is running.  There is no counterpart in the reference, which
// runs one CalcNonstat3DLine process per model.
//
// Batched time steps: requests submitted with the same batch key (the caller's
// statement that their models differ only in sources and receivers, e.g. transmitter
// positions of one survey over one earth model) and the same options are merged,
// up to batch_max at a time, when the plan thread takes the first of them: one
// run solves all their sources as one n x k block per step on one factorization per
// step size (merge_models checks the claim; a mismatch plans them one by one).  Each
// request gets its own receivers' values.  Requests that ask for output files are not
// merged (the files are numbered per run).
#pragma once
#include <array>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "driver.h"

namespace tdem {

struct ServerOptions {
  int device = 0;
  int max_active = 4;          // requests on the device at once
  int prep_threads = 2;        // host threads planning requests
  int64_t hbm_budget = 0;      // bytes; 0 = 85% of the device memory free at start
  int batch_max = 0;           // requests merged into one run (0 or 1: none)
};

struct RequestResult {
  std::string error;           // "" when the request succeeded
  double submit_s = 0, admit_s = 0, done_s = 0;  // steady-clock seconds
  int64_t device_bytes = 0;    // admission footprint
  int first_layer = 0, last_layer = 0, n_rec_b = 0, n_rec_e = 0, n_sources = 0;
  int steps = 0, factorizations = 0;
  int batch_size = 1;          // requests solved by the run that solved this one
  double run_gpu_ms = 0;
  std::vector<double> eall, emf, ball;  // reference units and signs, [layer][comp][receiver]
};

struct ServerStats {
  int64_t submitted = 0, completed = 0, failed = 0;
  double latency_p50_s = 0, latency_p99_s = 0, makespan_s = 0, solves_per_s = 0;
  int64_t peak_device_bytes = 0;
  int peak_active = 0;
  int64_t merged_runs = 0, merged_requests = 0;  // runs that solved several requests, and those requests
};

class Server {
 public:
  Server() = default;
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  std::string start(const ServerOptions& opt);
  // Queues a request; returns its id (> 0).
  int64_t submit(const std::string& dir, const RunOptions& opt, bool write_outputs,
                 const std::string& batch_key = "");
  // Blocks until the request has finished; false for an unknown id.
  bool wait(int64_t id, RequestResult* out);
  ServerStats stats();

 private:
  struct Request {
    std::string dir;
    RunOptions opt;
    bool write_outputs = false;
    std::string key;                      // batch key ("" = never merged)
    std::vector<int64_t> members;         // a merged run: the requests it solves, this one first
    std::vector<std::array<int, 3>> part_info;  // their (sources, B receivers, E receivers)
    std::unique_ptr<TransientSolve> solve;
    int64_t bytes = 0;
    bool done = false;
    RequestResult res;
  };
  void plan_loop();
  void run_loop();
  // a finished merged run: each member's share of the leader's results
  void split_results(Request& lead);
  static bool same_options(const RunOptions& a, const RunOptions& b);

  ServerOptions opt_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<int64_t> to_plan_, planned_;
  std::map<int64_t, std::unique_ptr<Request>> reqs_;
  int64_t next_id_ = 1, used_ = 0, peak_used_ = 0;
  int active_ = 0, peak_active_ = 0;
  int64_t merged_runs_ = 0, merged_requests_ = 0;
  bool stop_ = false;
  std::vector<std::thread> threads_;
};

}  // namespace tdem
