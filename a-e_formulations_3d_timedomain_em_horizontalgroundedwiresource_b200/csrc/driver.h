// Transient edge-FEM forward solve on one GPU: the B200 counterpart of the
// reference's CalcNonstat3DLine (CalcNonstat3DLine/TaskSP.cpp:445-711 CalcSP,
// time_approx.cpp:289-1152 Prepare_To_Schema / Two_Layers_Schema /
// Three_Layers_Schema, give_out_vec_loop.cpp:240-615 Gather_edsall).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "gpu_cholesky.h"
#include "model.h"
#include "receivers.h"
#include "symbolic.h"

namespace tdem {

struct RunOptions {
  int formulation = 0;   // 0 = A (vector potential), 1 = E (electric field)
  int scheme = 2;        // 2 = two-point (backward Euler), 3 = three-point (BDF2)
  int leaf_size = 128;   // nested-dissection leaf size
  // precision 32, the factorization: 0 FP64 (factor held rounded to FP32), 1 FP32 with
  // CUDA-core updates, 2 FP32 with tensor-core (tcgen05 3xTF32) updates
  int fp32_update = 0;
  // 64: FP64 factor, one direct solve per step.  32: FP32 factor used as the
  // preconditioner of an FP64 conjugate-gradient solve on the FP64 system, run to
  // a relative residual of refine_tol in every column.
  int precision = 64;
  double refine_tol = 1e-10;
  int refine_maxit = 200;
  // Numeric factors held on the device (precision 64): 2 factors the next time
  // step size on a low-priority stream while the current decade's steps run on a
  // high-priority one; 1 runs them in turn; 0 chooses 2 when free device memory
  // holds the second factor with room to spare.  Results are the same either way.
  int factor_slots = 0;
  const volatile int* cancel = nullptr;  // checked between time steps when set
  // Drop-in module behaviour (tdem_run_directory and the executable).
  // stop_file: a file whose presence ends the run before the next time step, as the
  // reference's `stop` file does (CheckStop, GeoCalculatorSP.cpp:27-39, polled per
  // step at time_approx.cpp:908).  time_watcher: file the phase marks are appended
  // to, one "<ticks>\t<label>" line each with the reference's labels
  // (TimeWatcher.cpp:37-44; TaskSP.cpp:459-701, time_approx.cpp:983-1131).
  std::string stop_file;
  std::string time_watcher;
};

struct PhaseTimes {
  double setup_s = 0, assemble_s = 0, factor_s = 0, steps_s = 0, output_s = 0;
  // device time of the last run() from CUDA events on the solver's stream
  // (factor_gpu_ms sums the factorizations, solve_gpu_ms the time-step spans;
  // with two factor slots they overlap and may add up to more than run_gpu_ms)
  double run_gpu_ms = 0, factor_gpu_ms = 0, solve_gpu_ms = 0;
  double ozaki_ms = 0;  // summed device time of the integer-pipe trailing updates
  int factorizations = 0, steps = 0, factor_slots = 1;
  int64_t h2d_bytes = 0, d2h_bytes = 0;   // host<->device traffic of prepare/run/results
  int refine_iters = 0, refine_iters_max = 0;  // CG iterations of the last run (mixed precision)
  double refine_worst = 0.0;              // largest final relative residual of the last run
};

class TransientSolve {
 public:
  TransientSolve();
  ~TransientSolve();

  // Loads and prepares everything that does not depend on the time step
  // (plan() followed by setup_device()).
  std::string prepare(const std::string& dir, const RunOptions& opt, cudaStream_t stream);
  // Host half: reads the inputs, builds the patterns, the analysis, the source
  // vectors and the receiver operators.  Touches no device.
  std::string plan(const std::string& dir, const RunOptions& opt);
  // plan() for several direct-mode model directories that differ only in their
  // sources and receivers (merge_models): one run solves all their sources as one
  // n x npls block per step, each source with its own initial field and receivers.
  // part_info receives each directory's (sources, B receivers, E receivers).
  std::string plan_merged(const std::vector<std::string>& dirs, const RunOptions& opt,
                          std::vector<std::array<int, 3>>* part_info = nullptr);
  // Device bytes setup_device() will allocate (valid after plan()).
  int64_t device_bytes_needed() const;
  // The analysis made by plan() (null before plan() and after setup_device()).
  const Symbolic* planned_symbolic() const { return sy_.get(); }
  // Device half: allocations, uploads and assembly on `stream`.
  std::string setup_device(cudaStream_t stream);
  // Runs every time step of every decade.
  std::string run();
  // Host copies of the output tables (A-form: E = -dA/dt, emf = dB/dt, B; E-form:
  // E, emf = -curl E, B = 0) indexed [layer - first][component][receiver].
  std::string results(std::vector<double>& eall, std::vector<double>& emf, std::vector<double>& ball);
  // Writes edsall_anom.N, ball_anom.N and eall_anom.N into the model directory.
  std::string write_outputs();

  // Device time of one time step's work on the factor the last run() ended with:
  // the history right-hand side and the triangular solves of every source, as one
  // n x npls block (block = true; the solve replayed from its CUDA graph, as run()
  // does) or as npls single-column steps issued one after another (block = false).
  // Average over reps repetitions, in ms.  The solution history is not changed.
  std::string time_step(bool block, int reps, double* ms);
  // Host phase mark (time_watcher only; also an NVTX mark).
  void mark_host(const std::string& label);
  // Appends the marks collected since the last call to the time_watcher file,
  // ordered by time.  Device marks must have completed.
  std::string flush_marks();

  const Model& model() const { return m_; }
  // Host products of plan(), until setup_device() moves them to the device: the source
  // vectors and the initial field (n x npls, column-major) and the receiver operators.
  const std::vector<double>& planned_sources() const { return S_; }
  const std::vector<double>& planned_initial_field() const { return u0_; }
  const ReceiverOperator& planned_receivers_b() const { return rop_b_; }
  const ReceiverOperator& planned_receivers_e() const { return rop_e_; }
  const PhaseTimes& times() const { return pt_; }
  int first_layer() const { return tlf_; }
  int last_layer() const { return tll_; }
  const GpuCholesky& cholesky() const { return *chol_; }
  int64_t n_interior() const { return n_int_; }
  int64_t nnz_full() const { return (int64_t)col_.size(); }
  int kernel_launches() const { return launches_; }

 private:
  // everything plan() does after the model is in m_
  std::string plan_model(const RunOptions& opt, double t0);
  Model m_;
  // merged plans: each directory with its source and receiver counts (its initial
  // field is read there, and its receivers are evaluated on their own neighbourhood)
  struct MergedPart {
    std::string dir;
    int npls = 0, nrec_b = 0, nrec_e = 0;
  };
  std::vector<MergedPart> parts_;
  RunOptions opt_;
  cudaStream_t s_ = nullptr;
  std::unique_ptr<GpuCholesky> chol_;
  cudaStream_t hs_ = nullptr;  // time steps during run() (highest priority)
  cudaStream_t fs_ = nullptr;  // factorizations ahead of use (lowest priority)
  int slot_ = 0;               // factor slot the time steps use
  // host results of plan() consumed by setup_device()
  bool planned_ = false;
  std::unique_ptr<Symbolic> sy_;
  std::vector<int> p2v_;
  std::vector<int64_t> src_;
  std::vector<uint8_t> diag_;
  std::vector<double> S_;
  PhaseTimes pt_;
  // phase marks (time_watcher only): host marks carry a wall time, device marks an
  // event on the stream doing the work, converted through mark_origin_ (recorded
  // at the start of run() together with its wall time)
  struct PhaseMark {
    std::string label;
    cudaEvent_t ev = nullptr;
    double wall_s = 0;
  };
  std::vector<PhaseMark> marks_;
  cudaEvent_t mark_origin_ = nullptr;
  double mark_origin_s_ = 0;
  std::string mark_device(const std::string& label, cudaStream_t s);
  int launches_ = 0;
  int n_ = 0, npls_ = 0, ntime_ = 0;
  int64_t n_int_ = 0;
  int tlf_ = 0, tll_ = 0;
  std::vector<int64_t> rowptr_;
  std::vector<int> col_;
  std::vector<int> dec_ig_;
  std::vector<int> vpre1_, vpre2_;
  std::vector<double> u0_;
  ReceiverOperator rop_b_, rop_e_;
  bool have_source_ = false;
  // primary-secondary mode (fdirect 0 with anomalous edges): C_dsigma on the full
  // pattern, the normal field of the current layer as edge values, its float copy
  // as read, the anomalous edges and their lengths
  bool ps_ = false;
  NormalField nf_;
  std::vector<float> ef_host_;   // A-form: one layer as read
  std::vector<double> en_host_;  // E-form: the step's source values on every edge
  double* d_Cds_ = nullptr;
  double* d_En_ = nullptr;
  float* d_Ef_ = nullptr;
  int* d_anom_ = nullptr;
  double* d_alen_ = nullptr;
  // device buffers
  int64_t* d_rowptr_ = nullptr;
  int* d_col_ = nullptr;
  double* d_C_ = nullptr;
  double* d_B_ = nullptr;
  int64_t* d_src_ = nullptr;   // interior lower entry -> full CSR index
  uint8_t* d_diag_ = nullptr;
  double* d_avals_ = nullptr;
  uint8_t* d_bound_ = nullptr;
  double* d_S_ = nullptr;      // source vectors
  double* d_hist_ = nullptr;   // ring of solution layers
  double* d_u0_ = nullptr;     // initial field (kept so run() can be repeated)
  cudaEvent_t ev_[6] = {};
  double* d_rhs_ = nullptr;
  double* d_x_ = nullptr;      // solve output (fixed, so the solve can be replayed as a graph)
  // mixed precision: FP64 system values per factor slot (the CG of a decade reads
  // its slot's while the next factorization writes the other) and CG work vectors
  double* d_Aslot_[kMaxSlots] = {};
  int factor_bytes() const { return (opt_.precision == 32 && opt_.fp32_update != 0) ? 4 : 8; }
  double *d_r_ = nullptr, *d_z_ = nullptr, *d_p_ = nullptr, *d_q_ = nullptr, *d_work_ = nullptr;
  double *d_rz_ = nullptr, *d_rzn_ = nullptr, *d_pq_ = nullptr, *d_rr_ = nullptr, *d_bn_ = nullptr;
  std::string refine(double* x);
  int ring_ = 8;
  // receivers
  int64_t* d_rb_ptr_ = nullptr; int* d_rb_col_ = nullptr; double* d_rb_val_ = nullptr; int* d_rb_src_ = nullptr;
  int64_t* d_re_ptr_ = nullptr; int* d_re_col_ = nullptr; double* d_re_val_ = nullptr; int* d_re_src_ = nullptr;
  double* d_vb_ = nullptr;     // B-type series (layers x rows)
  double* d_ve_ = nullptr;     // E-type series
  double* d_time_ = nullptr;
  int* d_vpre1_ = nullptr;
  int* d_vpre2_ = nullptr;
  std::vector<void*> allocs_;

  std::string alloc(void** p, size_t bytes);
  template <class T>
  std::string upload(T** d, const std::vector<T>& h);
  double* layer(int t) { return d_hist_ + (int64_t)(t % ring_) * n_ * npls_; }
  std::string factor_with(double mult, int slot, cudaStream_t s);
  // source vectors and receiver operators of the planned model (reads the model only)
  std::string build_sources_and_receivers();
  std::string step(int itime, int t1, int t2, double m1, double m2, double coef);
  // adds C_dsigma times the normal field of layer itime (A) or minus its rate over
  // the step's history layers (E) to the step's right-hand side (primary-secondary mode)
  std::string anomaly_source(int itime, int t1, int t2);
  void eval_receivers(int t);
  double source_coef(int itime, bool two_layer, double dt) const;
};

// Decade starts: layers where the step length changes (TaskSP.cpp:351-398).
std::vector<int> decade_starts(const std::vector<double>& time);
// Layer whose time equals val within a relative 1e-6 (TaskSP.cpp:326-349).
int find_time_layer(const std::vector<double>& time, double val);

}  // namespace tdem
