// GPU supernodal multifrontal Cholesky (FP64) and multi-RHS triangular solves.
//
// Replaces the numeric half of MKL PARDISO in the reference (phase 12 numeric
// factorization and phase 33 solve, CalcNonstat3DLine/pardiso.cpp:69-120).  The
// symbolic plan (symbolic.h) is uploaded once per sparsity pattern; factor() may
// be called again with new values (one factorization per time-step size), and
// solve() any number of times in between.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "ozaki_update.h"
#include "symbolic.h"

namespace tdem {

constexpr int kMaxRhs = 64;    // right-hand sides per solve
constexpr int kMaxSlots = 2;   // numeric factors held at once (one factored while the other solves)

// How a solve of several right-hand sides is scheduled (chosen per column count by
// the solve autotuner, GpuCholesky::tune_solve).
struct SolveSchedule {
  int kind = 0;   // 0: fused level solves (one launch per tree level and direction,
                  //    one unit per CTA); 1: panel solves (launches per 64-column panel
                  //    and level); 2: persistent fused level solves (FP64, 3..32
                  //    columns per group: CTAs stay resident and stream their units'
                  //    blocks through shared-memory stages)
  int split = 1;  // the columns are solved in this many groups one after another
  float ms = 0;   // measured device time of one solve with this schedule (0: not measured)
};

class GpuCholesky {
 public:
  GpuCholesky() = default;
  ~GpuCholesky();
  GpuCholesky(const GpuCholesky&) = delete;
  GpuCholesky& operator=(const GpuCholesky&) = delete;

  // Takes ownership of the analysis and allocates device memory for nrhs_max
  // right-hand sides.  perm_to_vec[p] is the position in the caller's vectors of
  // permuted unknown p (lets the solve read and write the caller's natural-order
  // vectors directly).  nslots numeric factors (1 or 2) are held: with two, one
  // can be factored (on its own stream) while solves use the other.
  // precision_bytes: element size of the held factors and of the solves (8 FP64,
  // 4 FP32).  factor_bytes: arithmetic of the factorization (0 = precision_bytes).
  // factor_bytes 8 with precision_bytes 4 factors in FP64 into one FP64 work
  // factor and stores each slot's factor (and inverted diagonal blocks) rounded
  // to FP32, for FP32 solves inside an FP64 refinement.
  std::string setup(Symbolic&& sy, const std::vector<int>& perm_to_vec, int nrhs_max,
                    cudaStream_t stream, int precision_bytes = 8, int nslots = 1, int factor_bytes = 0);

  // Device bytes setup() allocates for this analysis (factor, workspaces, plans).
  static int64_t bytes_needed(const Symbolic& sy, int nrhs_max, int precision_bytes, int nslots = 1,
                              int factor_bytes = 0);
  // Device bytes of one numeric factor slot (factor entries + inverted diagonal blocks).
  static int64_t slot_bytes(const Symbolic& sy, int precision_bytes);
  // True when the factorization runs in FP64 and the slots hold FP32 copies.
  bool demoted() const { return fac_elem_ == 8 && elem_ == 4; }
  int slots() const { return nslots_; }

  // Numeric factorization into factor slot `slot`.  d_lower_vals holds the
  // lower-CSR values of the analysed pattern (device, nnz_lower doubles).
  // Errors (non-positive pivot) are reported through status() after the stream
  // is synchronised.  Factorizations share one update workspace: they must not
  // run concurrently with each other (solves may).
  void factor(const double* d_lower_vals, cudaStream_t stream, int slot = 0);

  // x = A^-1 b for nrhs columns with the factor in `slot`.  b and x are device
  // arrays with leading dimension ld (positions given by perm_to_vec); x rows
  // not covered by the system are left untouched.  b and x may alias.  Solves
  // share their work vectors: they must not run concurrently with each other.
  void solve(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t stream, int slot = 0);
  // Same as solve(), replayed from a CUDA graph captured on first use for these
  // buffers and slot (the factor values may change between calls; the pointers
  // may not).
  std::string solve_graph(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t stream,
                          int slot = 0);
  int precision_bytes() const { return elem_; }

  // 0 = ok, otherwise 1-based permuted column of the first non-positive pivot.
  int status(cudaStream_t stream);
  // 0 = ok; 1 = a wait of the level solves gave up, 2 = a wait of the
  // tensor-core update gave up (results since setup are not valid).
  int solve_status(cudaStream_t stream);
  // FP32 factor: trailing updates on the tensor cores (3xTF32) or on the
  // CUDA cores (default).  Takes effect at setup().
  void set_tensor_core_update(bool on) { tc_update_ = on; }
  // FP64 factorization: the trailing updates the analysis planned for it (large
  // outer panels, kOzRowsCap rows per launch at most) run on the integer tensor
  // pipe by digit splitting (ozaki_update.h) instead of the FP64 tensor pipe.  On
  // by default; takes effect at setup().
  void set_ozaki(bool on) { ozaki_ = on; }
  bool ozaki() const { return oz_.slices != nullptr; }
  // Records CUDA events around every integer-pipe update launch of the following
  // factorizations; take_ozaki_ms() returns their summed device time (after the
  // stream has completed them) and starts over.
  void set_ozaki_timing(bool on) { oz_timing_ = on; }
  // FP64 factorizations: the panel chain's look-ahead on a side stream (default on)
  void set_lookahead(bool on) { lookahead_ = on; }
  double take_ozaki_ms();
  // Selects the per-panel solve (one launch per 64-column panel and level) instead
  // of the fused level solves; both compute the same triangular solves.  Turns the
  // autotuner off.
  void set_panel_solve(bool on) { panel_solve_ = on; }
  // Solve autotuner: the first graph-replayed solve of more than two right-hand
  // sides times every candidate schedule (fused, panel or persistent fused solves,
  // the columns in 1, 2 or 4 groups) on the factor at hand and keeps the fastest for that column
  // count; later solves of that count use it.  Every schedule computes the same
  // triangular solves (bitwise the same per column as the schedule solving the
  // columns together, not across schedules).  On by default.
  void set_autotune(bool on) { autotune_ = on; }
  // Uses this schedule for every solve of more than two columns (no tuning).
  void force_schedule(const SolveSchedule& sc) { forced_ = sc; has_forced_ = true; }
  // The schedule used for nrhs columns (tuned or default) and the tuner's record.
  SolveSchedule schedule_for(int nrhs) const;
  const std::vector<std::pair<int, std::vector<SolveSchedule>>>& tune_log() const { return tune_log_; }
  // Caps the persistent level-solve kernels at this many CTAs per SM (0 = as many
  // as fit): with one, half of every SM stays free for a factorization running
  // beside the solves.  Takes effect for solves captured or launched afterwards.
  void set_solve_ctas_per_sm(int n) { solve_ctas_cap_ = n; }

  const Symbolic& symbolic() const { return sy_; }
  size_t device_bytes() const { return bytes_; }
  int kernel_launches_factor() const { return launches_factor_; }
  int kernel_launches_solve() const { return launches_solve_; }

 private:
  Symbolic sy_;
  int nrhs_max_ = 0;
  size_t bytes_ = 0;
  int launches_factor_ = 0, launches_solve_ = 0;
  bool ozaki_ = true;
  OzakiBuffers oz_;
  bool oz_timing_ = false;
  std::vector<cudaEvent_t> oz_events_;  // start/stop pairs, the first 2 * oz_used_ recorded
  size_t oz_used_ = 0;
  int64_t* d_task_aux_ = nullptr;
  bool lookahead_ = true;
  cudaStream_t la_side_ = nullptr;   // side stream of the look-ahead, priority la_prio_
  int la_prio_ = 0;
  cudaEvent_t la_ev_[3] = {nullptr, nullptr, nullptr};
  // the side stream at the priority of s (created or re-created on first use)
  bool lookahead_ready(cudaStream_t s);
  bool autotune_ = true;
  bool has_forced_ = false;
  SolveSchedule forced_;
  std::vector<std::pair<int, SolveSchedule>> tuned_;  // (column count, chosen schedule)
  std::vector<std::pair<int, std::vector<SolveSchedule>>> tune_log_;  // every candidate measured
  void solve_with(const SolveSchedule& sc, const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s,
                  int slot);
  std::string tune_solve(int nrhs, int64_t ld, cudaStream_t s, int slot);
  int elem_ = 8;                 // bytes per held factor entry and solve value (8 = FP64, 4 = FP32)
  int fac_elem_ = 8;             // bytes per entry of the factorization's arithmetic
  void* d_Lw_ = nullptr;         // FP64 work factor of a demoted setup (slots hold FP32 copies)
  void* d_dinvw_ = nullptr;      // its inverted diagonal blocks
  int nslots_ = 1;
  bool panel_solve_ = false;
  bool tc_update_ = false;
  int resident_[2][2] = {};      // resident CTAs of the streaming level solves [NR 1, 2][fwd, bwd]
  int resident_mr_[2] = {};      // resident CTAs of the persistent many-column level solves [fwd, bwd]
  int sms_ = 0;                  // SMs of the device
  int solve_ctas_cap_ = 0;       // CTAs per SM of the level solves (0 = occupancy limit)
  struct SolveGraph {
    cudaGraphExec_t exec = nullptr;
    const double* b = nullptr;
    double* x = nullptr;
    int64_t ld = 0;
    int nrhs = 0;
  };
  SolveGraph graph_[kMaxSlots];
  // device arrays
  void* d_L_[kMaxSlots] = {};    // factor entries per slot
  void* d_U_ = nullptr;
  void* d_W_ = nullptr;          // solve front vectors (sum m) x nrhs_max
  void* d_part_ = nullptr;       // backward partial sums
  int64_t* d_l_off_ = nullptr;
  int64_t* d_u_off_ = nullptr;
  int64_t* d_w_off_ = nullptr;
  int* d_m_ = nullptr;
  int* d_k_ = nullptr;
  int64_t* d_entry_ = nullptr;
  int64_t* d_rel_off_ = nullptr;
  int* d_rel_ = nullptr;
  int64_t* d_rows_off_ = nullptr;
  int* d_rows_ = nullptr;        // rows_all mapped to caller vector positions
  int* d_tasks_ = nullptr;
  int64_t* d_prefix_ = nullptr;
  int* d_parent_ = nullptr;
  int* d_c0_ = nullptr;
  int* d_err_ = nullptr;         // [0] first non-positive pivot, [1] level-solve wait gave up,
                                 // [2] tensor-core update wait gave up
  int* d_items_ = nullptr;       // solve / inversion items (front, block)
  int64_t* d_dinv_off_ = nullptr;
  void* d_dinv_[kMaxSlots] = {};  // inverted diagonal blocks per slot
  int* d_sync_ = nullptr;        // level tickets + pivot-block flags + row counters of one solve
  int* d_units_ = nullptr;       // level-solve units
  void* d_spart_ = nullptr;      // level-solve partial sums (slots x 64 x nrhs)
  std::vector<void*> allocs_;
  template <class T>
  std::string upload(T** dst, const std::vector<T>& src, cudaStream_t s);
  std::string alloc(void** p, size_t bytes);
};

}  // namespace tdem
