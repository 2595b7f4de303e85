/*
 * C-ABI of the B200-native transient edge-FEM forward solve (libtdem_b200.so).
 *
 * Plain C types only.  Every entry point returns a tdem_status; the message of
 * the last failure of a solver object is available from tdem_solver_error().
 * Calls on one solver object are not thread-safe; separate objects are
 * independent.  Each solver object owns its device memory and CUDA stream on
 * the device it was created for.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - the process boundary of CalcNonstat3DLine: GeoCalculatorSP runs the
 *     executable in the Calculations directory
 *     (CODE/programs to folder Modules/GeoCalculatorSP/GeoCalculatorSP.cpp:1656-1662),
 *     whose main enters CalcSP
 *     (.../CalcNonstat3DLine/GeoCalculatorSP.cpp:56, TaskSP.cpp:445-711)
 *     -> tdem_run_directory / tdem_solver_*;
 *   - the in-process sparse solver boundary: MKL's pardiso_64 as called by
 *     pardiso_solver (.../CalcNonstat3DLine/pardiso.cpp:69-126, pardiso.h:25-53)
 *     -> pardiso_64 / tdem_pardiso_64 below.
 */
#ifndef TDEM_B200_H
#define TDEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tdem_status {
  TDEM_OK = 0,
  TDEM_ERR_ARGUMENT = 1,  /* bad argument (null pointer, unknown formulation / scheme) */
  TDEM_ERR_INPUT = 2,     /* missing, truncated or inconsistent input files */
  TDEM_ERR_CUDA = 3,      /* CUDA runtime error (no device, out of memory, launch failure) */
  TDEM_ERR_NUMERIC = 4,   /* non-positive pivot: the system is not positive definite */
  TDEM_ERR_CANCELLED = 5, /* tdem_solver_cancel() was called during tdem_solver_run() */
  TDEM_ERR_STATE = 6,     /* call out of order (e.g. results before run) */
  TDEM_ERR_HOST = 7       /* host-side failure: host memory exhausted or another internal error */
} tdem_status;

/* formulation: 0 = A (vector potential, CalcNonstat3DLine "A-formulation"),
 *              1 = E (electric field, "E-formulation").
 * scheme:      2 = two-point implicit (backward Euler),
 *              3 = three-point implicit (BDF2). */

/* Drop-in for one run of the reference's CalcNonstat3DLine in `workdir`: reads the
 * direct-mode input files there, runs the transient on CUDA device `device` and
 * writes edsall_anom.N, ball_anom.N and eall_anom.N (N = 1-based source index) in
 * the reference's text format.  errbuf (may be NULL) receives a message on failure.
 * Primary-secondary mode (fdirect 0 with mtrsizeforE0 flagging anomalous edges): the
 * normal field of each time layer is read from the file m<PName>.enor.NNNN in
 * `workdir` (float32 per anomalous edge and source), the stand-in for the named
 * shared memory the reference maps (time_approx.cpp:1263-1348); the E-formulation
 * also reads the normal potential v3n.dat for layer 0.
 * As the reference's module does: a file named `stop` in `workdir` ends the run
 * (before it starts, or before the next time step; CheckStop,
 * GeoCalculatorSP.cpp:27-39, TaskSP.cpp:462, time_approx.cpp:908) with
 * TDEM_ERR_CANCELLED and no outputs; phase marks are appended to
 * `workdir`/TimeWatcher.log as "<clock ticks>\t<label>" lines with the
 * reference's labels (TimeWatcher.cpp:37-44: Start CalcSP, Start/Finish
 * Prepare_To_Schema, Start decade / Start schema / Processing decade results /
 * Finish decade iDec= N, Start prepare matrix for new decade, Start/Finish
 * factorization, Start/Finish Direct-Inverse, Start/Finish Resultant); the times
 * of device work are taken from CUDA events on the streams that do it, and the
 * same labels are NVTX marks.
 * Replaces: GeoCalculatorSP.cpp:1656-1662 -> CalcNonstat3DLine main -> CalcSP
 * (TaskSP.cpp:445-711). */
tdem_status tdem_run_directory(const char* workdir, int formulation, int scheme, int device,
                               char* errbuf, size_t errlen);

/* Drop-in for one run of the reference's CalcStat3D_3T_A in `workdir` (the
 * grounded-wire stationary initial field, direct mode): reads inftry.dat, xyz.dat,
 * nver.dat, nvkat.dat, l13d.dat, sig3d, group, sours and the optional nSrsRazb and
 * ImpStatCur, solves the nodal potential V and the initial vector potential A0 with
 * both factorizations and all solves on CUDA device `device` (FP64), and writes
 * v3n.dat, v3a.dat and a0.dat in the reference's binary layout.
 * Replaces: GeoCalculatorSP.cpp:1562 -> CalcStat3D_3T_A main -> CalcSP ->
 * SolveStationarProblem3d(".", true, true) (MOD/CalcStat3D_3T_A/TaskSP.cpp:1625-2208). */
tdem_status tdem_stationary_directory(const char* workdir, int device, char* errbuf, size_t errlen);

/* ---- Time-grid modules run before CalcNonstat3DLine (host only, no GPU) ---------------
 * Drop-in for the reference's TimeDirectSolver in `workdir`: reads tcff (step growth
 * factor) and infite.0, replaces the times by a piecewise-uniform grid whose step grows
 * by tcff from one interval to the next, and interpolates currentfunction and
 * deltafunction onto it; the three files are rewritten (the old ones renamed with a
 * leading "!"), byte-identical to the reference's.  Replaces: GeoCalculatorSP.cpp:2111
 * -> TimeDirectSolver main (TimeDirectSolver/main.cpp:98-219, TimeStep.cpp:37-168). */
tdem_status tdem_time_direct_solver(const char* workdir, char* errbuf, size_t errlen);

/* Drop-in for the reference's CorrectTimeMesh in `workdir`: decades of the grid in
 * infite.0 that are too short for their step (fewer than 1/tcff of the previous
 * decade's times) are refilled with the previous decade's step; infite.0, deltafunction
 * and currentfunction are rewritten on the corrected times (old ones renamed with a
 * leading "!!"; both function files carry deltafunction's values, as in the reference),
 * byte-identical to the reference's.  Replaces: GeoCalculatorSP.cpp:2120 ->
 * CorrectTimeMesh main (CorrectTimeMesh/main.cpp:87-269). */
tdem_status tdem_correct_time_mesh(const char* workdir, char* errbuf, size_t errlen);

/* ---- Post-processing modules run after CalcNonstat3DLine (host only, no GPU) ----------
 * Drop-in for the reference's SumNonstat3DOnly in `workdir`: reads group,
 * timeintervalforprint, infite.0, xyzVectorB / recvsb, xyzVectorE / recvse and the
 * results ball_anom.N, edsall_anom.N, eall_anom.N, and writes one file per component
 * (Bxall.N, Byall.N, Bzall.N, Edsxall.N, Edsyall.N, Edsall.N, Exall.N, Eyall.N,
 * Ezall.N: t in ms, normal part 0, anomalous part, total), byte-identical to the
 * reference's.  Transmitters are processed on parallel host threads.
 * Replaces: GeoCalculatorSP.cpp:1673 -> SumNonstat3DOnly main
 * (SumNonstat3DOnly/main.cpp:171-384). */
tdem_status tdem_sum_nonstat_3d_only(const char* workdir, char* errbuf, size_t errlen);

/* Drop-in for the reference's SummatorEDMN in `workdir` (arguments as its command
 * line: WithDDV, profile number, place number): the voltage of each receiver line MN
 * of that transmitter, dV(t) = sum over the line's points of E(t) . dl, from
 * exall<profile>_<place>, eyall.., ezall.., xyzmn<place+1>_<profile> and
 * xyzVectorElin<place+1>_<profile>; writes edmnall<profile>_<place> and, when with_ddv
 * is nonzero, edmoonall<profile>_<place> (first half of the line minus the second),
 * byte-identical to the reference's.  Does nothing when xyzmn lists no lines.
 * Replaces: GeoCalculatorSP.cpp:2312-2314 -> SummatorEDMN main
 * (SummatorEDMN/main.cpp:37-294). */
tdem_status tdem_summator_edmn(const char* workdir, int with_ddv, int profile, int place, char* errbuf,
                               size_t errlen);

/* ---- The module sequence of a direct-mode 3D-only run --------------------------------
 * Runs, in `workdir` and in one process, the modules GeoCalculatorSP starts one after
 * another for a direct-mode (fdirect 1) run without the 2D chain, on a model directory
 * whose mesh files are already there (GeoCalculatorSP.cpp:2111-2126 Calc1Loop, then
 * CalcMainTask :1327-1709):
 *   TDEM_PIPE_TIME_GRID  TimeDirectSolver then CorrectTimeMesh (when `tcff` exists);
 *   TDEM_PIPE_STATIONARY CalcStat3D_3T_A (the grounded-wire initial field);
 *   always               xyzVectorE0 with 0 points when absent (:1579-1583), then
 *                        CalcNonstat3DLine (:1648-1655);
 *   TDEM_PIPE_SPLIT      SumNonstat3DOnly (:1664-1673).
 * Stops at the first module that fails and returns its status; errbuf then names the
 * module.  Unlike GeoCalculatorSP it builds no mesh (RegularMeshBuilder / p.bat), starts
 * no process and maps no shared memory; the line voltages (SummatorEDMN, per
 * transmitter and profile) stay a separate call.  A `stop` file ends the run as in the
 * modules themselves. */
enum {
  TDEM_PIPE_TIME_GRID = 1,
  TDEM_PIPE_STATIONARY = 2,
  TDEM_PIPE_SPLIT = 4
};
tdem_status tdem_pipeline_directory(const char* workdir, int formulation, int scheme, int device, int flags,
                                    char* errbuf, size_t errlen);

typedef struct tdem_solver tdem_solver;

typedef struct tdem_info {
  int64_t n_edges;          /* unknowns incl. Dirichlet edges */
  int64_t n_interior;       /* unknowns of the factorized system */
  int64_t nnz_matrix;       /* entries of the full symmetric system pattern */
  int64_t nnz_factor;       /* stored factor entries (dense front blocks) */
  double factor_flops;      /* flops of one numeric factorization */
  int64_t device_bytes;     /* device memory held by the factorization */
  int n_sources;            /* transmitter positions solved together (RHS columns) */
  int n_times;              /* time layers incl. t0 */
  int first_layer;          /* first printed layer */
  int last_layer;           /* last printed layer */
  int n_rec_b;              /* B / emf receivers */
  int n_rec_e;              /* E receivers */
  int factorizations;       /* numeric factorizations done by the last run */
  int steps;                /* time steps done by the last run */
  int kernel_launches;      /* kernels launched by the last run */
  double t_setup_s, t_assemble_s, t_factor_s, t_steps_s, t_output_s;
  /* device time of the last tdem_solver_run from CUDA events on the solver's stream */
  double run_gpu_ms, factor_gpu_ms, solve_gpu_ms;
  int64_t h2d_bytes;        /* host->device bytes copied so far by this solver */
  int64_t d2h_bytes;        /* device->host bytes copied so far by this solver */
  int precision;            /* 64 = FP64 factor; 32 = FP32 factor + FP64 refinement */
  int refine_iters;         /* conjugate-gradient iterations of the last run (precision 32) */
  int refine_iters_max;     /* most iterations any time step needed */
  double refine_worst;      /* largest final relative residual of any step / column */
  int factor_slots;         /* numeric factors held (2: factorizations overlapped the steps;
                               factor_gpu_ms and solve_gpu_ms then overlap in run_gpu_ms) */
  int solve_schedule;       /* per-step solve of the n_sources columns: 0 fused level solves,
                               1 panel solves, 2 persistent fused level solves (chosen by the
                               solve autotuner for more than two columns, measured on the first
                               step of the first run) */
  int solve_split;          /* column groups that solve is split into */
  int solve_candidates;     /* schedules the autotuner measured (0: not tuned) */
  double solve_tuned_ms;    /* the chosen schedule's measured device time per solve */
  double ozaki_ms;          /* device time of the last run's trailing updates on the integer
                               tensor pipe (CUDA events around each launch) */
  double ozaki_macs;        /* 8-bit multiply-adds one factorization issues there */
} tdem_info;

/* Options of tdem_solver_create_ex (zero-initialise, then set what differs). */
typedef struct tdem_options {
  int precision;            /* 64 (default when 0): FP64 factorization, one direct solve per
                               step.  32: the per-step triangular solves run in FP32 on an FP32
                               factor, as the preconditioner of an FP64 conjugate-gradient
                               solve on the FP64 system (residuals, history and receivers in
                               FP64); the factor is the FP64 factorization rounded to FP32
                               unless fp32_update asks for an FP32 factorization */
  double refine_tol;        /* relative residual to reach per step and column (default 1e-10) */
  int refine_maxit;         /* iteration cap; exceeding it is TDEM_ERR_NUMERIC (default 200) */
  int leaf_size;            /* nested-dissection leaf size (default 128) */
  int fp32_update;          /* precision 32, the factorization: 0 = FP64 factorization (FP64
                               tensor pipe), its factor held rounded to FP32; 1 = FP32
                               factorization with FP32 FMA trailing updates; 2 = FP32
                               factorization with tensor-core trailing updates (tcgen05, 3xTF32,
                               FP32 accumulation).  1 and 2 break down (non-positive pivot) on
                               systems whose condition number is beyond FP32, as the benchmark
                               models' air (1e-8 S/m) makes them */
  int factor_slots;         /* numeric factors held on the device.  2 factors the
                               next time-step size on a low-priority stream while the current
                               decade's steps run (same results, a second factor's memory);
                               1 factors between the decades; 0 (default) = 2 when free device
                               memory holds it with room to spare.  The server treats 0 as 1. */
} tdem_options;

/* Creates a solver for the model in `workdir` (reads the input files, analyses
 * the sparsity pattern, assembles the FEM matrices on the device and prepares the
 * receiver operators).  Replaces Read_data + Prepare_To_Schema
 * (time_approx.cpp:169-557). */
tdem_status tdem_solver_create(const char* workdir, int formulation, int scheme, int device,
                               tdem_solver** out);
/* tdem_solver_create with options (opts may be NULL for the defaults). */
tdem_status tdem_solver_create_ex(const char* workdir, int formulation, int scheme, int device,
                                  const tdem_options* opts, tdem_solver** out);
/* Host-only planning of a forward solve: reads the inputs of `workdir` and analyses
 * the sparsity pattern (nested-dissection ordering, assembly tree, launch plans,
 * including the check that every level-solve unit waits only for units queued
 * before it) without touching a GPU.  For sizing runs and admission decisions; no
 * counterpart in the reference.  err (may be NULL) receives the message of a
 * failure. */
typedef struct tdem_plan_info {
  int64_t n_edges;          /* unknowns incl. Dirichlet edges */
  int64_t n_interior;       /* unknowns of the factorized system */
  int64_t nnz_matrix;       /* entries of the full symmetric system pattern */
  int64_t nnz_factor;       /* stored factor entries (dense front blocks) */
  double factor_flops;      /* flops of one numeric factorization */
  int64_t device_bytes;     /* device memory tdem_solver_create allocates with one factor slot */
  int64_t factor_slot_bytes;/* device memory of one more factor slot */
  int64_t solve_units;      /* level-solve units (forward + backward) */
  int n_fronts;             /* fronts of the assembly tree */
  int tree_levels;          /* levels of the assembly tree */
  int n_sources;            /* right-hand-side columns per step */
  int n_times;              /* time layers incl. t0 */
  double plan_seconds;      /* host time of the planning (inputs, patterns, analysis) */
  uint64_t digest;          /* hash of the elimination order, the fronts, the entry map and the
                               solve units: equal digests mean identical launch plans */
  double ozaki_flops;       /* flops of the trailing updates planned on the integer tensor
                               pipe (FP64 products by digit splitting; FP64 solvers) */
  int64_t ozaki_rows;       /* rows of the digit buffer those updates need */
  int64_t solve_chain;      /* 64-wide pivot blocks on the critical path of one triangular
                               solve direction: the sum over the tree levels of the largest
                               front's pivot blocks (each is one dependent link) */
} tdem_plan_info;
tdem_status tdem_solver_plan(const char* workdir, int formulation, int scheme, const tdem_options* opts,
                             tdem_plan_info* out, char* err, size_t err_len);
/* Runs all decades / time steps (TaskSP.cpp:628-702, Three_Layers_Schema). */
tdem_status tdem_solver_run(tdem_solver* s);
/* Writes the reference output files into the model directory (Gather_edsall,
 * give_out_vec_loop.cpp:240-615). */
tdem_status tdem_solver_write_outputs(tdem_solver* s);
/* Copies the output tables to host arrays of nlayers * 3 * nrec doubles laid out
 * [layer][component][receiver] (layers first_layer .. last_layer): eall = E (mV),
 * emf = emf (mV), ball = B (mTl), with the reference's units and signs as written
 * to the files.  Any pointer may be NULL. */
tdem_status tdem_solver_results(tdem_solver* s, double* eall, double* emf, double* ball);
tdem_status tdem_solver_info(const tdem_solver* s, tdem_info* info);
/* Device time of one time step's work on the factor the last tdem_solver_run ended
 * with (FP64 solvers): the history right-hand side and the triangular solves of
 * every source, either as one n x npls block (block != 0: the solve replayed from
 * its CUDA graph, as the run does) or as npls single-column steps issued one after
 * another (block == 0).  Average of reps repetitions in *ms_per_step; the solution
 * history and the results are not changed.  TDEM_ERR_STATE before a completed run.
 * No counterpart in the reference: it lets a caller compare the batched step with
 * sequential per-source solves (pardiso.cpp:113-120 solves npls columns per call). */
tdem_status tdem_solver_time_step(tdem_solver* s, int block, int reps, double* ms_per_step);
/* The solve autotuner's measurements for the solver's column count (n_sources):
 * up to max entries of (schedule kind, column groups, device ms per solve), in the
 * order measured; *count receives how many there are (0 before the first run, or
 * when the count is not tuned).  No counterpart in the reference. */
tdem_status tdem_solver_tune_log(const tdem_solver* s, int* kinds, int* splits, double* ms, int max, int* count);
/* Requests cancellation of a running tdem_solver_run (checked between time steps;
 * the reference polls a file named "stop", GeoCalculatorSP.cpp:27-39). */
tdem_status tdem_solver_cancel(tdem_solver* s);
const char* tdem_solver_error(const tdem_solver* s);
void tdem_solver_destroy(tdem_solver* s);

/* ---- Serving: a stream of forward-modelling requests on one GPU --------------------
 * Requests (one model directory each, any mesh size, A/E, two/three-point) are planned
 * on host threads (inputs, analysis), admitted first-in first-out when the device
 * memory their analysis needs fits the HBM budget next to the running requests, and
 * run concurrently on their own CUDA streams with factors and field histories resident
 * until they finish.  Results are independent of what else runs (deterministic
 * kernels).  No counterpart in the reference, which runs one CalcNonstat3DLine process
 * per model (GeoCalculatorSP.cpp:1656-1662). */
typedef struct tdem_server tdem_server;
typedef struct tdem_server_options {
  int device;               /* CUDA device */
  int max_active;           /* requests on the device at once (default 4 when 0) */
  int prep_threads;         /* host threads planning requests (default 2 when 0) */
  int64_t hbm_budget_bytes; /* admission budget (default: 85% of the free device memory) */
  int batch_max;            /* requests of one batch key merged into one run (0 or 1: none);
                               see tdem_server_submit_keyed */
} tdem_server_options;
typedef struct tdem_request_info {
  int status;               /* tdem_status of the request */
  int first_layer, last_layer, n_rec_b, n_rec_e, n_sources, steps, factorizations;
  double submit_s, admit_s, done_s;  /* steady-clock seconds */
  double run_gpu_ms;        /* device time of the request's time stepping */
  int64_t device_bytes;     /* admission footprint (0 for the later requests of a merged run) */
  int batch_size;           /* requests solved by the run that solved this one */
} tdem_request_info;
typedef struct tdem_server_stats {
  int64_t submitted, completed, failed;
  double latency_p50_s, latency_p99_s; /* submit -> done */
  double makespan_s, solves_per_s;     /* first submit -> last completion */
  int64_t peak_device_bytes;
  int peak_active;
  int64_t merged_runs, merged_requests; /* runs that solved several requests, and those requests */
} tdem_server_stats;
tdem_status tdem_server_create(const tdem_server_options* opts, tdem_server** out);
/* Queues one request (write_outputs != 0: also write the reference output files into
 * workdir); *request_id receives its id. */
tdem_status tdem_server_submit(tdem_server* srv, const char* workdir, int formulation, int scheme,
                               const tdem_options* opts, int write_outputs, int64_t* request_id);
/* tdem_server_submit with a batch key: queued requests with the same non-empty key,
 * the same formulation, scheme and options, and no output files are merged (up to
 * the server's batch_max) into one run that solves all their sources as one n x k
 * block per time step on one factorization per step size; each request receives its
 * own receivers' values.  The key states that the models differ only in their sources
 * and receivers (sours, group, recvsb/recvse and the receiver files, the initial
 * fields); the server checks it on the loaded models and runs them one by one when it
 * does not hold.  No counterpart in the reference, which solves the sources of one
 * model directory as npls right-hand sides (time_approx.cpp:1087). */
tdem_status tdem_server_submit_keyed(tdem_server* srv, const char* workdir, int formulation, int scheme,
                                     const tdem_options* opts, int write_outputs, const char* batch_key,
                                     int64_t* request_id);
/* Blocks until the request has finished; returns its status.  info may be NULL. */
tdem_status tdem_server_wait(tdem_server* srv, int64_t request_id, tdem_request_info* info);
/* Output tables of a finished request, as tdem_solver_results. */
tdem_status tdem_server_results(tdem_server* srv, int64_t request_id, double* eall, double* emf, double* ball);
/* Error message of a finished request ("" when it succeeded); valid until the server
 * is destroyed. */
const char* tdem_server_error(tdem_server* srv, int64_t request_id);
tdem_status tdem_server_stats_get(tdem_server* srv, tdem_server_stats* st);
/* Runs every queued request to completion, then releases the server. */
void tdem_server_destroy(tdem_server* srv);

/* GPU-backed stand-in for MKL's pardiso_64 with the semantics the reference uses
 * (pardiso.cpp:69-126): mtype = 2 (real SPD), upper-triangular CSR with 1-based
 * int64 indices, phase 12 (analysis + numeric factorization; the analysis is
 * reused while the pattern is unchanged), phase 33 (solve for nrhs column-major
 * right-hand sides b -> x), phase -1 (release).  The handle lives in pt[0];
 * maxfct, mnum, perm, iparm and msglvl are accepted and ignored.  *error: 0 ok,
 * -1 bad input / unsupported phase or mtype, -2 out of memory or CUDA error,
 * -4 non-positive pivot.  Runs on CUDA device 0 unless TDEM_PARDISO_DEVICE is set.
 * The reference zeroes pt before every phase 12 (pardiso_solver::init,
 * pardiso.cpp:43-58, 76): the handle is also kept by the address of pt, so a
 * phase 12 on a zeroed pt reuses the analysis, factor memory and stream made
 * for that array, and phase -1 releases them.  A phase 33 with more columns than
 * the analysing phase 12 was given (the reference analyses with nrhs = 1 and
 * solves npls columns) widens the solve once, refactoring from the values
 * already on the device. */
void tdem_pardiso_64(void* pt, const long long* maxfct, const long long* mnum, const long long* mtype,
                     const long long* phase, const long long* n, const void* a, const long long* ia,
                     const long long* ja, long long* perm, const long long* nrhs, long long* iparm,
                     const long long* msglvl, void* b, void* x, long long* error);
/* Same function under MKL's name, so a maintainer can link the reference's
 * pardiso_solver against this library unchanged. */
void pardiso_64(void* pt, const long long* maxfct, const long long* mnum, const long long* mtype,
                const long long* phase, const long long* n, const void* a, const long long* ia,
                const long long* ja, long long* perm, const long long* nrhs, long long* iparm,
                const long long* msglvl, void* b, void* x, long long* error);
/* MKL threading call made by pardiso_solver::factorize (pardiso.cpp:83); no-op here. */
void mkl_set_num_threads(int n);
/* Live pardiso_64 handles (made by phase 12, released by phase -1).  No counterpart
 * in the reference: lets a caller check that repeated factorizations through the
 * boundary hold one handle per pt array. */
int tdem_pardiso_handles(void);

/* Residual norms of a block of solutions, computed on CUDA device `device`:
 * norms[2j] = ||b_j - A x_j||_2 and norms[2j+1] = ||b_j||_2 for j < ncols.
 * A is n x n in full CSR (both triangles), 0-based: rowptr (n+1 int64), col
 * (int32), val (FP64).  x, b: column-major n x ncols with leading dimension ld.
 * Every pointer is device memory; the work is queued on `stream` (a cudaStream_t,
 * NULL for the legacy default stream) and norms are valid once it completes.
 * 1 <= ncols <= 64.  The result is deterministic (fixed reduction order).
 * Scratch is taken from the stream-ordered allocator for each call.
 * No counterpart in the reference: pardiso_solver::solve_nrhs (pardiso.cpp:113-120)
 * never checks its solutions; this lets a caller of the solver boundary do so. */
tdem_status tdem_residual_norms(int device, int64_t n, const int64_t* rowptr, const int* col,
                                const double* val, const double* x, const double* b, int64_t ld,
                                int ncols, double* norms, void* stream);

/* tdem_residual_norms without any device allocation, for callers that may not
 * allocate: code being captured into a CUDA graph (cudaMallocAsync inside a capture
 * becomes part of the graph) and callers that run against a fixed memory budget.
 * The scratch is a static device array of 303,104 bytes in the library (296 x 64 x 2
 * doubles), so ncols is limited to 64 (larger is TDEM_ERR_ARGUMENT).  Every call
 * looks up the array's address on its device (cudaGetSymbolAddress; the first call
 * on a device may load the module, so make it before any stream capture), so the
 * address is never stale, also after a cudaDeviceReset.  The scratch needs no
 * initial contents.  Calls whose executions overlap on one device share the scratch
 * and race: issue them on one stream or synchronise between them.  Same arguments
 * and results as tdem_residual_norms.
 * No counterpart in the reference. */
tdem_status tdem_residual_norms_noalloc(int device, int64_t n, const int64_t* rowptr, const int* col,
                                        const double* val, const double* x, const double* b, int64_t ld,
                                        int ncols, double* norms, void* stream);

/* Library version string. */
const char* tdem_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TDEM_B200_H */
