"""B200-native 3D time-domain EM edge-FEM forward solve (horizontal grounded-wire source).

Python mirror of the C-ABI in include/tdem.h.  The product path is the native
library lib/libtdem_b200.so (CUDA kernels for sm_100a + C++ host code); this
module only loads it with ctypes.  There is no CPU fallback: every entry point
raises RuntimeError when the library is missing or no CUDA device is usable.

Reference interfaces mirrored:
  * run_directory(workdir, "A"|"E", 2|3)  ~ running CalcNonstat3DLine in the
    Calculations directory (GeoCalculatorSP.cpp:1656-1662 -> CalcSP, TaskSP.cpp:445);
  * Solver                               ~ Read_data / Prepare_To_Schema /
    the decade loop / Gather_edsall of CalcNonstat3DLine;
  * pardiso_64(...)                      ~ MKL's pardiso_64 as called by
    pardiso_solver (pardiso.cpp:69-126), backed by the GPU factorization.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtdem_b200.so")
EXE_PATH = os.path.join(_HERE, "lib", "tdem_calcnonstat3dline")

FORMULATIONS = {"A": 0, "E": 1, 0: 0, 1: 1}

STATUS = {
    0: "TDEM_OK",
    1: "TDEM_ERR_ARGUMENT",
    2: "TDEM_ERR_INPUT",
    3: "TDEM_ERR_CUDA",
    4: "TDEM_ERR_NUMERIC",
    5: "TDEM_ERR_CANCELLED",
    6: "TDEM_ERR_STATE",
    7: "TDEM_ERR_HOST",
}


class TdemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("%s: %s" % (STATUS.get(status, status), message))
        self.status = status


class TdemInfo(ctypes.Structure):
    _fields_ = [
        ("n_edges", ctypes.c_int64),
        ("n_interior", ctypes.c_int64),
        ("nnz_matrix", ctypes.c_int64),
        ("nnz_factor", ctypes.c_int64),
        ("factor_flops", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
        ("n_sources", ctypes.c_int),
        ("n_times", ctypes.c_int),
        ("first_layer", ctypes.c_int),
        ("last_layer", ctypes.c_int),
        ("n_rec_b", ctypes.c_int),
        ("n_rec_e", ctypes.c_int),
        ("factorizations", ctypes.c_int),
        ("steps", ctypes.c_int),
        ("kernel_launches", ctypes.c_int),
        ("t_setup_s", ctypes.c_double),
        ("t_assemble_s", ctypes.c_double),
        ("t_factor_s", ctypes.c_double),
        ("t_steps_s", ctypes.c_double),
        ("t_output_s", ctypes.c_double),
        ("run_gpu_ms", ctypes.c_double),
        ("factor_gpu_ms", ctypes.c_double),
        ("solve_gpu_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
        ("precision", ctypes.c_int),
        ("refine_iters", ctypes.c_int),
        ("refine_iters_max", ctypes.c_int),
        ("refine_worst", ctypes.c_double),
        ("factor_slots", ctypes.c_int),
        ("solve_schedule", ctypes.c_int),
        ("solve_split", ctypes.c_int),
        ("solve_candidates", ctypes.c_int),
        ("solve_tuned_ms", ctypes.c_double),
        ("ozaki_ms", ctypes.c_double),
        ("ozaki_macs", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class TdemOptions(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("refine_tol", ctypes.c_double),
        ("refine_maxit", ctypes.c_int),
        ("leaf_size", ctypes.c_int),
        ("fp32_update", ctypes.c_int),
        ("factor_slots", ctypes.c_int),
    ]


class TdemPlanInfo(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_int64), ("n_interior", ctypes.c_int64), ("nnz_matrix", ctypes.c_int64),
                ("nnz_factor", ctypes.c_int64), ("factor_flops", ctypes.c_double), ("device_bytes", ctypes.c_int64),
                ("factor_slot_bytes", ctypes.c_int64), ("solve_units", ctypes.c_int64), ("n_fronts", ctypes.c_int),
                ("tree_levels", ctypes.c_int), ("n_sources", ctypes.c_int), ("n_times", ctypes.c_int),
                ("plan_seconds", ctypes.c_double), ("digest", ctypes.c_uint64), ("ozaki_flops", ctypes.c_double),
                ("ozaki_rows", ctypes.c_int64), ("solve_chain", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class TdemServerOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_active", ctypes.c_int), ("prep_threads", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_int64), ("batch_max", ctypes.c_int)]


class TdemRequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("first_layer", ctypes.c_int), ("last_layer", ctypes.c_int),
                ("n_rec_b", ctypes.c_int), ("n_rec_e", ctypes.c_int), ("n_sources", ctypes.c_int),
                ("steps", ctypes.c_int), ("factorizations", ctypes.c_int), ("submit_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double), ("run_gpu_ms", ctypes.c_double),
                ("device_bytes", ctypes.c_int64), ("batch_size", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class TdemServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("latency_p50_s", ctypes.c_double), ("latency_p99_s", ctypes.c_double),
                ("makespan_s", ctypes.c_double), ("solves_per_s", ctypes.c_double),
                ("peak_device_bytes", ctypes.c_int64), ("peak_active", ctypes.c_int),
                ("merged_runs", ctypes.c_int64), ("merged_requests", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib: Optional[ctypes.CDLL] = None

EXPORTED = [
    "tdem_run_directory",
    "tdem_stationary_directory",
    "tdem_time_direct_solver",
    "tdem_correct_time_mesh",
    "tdem_sum_nonstat_3d_only",
    "tdem_summator_edmn",
    "tdem_pipeline_directory",
    "tdem_solver_create",
    "tdem_solver_create_ex",
    "tdem_solver_plan",
    "tdem_solver_run",
    "tdem_solver_write_outputs",
    "tdem_solver_results",
    "tdem_solver_info",
    "tdem_solver_cancel",
    "tdem_solver_time_step",
    "tdem_solver_tune_log",
    "tdem_solver_error",
    "tdem_solver_destroy",
    "tdem_pardiso_64",
    "pardiso_64",
    "mkl_set_num_threads",
    "tdem_pardiso_handles",
    "tdem_residual_norms",
    "tdem_server_create",
    "tdem_server_submit",
    "tdem_server_submit_keyed",
    "tdem_server_wait",
    "tdem_server_results",
    "tdem_server_error",
    "tdem_server_stats_get",
    "tdem_server_destroy",
    "tdem_version",
]


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libtdem_b200.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("native library %s not found: run __graft_entry__.build() "
                           "(or python -m <package>.build) first" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.tdem_run_directory.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_char_p, ctypes.c_size_t]
    lib.tdem_run_directory.restype = ctypes.c_int
    lib.tdem_pipeline_directory.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_char_p, ctypes.c_size_t]
    lib.tdem_pipeline_directory.restype = ctypes.c_int
    lib.tdem_stationary_directory.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    lib.tdem_stationary_directory.restype = ctypes.c_int
    for name in ("tdem_time_direct_solver", "tdem_correct_time_mesh"):
        getattr(lib, name).argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        getattr(lib, name).restype = ctypes.c_int
    lib.tdem_sum_nonstat_3d_only.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.tdem_sum_nonstat_3d_only.restype = ctypes.c_int
    lib.tdem_summator_edmn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                       ctypes.c_size_t]
    lib.tdem_summator_edmn.restype = ctypes.c_int
    lib.tdem_solver_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(P)]
    lib.tdem_solver_create.restype = ctypes.c_int
    lib.tdem_solver_create_ex.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(TdemOptions), ctypes.POINTER(P)]
    lib.tdem_solver_create_ex.restype = ctypes.c_int
    lib.tdem_solver_plan.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TdemOptions),
                                     ctypes.POINTER(TdemPlanInfo), ctypes.c_char_p, ctypes.c_size_t]
    lib.tdem_solver_plan.restype = ctypes.c_int
    for name in ("tdem_solver_run", "tdem_solver_write_outputs", "tdem_solver_cancel"):
        getattr(lib, name).argtypes = [P]
        getattr(lib, name).restype = ctypes.c_int
    lib.tdem_solver_time_step.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.tdem_solver_time_step.restype = ctypes.c_int
    lib.tdem_solver_tune_log.argtypes = [P, P, P, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.tdem_solver_tune_log.restype = ctypes.c_int
    lib.tdem_solver_results.argtypes = [P, P, P, P]
    lib.tdem_solver_results.restype = ctypes.c_int
    lib.tdem_solver_info.argtypes = [P, ctypes.POINTER(TdemInfo)]
    lib.tdem_solver_info.restype = ctypes.c_int
    lib.tdem_solver_error.argtypes = [P]
    lib.tdem_solver_error.restype = ctypes.c_char_p
    lib.tdem_solver_destroy.argtypes = [P]
    lib.tdem_solver_destroy.restype = None
    lib.tdem_version.restype = ctypes.c_char_p
    pi = ctypes.POINTER(ctypes.c_longlong)
    for name in ("tdem_pardiso_64", "pardiso_64"):
        f = getattr(lib, name)
        f.argtypes = [P, pi, pi, pi, pi, pi, P, pi, pi, pi, pi, pi, pi, P, P, pi]
        f.restype = None
    lib.tdem_pardiso_handles.argtypes = []
    lib.tdem_pardiso_handles.restype = ctypes.c_int
    lib.tdem_residual_norms.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P, P, P, ctypes.c_int64,
                                        ctypes.c_int, P, P]
    lib.tdem_residual_norms.restype = ctypes.c_int
    lib.tdem_server_create.argtypes = [ctypes.POINTER(TdemServerOptions), ctypes.POINTER(P)]
    lib.tdem_server_create.restype = ctypes.c_int
    lib.tdem_server_submit.argtypes = [P, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TdemOptions),
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    lib.tdem_server_submit.restype = ctypes.c_int
    lib.tdem_server_submit_keyed.argtypes = [P, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(TdemOptions), ctypes.c_int, ctypes.c_char_p,
                                             ctypes.POINTER(ctypes.c_int64)]
    lib.tdem_server_submit_keyed.restype = ctypes.c_int
    lib.tdem_server_wait.argtypes = [P, ctypes.c_int64, ctypes.POINTER(TdemRequestInfo)]
    lib.tdem_server_wait.restype = ctypes.c_int
    lib.tdem_server_results.argtypes = [P, ctypes.c_int64, P, P, P]
    lib.tdem_server_results.restype = ctypes.c_int
    lib.tdem_server_error.argtypes = [P, ctypes.c_int64]
    lib.tdem_server_error.restype = ctypes.c_char_p
    lib.tdem_server_stats_get.argtypes = [P, ctypes.POINTER(TdemServerStats)]
    lib.tdem_server_stats_get.restype = ctypes.c_int
    lib.tdem_server_destroy.argtypes = [P]
    lib.tdem_server_destroy.restype = None
    _lib = lib
    return lib


def _form(formulation) -> int:
    if formulation not in FORMULATIONS:
        raise ValueError("formulation must be 'A' or 'E'")
    return FORMULATIONS[formulation]


def run_directory(workdir: str, formulation="A", scheme: int = 2, device: int = 0) -> None:
    """One drop-in run of CalcNonstat3DLine in workdir (writes edsall/ball/eall_anom.N)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_run_directory(os.fsencode(workdir), _form(formulation), int(scheme), int(device), buf,
                                len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


PIPE_TIME_GRID, PIPE_STATIONARY, PIPE_SPLIT = 1, 2, 4


def pipeline_directory(workdir: str, formulation="A", scheme: int = 2, device: int = 0,
                       flags: int = PIPE_TIME_GRID | PIPE_STATIONARY | PIPE_SPLIT) -> None:
    """The direct-mode 3D-only module sequence of GeoCalculatorSP in workdir: time
    grid (when tcff exists), stationary initial field, transient, component split."""
    lib = load_library()
    err = ctypes.create_string_buffer(1024)
    st = lib.tdem_pipeline_directory(os.fsencode(workdir), _form(formulation), int(scheme), int(device), int(flags),
                                     err, len(err))
    if st != 0:
        raise TdemError(st, err.value.decode(errors="replace"))


def stationary_directory(workdir: str, device: int = 0) -> None:
    """Drop-in run of CalcStat3D_3T_A in workdir: the grounded-wire stationary
    initial field on the GPU (writes v3n.dat, v3a.dat and a0.dat)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_stationary_directory(os.fsencode(workdir), int(device), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


def time_direct_solver(workdir: str) -> None:
    """Drop-in run of TimeDirectSolver in workdir (host only): infite.0 becomes the
    piecewise-uniform grid with step growth tcff; currentfunction and deltafunction
    are interpolated onto it."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_time_direct_solver(os.fsencode(workdir), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


def correct_time_mesh(workdir: str) -> None:
    """Drop-in run of CorrectTimeMesh in workdir (host only): short decades of
    infite.0 are refilled with the previous decade's step."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_correct_time_mesh(os.fsencode(workdir), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


def sum_nonstat_3d_only(workdir: str) -> None:
    """Drop-in run of SumNonstat3DOnly in workdir (host only): the per-component
    files Bxall.N .. Ezall.N from ball_anom.N, edsall_anom.N and eall_anom.N."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_sum_nonstat_3d_only(os.fsencode(workdir), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


def summator_edmn(workdir: str, with_ddv: bool, profile: int, place: int) -> None:
    """Drop-in run of SummatorEDMN in workdir (host only): line voltages
    edmnall<profile>_<place> (and edmoonall.. with with_ddv)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_summator_edmn(os.fsencode(workdir), int(bool(with_ddv)), int(profile), int(place), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))


def plan(workdir: str, formulation="A", scheme: int = 2, precision: int = 64, leaf_size: int = 128,
         factor_slots: int = 0) -> dict:
    """Host-only planning of a forward solve (no GPU): sizes of the system and its
    factor, factorization flops and the device memory a Solver would allocate."""
    lib = load_library()
    opts = TdemOptions(int(precision), 1e-10, 200, int(leaf_size), 0, int(factor_slots))
    info = TdemPlanInfo()
    buf = ctypes.create_string_buffer(2048)
    st = lib.tdem_solver_plan(os.fsencode(workdir), _form(formulation), int(scheme), ctypes.byref(opts),
                              ctypes.byref(info), buf, len(buf))
    if st != 0:
        raise TdemError(st, buf.value.decode(errors="replace"))
    return info.as_dict()


class Solver:
    """A transient forward solve held on one GPU: create -> run -> results / write_outputs."""

    def __init__(self, workdir: str, formulation="A", scheme: int = 2, device: int = 0, precision: int = 64,
                 refine_tol: float = 1e-10, refine_maxit: int = 200, leaf_size: int = 128,
                 fp32_update: str = "default", factor_slots: int = 0):
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        engines = {"default": 0, "cuda_cores": 1, "tensor_cores": 2}
        if fp32_update not in engines:
            raise ValueError("fp32_update must be one of %s" % sorted(engines))
        opts = TdemOptions(int(precision), float(refine_tol), int(refine_maxit), int(leaf_size),
                           engines[fp32_update], int(factor_slots))
        st = self._lib.tdem_solver_create_ex(os.fsencode(workdir), _form(formulation), int(scheme), int(device),
                                             ctypes.byref(opts), ctypes.byref(self._h))
        if st != 0:
            msg = self.error()
            self.close()
            raise TdemError(st, msg)

    def error(self) -> str:
        if not self._h:
            return "no solver"
        return (self._lib.tdem_solver_error(self._h) or b"").decode(errors="replace")

    def _check(self, st: int) -> None:
        if st != 0:
            raise TdemError(st, self.error())

    def run(self) -> "Solver":
        self._check(self._lib.tdem_solver_run(self._h))
        return self

    def cancel(self) -> None:
        self._check(self._lib.tdem_solver_cancel(self._h))

    def time_step(self, block: bool = True, reps: int = 5) -> float:
        """Device ms of one time step's RHS + solves of every source on the last
        run's factor: one n x npls block, or npls single-column steps in turn."""
        ms = ctypes.c_double(0.0)
        self._check(self._lib.tdem_solver_time_step(self._h, 1 if block else 0, int(reps), ctypes.byref(ms)))
        return ms.value

    def tune_log(self) -> list:
        """The solve autotuner's candidates for this solver's column count:
        [(kind, column groups, device ms per solve), ...]."""
        kinds = (ctypes.c_int * 16)()
        splits = (ctypes.c_int * 16)()
        ms = (ctypes.c_double * 16)()
        n = ctypes.c_int(0)
        self._check(self._lib.tdem_solver_tune_log(self._h, ctypes.cast(kinds, ctypes.c_void_p),
                                                   ctypes.cast(splits, ctypes.c_void_p),
                                                   ctypes.cast(ms, ctypes.c_void_p), 16, ctypes.byref(n)))
        return [(kinds[i], splits[i], ms[i]) for i in range(min(n.value, 16))]

    def write_outputs(self) -> None:
        self._check(self._lib.tdem_solver_write_outputs(self._h))

    def info(self) -> dict:
        inf = TdemInfo()
        self._check(self._lib.tdem_solver_info(self._h, ctypes.byref(inf)))
        return inf.as_dict()

    def results(self):
        """(eall, emf, ball): arrays [layer][component][receiver] in mV, mV, mTl."""
        inf = self.info()
        nl = inf["last_layer"] - inf["first_layer"] + 1
        e = np.zeros((nl, 3, inf["n_rec_e"]))
        m = np.zeros((nl, 3, inf["n_rec_b"]))
        b = np.zeros((nl, 3, inf["n_rec_b"]))
        self._check(self._lib.tdem_solver_results(self._h, e.ctypes.data, m.ctypes.data, b.ctypes.data))
        return e, m, b

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tdem_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pardiso_64(handle: np.ndarray, phase: int, a, ia, ja, nrhs: int = 1, b=None, x=None) -> int:
    """Calls the GPU-backed pardiso_64 with MKL's argument conventions (mtype 2,
    1-based upper CSR with int64 indices).  handle is a 64-entry int64 array
    (MKL's pt); returns MKL's error code."""
    lib = load_library()
    pi = ctypes.POINTER(ctypes.c_longlong)

    def ll(v):
        return ctypes.byref(ctypes.c_longlong(v))

    n = len(ia) - 1
    err = ctypes.c_longlong(0)
    iparm = np.zeros(64, dtype=np.int64)
    perm = np.zeros(max(n, 1), dtype=np.int64)
    ia = np.ascontiguousarray(ia, dtype=np.int64)
    ja = np.ascontiguousarray(ja, dtype=np.int64)
    a = np.ascontiguousarray(a, dtype=np.float64)
    lib.pardiso_64(handle.ctypes.data, ll(1), ll(1), ll(2), ll(phase), ll(n), a.ctypes.data,
                   ia.ctypes.data_as(pi), ja.ctypes.data_as(pi), perm.ctypes.data_as(pi), ll(nrhs),
                   iparm.ctypes.data_as(pi), ll(0), None if b is None else b.ctypes.data,
                   None if x is None else x.ctypes.data, ctypes.byref(err))
    return int(err.value)


def residual_norms(device: int, n: int, rowptr: int, col: int, val: int, x: int, b: int, ld: int,
                   ncols: int, norms: int, stream: int = 0) -> None:
    """tdem_residual_norms on device pointers (integers, e.g. torch's data_ptr()):
    norms[2j] = ||b_j - A x_j||, norms[2j+1] = ||b_j|| for the full-CSR matrix A.
    Queued on `stream` (a cudaStream_t handle, 0 for the default stream)."""
    st = load_library().tdem_residual_norms(device, n, rowptr, col, val, x, b, ld, ncols, norms, stream)
    if st != 0:
        raise TdemError(st, "tdem_residual_norms failed (status %d)" % st)


class Server:
    """Serving loop on one GPU (tdem_server_*): submit model directories, wait for
    their transients; requests are admitted by the device memory their analysis
    needs and run concurrently on their own streams; with batch_max > 1, queued
    requests submitted with the same batch key are merged into one run."""

    def __init__(self, device: int = 0, max_active: int = 4, prep_threads: int = 2, hbm_budget_bytes: int = 0,
                 batch_max: int = 0):
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        o = TdemServerOptions(int(device), int(max_active), int(prep_threads), int(hbm_budget_bytes),
                              int(batch_max))
        st = self._lib.tdem_server_create(ctypes.byref(o), ctypes.byref(self._h))
        if st != 0:
            raise TdemError(st, "tdem_server_create failed")

    def submit(self, workdir: str, formulation="A", scheme: int = 2, precision: int = 64,
               write_outputs: bool = False, batch_key: str = "") -> int:
        opts = TdemOptions(int(precision), 1e-10, 200, 128, 0, 0)
        rid = ctypes.c_int64(0)
        st = self._lib.tdem_server_submit_keyed(self._h, os.fsencode(workdir), _form(formulation), int(scheme),
                                                ctypes.byref(opts), int(bool(write_outputs)),
                                                batch_key.encode() if batch_key else None, ctypes.byref(rid))
        if st != 0:
            raise TdemError(st, "tdem_server_submit failed")
        return int(rid.value)

    def wait(self, request_id: int) -> dict:
        """Blocks until the request is done; returns its info (raises on failure)."""
        info = TdemRequestInfo()
        st = self._lib.tdem_server_wait(self._h, int(request_id), ctypes.byref(info))
        if st != 0:
            raise TdemError(st, self._lib.tdem_server_error(self._h, int(request_id)).decode(errors="replace"))
        return info.as_dict()

    def results(self, request_id: int, info: dict):
        nl = info["last_layer"] - info["first_layer"] + 1
        e = np.zeros((nl, 3, info["n_rec_e"]))
        m = np.zeros((nl, 3, info["n_rec_b"]))
        b = np.zeros((nl, 3, info["n_rec_b"]))
        st = self._lib.tdem_server_results(self._h, int(request_id), e.ctypes.data, m.ctypes.data, b.ctypes.data)
        if st != 0:
            raise TdemError(st, "tdem_server_results failed")
        return e, m, b

    def stats(self) -> dict:
        s = TdemServerStats()
        self._lib.tdem_server_stats_get(self._h, ctypes.byref(s))
        return s.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.tdem_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
