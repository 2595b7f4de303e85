#!/usr/bin/env python
"""Benchmark of the B200 transient edge-FEM forward solve.

Metric: forward solves per second (one solve = one transmitter position's whole
transient: every factorization, every time step, every receiver), on the 80^3
three-layer-plus-block model with the E-formulation and the three-point (BDF2)
scheme, 160 steps over 1e-6 .. 1e-1 s (the configuration the headline metric is
quoted on).  Synthetic inputs are generated by the package's model generator;
the grounded-wire initial field is the analytic half-space field
(modelgen.write_analytic_initial_field).

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                        [--config c2|c1|c3|c5]
Multi-GPU (one process per GPU, replicas: every rank solves its own copy of the
workload, no data-path collective) is launched by torch.distributed.run.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
PKG = "a-e_formulations_3d_timedomain_em_horizontalgroundedwiresource_b200"
METRIC = "forward solves/s + p50/p99 latency, mixed vs FP64 GPU, ≤1e-5 rel. error"
# k_oz_update, one launch of the 40^3 half-space (ncu --set full, profiles/k_oz_update_c1.md):
# DRAM bytes read + written and 8-bit tensor ops of that launch
OZ_CAPTURE_DRAM_BYTES = 342.647296e6 + 200.931328e6
OZ_CAPTURE_OPS = 493753466880.0


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def make_spec(cfg: str, mg, n_steps_override=None):
    if cfg == "c1":
        spec = mg.halfspace_model()
        return spec, "A", 2, "40^3 half-space, A-form, two-point, 120 steps, 1 wire, 21 receivers"
    if cfg == "c2":
        spec = mg.layered_block_model()
        return spec, "E", 3, "80^3 three-layer + 0.1 S/m block, E-form, BDF2, 160 steps, 1 wire, 21 receivers"
    if cfg == "c3":
        spec = mg.layered_block_model(sources=mg.wire_grid_sources())
        return spec, "A", 3, "80^3 three-layer + block, A-form, BDF2, 160 steps, 32 wires as one n x 32 block"
    if cfg == "c5":
        spec = mg.largest_model(20261203)
        return spec, "A", 3, ("120x120x100 three-layer + 5 random 0.05-1 S/m blocks (PCG64(20261203)), A-form, "
                              "BDF2, 200 steps to 1 s, 200 m wire, 21 receivers")
    raise ValueError(cfg)


def write_workload(cfg: str, path: str, air_sigma=None):
    mg = importlib.import_module(PKG + ".modelgen")
    spec, form, scheme, desc = make_spec(cfg, mg)
    if air_sigma is not None:
        # well-conditioned variant for the FP32-factor path (air of air_sigma S/m)
        spec.sigma_air = air_sigma
        desc += ", air %g S/m" % air_sigma
    info = mg.write_model(path, spec)
    mg.write_analytic_initial_field(path, spec)
    return spec, form, scheme, desc, info


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY, "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz = float(p[1].split()[0])
                smax = float(p[2].split()[0])
            except ValueError:
                continue
            sm.append(mhz)
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": ["no samples"]}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = os.environ.get("TDEM_BENCH_BACKEND", "nccl")
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=1800))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_units(total: int, world: int, rank: int):
    """Forward solves assigned to one rank when total solves are spread over world ranks."""
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


# ---------------------------------------------------------------------------
# measurements
# ---------------------------------------------------------------------------
def fp64_peak_tflops(device: int) -> float:
    """Measured cuBLAS DGEMM throughput (8192^3, best of 3) -- the FP64 roofline."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda:%d" % device)
    b = torch.randn(n, n, dtype=torch.float64, device="cuda:%d" % device)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def measured_peaks() -> dict:
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


def count_factorizations(times, scheme: int):
    """Factorizations of a full solve: one per distinct step length, plus the
    two-point start-up factorization of the three-point scheme."""
    h = [times[i + 1] - times[i] for i in range(len(times) - 1)]
    distinct = 1 + sum(1 for i in range(1, len(h)) if abs(1 - h[i - 1] / h[i]) > 1e-3)
    return distinct + (1 if scheme == 3 else 0)


def cpu_baseline(cfg: str, spec, form: str, scheme: int, workdir: str, full_factorizations: int,
                 full_steps: int, threads: int) -> dict:
    """Times the reference's own CalcNonstat3DLine (built from source, oracle/_ref)
    on a bounded sample of the same workload: the same variant, mesh and matrices
    with the time grid cut to its first 3 steps (one factorization for the
    two-point scheme; two for the three-point one, which takes its first two steps
    with the two-point formula), so that 3 time layers are printed.  The per-call
    wall times logged by the pardiso_64 stand-in split the run into set-up,
    factorization and per-step time; the full solve's time is extrapolated from
    them (set-up + factorizations x mean factor time + steps x step time) and
    labelled as such.  The sample's outputs stay in workdir."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import run_ref  # noqa: E402  (oracle: baseline leg only)
    mg = importlib.import_module(PKG + ".modelgen")
    variant = form + str(scheme)  # the same variant as the GPU run
    if not run_ref.available("CalcNonstat3DLine_" + variant):
        return {"value": None, "unit": "forward solves/s", "cores": threads, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    import copy
    s2 = copy.deepcopy(spec)
    cut = 4
    s2.times = spec.times[:cut]
    s2.print_interval = (float(s2.times[1]), float(s2.times[cut - 1]))
    mg.write_model(workdir, s2)
    mg.write_analytic_initial_field(workdir, s2)
    timing = os.path.join(workdir, "pardiso_calls.txt")
    if os.path.exists(timing):
        os.unlink(timing)
    env = run_ref.ref_env(threads)
    env["TDEM_ORACLE_TIMING"] = timing
    t0 = time.time()
    with open(os.path.join(workdir, "ref.log"), "w") as log:
        subprocess.run([run_ref.binary("CalcNonstat3DLine_" + variant)], cwd=workdir, env=env, stdout=log,
                       stderr=subprocess.STDOUT, check=True, timeout=3600)
    wall = time.time() - t0
    n_big = spec.n_edges
    fac, sol = [], []
    first = None
    last_end = 0.0
    with open(timing) as f:
        for line in f:
            ph, n, nrhs, a, b = line.split()
            if int(n) != n_big:
                continue
            a, b = float(a), float(b)
            if int(ph) == 12:
                fac.append(b - a)
                first = a if first is None else first
            if int(ph) == 33:
                sol.append(b - a)
                last_end = b
    t_fact = sum(fac) / max(len(fac), 1)
    steps = len(sol)
    t_after = (last_end - (first + sum(fac))) if first is not None else 0.0
    t_step = t_after / max(steps, 1)
    t_setup = wall - t_fact * len(fac) - t_after
    full = t_setup + full_factorizations * t_fact + full_steps * t_step
    return {"value": 1.0 / full, "unit": "forward solves/s", "cores": threads, "kind": "reference",
            "extrapolated": True, "measured_wall_s": wall, "sampled_steps": steps,
            "sampled_factorizations": len(fac), "setup_s": t_setup, "factor_s": t_fact, "step_s": t_step,
            "extrapolated_solve_s": full, "full_factorizations": full_factorizations, "full_steps": full_steps,
            "sample": "reference CalcNonstat3DLine_%s (built from source, CPU FP64 Cholesky stand-in for "
                      "MKL PARDISO) on the same mesh, time grid cut to %d steps: wall %.1f s = set-up %.1f s + "
                      "%d factorization(s) x %.2f s + %d steps x %.3f s; extrapolated to %d factorizations + "
                      "%d steps = %.1f s per forward solve" % (variant, steps, wall, t_setup, len(fac), t_fact,
                                                               steps, t_step, full_factorizations, full_steps,
                                                               full)}


def gpu_parity(pkg, outs, ref_dir: str, work: str, form: str, scheme: int, device: int, label: str) -> dict:
    """Runs the GPU solver on the inputs of a reference run (ref_dir, outputs
    present) and compares every result file: the largest deviation of any component
    from the reference, relative to the peak of that receiver's vector transient
    (outputs.compare_files)."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import run_ref  # noqa: E402  (oracle: the checker)
    run_ref.copy_inputs(ref_dir, work)
    with pkg.Solver(work, form, scheme, device=device) as s:
        s.run()
        s.write_outputs()
        npls = s.info()["n_sources"]
    worst = 0.0
    for p in range(1, npls + 1):
        for stem in ("eall_anom", "edsall_anom", "ball_anom"):
            name = "%s.%d" % (stem, p)
            worst = max(worst, outs.compare_files(os.path.join(work, name), os.path.join(ref_dir, name)))
    return {"case": label, "max_rel_err": worst, "files": 3 * npls}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference_arm(args, world, rank, local):
    """The reference's own CalcNonstat3DLine on the host cores.  A full solve of the
    80^3 workload takes ~13 min on 16 cores, so each sample runs the workload cut to
    its first 3 steps and the full solve is extrapolated (labelled so in the line,
    with the measured phases); the extrapolation is checked once per run against a
    full reference solve of the 40^3 half-space (A-form, two-point, 120 steps),
    extrapolated and measured side by side."""
    if rank != 0:
        return
    mg = importlib.import_module(PKG + ".modelgen")
    spec, form, scheme, desc = make_spec(args.config, mg)
    threads = os.cpu_count() or 1
    n_fact = count_factorizations(spec.times, scheme)
    n_steps = len(spec.times) - 1
    samples = max(1, min(args.steps, args.ref_samples))
    base = tempfile.mkdtemp(prefix="tdem_ref_")
    vals = []
    check = None
    try:
        t_run = time.time()
        for i in range(samples):
            d = os.path.join(base, "s%d" % i)
            os.makedirs(d)
            vals.append(cpu_baseline(args.config, spec, form, scheme, d, n_fact, n_steps, threads))
            shutil.rmtree(d, ignore_errors=True)
        if not args.no_ref_check and vals and vals[0].get("value"):
            sys.path.insert(0, os.path.join(HERE, "oracle"))
            import run_ref  # noqa: E402  (oracle: reference arm only)
            c1 = mg.halfspace_model()
            d = os.path.join(base, "c1_cut")
            os.makedirs(d)
            est = cpu_baseline("c1", c1, "A", 2, d, count_factorizations(c1.times, 2), len(c1.times) - 1, threads)
            d = os.path.join(base, "c1_full")
            mg.write_model(d, c1)
            mg.write_analytic_initial_field(d, c1)
            meas = run_ref.run_transient(d, "A2", threads=threads)
            check = {"workload": "40^3 half-space, A-form, two-point, 120 steps (full reference solve)",
                     "extrapolated_s": est["extrapolated_solve_s"], "measured_s": meas,
                     "measured_over_extrapolated": meas / est["extrapolated_solve_s"]}
        ref_wall = time.time() - t_run
    finally:
        shutil.rmtree(base, ignore_errors=True)
    ok = [x for x in vals if x.get("value")]
    v = sum(x["value"] for x in ok) / len(ok) if ok else None
    last = dict(vals[-1]) if vals else None
    line = {"metric": METRIC, "value": v, "unit": "forward solves/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": len(vals), "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "extrapolated": True,
            "ms_per_step": (1000.0 * sum(x["measured_wall_s"] for x in ok) / len(ok)) if ok else None,
            "ms_per_step_is": "measured wall time of one sample (the workload cut to its first 3 steps)",
            "extrapolated_ms_per_solve": (1000.0 / v) if v else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "parallelism": "host cores (%d threads)" % threads},
            "cpu_baseline": last, "extrapolation_check": check, "wall_s": ref_wall,
            "e2e": {"value": v, "unit": "forward solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    pkg = importlib.import_module(PKG)
    torch.cuda.set_device(local)
    base = tempfile.mkdtemp(prefix="tdem_bench_r%d_" % rank)
    try:
        wdir = os.path.join(base, "model")
        spec, form, scheme, desc, winfo = write_workload(args.config, wdir, args.air_sigma)
        sopts = dict(precision=args.precision, fp32_update=args.fp32_update, factor_slots=args.factor_slots)
        solver = pkg.Solver(wdir, form, scheme, device=local, **sopts)
        # one run solves every transmitter position of the model (one RHS column each)
        per_run = solver.info()["n_sources"]
        for _ in range(args.warmup):
            solver.run()
        # replicas: every rank solves its own copy of the workload
        units = args.steps
        sampler = ClockSampler(local)
        sampler.start()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gpu_ms = factor_ms = solve_ms = oz_ms = 0.0
        launches = 0
        lat = []
        for _ in range(units):
            solver.run()
            inf = solver.info()
            gpu_ms += inf["run_gpu_ms"]
            factor_ms += inf["factor_gpu_ms"]
            solve_ms += inf["solve_gpu_ms"]
            oz_ms += inf["ozaki_ms"]
            launches += inf["kernel_launches"]
            lat.append(inf["run_gpu_ms"])
        torch.cuda.synchronize()
        barrier(world)
        wall = time.perf_counter() - t0
        clocks = sampler.stop()
        t_job = max_over_ranks(world, gpu_ms * 1e-3)
        value = world * units * per_run / t_job
        inf = solver.info()
        fp64_results = solver.results() if (args.precision == 64 and args.config == "c2" and not args.no_mixed) \
            else None
        solver.close()

        # e2e through the drop-in C-ABI path: files on the host -> device -> results on the host
        e2e_steps = max(1, min(args.steps, 2))
        barrier(world)
        te = time.perf_counter()
        h2d = d2h = 0
        create_s = plan_s = 0.0
        for _ in range(e2e_steps):
            tc = time.perf_counter()
            with pkg.Solver(wdir, form, scheme, device=local, **sopts) as s:
                create_s += time.perf_counter() - tc
                s.run()
                s.results()
                ii = s.info()
                h2d += ii["h2d_bytes"]
                d2h += ii["d2h_bytes"]
                plan_s += ii["t_setup_s"]
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(world, time.perf_counter() - te)
        e2e = {"value": world * e2e_steps * per_run / t_e2e, "unit": "forward solves/s",
               "h2d_bytes_per_step": h2d // e2e_steps, "d2h_bytes_per_step": d2h // e2e_steps,
               "path": "tdem_solver_create (reads the input files, analysis, H2D) + run + results (D2H)",
               "create_s_per_step": create_s / e2e_steps,
               "setup_s_per_step": plan_s / e2e_steps}

        if rank == 0:
            peaks = measured_peaks()
            fp64 = fp64_peak_tflops(local)
            n_fact = inf["factorizations"]
            fac_ms_avg = factor_ms / max(units * n_fact, 1)
            achieved = inf["factor_flops"] / (fac_ms_avg * 1e-3) / 1e12
            # per-step HBM roofline of the solve phase: the factor is streamed twice per step
            steps_per_run = inf["steps"]
            solve_ms_step = solve_ms / max(units * steps_per_run, 1)
            solve_bytes = 2.0 * 8.0 * inf["nnz_factor"] + 20.0 * inf["nnz_matrix"]
            hbm_measured = peaks.get("hbm_gbs")
            hbm = hbm_measured or 6650.0  # the pool's earlier copy measurement when the file is absent
            roof = {"bound": "tensor", "kernel": "multifrontal FP64 factorization (dense front updates)",
                    "achieved": achieved, "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64,
                    "peak_source": "measured on this GPU in bench.py: cuBLAS DGEMM 8192^3 (FP64 has no "
                                   "entry in MEASURED_PEAKS.json)",
                    "flops_per_launch": inf["factor_flops"], "avg_launch_ms": fac_ms_avg,
                    "traffic": None}
            roof_solve = {"bound": "hbm", "kernel": "per-step RHS + triangular solves",
                          "achieved": solve_bytes / (solve_ms_step * 1e-3) / 1e9,
                          "peak": hbm, "unit": "GB/s",
                          "frac": solve_bytes / (solve_ms_step * 1e-3) / 1e9 / hbm,
                          "bytes_per_step": solve_bytes, "avg_step_ms": solve_ms_step,
                          "peak_source": ("MEASURED_PEAKS.json hbm_gbs (measured)" if hbm_measured
                                          else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)")}
            roof_oz = None
            if inf["ozaki_macs"] > 0 and oz_ms > 0:
                # the integer tensor pipe: 8-bit multiply-adds of the digit products per launch
                # time; peak = twice the measured dense bf16 rate (B200's 8-bit dense rate is
                # twice its bf16 rate)
                bf16 = peaks.get("bf16_tflops")
                ops = 2.0 * inf["ozaki_macs"] * n_fact * units
                ach = ops / (oz_ms * 1e-3) / 1e12
                pk = 2.0 * bf16 if bf16 else 2.0 * 1590.0
                # DRAM bytes per 8-bit op of one captured launch (ncu, 40^3 half-space:
                # profiles/k_oz_update_c1.md), scaled to a factorization's ops: the traffic is
                # the read-modify-write of the trailing tiles, which grows with the tiles as the
                # ops do
                traffic = OZ_CAPTURE_DRAM_BYTES / OZ_CAPTURE_OPS * 2.0 * inf["ozaki_macs"]
                roof_oz = {"bound": "tensor", "kernel": "k_oz_update (tcgen05 kind::i8, FP64 trailing updates by "
                                                        "digit splitting; the dominant kernel)",
                           "achieved": ach, "peak": pk, "unit": "TOP/s (int8)", "frac": ach / pk,
                           "ops_per_launch": 2.0 * inf["ozaki_macs"],
                           "launch": "all k_oz_update launches of one factorization",
                           "avg_launch_ms": oz_ms / max(units * n_fact, 1),
                           "traffic": traffic,
                           "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 40^3 launch "
                                             "(profiles/k_oz_update_c1.md), scaled by 8-bit ops",
                           "peak_source": ("2 x MEASURED_PEAKS.json bf16_tflops (measured bf16 burst; B200's dense "
                                           "8-bit rate is twice its bf16 rate)" if bf16
                                           else "2 x fallback 1590 TF/s bf16")}
            cpu = None
            parity = None
            if not args.no_cpu_baseline:
                d = os.path.join(base, "cpu_sample")
                os.makedirs(d)
                try:
                    cpu = cpu_baseline(args.config, spec, form, scheme, d, n_fact, steps_per_run,
                                       os.cpu_count() or 1)
                except Exception as ex:  # the baseline is reported, never required
                    cpu = {"value": None, "unit": "forward solves/s", "cores": os.cpu_count(),
                           "kind": "reference", "sample": "failed: %s" % ex}
                if cpu.get("value"):
                    # the GPU path on the very inputs the reference sample ran: its outputs
                    # against the reference's own, file by file
                    outs = importlib.import_module(PKG + ".outputs")
                    try:
                        pc = gpu_parity(pkg, outs, d, os.path.join(base, "gpu_on_cpu_sample"), form, scheme,
                                        local, "%s mesh (%d edges), %s%d, time grid cut to its first 3 steps" %
                                        (args.config, winfo["n_edges"], form, scheme))
                        parity = {"max_rel_err": pc["max_rel_err"], "tol": 1e-9,
                                  "pass": pc["max_rel_err"] <= 1e-9, "cases": [pc],
                                  "measure": "max over receivers, time and components of |gpu - ref| / peak "
                                             "of the reference receiver's vector transient"}
                    except Exception as ex:
                        parity = {"max_rel_err": None, "tol": 1e-9, "pass": False, "error": str(ex)}
            lat.sort()
            line = {
                "metric": METRIC,
                "value": value,
                "unit": "forward solves/s",
                "n_gpus": world,
                "steps": args.steps,
                "warmup": args.warmup,
                "ms_per_step": t_job * 1000.0 / units,
                "solves_per_step": per_run,
                "higher_is_better": True,
                "scaling": "weak",
                "vs_baseline": None,
                "dtype": "f64" if args.precision == 64 else "f32 factor + f64 refinement",
                "data": "synthetic",
                "config": {"workload": desc, "n_edges": winfo["n_edges"], "n_interior": inf["n_interior"],
                           "nnz_matrix": inf["nnz_matrix"], "nnz_factor": inf["nnz_factor"],
                           "factorizations_per_solve": n_fact, "steps_per_solve": steps_per_run,
                           "parallelism": "replicas x%d" % world, "precision": ("FP64 factor + FP64 solves" if args.precision == 64 else
                                         "FP32 factor (%s) + FP64 CG to 1e-10 relative residual" % args.fp32_update),
                           "l2": "inputs larger than L2 (factor %.1f GB)" % (8e-9 * inf["nnz_factor"]),
                           "factor_slots": inf["factor_slots"],
                           "overlap": ("factorization k+1 runs beside the time steps of decade k (phase times "
                                       "overlap)") if inf["factor_slots"] > 1 else "none"},
                "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                               "what": "device time per forward solve with requests one at a time (the served "
                                       "stream's latency is --config c4)"},
                "phase_ms_per_solve": {"factor": factor_ms / units, "steps": solve_ms / units},
                "wall_s": wall,
                "gpu_launches": launches,
                "clocks": clocks,
                # the dominant kernel: the integer-pipe trailing update when the factorization
                # uses it, else the factorization as a whole on the FP64 pipes
                "roofline": roof_oz if roof_oz else roof,
                "roofline_factorization": roof,
                "roofline_solve": roof_solve,
                "cpu_baseline": cpu,
                "parity": parity,
                "e2e": e2e,
            }
            if args.config == "c2" and not args.no_batched:
                line["batched"] = batched_leg(args, pkg, base, form, scheme, local, value)
            if fp64_results is not None:
                line["mixed_vs_fp64"] = mixed_leg(args, pkg, wdir, form, scheme, local, value, fp64_results)
            print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(base, ignore_errors=True)


def peak_rel_err(got, ref) -> float:
    """Largest |got - ref| over time and components of a receiver, relative to the
    peak of that receiver's reference transient, over all receivers and tables."""
    import numpy as np
    worst = 0.0
    for a, b in zip(got, ref):
        for i in range(b.shape[2]):
            sc = np.abs(b[:, :, i]).max()
            if sc > 0:
                worst = max(worst, float(np.abs(a[:, :, i] - b[:, :, i]).max() / sc))
    return worst


def mixed_leg(args, pkg, wdir: str, form: str, scheme: int, device: int, fp64_value: float, fp64_results) -> dict:
    """The same workload with precision 32: FP64 factorization held rounded to FP32,
    FP32 triangular solves inside an FP64 conjugate gradient to a 1e-10 relative
    residual per step.  Forward solves/s against the FP64 path of this run, and the
    largest receiver deviation from the FP64 transients."""
    with pkg.Solver(wdir, form, scheme, device=device, precision=32) as s:
        s.run()  # warm-up
        runs = []
        for _ in range(max(1, args.batched_runs)):
            s.run()
            runs.append(s.info()["run_gpu_ms"])
        inf = s.info()
        got = s.results()
    ms = sum(runs) / len(runs)
    v = inf["n_sources"] / (ms * 1e-3)
    return {"workload": "same model and scheme, precision 32 (FP64 factorization held in FP32, FP32 solves, "
                        "FP64 CG to 1e-10 per step)",
            "value": v, "unit": "forward solves/s", "vs_fp64": v / fp64_value, "ms_per_run": ms,
            "max_rel_err_vs_fp64": peak_rel_err(got, fp64_results), "accept": 1e-5,
            "cg_iterations": inf["refine_iters"], "cg_iterations_max_per_step": inf["refine_iters_max"],
            "worst_relative_residual": inf["refine_worst"], "steps": inf["steps"],
            "factor_gpu_ms_per_run": inf["factor_gpu_ms"], "solve_gpu_ms_per_run": inf["solve_gpu_ms"]}


def batched_leg(args, pkg, base: str, form: str, scheme: int, device: int, single_value: float) -> dict:
    """The same model, formulation and scheme with 32 wires (centres on a 4 x 8
    surface grid, 100 m apart) solved as one n x 32 block per time step, FP64: forward
    solves/s of the block run against the single-wire FP64 rate of this run, and one
    time step's device time as the graph-replayed block against 32 single-column
    steps issued in turn on the same factor."""
    mg = importlib.import_module(PKG + ".modelgen")
    d = os.path.join(base, "batched")
    spec = mg.layered_block_model(sources=mg.wire_grid_sources())
    mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    with pkg.Solver(d, form, scheme, device=device) as s:
        s.run()  # warm-up
        runs = []
        for _ in range(max(1, args.batched_runs)):
            s.run()
            runs.append(s.info()["run_gpu_ms"])
        inf = s.info()
        step_block = s.time_step(True, 5)
        step_seq = s.time_step(False, 2)
        tune = s.tune_log()
    ms = sum(runs) / len(runs)
    npls = inf["n_sources"]
    return {"workload": "same model, %s-form, %s, %d wires as one n x %d block per step, FP64" %
                        (form, "BDF2" if scheme == 3 else "backward Euler", npls, npls),
            "value": npls / (ms * 1e-3), "unit": "forward solves/s", "ms_per_run": ms, "runs": len(runs),
            "vs_single_wire_fp64": npls / (ms * 1e-3) / single_value,
            "step_ms": {"block_graph": step_block, "sequential_single_column": step_seq,
                        "sequential_over_block": step_seq / step_block},
            "factor_gpu_ms_per_run": inf["factor_gpu_ms"], "solve_gpu_ms_per_run": inf["solve_gpu_ms"],
            "steps": inf["steps"], "factorizations": inf["factorizations"],
            "autotuner": {"chosen": {"kind": inf["solve_schedule"], "split": inf["solve_split"],
                                     "ms": inf["solve_tuned_ms"]},
                          "kinds": "0 fused level solves, 1 panel solves, 2 persistent fused level solves",
                          "candidates": [{"kind": a, "split": b, "ms": c} for a, b, c in tune]}}


def write_request(job):
    """Inputs of one served request (seed, cells lo, cells hi, directory, transmitter
    index); runs in a worker process.  Transmitter t > 0 moves the model's wires and
    receivers 100 t m along y (the same earth model and mesh: a survey's next
    transmitter position).  Returns (directory, formulation, scheme, edges)."""
    import dataclasses
    seed, lo, hi, d, tx = job
    sys.path.insert(0, HERE)
    mg = importlib.import_module(PKG + ".modelgen")
    spec, form, scheme = mg.random_request_model(seed, lo, hi)
    if tx:
        dy = 100.0 * tx
        mv = lambda p: (p[0], p[1] + dy, p[2])
        spec = dataclasses.replace(spec, sources=[(mv(a), mv(b)) for a, b in spec.sources],
                                   receivers_b=[[mv(p) for p in r] for r in spec.receivers_b],
                                   receivers_e=[[mv(p) for p in r] for r in spec.receivers_e])
    info = mg.write_model(d, spec)
    mg.write_analytic_initial_field(d, spec)
    return d, form, scheme, info["n_edges"]


def run_serving(args, world, rank, local):
    """Config c4: a Poisson stream of random forward-modelling requests through
    the serving loop (tdem_server_*) on one GPU; prints solves/s and p50/p99 latency."""
    import numpy as np
    import torch
    pkg = importlib.import_module(PKG)
    mg = importlib.import_module(PKG + ".modelgen")
    torch.cuda.set_device(local)
    lo, hi = (int(v) for v in args.c4_cells.split(","))
    s0 = 20261203
    base = tempfile.mkdtemp(prefix="tdem_serve_r%d_" % rank)
    try:
        # request inputs written by a spawned process pool (no CUDA state is shared)
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        # --c4-survey K: requests in groups of K transmitter positions over one model,
        # submitted with the group's batch key (the server merges queued ones)
        K = max(1, args.c4_survey)
        jobs = [(s0 + i // K, lo, hi, os.path.join(base, "req%03d" % i), i % K) for i in range(args.c4_requests)]
        t_gen = time.perf_counter()
        with ProcessPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1)),
                                 mp_context=mp.get_context("spawn")) as ex:
            reqs = list(ex.map(write_request, jobs))
        t_gen = time.perf_counter() - t_gen
        # single-stream service rate from the first requests run alone
        t_alone = []
        for d, form, scheme, _ in reqs[:2]:
            t0 = time.perf_counter()
            with pkg.Solver(d, form, scheme, device=local) as sv:
                sv.run()
                sv.results()
            t_alone.append(time.perf_counter() - t0)
        lam = 1.2 / (sum(t_alone) / len(t_alone))
        rng = np.random.Generator(np.random.PCG64(s0))
        if K > 1:
            # a survey's transmitter positions arrive together (one client submits them),
            # the surveys as a Poisson stream at the same request rate
            ng = (len(reqs) + K - 1) // K
            arrivals = np.repeat(np.cumsum(rng.exponential(K / lam, ng)), K)[:len(reqs)]
        else:
            arrivals = np.cumsum(rng.exponential(1.0 / lam, len(reqs)))
        sampler = ClockSampler(local)
        sampler.start()
        bmax = K if args.c4_batch_max < 0 else args.c4_batch_max
        with pkg.Server(device=local, max_active=args.c4_active, batch_max=bmax) as srv:
            t0 = time.perf_counter()
            ids = []
            for i, ((d, form, scheme, _), ta) in enumerate(zip(reqs, arrivals)):
                delay = t0 + ta - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                ids.append(srv.submit(d, form, scheme, batch_key="model%d" % (i // K) if K > 1 else ""))
            infos = [srv.wait(i) for i in ids]
            st = srv.stats()
        clocks = sampler.stop()
        line = {"metric": "served forward solves/s + p50/p99 latency", "value": st["solves_per_s"],
                "unit": "forward solves/s", "n_gpus": 1, "steps": len(reqs), "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "served stream: %d requests, %d^3..%d^3 cells, random A/E x 2/3-point, "
                                       "1-3 layers + 1-3 boxes, 60-200 steps, PCG64(%d + i)" % (len(reqs), lo, hi, s0)
                                       + ("" if K == 1 else ", %d transmitter positions per model arriving "
                                          "together (batch key per model, up to %d requests merged per run)"
                                          % (K, bmax)),
                           "arrival_rate_per_s": lam, "single_stream_service_s": t_alone,
                           "max_active": args.c4_active,
                           "edges_min_max": [min(r[3] for r in reqs), max(r[3] for r in reqs)]},
                "latency_s": {"p50": st["latency_p50_s"], "p99": st["latency_p99_s"]},
                "makespan_s": st["makespan_s"], "completed": st["completed"], "failed": st["failed"],
                "peak_device_gb": st["peak_device_bytes"] / 1e9, "peak_active": st["peak_active"],
                "merged_runs": st["merged_runs"], "merged_requests": st["merged_requests"],
                "queue_wait_s_max": max(i["admit_s"] - i["submit_s"] for i in infos),
                "inputs_written_s": t_gen,
                "clocks": clocks}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(base, ignore_errors=True)


# ---------------------------------------------------------------------------
# post-processing modules (host): SumNonstat3DOnly + SummatorEDMN
# ---------------------------------------------------------------------------
def write_postprocess_workload(path: str, npls=32, nb=21, npts=21, nlines=5, per_line=20, nt=160, seed=7):
    """Result files of a 32-transmitter run (the 32-wire configuration's shape): per
    transmitter nb B receivers, npts E point receivers plus nlines lines of per_line
    points, nt printed layers; values seeded, in CalcNonstat3DLine's text layout."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = np.concatenate([[0.0], np.cumsum(np.repeat(1e-6 * 2.0 ** np.arange(8), nt // 8 + 1)[:nt - 1])])
    hdr = ["    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n" % (nt, nt),
           "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n",
           "       u0=   0.00000e+000\n", " T I M E :\n"]
    hdr += ["".join(" %.13e;" % v for v in t[i:i + 5]) + "\n" for i in range(0, nt, 5)]
    files = {"infite.0": "".join(hdr), "timeintervalforprint": "%.13e %.13e\n" % (t[0], t[-1]),
             "group": "1\n1 0 %d\n" % (npls - 1)}
    ne = npts + nlines * per_line
    pts_b = rng.uniform(-1000, 1000, (npls, nb, 3))
    pts_e = rng.uniform(-1000, 1000, (npls, ne, 3))
    files["xyzVectorB"] = "%d\n" % (npls * nb) + "".join("%.6f %.6f %.6f\n" % tuple(q) for q in pts_b.reshape(-1, 3))
    files["xyzVectorE"] = "%d\n" % (npls * ne) + "".join("%.6f %.6f %.6f\n" % tuple(q) for q in pts_e.reshape(-1, 3))
    files["recvsb"] = ("%d\n" % nb) * npls
    files["recvse"] = ("%d\n" % ne) * npls
    files["xyzmn"] = "%d\n" % (npls * nlines)
    t_ms = t * 1000.0

    def block(pts, legend):
        out = []
        for q in pts:
            out.append("%d %d\n%.16e %.16e %.16e\n1\n1 1 1 1\n1\n%s\n" % (int(q[0]), int(q[1]), q[0], q[1], q[2],
                                                                          legend))
            v = rng.standard_normal((nt, 3)) * 10.0 ** rng.integers(-6, 2)
            out.append("".join("%.16e\t%.16e\t%.16e\t%.16e\n" % (t_ms[k], v[k, 0], v[k, 1], v[k, 2])
                               for k in range(nt)))
        return "".join(out)

    legs = {"ball_anom": "      t (ms)        Bx_anom (mTl)     By_anom (mTl)     Bz_anom (mTl)",
            "edsall_anom": "      t (ms)         Emfx_anom (mV)     Emfy_anom (mV)     Emfz_anom (mV)",
            "eall_anom": "      t (ms)         Ex_anom n (mV)     Ey_anom a (mV)     Ez_anom s (mV)"}
    for p in range(npls):
        files["ball_anom.%d" % (p + 1)] = block(pts_b[p], legs["ball_anom"])
        files["edsall_anom.%d" % (p + 1)] = block(pts_b[p], legs["edsall_anom"])
        files["eall_anom.%d" % (p + 1)] = block(pts_e[p], legs["eall_anom"])
        ab = rng.uniform(-1000, 1000, (nlines, 6))
        files["xyzmn%d_1" % (p + 1)] = "%d\n" % nlines + "".join(" ".join("%.16e" % v for v in r) + "\n" for r in ab)
        files["xyzVectorElin%d_1" % (p + 1)] = "%d\n" % (nlines * per_line) + "".join(
            "%.16e %.16e %.16e\n" % tuple(q) for q in pts_e[p, npts:])
    os.makedirs(path, exist_ok=True)
    for name, text in files.items():
        with open(os.path.join(path, name), "w") as f:
            f.write(text)
    return npls


def time_grid_timing(pkg, ref_bin, root):
    """TimeDirectSolver + CorrectTimeMesh on a 200-time log-spaced grid (1e-7 .. 1 s,
    tcff 2), the package's modules against the reference programs."""
    import numpy as np
    t = np.concatenate([[0.0], np.geomspace(1e-7, 1.0, 200)])
    files = {"tcff": "2\n", "currentfunction": "".join("%.13e\t%.13e\n" % (v, 1.0 if i == 0 else 0.0)
                                                      for i, v in enumerate(t)),
             "deltafunction": "50.0\n%d\n" % len(t) + "".join("%.13e %.13e\n" % (v, np.exp(-v)) for v in t)}
    hdr = ["    ktime=  %d;  ntstop=  %d;   kiter=    1;   ntime=    1;   niter=    1;\n" % (len(t), len(t)),
           "   kprogm=    1;  kpropi=    1;  kpropt=   -1;  kitrel=  250;              ;\n",
           "       u0=   0.00000e+000\n", " T I M E :\n"]
    files["infite.0"] = "".join(hdr + ["".join(" %.13e;" % v for v in t[i:i + 5]) + "\n" for i in range(0, len(t), 5)])

    def one(run):
        d = os.path.join(root, "grid")
        shutil.rmtree(d, ignore_errors=True)
        os.makedirs(d)
        for k, v in files.items():
            with open(os.path.join(d, k), "w") as f:
                f.write(v)
        t0 = time.perf_counter()
        run(d)
        dt = time.perf_counter() - t0
        out = {}
        for k in ("infite.0", "currentfunction", "deltafunction"):
            with open(os.path.join(d, k), "rb") as f:
                out[k] = f.read()
        return dt, out

    def ours(d):
        pkg.time_direct_solver(d)
        pkg.correct_time_mesh(d)

    t_ours = min(one(ours)[0] for _ in range(5))
    res = {"workload": "200-time log grid 1e-7..1 s, tcff 2", "ms": 1000 * t_ours}
    if all(os.path.exists(os.path.join(ref_bin, n)) for n in ("TimeDirectSolver", "CorrectTimeMesh")):
        def ref(d):
            for n in ("TimeDirectSolver", "CorrectTimeMesh"):
                subprocess.run([os.path.join(ref_bin, n)], cwd=d, check=True, capture_output=True)
        t_ref, out_ref = one(ref)
        res["reference_ms"] = 1000 * t_ref
        res["identical_outputs"] = out_ref == one(ours)[1]
    return res


def run_postprocess(args):
    """Times SumNonstat3DOnly + SummatorEDMN (WithDDV = 1, every transmitter) on the
    32-transmitter workload: the package's host modules against the reference's
    programs compiled from source (oracle/_ref), outputs compared byte for byte."""
    pkg = importlib.import_module(PKG)
    ref_bin = os.path.join(HERE, "oracle", "_ref")
    have_ref = all(os.path.exists(os.path.join(ref_bin, n)) for n in ("SumNonstat3DOnly", "SummatorEDMN"))
    root = tempfile.mkdtemp(prefix="tdem_post_")
    try:
        base = os.path.join(root, "in")
        npls = write_postprocess_workload(base)

        def stage_lines(d, prefix):
            for p in range(npls):
                for c in "xyz":
                    shutil.copy(os.path.join(d, "E%sall.%d" % (c, p + 1)), os.path.join(d, prefix + "e%sall1_%d" % (c, p)))

        def one(run_split, run_lines, prefix):
            d = os.path.join(root, "run")
            shutil.rmtree(d, ignore_errors=True)
            shutil.copytree(base, d)
            t0 = time.perf_counter()
            run_split(d)
            t1 = time.perf_counter()
            stage_lines(d, prefix)  # the pipeline's renaming, not timed
            t2 = time.perf_counter()
            for p in range(npls):
                run_lines(d, p)
            t3 = time.perf_counter()
            outs = {}
            for p in range(npls):
                for stem in ("Exall.%d" % (p + 1), "Bzall.%d" % (p + 1), "Edsall.%d" % (p + 1)):
                    with open(os.path.join(d, stem), "rb") as f:
                        outs[stem] = f.read()
                for stem in ("edmnall1_%d" % p, "edmoonall1_%d" % p):
                    with open(os.path.join(d, prefix + stem), "rb") as f:
                        outs[stem] = f.read()
            return (t1 - t0) + (t3 - t2), outs

        def ours():
            return one(pkg.sum_nonstat_3d_only, lambda d, p: pkg.summator_edmn(d, 1, 1, p), "")

        def ref():
            # the reference's SummatorEDMN names its files ".\\<name>" (a backslash-joined path)
            return one(lambda d: subprocess.run([os.path.join(ref_bin, "SumNonstat3DOnly")], cwd=d, check=True,
                                                capture_output=True),
                       lambda d, p: subprocess.run([os.path.join(ref_bin, "SummatorEDMN"), "1", "1", str(p)], cwd=d,
                                                   check=True, capture_output=True), ".\\")

        for _ in range(max(1, args.warmup)):
            ours()
        t_ours = []
        for _ in range(max(1, args.steps)):
            dt, out_ours = ours()
            t_ours.append(dt)
        t_best = min(t_ours)
        line = {"metric": "post-processing (SumNonstat3DOnly + SummatorEDMN) transmitters/s", "unit": "transmitters/s",
                "value": npls / t_best, "ms_per_step": 1000 * t_best, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "32 transmitters x (21 B + 21 E point receivers + 5 lines x 20 points), "
                                       "160 layers", "device": "host (text transforms, no GPU)",
                           "host_threads": os.cpu_count()}}
        if have_ref:
            t_ref, out_ref = ref()
            line["reference"] = {"value": npls / t_ref, "unit": "transmitters/s", "cores": 1,
                                 "kind": "reference programs built from source (oracle/_ref)"}
            line["identical_outputs"] = out_ref == out_ours
        else:
            line["reference"] = {"unavailable": "oracle/_ref programs not built"}
        line["time_grid"] = time_grid_timing(pkg, ref_bin, root)
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(root, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--c4-requests", type=int, default=16, help="served-stream length (config c4)")
    ap.add_argument("--c4-cells", default="30,60", help="mesh cells per side, lo,hi (config c4; 30,100 in full)")
    ap.add_argument("--c4-active", type=int, default=4, help="requests on the device at once (config c4)")
    ap.add_argument("--c4-survey", type=int, default=1,
                    help="transmitter positions per earth model (config c4; > 1 batches their time steps)")
    ap.add_argument("--c4-batch-max", type=int, default=-1,
                    help="requests merged per run (config c4; default: --c4-survey; 0 turns merging off)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 32-wire block leg (config c2)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the precision-32 leg (config c2)")
    ap.add_argument("--batched-runs", type=int, default=1, help="timed runs of the 32-wire block leg")
    ap.add_argument("--ref-samples", type=int, default=2,
                    help="reference arm: samples of the cut workload (at most --steps)")
    ap.add_argument("--no-ref-check", action="store_true",
                    help="reference arm: skip the full 40^3 solve that checks the extrapolation")
    ap.add_argument("--precision", type=int, default=64, choices=[64, 32],
                    help="64: FP64 factor and solves; 32: FP32 solves preconditioning an FP64 CG")
    ap.add_argument("--fp32-update", default="default", choices=["default", "cuda_cores", "tensor_cores"],
                    help="precision 32: default = FP64 factorization held in FP32; cuda_cores / tensor_cores = "
                         "FP32 factorization")
    ap.add_argument("--factor-slots", type=int, default=0, choices=[0, 1, 2],
                    help="numeric factors held: 2 overlaps the next factorization with the steps, 0 = auto")
    ap.add_argument("--air-sigma", type=float, default=None,
                    help="conductivity of the air cells (default 1e-8 S/m as the reference's mesh builder)")
    ap.add_argument("--postprocess", action="store_true",
                    help="time the host modules around the solve (SumNonstat3DOnly, SummatorEDMN, "
                         "TimeDirectSolver, CorrectTimeMesh) instead")
    args = ap.parse_args()
    if args.postprocess:
        run_postprocess(args)
        return
    world, rank, local = dist_init(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank, local)
        elif args.config == "c4":
            run_serving(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
