"""Benchmark of the B200-native bld_mult solver.

Default workload: a single large plain solve, x=1024, y=1024, z=64 (67M-element
S, 512 MiB in FP64), 100 psi_appr iterations per step, FP64 storage.  A step is
one 100-iteration solve; steps continue from the previous step's S, so every
step does the same work.  S is larger than L2, so no L2 flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--dtype f64|f32]

--impl reference times the reference algorithm's CPU path on this machine's
host cores: the reference itself cannot be compiled here (it needs Eigen3 and
GSL), so its OpenMP restatement in oracle/ stands in for it.

With N > 1 (torchrun, one process per GPU) each rank solves its own replica:
the solver does not shard (replicas only); value = all ranks' updates / the
slowest rank's time.
"""

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "bnmf-algs_b200")
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def load_package():
    if "bnmf_algs_b200" in sys.modules:
        return sys.modules["bnmf_algs_b200"]
    spec = importlib.util.spec_from_file_location(
        "bnmf_algs_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bnmf_algs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_value(name, key="traffic_bytes_per_launch"):
    """A per-launch figure of the sweep (`key: value` line) from a committed ncu
    summary under profiles/, with where it came from: these figures are read
    from the capture, not measured by this run."""
    path = os.path.join(ROOT, "profiles", name)
    val, kernel_build = None, None
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                val = float(line.split(":")[1])
            if line.startswith("kernel_source_sha:"):
                kernel_build = line.split(":", 1)[1].strip()
    except OSError:
        pass
    if val is None:
        return None, None
    src = f"profiles/{name} (ncu capture"
    src += f" of kernel sources {kernel_build})" if kernel_build else ")"
    return val, src


def kernel_source_sha():
    """Digest of the files that hold the update sweep's code (the tile function,
    the digamma and bulk-copy helpers, the finalize it includes), to compare
    with a profile's kernel_source_sha line: equal means the capture is of this
    build's kernel."""
    import hashlib
    h = hashlib.sha256()
    for f in ("bldm_sweep_kernels.cuh", "bldm_device.cuh", "bldm_finalize.cuh"):
        with open(os.path.join(PKG_DIR, "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:12]


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


# Nominal FP64 vector peak of a B200: 148 SMs x 64 DFMA lanes per cycle x 2 flops x 1965 MHz.
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        rows = []
        for l in self.lines:
            p = [s.strip() for s in l.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def cpu_baseline_oracle(prob, target_s=10.0, threads=0, small=None):
    """The oracle (reference restatement, OpenMP) on a bounded sample: whole
    iterations of the same workload, as many as fit in about target_s; with
    `small`, also the CPU-runnable 64x48x8 workload's whole 200-iteration solve."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = O.set_threads(threads)
    X, z = prob["X"], prob["z"]
    S0 = O.init_S(X, z, 0)
    t0 = time.perf_counter()
    O.bld_mult(X, z, prob["alpha"], prob["beta"], 1, O.PSI_APPR, 1e-50, S0=S0)
    one = time.perf_counter() - t0
    n = max(1, min(int(target_s / max(one, 1e-6)), 50))
    t0 = time.perf_counter()
    O.bld_mult(X, z, prob["alpha"], prob["beta"], n, O.PSI_APPR, 1e-50, S0=S0)
    dt = time.perf_counter() - t0
    upd = X.size * z * n
    out = {"value": upd / dt, "unit": "S-updates/s", "cores": cores, "kind": "port",
           "cpu_model": cpu_model(), "nproc": os.cpu_count(),
           "sample": f"{n} iterations of the full {X.shape[0]}x{X.shape[1]}x{z} workload "
                     f"({dt:.1f} s, FP64, psi_appr, OpenMP {cores} threads)"}
    if small is not None:
        Xs, zs, it = small["X"], small["z"], small["iters"]
        S0s = O.init_S(Xs, zs, 0)
        reps, t_all = 0, 0.0
        while t_all < 1.0 and reps < 200:
            t0 = time.perf_counter()
            O.bld_mult(Xs, zs, small["alpha"], small["beta"], it, O.PSI_APPR, 1e-50, S0=S0s)
            t_all += time.perf_counter() - t0
            reps += 1
        out["plain_64x48x8"] = {"ms_per_solve": t_all * 1e3 / reps,
                                "value": Xs.size * zs * it * reps / t_all,
                                "unit": "S-updates/s", "iters": it, "solves_timed": reps}
    return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    load_package()
    import bnmf_algs_b200.workloads as W
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    prob = W.plain_large(1)
    X, z = prob["X"], prob["z"]
    cores = O.set_threads(0)
    S = O.init_S(X, z, 0)
    # iterations of the full workload per step (a bounded sample: the call's
    # fixed cost -- the sums of S0 and the copies of S in and out -- is spread
    # over a few iterations as in a solve)
    per_step = 4
    for _ in range(args.warmup):
        S = O.bld_mult(X, z, prob["alpha"], prob["beta"], per_step, O.PSI_APPR, 1e-50, S0=S)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        S = O.bld_mult(X, z, prob["alpha"], prob["beta"], per_step, O.PSI_APPR, 1e-50, S0=S)
    dt = time.perf_counter() - t0
    value = X.size * z * per_step * args.steps / dt
    line = {"impl": "reference", "metric": "S_elem_updates_per_s", "value": value,
            "unit": "S-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plain_1024x1024x64", "x": 1024, "y": 1024, "z": 64,
                       "iters_per_step": per_step, "psi": "psi_appr", "storage": "f64",
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "S-updates/s", "cores": cores,
                             "kind": "port", "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                             "sample": f"{per_step} iteration(s) of the full 1024x1024x64 "
                                       "workload per step; the reference is not buildable here "
                                       "(Eigen3/GSL absent), its OpenMP restatement runs"},
            "e2e": {"value": value, "unit": "S-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_sharded(args):
    """The headline solve (1024x1024x64 FP64, 100 iterations) row-sharded over
    the ranks: strong scaling, one NCCL all-reduce of y*z + z values per
    iteration.  Works with one rank; it has not run on more than one GPU here."""
    import datetime
    import torch
    import torch.distributed as dist
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29517")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), rank=rank,
                            world_size=world, device_id=torch.device("cuda", local))
    pkg = load_package()
    import bnmf_algs_b200.multi as M
    import bnmf_algs_b200.workloads as W
    prob = W.plain_large(1)
    X, z, iters = prob["X"], prob["z"], prob["iters"]
    x, y = X.shape
    i0, i1 = M.row_shards(x, world)[rank]
    dev = torch.device("cuda", local)
    plan = pkg.Plan(i1 - i0, y, z, pkg.F64)
    dX = torch.as_tensor(X[i0:i1]).to(dev)
    da = torch.as_tensor(prob["alpha"][i0:i1]).to(dev)
    db = torch.as_tensor(prob["beta"]).to(dev)
    dS = torch.empty((i1 - i0, y, z), dtype=torch.float64, device=dev)
    red = torch.empty(plan.shard_red_size(), dtype=torch.float64, device=dev)
    sh = M.Shard(plan, dX, da, db, dS, red)
    reduce = M.collective_allreduce(dist)
    stream = torch.cuda.current_stream()

    def step():
        plan.init_S(dX, dS, seed=rank)
        M.sharded_solve([sh], iters, pkg.PSI_APPR, 1e-50, reduce)

    for _ in range(args.warmup):
        step()
    plan.check(stream)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    plan.check(stream)
    ms = torch.tensor([e0.elapsed_time(e1) / args.steps], dtype=torch.float64, device=dev)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms.item())
    if rank == 0:
        print(json.dumps({"metric": "S_elem_updates_per_s", "value": x * y * z * iters / (ms_max / 1e3),
                          "unit": "S-updates/s", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic",
                          "config": {"workload": "plain_1024x1024x64", "iters_per_step": iters,
                                     "parallelism": f"row-sharded over {world} ranks",
                                     "exchange_doubles_per_iteration": y * z + z}}))
    plan.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def plain_measure(pkg, torch, prob, f64, steps, warmup, dev, stream, dist, world,
                  with_skip=True, with_e2e_S0=True):
    """The plain solve of `prob` on one device: device-resident rate, roofline of
    the update sweep, the skip_zero_rows variant and the drop-in host-buffer e2e.
    Returns (result dict, plan, dX, dS) with the plan still open."""
    X, z, iters = prob["X"], prob["z"], prob["iters"]
    x, y = X.shape
    dt_t = torch.float64 if f64 else torch.float32
    dtype = pkg.F64 if f64 else pkg.F32
    es = 8 if f64 else 4
    dtn = "f64" if f64 else "f32"
    dX = torch.as_tensor(X).to(dev, dt_t)
    dalpha = torch.as_tensor(prob["alpha"]).to(dev)
    dbeta = torch.as_tensor(prob["beta"]).to(dev)
    dS = torch.empty((x, y, z), dtype=dt_t, device=dev)
    plan = pkg.Plan(x, y, z, dtype)
    plan.init_S(dX, dS, seed=0)
    mode = pkg.PSI_APPR

    def step():
        plan.run(dX, dalpha, dbeta, dS, iters, mode, 1e-50, stream)

    for _ in range(warmup):
        step()
    plan.check(stream)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = plan.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index or 0) as clk:
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = plan.launch_count() - launches0
    plan.check(stream)
    ms = e0.elapsed_time(e1) / steps
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if dist:
        dist.barrier()
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    upd_step = x * y * z * iters
    value = upd_step * world / (ms_max / 1e3)
    conservation = plan.conservation(dX, dS, stream)

    # Roofline of the fused update sweep: CUDA events around each launch.
    kern_ms, iter_ms = plan.profile(dX, dalpha, dbeta, dS, 20, mode, 1e-50, stream)
    alg_bytes = 2 * x * y * z * es + x * y * es
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    peak, peak_src = hbm_peak()
    prof = f"sweep_update_plain_{x}x{y}x{z}_{dtn}.md"
    traffic, traffic_src = profile_value(prof)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src,
                "traffic": traffic, "traffic_source": traffic_src,
                "kernel_source_sha": kernel_source_sha(),
                "kernel": "sweep_kernel<UPDATE>", "kernel_ms": kern_ms,
                "algorithmic_bytes_per_launch": alg_bytes,
                "iteration_ms": iter_ms,
                "iteration_frac": alg_bytes / (iter_ms / 1e3) / 1e9 / peak}
    # The secondary ceiling: FP64 arithmetic of the same launch (flops counted by
    # ncu on the committed capture of this workload, 2*DFMA + DADD + DMUL).
    fp64 = None
    flop, flop_src = profile_value(prof, "fp64_flop_per_launch")
    if flop and f64:
        fp64 = {"flop_per_launch": flop, "flop_source": flop_src,
                "achieved_tflops": flop / (kern_ms / 1e3) / 1e12,
                "peak_tflops": FP64_NOMINAL_TFLOPS, "peak_source": "nominal",
                "frac": flop / (kern_ms / 1e3) / 1e12 / FP64_NOMINAL_TFLOPS}

    zero_row_skip = None
    if with_skip:
        # The same solve with skip_zero_rows: bitwise the same S; after the first
        # update, rows whose band segment of X is all zero are neither read nor
        # written and zeros are not stored again.  Its rate counts all x*y*z
        # updates of an iteration; the roofline above stays the streaming kernel's.
        plan_skip = pkg.Plan(x, y, z, dtype, skip_zero_rows=True)
        dS2 = torch.empty_like(dS)
        plan_skip.init_S(dX, dS2, seed=0)
        for _ in range(2):
            plan_skip.run(dX, dalpha, dbeta, dS2, iters, mode, 1e-50, stream)
        plan_skip.check(stream)
        n_skip = max(1, steps // 3)
        e0.record(stream)
        for _ in range(n_skip):
            plan_skip.run(dX, dalpha, dbeta, dS2, iters, mode, 1e-50, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        plan_skip.check(stream)
        skip_ms = e0.elapsed_time(e1) / n_skip
        skip_kern, _ = plan_skip.profile(dX, dalpha, dbeta, dS2, 20, mode, 1e-50, stream)
        zero_row_skip = {"value": upd_step / (skip_ms / 1e3), "unit": "S-updates/s",
                         "ms_per_step": skip_ms, "speedup": ms_max / skip_ms,
                         "update_kernel_ms": skip_kern, "steps": n_skip,
                         "fibers_with_X_nonzero": float(np.mean(X != 0)),
                         "note": "bldm_tuning.skip_zero_rows; bitwise the same S"}
        plan_skip.close()
        del dS2

    # End to end through the public host-buffer C ABI, as the drop-in call
    # bld_mult_cuda(X, z, params, max_iter, true) makes it: pinned host X in,
    # the seeded initial S drawn on the device, S out (H2D of X, alpha, beta and
    # D2H of S inside every step).  A second measurement passes a host S0 as
    # well (its H2D inside the step).
    hX = torch.as_tensor(X.astype(np.float64 if f64 else np.float32)).pin_memory()
    hS0 = dS.cpu().pin_memory()
    hS = torch.empty_like(hS0).pin_memory()
    params = pkg.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    cp = params.c_struct()
    L = pkg.lib()
    solve = L.bldm_solve_f64 if f64 else L.bldm_solve_f32
    ptr_t = ctypes.POINTER(ctypes.c_double if f64 else ctypes.c_float)
    st = pkg.bldm_stats()

    def e2e_step(with_S0):
        s0 = ctypes.cast(hS0.data_ptr(), ptr_t) if with_S0 else None
        rc = solve(ctypes.cast(hX.data_ptr(), ptr_t), x, y, z, ctypes.byref(cp), iters, mode,
                   1e-50, s0, 0, ctypes.cast(hS.data_ptr(), ptr_t), ctypes.byref(st))
        if rc != 0:
            raise RuntimeError(f"bldm_solve failed with status {rc}")

    def e2e_time(with_S0, n):
        for _ in range(max(1, warmup)):
            e2e_step(with_S0)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(n):
            e2e_step(with_S0)
        sec = (time.perf_counter() - t0) / n
        t = torch.tensor([sec], device=dev, dtype=torch.float64)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    e2e_s = e2e_time(False, steps)
    h2d = x * y * es + (x + z) * 8
    d2h = x * y * z * es
    e2e = {"value": upd_step * world / e2e_s, "unit": "S-updates/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3,
           "conservation_residual_last_call": st.conservation_residual,
           "call": f"bldm_solve_{dtn} (host X in, device-seeded S0, host S out)"}
    e2e_from_S0 = None
    if with_e2e_S0:
        e2e_s0_s = e2e_time(True, max(1, steps // 3))
        e2e_from_S0 = {"value": upd_step * world / e2e_s0_s, "unit": "S-updates/s",
                       "h2d_bytes_per_step": h2d + x * y * z * es, "d2h_bytes_per_step": d2h,
                       "ms_per_step": e2e_s0_s * 1e3}
    res = {"value": value, "ms_per_step": ms_max, "launches": launches,
           "upd_step": upd_step, "alg_bytes": alg_bytes,
           "hbm_gbs_iteration": alg_bytes / (ms_max / 1e3 / iters) / 1e9,
           "roofline": roofline, "fp64_arith": fp64, "zero_row_skip": zero_row_skip,
           "e2e": e2e, "e2e_from_host_S0": e2e_from_S0, "clocks": clk.summary(),
           "conservation_residual": conservation}
    return res, plan, dX, dS


def parity_block(pkg, torch, prob, dS64, plan64, stream):
    """Parity of this build on the benchmark's own inputs, measured in the run:
    (1) the CPU-runnable 64x48x8 workload, 200 iterations through the drop-in
    call against the oracle (max-norm relative error of S); (2) the timed
    solve's conservation residual (filled in by the caller); (3) FP32 storage
    against FP64 on the headline workload from the same initial S, 100
    iterations: log-marginal gap and S error."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import bnmf_algs_b200.workloads as W
    small = W.plain_small(0)
    Xs, zs = small["X"], small["z"]
    S0s = O.init_S(Xs, zs, 0)
    ref = O.bld_mult(Xs, zs, small["alpha"], small["beta"], small["iters"], O.PSI_APPR, 1e-50,
                     S0=S0s)
    ps = pkg.Params(small["a"], small["b"], small["alpha"], small["beta"])
    got = pkg.bld_mult_cuda(Xs, zs, ps, small["iters"], use_psi_appr=True, S0=S0s)
    err_small = float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300))
    # FP32 vs FP64 on the headline workload from one initial S
    X, z, iters = prob["X"], prob["z"], prob["iters"]
    x, y = X.shape
    dX64 = torch.as_tensor(X).cuda()
    da = torch.as_tensor(prob["alpha"]).cuda()
    db = torch.as_tensor(prob["beta"]).cuda()
    S64 = torch.empty((x, y, z), dtype=torch.float64, device="cuda")
    plan64.init_S(dX64, S64, seed=7, stream=stream)
    S32 = S64.float()
    p32 = pkg.Plan(x, y, z, pkg.F32)
    plan64.run(dX64, da, db, S64, iters, pkg.PSI_APPR, 1e-50, stream)
    p32.run(dX64.float(), da, db, S32, iters, pkg.PSI_APPR, 1e-50, stream)
    plan64.check(stream)
    p32.check(stream)
    params = pkg.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    lm64 = pkg.log_marginal_S(S64, params, stream=stream)
    lm32 = pkg.log_marginal_S(S32, params, dtype=pkg.F32, stream=stream)
    mask = S64 > 1e-6 * dX64.unsqueeze(2)
    rel = ((S32.double() - S64).abs() / S64.abs().clamp_min(1e-300))[mask]
    p32.close()
    out = {"plain_64x48x8_fp64_max_rel_err_S_vs_oracle": err_small,
           "plain_64x48x8_iters": small["iters"], "plain_64x48x8_tolerance": 1e-9,
           "fp32_vs_fp64_log_marginal_rel_gap": abs(lm32 - lm64) / abs(lm64),
           "fp32_vs_fp64_log_marginal_tolerance": 1e-5,
           "fp32_vs_fp64_max_rel_err_S": float(rel.max()) if rel.numel() else 0.0,
           "fp32_vs_fp64_median_rel_err_S": float(rel.median()) if rel.numel() else 0.0,
           "fp32_vs_fp64_workload": f"{x}x{y}x{z}, {iters} iterations from one initial S "
                                    "(S error over S > 1e-6 X)"}
    del S64, S32, dX64
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    pkg = load_package()
    import bnmf_algs_b200.workloads as W
    prob = W.plain_large(1)
    X, z, iters = prob["X"], prob["z"], prob["iters"]
    x, y = X.shape
    f64 = args.dtype == "f64"
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    head, plan, dX, dS = plain_measure(pkg, torch, prob, f64, args.steps, args.warmup, dev,
                                       stream, dist, world)
    # The extra blocks are one-GPU measurements of the other benchmark workloads;
    # with several ranks only the headline replicas run.
    extra = world == 1 and not args.headline_only
    parity = fp32 = batch = serving = None
    if extra:
        parity = parity_block(pkg, torch, prob, dS, plan, stream)
        parity["headline_conservation_residual"] = head["conservation_residual"]
        parity["headline_e2e_conservation_residual"] = head["e2e"][
            "conservation_residual_last_call"]
    plan.close()
    del dX, dS
    torch.cuda.empty_cache()
    if extra and f64:
        r32, p32, dX32, dS32 = plain_measure(pkg, torch, prob, False, args.steps, args.warmup,
                                             dev, stream, None, 1, with_skip=False,
                                             with_e2e_S0=False)
        p32.close()
        del dX32, dS32
        torch.cuda.empty_cache()
        fp32 = {"value": r32["value"], "unit": "S-updates/s", "ms_per_step": r32["ms_per_step"],
                "roofline": r32["roofline"], "e2e": r32["e2e"],
                "conservation_residual": r32["conservation_residual"],
                "vs_fp64_plain": r32["value"] / head["value"], "gpu_launches": r32["launches"],
                "clocks": r32["clocks"]}
    if extra:
        batch = batch_measure(pkg, torch, args, steps=max(3, args.steps // 3), loop_reps=1)
        batch["vs_plain_fp64_S_updates_per_s"] = batch["S_updates_per_s"] / head["value"]
        if fp32:
            batch["vs_plain_fp32_S_updates_per_s"] = batch["S_updates_per_s"] / fp32["value"]
        torch.cuda.empty_cache()
        serving = serve_measure(pkg, torch, args.serve_sample_rate, args.serve_sample_seconds,
                                fp64_sample=4, dtype_name="f32")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_oracle(prob, target_s=args.cpu_seconds, small=W.plain_small(0))

    if rank == 0:
        line = {"metric": "S_elem_updates_per_s", "value": head["value"], "unit": "S-updates/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
                "config": {"workload": "plain_1024x1024x64", "x": x, "y": y, "z": z,
                           "iters_per_step": iters, "psi": "psi_appr", "storage": args.dtype,
                           "X_zero_fraction": float(np.mean(X == 0)),
                           "l2": "inputs larger than L2 (S is 512 MiB in f64)",
                           "parallelism": "replicas" if world > 1 else "single GPU"},
                "hbm_gbs_iteration": head["hbm_gbs_iteration"],
                "roofline": head["roofline"], "fp64_arith": head["fp64_arith"],
                "zero_row_skip": head["zero_row_skip"],
                "cpu_baseline": cpu, "e2e": head["e2e"],
                "e2e_from_host_S0": head["e2e_from_host_S0"],
                "gpu_launches": head["launches"], "clocks": head["clocks"],
                "parity": parity, "fp32_plain": fp32, "batch": batch, "serving": serving}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile(args):
    """One untimed solve of --profile-iters iterations (for ncu captures)."""
    import torch
    pkg = load_package()
    import bnmf_algs_b200.workloads as W
    x, y, z = (int(v) for v in args.shape.split("x"))
    rng = np.random.default_rng(1)
    if args.x_kind == "model":
        X = W.allocation_model_X(x, y, z, 5.0, 0.01 if x * y >= 1 << 20 else 0.1, rng)
    else:
        X = make_X(args.x_kind, x, y, z, rng)
    f64 = args.dtype == "f64"
    dt_t = torch.float64 if f64 else torch.float32
    dX = torch.as_tensor(X).to("cuda", dt_t)
    dalpha = torch.ones(x, dtype=torch.float64, device="cuda")
    dbeta = torch.ones(z, dtype=torch.float64, device="cuda")
    dS = torch.empty((x, y, z), dtype=dt_t, device="cuda")
    plan = pkg.Plan(x, y, z, pkg.F64 if f64 else pkg.F32, skip_zero_rows=args.skip_zero_rows)
    plan.init_S(dX, dS, seed=0)
    plan.run(dX, dalpha, dbeta, dS, args.profile_iters, pkg.PSI_APPR, 1e-50)
    plan.check()
    plan.close()
    print(f"profile run ok: {x}x{y}x{z} {args.dtype}, {args.profile_iters} iterations"
          f"{' (skip_zero_rows)' if args.skip_zero_rows else ''}")
    return 0


def run_batch_probe(args):
    """The uneven batch of --batch run for --profile-iters iterations twice,
    without the CUDA graph (for ncu captures of the class kernels)."""
    import torch
    pkg = load_package()
    import bnmf_algs_b200.workloads as W
    shapes = W.batch_shapes(args.batch_n, 3)
    f64 = args.dtype == "f64"
    b = pkg.Batch(shapes, dtype=pkg.F64 if f64 else pkg.F32, rows_per_tile=args.rows_per_tile)
    for k, (x, y, z) in enumerate(shapes):
        pr = W.batch_instance((x, y, z), 1000 + 3 * 100003 + k)
        b.set(k, pr["X"], pr["alpha"], pr["beta"], None, seed=k)
    stream = torch.cuda.Stream()
    for _ in range(2):
        b.run(args.profile_iters, pkg.PSI_APPR, 1e-50, False, stream)
    b.check(stream)
    print(f"batch probe ok: {len(shapes)} instances, {b.info()['classes']} classes, "
          f"{args.profile_iters} iterations twice")
    b.close()
    return 0


def batch_measure(pkg, torch, args, steps, loop_reps=2, autotune=True):
    """Batched uneven solves (512 instances, FP32 unless --dtype f64, 150
    iterations, one graph-captured run per step) against a loop of the plain
    per-instance solver over the same instances."""
    import bnmf_algs_b200.workloads as W
    shapes = W.batch_shapes(args.batch_n, 3)
    iters = 150
    f64 = args.batch_dtype == "f64"
    dtype = pkg.F64 if f64 else pkg.F32
    es = 8 if f64 else 4
    upd = sum(x * y * z for x, y, z in shapes) * iters
    t0 = time.perf_counter()
    b = pkg.Batch(shapes, dtype=dtype, rows_per_tile=args.rows_per_tile)
    probs = []
    for k, (x, y, z) in enumerate(shapes):
        pr = W.batch_instance((x, y, z), 1000 + 3 * 100003 + k)
        b.set(k, pr["X"], pr["alpha"], pr["beta"], None, seed=k)
        probs.append(pr)
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    tune = None
    if autotune:
        t1 = time.perf_counter()
        d_ms, t_ms = b.autotune(probe_iters=6, psi_mode=pkg.PSI_APPR, eps=1e-50, stream=stream)
        tune = {"seconds": time.perf_counter() - t1, "probe_iters": 6,
                "default_probe_ms": d_ms, "tuned_probe_ms": t_ms,
                "classes": [{k: c[k] for k in ("vec", "lanes_per_fiber", "chunks", "multirow",
                                               "rows_per_tile", "stages", "tiles", "instances")}
                            for c in b.classes()]}
    for _ in range(args.warmup):
        b.run(iters, pkg.PSI_APPR, 1e-50, True, stream)
    b.check(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.info()["launches"]
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(steps):
            b.run(iters, pkg.PSI_APPR, 1e-50, True, stream)
        e1.record(stream)
        torch.cuda.synchronize()
    b.check(stream)
    ms = e0.elapsed_time(e1) / steps
    launches = b.info()["launches"] - l0
    # the same runs in the persistent form (one launch per class for a whole
    # run), for comparison; S continues
    persist = None
    b.set_launch_mode(True)
    if b.persistent():
        b.run(iters, pkg.PSI_APPR, 1e-50, True, stream)
        n_p = max(2, steps // 3)
        lp0 = b.info()["launches"]
        e0.record(stream)
        for _ in range(n_p):
            b.run(iters, pkg.PSI_APPR, 1e-50, True, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        b.check(stream)
        p_ms = e0.elapsed_time(e1) / n_p
        persist = {"ms_per_step": p_ms, "solves_per_s": len(shapes) / (p_ms / 1e3),
                   "steps": n_p, "gpu_launches_per_run": (b.info()["launches"] - lp0) / n_p,
                   "vs_per_iteration_form": ms / p_ms}
    b.set_launch_mode(False)
    cons = b.conservation(stream)
    # loop of the plain per-instance solver (one plan per distinct shape)
    plans = {}
    dev = []
    tt = torch.float64 if f64 else torch.float32
    for (x, y, z), pr in zip(shapes, probs):
        if (x, y, z) not in plans:
            plans[(x, y, z)] = pkg.Plan(x, y, z, dtype)
        dX = torch.as_tensor(pr["X"]).to("cuda", tt)
        dS = torch.empty((x, y, z), dtype=tt, device="cuda")
        plans[(x, y, z)].init_S(dX, dS, seed=0)
        dev.append((plans[(x, y, z)], dX, torch.as_tensor(pr["alpha"]).cuda(),
                    torch.as_tensor(pr["beta"]).cuda(), dS))

    def loop():
        for plan, dX, da, db, dS in dev:
            plan.run(dX, da, db, dS, iters, pkg.PSI_APPR, 1e-50, stream)
    loop()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(loop_reps):
        loop()
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1) / loop_reps
    for p in plans.values():
        p.close()
    del dev
    alg_bytes = sum(2 * x * y * z * es + x * y * es for x, y, z in shapes) * iters
    peak, _ = hbm_peak()
    out = {"metric": "batched_solves_per_s", "value": len(shapes) / (ms / 1e3),
           "unit": "solves/s", "ms_per_step": ms, "steps": steps, "dtype": args.batch_dtype,
           "config": {"workload": f"batch_{len(shapes)}_uneven", "iters": iters,
                      "x_y": "log-uniform [32,512]", "z": "{4,8,16,32,64}",
                      "total_S_elements": sum(x * y * z for x, y, z in shapes),
                      "rows_per_tile": "autotuned per class" if tune else
                      (args.rows_per_tile or 64), "graph": True},
           "S_updates_per_s": upd / (ms / 1e3),
           "hbm_gbs_algorithmic": alg_bytes / (ms / 1e3) / 1e9,
           "frac_of_hbm_peak": alg_bytes / (ms / 1e3) / 1e9 / peak,
           "plain_loop": {"ms": loop_ms, "solves_per_s": len(shapes) / (loop_ms / 1e3),
                          "S_updates_per_s": upd / (loop_ms / 1e3)},
           "speedup_vs_plain_loop": loop_ms / ms,
           "conservation_residual_max": float(np.max(cons)),
           "conservation_residual_median": float(np.median(cons)),
           "launch_form": "per iteration: a sweep launch per class, one finalize launch",
           "persistent_form": persist,
           "classes": b.info()["classes"], "gpu_launches": launches,
           "gpu_launches_per_solve_iteration": launches / (steps * iters),
           "setup_s": setup_s, "autotune": tune, "clocks": clk.summary()}
    b.close()
    return out


def run_batch(args):
    import torch
    pkg = load_package()
    out = batch_measure(pkg, torch, args, args.steps)
    line = {"metric": out.pop("metric"), "value": out.pop("value"), "unit": out.pop("unit"),
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic"}
    line.update(out)
    print(json.dumps(line))
    return 0


def serve_measure(pkg, torch, rate, duration, fp64_sample=16, dtype_name="f32"):
    """Continuous-batching server under Poisson arrivals at `rate` req/s for
    `duration` s of traffic: latency percentiles, throughput, and per-request
    log-marginal error against an FP64 solve of the same request."""
    import queue as _queue
    import bnmf_algs_b200.workloads as W
    rng = np.random.default_rng(11)
    # request templates: the batch size distribution plus the 4096x4096x32 tail
    reg = [W.batch_instance(s, 5000 + k) for k, s in enumerate(W.batch_shapes(96, 21))]
    tail = [W.batch_instance((4096, 4096, 32), 9000 + k) for k in range(2)]
    n_max = int(rate * duration * 1.5) + 16
    times, _ = W.serving_requests(n_max, rate, seed=4)
    times = times[times < duration]
    picks = []
    for _ in range(len(times)):
        picks.append(tail[rng.integers(len(tail))] if rng.random() < 0.02
                     else reg[rng.integers(len(reg))])
    dtype = pkg.F64 if dtype_name == "f64" else pkg.F32
    srv = pkg.Server(dtype=dtype, tol=1e-6, max_iter=500, iters_per_round=10, max_active=256)
    pending = _queue.Queue()
    results = []
    n_keep_S = fp64_sample

    def consume():
        # fetches in submission order as results complete; S only for the
        # requests the FP64 comparison uses (the tail's S is 2 GiB)
        kept = 0
        while True:
            item = pending.get()
            if item is None:
                return
            rid, k, pr = item
            srv.wait(rid, 900.0)
            want = kept < n_keep_S and pr["X"].shape != (4096, 4096)
            S, st = srv.fetch(rid, want_S=want)
            kept += 1 if want else 0
            results.append((k, pr, S, st))

    fetcher = threading.Thread(target=consume)
    fetcher.start()
    t0 = time.perf_counter()
    with ClockSampler(0) as clk:
        for k, (t, pr) in enumerate(zip(times, picks)):
            now = time.perf_counter() - t0
            if t > now:
                time.sleep(t - now)
            rid = srv.submit(pr["X"], pr["z"], pkg.Params(pr["a"], pr["b"], pr["alpha"],
                                                          pr["beta"]), seed=k)
            pending.put((rid, k, pr))
        pending.put(None)
        fetcher.join()
    wall = time.perf_counter() - t0
    sstats = srv.stats()
    srv.close()
    ok = [r for r in results if r[3]["status"] == 0]
    lat = np.array([r[3]["latency_ms"] for r in ok])
    tail_lat = np.array([r[3]["latency_ms"] for r in ok if r[1]["X"].shape == (4096, 4096)])
    reg_lat = np.array([r[3]["latency_ms"] for r in ok if r[1]["X"].shape != (4096, 4096)])
    iters = np.array([r[3]["iterations"] for r in ok])
    cons = np.array([r[3]["conservation_residual"] for r in ok])
    upd = sum(r[1]["X"].size * r[1]["z"] * r[3]["iterations"] for r in ok)
    # per-request log-marginal error vs an FP64 solve of the same request
    errs = []
    sample = [r for r in ok if r[2] is not None][:fp64_sample]
    for k, pr, S, st in sample:
        x, y = pr["X"].shape
        z = pr["z"]
        plan = pkg.Plan(x, y, z, pkg.F64)
        dX = torch.as_tensor(pr["X"]).cuda()
        dS = torch.empty((x, y, z), dtype=torch.float64, device="cuda")
        plan.init_S(dX, dS, seed=k)
        plan.run(dX, torch.as_tensor(pr["alpha"]).cuda(), torch.as_tensor(pr["beta"]).cuda(),
                 dS, int(st["iterations"]), pkg.PSI_APPR)
        plan.check()
        lm64 = pkg.log_marginal_S(dS, pkg.Params(pr["a"], pr["b"], pr["alpha"], pr["beta"]))
        errs.append(abs(st["log_marginal"] - lm64) / abs(lm64))
        plan.close()
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    return {"metric": "serving_latency_p50_p99", "value": pct(lat, 50), "unit": "ms (p50)",
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "higher_is_better": False,
            "dtype": dtype_name,
            "config": {"workload": "serving_poisson", "offered_rate_per_s": rate,
                       "duration_s": duration, "tol": 1e-6, "max_iter": 500,
                       "iters_per_round": 10, "sizes": "batch distribution + 2% 4096x4096x32"},
            "requests": len(results), "completed": len(ok), "solves_per_s": len(ok) / wall,
            "S_updates_per_s": upd / wall, "wall_s": wall,
            "regular_p50_ms": pct(reg_lat, 50), "regular_p99_ms": pct(reg_lat, 99),
            "tail_requests": int(len(tail_lat)), "tail_p50_ms": pct(tail_lat, 50),
            "iterations_p50": pct(iters, 50),
            "iterations_max": int(iters.max()) if len(iters) else 0,
            "conservation_residual_max": float(cons.max()) if len(cons) else None,
            "log_marginal_rel_err_vs_fp64": {"max": max(errs) if errs else None,
                                             "median": float(np.median(errs)) if errs else None,
                                             "n": len(errs)},
            "gpu_busy_frac": sstats["gpu_ms"] / 1e3 / wall,
            "gpu_busy_frac_lanes": {"small": (sstats["gpu_ms"] - sstats["gpu_ms_large"]) / 1e3
                                    / wall, "large": sstats["gpu_ms_large"] / 1e3 / wall},
            "server": sstats, "clocks": clk.summary()}


def run_serve(args):
    import torch
    pkg = load_package()
    out = serve_measure(pkg, torch, args.rate, args.duration, args.fp64_sample, args.dtype)
    line = {"metric": out.pop("metric"), "value": out.pop("value"), "unit": out.pop("unit"),
            "n_gpus": 1, "data": "synthetic"}
    line.update(out)
    print(json.dumps(line))
    return 0


def run_precision(args):
    """FP32 storage with compensated axis sums against the FP64 path."""
    import torch
    pkg = load_package()
    import bnmf_algs_b200.workloads as W
    base = W.precision_study(2)
    X, z = base["X"], base["z"]
    x, y = X.shape
    # as specified, and the same draws mapped onto U(1,2) (grad_plus >= 0 there)
    variants = [("alpha,beta~U(0.5,2)", base["alpha"], base["beta"]),
                ("alpha,beta~U(1,2)", 1.0 + (base["alpha"] - 0.5) / 1.5,
                 1.0 + (base["beta"] - 0.5) / 1.5)]
    out = []
    for name, alpha, beta in variants:
        params = pkg.Params(base["a"], base["b"], alpha, beta)
        da = torch.as_tensor(alpha).cuda()
        db = torch.as_tensor(beta).cuda()
        dX64 = torch.as_tensor(X).cuda()
        dX32 = dX64.float()
        p64 = pkg.Plan(x, y, z, pkg.F64)
        p32 = pkg.Plan(x, y, z, pkg.F32)
        S64 = torch.empty((x, y, z), dtype=torch.float64, device="cuda")
        p64.init_S(dX64, S64, seed=0)
        S32 = S64.float()
        Xf = dX64.unsqueeze(2)
        rows = []
        done = 0
        for ck in range(25, base["iters"] + 1, 25):
            p64.run(dX64, da, db, S64, ck - done, pkg.PSI_APPR)
            p32.run(dX32, da, db, S32, ck - done, pkg.PSI_APPR)
            p64.check()
            p32.check()
            done = ck
            finite64 = bool(torch.isfinite(S64).all())
            finite32 = bool(torch.isfinite(S32).all())
            row = {"iteration": ck, "fp64_finite": finite64, "fp32_finite": finite32,
                   "fp64_negative": int((S64 < 0).sum())}
            if finite64 and finite32:
                mask = S64 > 1e-6 * Xf
                rel = ((S32.double() - S64).abs() / S64.abs().clamp_min(1e-300))[mask]
                row["max_rel_err_S"] = float(rel.max()) if rel.numel() else 0.0
                row["median_rel_err_S"] = float(rel.median()) if rel.numel() else 0.0
                den = dX64.clamp_min(1.0)
                row["conservation_fp64"] = float(((S64.sum(2) - dX64).abs() / den).max())
                row["conservation_fp32"] = float(((S32.double().sum(2) - dX64).abs() / den).max())
                lm64 = pkg.log_marginal_S(S64, params)
                lm32 = pkg.log_marginal_S(S32, params, dtype=pkg.F32)
                row["log_marginal_fp64"] = lm64
                row["log_marginal_gap_rel"] = abs(lm32 - lm64) / abs(lm64)
            rows.append(row)
        out.append({"params": name, "checkpoints": rows})
        p64.close()
        p32.close()
    line = {"metric": "precision_fp32_vs_fp64", "dtype": "f32 vs f64", "data": "synthetic",
            "config": {"workload": "precision_2048x2048x32", "iters": base["iters"],
                       "X": "30% zeros; otherwise Poisson(rate_i) conditioned on >= 1, "
                            "rate_i~LogNormal(0,1.5)",
                       "zero_fraction": float(np.mean(X == 0))},
            "results": out}
    print(json.dumps(line))
    return 0


def make_X(kind, x, y, z, rng):
    """X kinds: 'model' (the plain workload's allocation-model draw), 'dense'
    (1 + Poisson(10), no zeros), 'zeros' (all zero)."""
    load_package()
    import bnmf_algs_b200.workloads as W
    if kind == "model":
        return W.allocation_model_X(x, y, z, 5.0, 0.01, rng)
    if kind == "dense":
        return 1.0 + rng.poisson(10.0, (x, y)).astype(np.float64)
    return np.zeros((x, y))


def run_kernel_matrix(args):
    import torch
    pkg = load_package()
    x, y, z = (int(v) for v in args.shape.split("x"))
    peak, _ = hbm_peak()
    knobs = [(0, 0, 0), (8, 1, 0), (3, 2, 0), (4, 2, 0), (2, 2, 0), (6, 1, 0)]
    for dt in ("f64", "f32"):
        f64 = dt == "f64"
        es = 8 if f64 else 4
        dt_t = torch.float64 if f64 else torch.float32
        for kind in ("model", "dense", "zeros"):
            X = make_X(kind, x, y, z, np.random.default_rng(1))
            dX = torch.as_tensor(X).to("cuda", dt_t)
            da = torch.ones(x, dtype=torch.float64, device="cuda")
            db = torch.ones(z, dtype=torch.float64, device="cuda")
            dS = torch.empty((x, y, z), dtype=dt_t, device="cuda")
            for st, cps, rr in knobs:
                try:
                    plan = pkg.Plan(x, y, z, pkg.F64 if f64 else pkg.F32, st, cps, rr)
                except Exception as e:
                    print(json.dumps({"dtype": dt, "x_kind": kind, "knobs": [st, cps, rr],
                                      "error": str(e)}))
                    continue
                plan.init_S(dX, dS, seed=0)
                plan.run(dX, da, db, dS, 3, pkg.PSI_APPR)
                kms, ims = plan.profile(dX, da, db, dS, 10, pkg.PSI_APPR)
                alg = 2 * x * y * z * es + x * y * es
                print(json.dumps({"dtype": dt, "x_kind": kind, "knobs": [st, cps, rr],
                                  "tuning": plan.tuning(), "kernel_ms": round(kms, 4),
                                  "iteration_ms": round(ims, 4),
                                  "frac": round(alg / (kms / 1e3) / 1e9 / peak, 3)}), flush=True)
                plan.close()
            del dX, dS
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dtype", choices=["f64", "f32"], default=None,
                    help="storage precision (default f64 for the plain solve, f32 for --batch "
                         "and --serve)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="untimed: set up the workload, run --profile-iters iterations, exit "
                         "(the command profiled by ncu)")
    ap.add_argument("--profile-iters", type=int, default=3)
    ap.add_argument("--skip-zero-rows", action="store_true",
                    help="--profile-run: the plan option skip_zero_rows")
    ap.add_argument("--x-kind", choices=["model", "dense", "zeros"], default="model",
                    help="X of --profile-run: the plain workload's draw, 1+Poisson(10), or zeros")
    ap.add_argument("--shape", default="1024x1024x64",
                    help="x*y*z of the plain workload for --profile-run / --kernel-matrix")
    ap.add_argument("--batch", action="store_true",
                    help="batched uneven solves: 512 instances, x,y log-uniform in [32,512], "
                         "z in {4..64}, FP32, 150 iterations; vs a loop of the plain solver")
    ap.add_argument("--batch-n", type=int, default=512)
    ap.add_argument("--headline-only", action="store_true",
                    help="default mode: skip the parity, FP32, batch and serving blocks")
    ap.add_argument("--serve-sample-rate", type=float, default=50.0,
                    help="offered rate (req/s) of the default run's serving sample")
    ap.add_argument("--serve-sample-seconds", type=float, default=12.0,
                    help="seconds of traffic of the default run's serving sample")
    ap.add_argument("--sharded", action="store_true",
                    help="the headline solve row-sharded over the torchrun ranks (NCCL)")
    ap.add_argument("--batch-probe", action="store_true",
                    help="build the --batch workload and run --profile-iters iterations twice "
                         "without a graph (for ncu)")
    ap.add_argument("--rows-per-tile", type=int, default=0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="--batch: keep the default tile height and stage depth")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop: Poisson arrivals at --rate req/s for --duration s; "
                         "p50/p99 latency, solves/s, log-marginal error vs FP64")
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--duration", type=float, default=60.0,
                    help="seconds of Poisson traffic for --serve (the serving workload runs 60 s)")
    ap.add_argument("--fp64-sample", type=int, default=16)
    ap.add_argument("--precision", action="store_true",
                    help="precision study: 2048x2048x32 heavy-tailed X, FP32 (compensated sums) "
                         "vs the FP64 path, 300 iterations, checkpoints every 25")
    ap.add_argument("--kernel-matrix", action="store_true",
                    help="time the update sweep (CUDA events) over X kinds, dtypes and launch "
                         "knobs; one JSON line each")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.dtype is None:
        args.dtype = "f32" if (args.batch or args.serve or args.batch_probe) else "f64"
    # the default run's batch block is the FP32-compensated batched form
    args.batch_dtype = args.dtype if (args.batch or args.batch_probe) else "f32"
    if args.batch_probe:
        return run_batch_probe(args)
    if args.sharded:
        return run_sharded(args)
    if args.profile_run:
        return run_profile(args)
    if args.kernel_matrix:
        return run_kernel_matrix(args)
    if args.batch:
        return run_batch(args)
    if args.serve:
        return run_serve(args)
    if args.precision:
        return run_precision(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
