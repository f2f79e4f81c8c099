"""Benchmark: EM iterations/s of the AMICA engine on one B200, or of one fit
sharded over N B200s.

Workload (the metric's configuration): n=128 channels, T=1,000,000 samples,
M=3 models, m=3 mixtures, synthetic FP32 data from cudamica_b200.synth
(config-2 recipe, seed 0).  A "step" is one full EM iteration over all T
samples: fused E-step + FP64 M-step.  The sphered data (512 MB) is larger than
L2 (126 MB), so every step reads it from HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line.  `value` is the mixed-precision (tcgen05 TF32)
form's iterations/s with the data resident in HBM, timed with CUDA events on
the engine's stream, max over ranks; the plain FP32 form is timed the same way
and reported beside it, with both forms' final LL after a fixed-length fit.
`e2e` runs a whole fit through the public C ABI from pinned host memory.
Under torchrun with N > 1 ranks the samples are split over the ranks (one
fit, strong scaling: each iteration is the shards' E-steps, one NCCL
all-reduce of the sufficient statistics, the same M-step on every rank);
`--replicas` runs N independent fits instead.
`--impl reference` times the reference's own implementation (its CUDA sources
compiled here for sm_100a, oracle/_ref/cudaamica_ref) on the same workload,
using its own per-iteration timer.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=128, T=1_000_000, M=3, m=3)
METRIC = "EM iters/s at n=128,T=1M,M=3: mixed-precision vs plain FP32, same final LL"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_over_ranks(values, pg, op: str, device: str = "cuda"):
    """Element-wise max or min of `values` over all ranks (every rank calls it,
    in the same order); identity without a process group."""
    if pg is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX if op == "max" else pg.ReduceOp.MIN)
    return [float(v) for v in t.cpu()]


def whole_job_rate(ms_per_step_max: float, ws: int) -> float:
    """Iterations per second of the whole job: every rank runs one iteration of
    its own replica per step; the step takes as long as the slowest rank."""
    return ws * 1000.0 / ms_per_step_max


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(prefix="clk_", suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
             "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        # median under load: ignore idle samples below half of max
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def make_data(seed: int = 0):
    from cudamica_b200 import synth
    d = synth.config2(seed=seed, n=WORKLOAD["n"], T=WORKLOAD["T"], M=WORKLOAD["M"], m=WORKLOAD["m"])
    A0, c0 = synth.norand_init(WORKLOAD["n"], WORKLOAD["M"])
    return d.x, A0, c0


def new_engine(x, A0, c0, precision, device, **over):
    from cudamica_b200.engine import Amica
    eng = Amica(WORKLOAD["n"], WORKLOAD["T"], WORKLOAD["M"], WORKLOAD["m"], precision=precision,
                device=device, maxiter=4000, **over)
    eng.load_data(x)
    eng.preprocess()
    eng.init(A0, c0)
    return eng


def traffic_per_launch():
    """DRAM bytes per E-step launch at the bench size, from the committed ncu
    summary of the tensor-core E-step (captured at T = 400,000 and scaled by
    samples, as that file states)."""
    p = os.path.join(ROOT, "profiles", "estep_tc_n128_T400k_M3_m3.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch_n128_T1e6:\s*(\d+)", open(p).read())
    return int(m.group(1)) if m else None


def roofline_for(estep_ms: float, T: int, clocks: dict, kernel: str) -> dict:
    """The binding (largest) of the algorithmic bounds of one E-step launch over
    T samples at the workload's n, M, m, against its CUDA-event time."""
    hbm, bf16, src = peaks()
    n, M, m = (WORKLOAD[k] for k in ("n", "M", "m"))
    est = estep_ms * 1e-3
    alg_bytes = 4 * n * T + 4 * M * T            # x read once + Lt write per iteration
    tc_flops = 4 * M * n * n * T                 # W x and g b^T
    mufu = (4 * m + 1) * M * n * T               # lg2, ex2, ex2, rcp per element + lg2 per (h, i, t)
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    mufu_peak = 16 * 148 * sm_mhz * 1e6          # ops/s
    tf32_peak = 0.5 * bf16 * 1e12                # flop/s
    bounds = {
        "hbm": {"time_s": alg_bytes / (hbm * 1e9), "achieved": alg_bytes / est / 1e9, "peak": hbm,
                "unit": "GB/s", "per_launch": alg_bytes},
        "tensor": {"time_s": tc_flops / tf32_peak, "achieved": tc_flops / est / 1e12,
                   "peak": tf32_peak / 1e12, "unit": "TFLOP/s", "per_launch": tc_flops},
        "sfu": {"time_s": mufu / mufu_peak, "achieved": mufu / est / 1e9, "peak": mufu_peak / 1e9,
                "unit": "Gop/s", "per_launch": mufu},
    }
    for v in bounds.values():
        v["frac"] = v["time_s"] / est
    bind = max(bounds, key=lambda k: bounds[k]["time_s"])
    b = bounds[bind]
    tr = traffic_per_launch()
    return {"bound": bind, "achieved": b["achieved"], "peak": b["peak"], "unit": b["unit"],
            "frac": b["frac"],
            "traffic": None if tr is None else int(tr * T / WORKLOAD["T"]),
            "kernel": kernel, "kernel_ms": estep_ms, "samples_per_launch": T,
            "all_bounds": bounds,
            "peaks_used": {
                "hbm": f"{hbm} GB/s, {src} copy bandwidth (MEASURED_PEAKS.json)",
                "tensor": f"TF32 = half of the {src} BF16 burst rate {bf16} TFLOP/s "
                          "(dense TF32 is half of dense BF16 on B200; TF32 not measured)",
                "sfu": f"16 MUFU ops/clk/SM x 148 SMs x {sm_mhz:.0f} MHz (sampled SM clock)"},
            "note": "the binding (largest) of the algorithmic bounds of one E-step launch, "
                    "divided by its CUDA-event time; FP32 non-tensor work is not among the "
                    "algorithmic counts"}


def time_form(x, A0, c0, precision, device, steps, warmup, fit_iters):
    """Returns a dict: ms per timed step, the final LL and parameters after
    fit_iters iterations, the E-step's own time (and, for the mixed form, with
    the split correction of phi switched on), kernel, launches per iteration and
    the E-step grid (as many clusters as the device holds at once)."""
    eng = new_engine(x, A0, c0, precision, device)
    eng.run(warmup)
    outs = eng.run(steps)                     # device time via CUDA events on the engine stream
    ms = float(np.mean([o.device_ms for o in outs]))
    rest = fit_iters - warmup - steps
    if rest > 0:
        outs2 = eng.run(rest)
        final_ll = outs2[-1].ll
    else:
        final_ll = outs[-1].ll
    est_ms, _ = eng.time_estep(5)
    res = {"ms": ms, "final_ll": final_ll, "estep_ms": est_ms, "kernel": eng.kernel,
           "lpi": eng.launches_per_iteration, "params": eng.params(),
           "iters": max(fit_iters, warmup + steps)}
    try:
        res["grid"] = eng.set_grid(0)         # the grid in effect (as many as fit)
    except Exception:                         # informational only
        res["grid"] = None
    eng.close()
    if precision == 1:
        # the same E-step with phi formed from hi + lo parts of both operands
        e2 = new_engine(x, A0, c0, precision, device, phi_split=1)
        res["estep_split_ms"], _ = e2.time_estep(5)
        e2.close()
    return res


def ll_at(x, A0, c0, precision, device, prm):
    """LL per sample and channel of one E-step of the given form at the given
    parameters (no M-step)."""
    n, T = WORKLOAD["n"], WORKLOAD["T"]
    eng = new_engine(x, A0, c0, precision, device)
    eng.set_params(**{k: prm[k] for k in ("A", "c", "gm", "alpha", "mu", "beta", "rho")})
    ll = float(eng.estep_stats()[0]) / (n * T)
    eng.close()
    return ll


def cpu_baseline_port(x, A0, c0, iters: int = 3):
    """The C oracle's EM iteration on the whole workload on every host core:
    `iters` full iterations in FP64 (after one untimed), and as many with the
    E-step's per-sample arithmetic in FP32 (sums FP64)."""
    from oracle import oracle as O
    xs = x.astype(np.float64)
    xs -= xs.mean(0)
    C = xs.T @ xs / xs.shape[0]
    d, V = np.linalg.eigh(C)
    S = (V * (2.0 / np.sqrt(d))) @ V.T
    xs = xs @ S.T
    cores = os.cpu_count() or 1
    out = {}
    for label, fp32 in (("fp64", False), ("fp32", True)):
        orc = O.Oracle(xs, WORKLOAD["M"], WORKLOAD["m"], A0, c0, 0.0, nthreads=cores, fp32=fp32)
        orc.step()                             # untimed first iteration
        t0 = time.perf_counter()
        for _ in range(iters):
            orc.step()
        dt = (time.perf_counter() - t0) / iters
        out[label] = {"value": 1.0 / dt, "s_per_iter": dt}
        del orc
    return {"value": out["fp64"]["value"], "unit": "iters/s", "cores": cores, "kind": "port",
            "sample": f"{iters} full EM iterations (n=128, T=1e6, M=3, m=3) of the C oracle on "
                      f"{cores} threads after one untimed iteration; FP64",
            "fp32": {**out["fp32"], "note": "same iteration, E-step per-sample arithmetic in FP32, "
                                            "sums FP64 (oracle/liboracle32.so)"}}


def pinned_copy(x):
    """The raw data in page-locked host memory (torch is used only as the
    allocator), as a user holding the recording for the fit would keep it."""
    import torch
    pin = torch.empty(x.shape, dtype=torch.float32, pin_memory=True)
    pin.numpy()[...] = x
    return pin


def e2e_run(pin, A0, c0, device, steps):
    """Whole fit through the public API from pinned host memory: H2D load,
    GPU sphering, init, `steps` iterations, D2H of the parameters."""
    from cudamica_b200.engine import Amica
    n, T = WORKLOAD["n"], WORKLOAD["T"]
    buf = pin.numpy()
    nbytes = buf.nbytes
    pinned = pin.is_pinned()
    eng = Amica(n, T, WORKLOAD["M"], WORKLOAD["m"], precision=1, device=device, maxiter=4000)
    t0 = time.perf_counter()
    eng.load_data(buf)
    eng.preprocess()
    eng.init(A0, c0)
    eng.run(steps)
    prm = eng.params()
    dt = time.perf_counter() - t0
    eng.close()
    d2h = sum(v.nbytes for v in prm.values()) + steps * 64
    return {"value": steps / dt, "unit": "iters/s", "h2d_bytes_per_step": nbytes / steps,
            "d2h_bytes_per_step": d2h / steps, "pinned_host": bool(pinned),
            "scope": f"load_data + preprocess + init + run({steps}) + get_params, wall clock"}


# ---------------------------------------------------------------- reference arm
def reference_arm(args):
    # the build without the per-iteration dumps of -DITERTEST (oracle/Makefile)
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "cudaamica_ref_timed")
    if not os.path.exists(ref_bin):
        return None
    from cudamica_b200 import synth
    x, A0, c0 = make_data()
    n, T, M, m = WORKLOAD["n"], WORKLOAD["T"], WORKLOAD["M"], WORKLOAD["m"]
    work = tempfile.mkdtemp(prefix="amica_refarm_")
    try:
        os.makedirs(os.path.join(work, "datasets"))
        os.makedirs(os.path.join(work, "out"))
        x.astype(np.float32).tofile(os.path.join(work, "data.fdt"))
        xd = x.astype(np.float64)
        mean = xd.mean(0)
        xd -= mean
        C = xd.T @ xd / T
        dd, V = np.linalg.eigh(C)
        S = (V * (2.0 / np.sqrt(dd))) @ V.T
        (xd @ S.T).tofile(os.path.join(work, "datasets", "whitened.fdt"))
        del xd
        mean.tofile(os.path.join(work, "datasets", "means.fdt"))
        A0[0].astype(np.float32).tofile(os.path.join(work, "datasets", "anorand.fdt"))
        c0[0].astype(np.float32).tofile(os.path.join(work, "datasets", "cnorand.fdt"))
        A0[1].astype(np.float32).tofile(os.path.join(work, "datasets", "anorand1.fdt"))
        c0[1].astype(np.float32).tofile(os.path.join(work, "datasets", "cnorand1.fdt"))
        iters = args.warmup + args.steps
        lines = ["datafile data.fdt", f"nchannels {n}", f"nsamples {T}", "do_sphere 1",
                 f"maxiter {iters}", f"nsdm {m}", f"nmmodels {M}", "spherefile out/sphere.fdt",
                 "block_size 5000", "fix_init on", "do_newton on", "newt_start_iter 50",
                 "rho_start_iter 1", "update_rho 1"]
        with open(os.path.join(work, "case.in"), "w") as f:
            f.write("\n".join(lines) + "\n")
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0"))
        proc = subprocess.run([ref_bin, "-f", "case.in"], cwd=work, capture_output=True, text=True,
                              timeout=1800, env=env)
        if proc.returncode != 0:
            return {"error": f"reference exited {proc.returncode}"}
        ms = [int(v) for v in re.findall(r"Iteration \d+ times = \d+ ticks, (\d+) ms", proc.stdout)]
        ll = [float(v) for v in re.findall(r"Iteration \d+: lrate \S+ LL (\S+)", proc.stdout)]
        timed = ms[args.warmup:]
        return {"ms": timed, "ll": ll}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def cohort_arm(args):
    """Cohort workload: subjects with n in {32, 64, 128} (in turn), T uniform in
    [100k, 800k] x scale, M = 1, m = 3, each from the single-model recipe with
    seed 1000 + i and cond(A) uniform in [10, 50]; fitted together in the mixed
    form with one persistent E-step launch per cohort iteration (the value), and
    as concurrent per-subject graphs with the autotuner's SM split (for
    comparison), against the same subjects fitted one after another on the whole
    GPU with the plain form.  Host wall clock; every subject runs warmup + steps
    iterations in every arm."""
    import torch
    from cudamica_b200 import synth
    from cudamica_b200.cohort import Cohort
    from cudamica_b200.engine import Amica
    rng = np.random.default_rng(7)
    S = args.cohort_subjects
    data, inits = [], []
    for i in range(S):
        n = (32, 64, 128)[i % 3]
        T = int(rng.uniform(100_000, 800_000) * args.cohort_scale)
        cond = float(rng.uniform(10.0, 50.0))
        d = synth.config1(seed=1000 + i, n=n, T=T, cond=cond)
        data.append(d.x.astype(np.float32))
        inits.append(synth.norand_init(n, 1))
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    coh = Cohort(data, M=1, m=3, precision=1, inits=inits, maxiter=4000, persistent=True)
    coh.run(args.warmup)
    outs, dt = coh.timed_run(args.steps)
    cohort_ll = [o[-1].ll for o in outs]
    device_ms = coh.last_ms
    coh.close()
    coh = Cohort(data, M=1, m=3, precision=1, inits=inits, sm_budget=nsm, maxiter=4000)
    coh.run(args.warmup)
    _, dt_streams = coh.timed_run(args.steps)
    grids = list(coh.grids)
    coh.close()
    seq_ms, seq_ll = 0.0, []
    for x, init in zip(data, inits):
        T, n = x.shape
        eng = Amica(n, T, 1, 3, precision=0, maxiter=4000)
        eng.load_data(x)
        eng.preprocess()
        eng.init(*init)
        eng.run(args.warmup)
        t0 = time.perf_counter()
        o = eng.run(args.steps)
        seq_ms += (time.perf_counter() - t0) * 1e3
        seq_ll.append(o[-1].ll)
        eng.close()
    value = args.steps / dt
    seq = 1000.0 * args.steps / seq_ms
    d_ll = [abs(a - b) for a, b in zip(cohort_ll, seq_ll)]
    return {
        "metric": "cohort EM iters/s (all subjects one iteration each)", "value": value,
        "unit": "cohort iters/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"cohort of {S} subjects, n in {{32,64,128}}, T ~ U[1e5, 8e5] x "
                               f"{args.cohort_scale}, M=1, m=3",
                   "subjects": S, "total_samples": int(sum(x.shape[0] for x in data)),
                   "parallelism": "single GPU: one persistent E-step launch over all subjects' "
                                  "tiles per cohort iteration, per-subject M-steps on their "
                                  "own streams, one CUDA graph"},
        "device_ms_per_step": device_ms,
        "streams": {"value": args.steps / dt_streams, "ms_per_step": 1000.0 * dt_streams / args.steps,
                    "grids": grids,
                    "note": "per-subject graphs on concurrent streams, grids from the autotuner"},
        "sequential_plain": {"value": seq, "ms_per_step": seq_ms / args.steps},
        "speedup_vs_sequential_plain": value / seq,
        "final_ll_abs_diff": {"max": max(d_ll), "median": float(np.median(d_ll)),
                              "note": "per subject, cohort (mixed) vs sequential (plain), "
                                      "after warmup + steps iterations"},
    }


def big_arm(args):
    """The 256-channel multi-model workload (synth.config4, seed 0: n=256,
    T=2,000,000, M=4, m=5): the split mixed form (tcgen05 TF32 contraction
    kernels around the density-only E-step) against plain FP32.  Device time per
    graph-captured iteration (CUDA events on the engine's stream), the E-step
    alone, and the LL of both forms after --big-fit-iters iterations from the
    same start (or the error that stopped a fit)."""
    from cudamica_b200 import synth
    from cudamica_b200.engine import Amica, AmicaError
    n, M, m = 256, 4, 5
    T = args.big_T
    x = np.ascontiguousarray(synth.config4(seed=0, n=n, T=T, M=M, m=m).x)
    A0, c0 = synth.norand_init(n, M)
    res = {}
    for precision in (1, 0):
        eng = Amica(n, T, M, m, precision=precision, maxiter=max(4000, args.big_fit_iters + 16))
        eng.load_data(x)
        eng.preprocess()
        eng.init(A0, c0)
        eng.run(args.warmup)
        outs = eng.run(args.steps)
        ms = float(np.mean([o.device_ms for o in outs]))
        ll, status = outs[-1].ll, "ok"
        rest = args.big_fit_iters - args.warmup - args.steps
        try:
            if rest > 0:
                ll = eng.run(rest)[-1].ll
        except AmicaError as e:
            status = str(e)
        est_ms, _ = eng.time_estep(3)
        res[eng.kernel] = {"ms_per_step": ms, "value": 1000.0 / ms, "estep_ms": est_ms,
                           "ll": ll, "fit_status": status}
        eng.close()
    sp, pl = res["split_tf32"], res["plain_fp32"]
    return {
        "metric": "EM iters/s at n=256,T=2M,M=4,m=5: split mixed form vs plain FP32",
        "value": sp["value"], "unit": "iters/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sp["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"n=256 T={T} M=4 m=5 (synth.config4), one EM iteration per step",
                   "n": n, "T": T, "M": M, "m": m, "kernel": "split_tf32",
                   "precision": "mixed: TF32 tensor-core GEMMs for b = W x and Psi, FP32 densities, "
                                "FP64 M-step", "parallelism": "single GPU"},
        "split_tf32": sp, "plain_fp32": pl, "split_over_plain": pl["ms_per_step"] / sp["ms_per_step"],
        "fit_iters": args.big_fit_iters,
    }


def profile_case(args):
    """A few E-step launches per form on the first T samples of the workload
    (or, with --profile-shape n,M,m, of the large multi-model recipe at that
    shape: synth.config4, seed 0)."""
    from cudamica_b200.engine import Amica
    T = args.T
    if args.profile_shape:
        from cudamica_b200 import synth
        n, M, m = (int(v) for v in args.profile_shape.split(","))
        x = synth.config4(seed=0, n=n, T=T, M=M, m=m).x
        A0, c0 = synth.norand_init(n, M)
    else:
        x, A0, c0 = make_data()
        n, M, m = WORKLOAD["n"], WORKLOAD["M"], WORKLOAD["m"]
    for precision in (1, 0):
        eng = Amica(n, T, M, m, precision=precision, device=0)
        eng.load_data(np.ascontiguousarray(x[:T]))
        eng.preprocess()
        eng.init(A0, c0)
        eng.estep_stats()
        ms, _ = eng.time_estep(2)
        print(f"{eng.kernel}: {ms:.3f} ms per E-step launch at T={T}")
        eng.close()
    return 0


def sharded_arm(args, ws: int, rank: int, local: int):
    """One fit of the workload with its samples split over the ranks (strong
    scaling): each rank loads its contiguous sample range, the sphering is
    formed from the column sums and scatters of all ranks, and every EM
    iteration is the shard's E-step, one NCCL all-reduce of the statistics
    vector and the same M-step on every rank (cudamica_b200.sharded).  A step
    is one iteration of the whole T-sample fit."""
    import torch
    import torch.distributed as dist
    from cudamica_b200.engine import Amica
    from cudamica_b200.sharded import EngineShard, ShardedFit, engine_shard_preprocess, shard_range
    n, T, M, m = (WORKLOAD[k] for k in ("n", "T", "M", "m"))
    dev = torch.device("cuda", local)
    x, A0, c0 = make_data()
    t0, t1 = shard_range(T, rank, ws)
    xs = np.ascontiguousarray(x[t0:t1])
    del x

    def fit_setup(data):
        eng = Amica(n, t1 - t0, M, m, precision=1, device=local, maxiter=4000)
        eng.load_data(data)
        engine_shard_preprocess(eng, T, group=dist.group.WORLD)
        eng.init(A0, c0)
        return eng, ShardedFit(EngineShard(eng), T, group=dist.group.WORLD, device=dev)

    eng, fit = fit_setup(xs)
    for _ in range(args.warmup):
        fit.step()
    st = fit.shard.torch_stream                 # the engine's stream, where the iteration runs
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(st)
        outs = fit.run(args.steps)
        e1.record(st)
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms_rank = e0.elapsed_time(e1) / args.steps
    est_ms, _ = eng.time_estep(5)
    # the exchange alone: the statistics all-reduce, 20 times
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    with fit.shard.stream():
        a0.record(st)
        for _ in range(20):
            dist.all_reduce(fit.buf, op=dist.ReduceOp.SUM)
        a1.record(st)
    torch.cuda.synchronize()
    ar_ms = a0.elapsed_time(a1) / 20
    kernel, lpi = eng.kernel, eng.launches_per_iteration
    eng.close()
    ms, est_max, ar_max = reduce_over_ranks([ms_rank, est_ms, ar_ms], dist, "max")
    e2e = None
    if not args.no_e2e:
        pin = pinned_copy(xs)
        dist.barrier()
        w0 = time.perf_counter()
        eng2, fit2 = fit_setup(pin.numpy())
        fit2.run(args.steps)
        prm = eng2.params()
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        eng2.close()
        del pin
        wall = reduce_over_ranks([wall], dist, "max")[0]
        e2e = {"value": args.steps / wall, "unit": "iters/s",
               "h2d_bytes_per_step": xs.nbytes * ws / args.steps,
               "d2h_bytes_per_step": (sum(v.nbytes for v in prm.values()) + args.steps * 64) * ws / args.steps,
               "scope": f"per rank: load_data of its shard from pinned memory, sharded sphering, init, "
                        f"{args.steps} sharded iterations, get_params; wall clock, max over ranks"}
    out = {
        "metric": METRIC, "value": 1000.0 / ms, "unit": "iters/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "n=128 T=1e6 M=3 m=3, one EM iteration of the whole fit per step", **WORKLOAD,
                   "precision": "mixed: tcgen05 TF32 contractions, FP32 densities, FP64 M-step",
                   "kernel": kernel, "parallelism": f"samples sharded over {ws} GPUs, "
                                                    "one FP64 all-reduce of the statistics per iteration",
                   "samples_per_rank": t1 - t0,
                   "l2": "inputs larger than L2 (512 MB sphered data in all, per step)"},
        "allreduce_ms": ar_max, "stats_bytes": int(fit.buf.numel() * 8),
        "final_ll": outs[-1].ll,
        "roofline": roofline_for(est_max, t1 - t0, clocks, kernel),
        "gpu_launches": lpi * args.steps,
        "clocks": clocks,
    }
    if e2e is not None:
        out["e2e"] = e2e
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fit-iters", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sharded", action="store_true",
                    help="the sample-sharded fit also on one rank (a one-member process group)")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 GPUs: N independent fits instead of one sample-sharded fit")
    ap.add_argument("--profile-case", action="store_true",
                    help="no timing: run a few fused E-step launches of both forms on a "
                         "T-sample slice (for ncu captures)")
    ap.add_argument("--T", type=int, default=WORKLOAD["T"])
    ap.add_argument("--profile-shape", default="",
                    help="n,M,m for --profile-case (data: the large multi-model recipe)")
    ap.add_argument("--cohort", action="store_true",
                    help="the cohort workload instead of the single-fit one")
    ap.add_argument("--cohort-subjects", type=int, default=48)
    ap.add_argument("--cohort-scale", type=float, default=1.0,
                    help="scale of the per-subject sample counts")
    ap.add_argument("--big", action="store_true",
                    help="the 256-channel workload (n=256, M=4, m=5), both forms")
    ap.add_argument("--big-T", type=int, default=2_000_000)
    ap.add_argument("--big-fit-iters", type=int, default=300)
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.cohort:
        print(json.dumps(cohort_arm(args)))
        return 0
    if args.big:
        print(json.dumps(big_arm(args)))
        return 0
    ws, rank, local = dist_env()
    pg = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    if args.impl == "reference":
        if rank != 0:
            return 0
        with Clocks(local) as clk:
            res = reference_arm(args)
        if res is None or "error" in res:
            why = "oracle/_ref/cudaamica_ref_timed not built" if res is None else res["error"]
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        ms = float(np.mean(res["ms"])) if res["ms"] else float("nan")
        v = 1000.0 / ms
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": "iters/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "n=128 T=1e6 M=3 m=3, one EM iteration per step", **WORKLOAD,
                       "l2": "inputs larger than L2 (1 GB FP64 whitened data)",
                       "implementation": "reference CUDA sources (fp64, cuBLAS + kernels) built "
                                         "for sm_100a with a MAGMA/MKL stand-in"},
            "cpu_baseline": {"value": v, "unit": "iters/s", "cores": 1, "kind": "reference",
                             "sample": f"reference's own per-iteration timer over {len(res['ms'])} "
                                       "iterations after warm-up; single host thread driving the GPU"},
            "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk.summary(),
            "ll_last": res["ll"][-1] if res["ll"] else None,
        }
        print(json.dumps(line))
        return 0

    if (ws > 1 and not args.replicas) or args.sharded:
        if pg is None:                          # --sharded on one rank: a one-member group
            import datetime
            import torch
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29533")
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=600))
            pg = dist
        out = sharded_arm(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(out))
        pg.barrier()
        pg.destroy_process_group()
        return 0

    import torch
    device = local
    torch.cuda.set_device(device)
    x, A0, c0 = make_data()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with Clocks(device) as clk:
        rm = time_form(x, A0, c0, 1, device, args.steps, args.warmup, args.fit_iters)
    clocks = clk.summary()
    rp = time_form(x, A0, c0, 0, device, args.steps, args.warmup, args.fit_iters)
    # "same final LL": the two fits follow different trajectories of a chaotic
    # map, so their LL at a fixed iteration differs by trajectory noise (the
    # control: the plain form refit from A0 perturbed by 1e-12).  What precision
    # alone does is measured at identical parameters: each form's E-step at the
    # other form's final parameters.
    ctrl = None
    if args.fit_iters > 0:
        rng = np.random.default_rng(123)
        A0p = A0 * (1.0 + 1e-12 * rng.standard_normal(A0.shape))
        ctrl = time_form(x, A0p, c0, 0, device, 1, 0, args.fit_iters)["final_ll"]
    same = {}
    for fit, prm in (("mixed_fit", rm["params"]), ("plain_fit", rp["params"])):
        lm, lp = ll_at(x, A0, c0, 1, device, prm), ll_at(x, A0, c0, 0, device, prm)
        same[fit] = {"mixed": lm, "plain": lp, "abs_diff": abs(lm - lp)}
    ms, t_plain = reduce_over_ranks([rm["ms"], rp["ms"]], pg, "max")
    value = whole_job_rate(ms, ws)
    roof = roofline_for(rm["estep_ms"], WORKLOAD["T"], clocks, rm["kernel"])
    out = {
        "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "n=128 T=1e6 M=3 m=3, one EM iteration per step", **WORKLOAD,
                   "precision": "mixed: tcgen05 TF32 contractions, FP32 densities, FP64 M-step",
                   "kernel": rm["kernel"], "l2": "inputs larger than L2 (512 MB sphered data per step)",
                   "parallelism": "independent replicas" if ws > 1 else "single GPU",
                   "estep_clusters": rm["grid"]},
        "plain_fp32": {"value": whole_job_rate(t_plain, ws), "ms_per_step": t_plain,
                       "kernel": rp["kernel"], "estep_ms": rp["estep_ms"], "estep_clusters": rp["grid"]},
        "mixed_over_plain": t_plain / ms,
        "estep_split_phi_ms": rm.get("estep_split_ms"),
        "final_ll": {"iters": rm["iters"], "mixed": rm["final_ll"], "plain": rp["final_ll"],
                     "abs_diff": abs(rm["final_ll"] - rp["final_ll"]),
                     "plain_perturbed_1e-12": ctrl,
                     "control_abs_diff": abs(ctrl - rp["final_ll"]) if ctrl is not None else None,
                     "note": "nats per sample and channel; control = plain form from A0*(1+1e-12 N(0,1))"},
        "same_ll_at_same_params": {
            **same, "max_abs_diff": max(v["abs_diff"] for v in same.values()), "band": 1e-5,
            "note": "one E-step of each form at each fit's final parameters (after its last "
                    "M-step): the LL difference that precision alone makes; nats per sample "
                    "and channel"},
        "roofline": roof,
        "gpu_launches": rm["lpi"] * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_port(x, A0, c0)
    if not args.no_e2e:
        # one untimed fit (first-launch costs), then three whole fits from the
        # same pinned buffer, the median reported
        pin = pinned_copy(x)
        e2e_run(pin, A0, c0, device, args.warmup)
        runs = [e2e_run(pin, A0, c0, device, args.steps) for _ in range(3)]
        del pin
        e2e = dict(sorted(runs, key=lambda r: r["value"])[1])
        e2e["runs"] = [r["value"] for r in runs]
        e2e["scope"] += ", median of 3 fits after one untimed fit"
        if pg:
            e2e["value"] = reduce_over_ranks([e2e["value"]], pg, "min")[0] * ws
        out["e2e"] = e2e
    if rank == 0:
        print(json.dumps(out))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
