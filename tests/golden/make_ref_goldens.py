"""Run the reference's own CUDA build (oracle/_ref/cudaamica_ref, made by
``make -C oracle ref``) on the parity cases and save its outputs as golden
fixtures (tests/golden/ref_<case>.npz).

Needs a GPU.  Usage:
    python tests/golden/make_ref_goldens.py --out DIR c0 m2 m3
    python tests/golden/make_ref_goldens.py --time-only --out DIR c1t c2t

The reference runs in its deterministic mode (-DNORAND -DITERTEST): it reads the
whitened data, the means and the initial A/c of every model from
``datasets/*.fdt`` in its working directory (src/amica.cu:314-322,731-734) and
dumps A, c, alpha, mu, beta and rho after every iteration
(src/amica.cu:2514-2532).  Its stdout carries the per-iteration log-likelihood
("Iteration %lu: lrate %.16f LL %.16f", src/amica.cu:1983) and its own
per-iteration wall time (src/amica.cu:2540).
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from golden.cases import CASES, Case, prepared, digest, sphere_numpy  # noqa: E402
from cudamica_b200 import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "cudaamica_ref")

TIMING = {
    # shape-only runs for the reference's own per-iteration time on the GPU
    "c1t": Case("c1t", 64, 500_000, 1, 3, 3, 50, True, "config1", 0, ()),
    "c2t": Case("c2t", 128, 1_000_000, 3, 3, 3, 50, True, "config2", 0, ()),
}


def write_config(path: str, case: Case, outdir: str) -> None:
    lines = [
        "datafile data.fdt",
        f"nchannels {case.n}",
        f"nsamples {case.T}",
        "do_sphere 1",
        f"maxiter {case.maxiter}",
        f"nsdm {case.m}",
        f"nmmodels {case.M}",
        f"spherefile {outdir}/sphere.fdt",
        "block_size 5000",
        "fix_init on",
        "do_newton on",
        f"newt_start_iter {case.newt_start_iter}",
        "rho_start_iter 1",
        f"weightsfile {outdir}/W.fdt",
        f"afile {outdir}/A.fdt",
        f"cfile {outdir}/c.fdt",
        f"llfile {outdir}/ll.fdt",
        f"ltallfile {outdir}/ltall.fdt",
        f"gmfile {outdir}/gm.fdt",
        f"alphafile {outdir}/alpha.fdt",
        f"mufile {outdir}/mu.fdt",
        f"betafile {outdir}/beta.fdt",
        f"rhofile {outdir}/rho.fdt",
    ]
    if case.update_rho:
        lines.append("update_rho 1")
    # no '#' comment lines: the reference's getters other than getString call
    # strstr() on the NULL entry a comment line leaves (src/params.c:12,263)
    with open(path, "w") as f:
        for ln in lines:
            f.write(ln + "\n")


def run_case(case: Case, workroot: str, keep_arrays: bool) -> dict:
    wd = os.path.join(workroot, case.name)
    os.makedirs(os.path.join(wd, "datasets"), exist_ok=True)
    os.makedirs(os.path.join(wd, "out"), exist_ok=True)
    if case.recipe == "config1":
        x = synth.config1(seed=case.seed, n=case.n, T=case.T).x
        xs, means, S, ldetS = sphere_numpy(x)
        A0, c0 = synth.norand_init(case.n, case.M)
        prep = dict(x=x, xs=xs, means=means, sphere=S, ldetS=ldetS, A0=A0, c0=c0)
    else:
        prep = prepared(case)
    prep["x"].astype(np.float32).tofile(os.path.join(wd, "data.fdt"))
    prep["xs"].astype(np.float64).tofile(os.path.join(wd, "datasets", "whitened.fdt"))
    prep["means"].astype(np.float64).tofile(os.path.join(wd, "datasets", "means.fdt"))
    A0, c0 = prep["A0"], prep["c0"]
    A0[0].astype(np.float32).tofile(os.path.join(wd, "datasets", "anorand.fdt"))
    c0[0].astype(np.float32).tofile(os.path.join(wd, "datasets", "cnorand.fdt"))
    h1 = 1 if case.M > 1 else 0
    A0[h1].astype(np.float32).tofile(os.path.join(wd, "datasets", "anorand1.fdt"))
    c0[h1].astype(np.float32).tofile(os.path.join(wd, "datasets", "cnorand1.fdt"))
    write_config(os.path.join(wd, "case.in"), case, "out")

    t0 = time.time()
    proc = subprocess.run([REF_BIN, "-f", "case.in"], cwd=wd, capture_output=True,
                          text=True, timeout=1800)
    wall = time.time() - t0
    log = proc.stdout
    if proc.returncode != 0:
        sys.stderr.write(log[-4000:] + proc.stderr[-4000:])
        raise RuntimeError(f"reference exited {proc.returncode} on {case.name}")

    ll = [float(v) for v in re.findall(r"Iteration \d+: lrate [-0-9.eE+]+ LL ([-0-9.eE+naninf]+)", log)]
    lrate = [float(v) for v in re.findall(r"Iteration \d+: lrate ([-0-9.eE+]+) LL", log)]
    ms = [int(v) for v in re.findall(r"Iteration \d+ times = \d+ ticks, (\d+) ms", log)]
    newton_fallbacks = log.count("Hessian non positive definite")
    res = dict(case=case.name, n=case.n, T=case.T, M=case.M, m=case.m,
               maxiter=case.maxiter, ll=np.array(ll), lrate=np.array(lrate),
               iter_ms=np.array(ms), wall_s=wall, newton_fallbacks=newton_fallbacks,
               xs_digest=digest(prep["xs"][:1000]))
    if not keep_arrays:
        return res

    n, M, m, T = case.n, case.M, case.m, case.T
    rd = lambda name, cnt: np.fromfile(os.path.join(wd, "out", name), dtype=np.float64, count=cnt)
    res.update(
        W=rd("W.fdt", M * n * n).reshape(M, n, n),
        A=rd("A.fdt", M * n * n).reshape(M, n, n),
        c=rd("c.fdt", M * n).reshape(M, n),
        gm=rd("gm.fdt", M),
        alpha=rd("alpha.fdt", M * m * n).reshape(M, m, n),
        mu=rd("mu.fdt", M * m * n).reshape(M, m, n),
        beta=rd("beta.fdt", M * m * n).reshape(M, m, n),
        rho=rd("rho.fdt", M * m * n).reshape(M, m, n),
        llfile=rd("ll.fdt", case.maxiter),
        sphere=rd("sphere.fdt", n * n).reshape(n, n),
        ltall_stride=rd("ltall.fdt", M * T).reshape(M, T)[:, ::97].copy(),
        ldetS=np.fromfile(os.path.join(wd, "datasets", "INPUT-ldets.fdt"), dtype=np.float64),
    )
    its = [k for k in case.keep_iters if k <= case.maxiter]
    res["keep_iters"] = np.array(its)
    for key, fn, shape in (("A", "A", (n, n)), ("c", "C", (n,)), ("alpha", "ALPHA", (m, n)),
                           ("mu", "MU", (m, n)), ("beta", "BETA", (m, n)), ("rho", "RHO", (m, n))):
        arr = np.empty((len(its), M) + shape)
        for a, it in enumerate(its):
            for h in range(M):
                p = os.path.join(wd, "datasets", f"FINAL-{fn}-i{it}-m{h}.fdt")
                arr[a, h] = np.fromfile(p, dtype=np.float64, count=int(np.prod(shape))).reshape(shape)
        res["iter_" + key] = arr
    return res


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="+")
    ap.add_argument("--out", required=True)
    ap.add_argument("--time-only", action="store_true")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if not os.path.exists(REF_BIN):
        raise SystemExit("build the reference first: make -C oracle ref")
    with tempfile.TemporaryDirectory(prefix="amica_ref_") as work:
        for name in args.cases:
            case = TIMING[name] if args.time_only else CASES[name]
            res = run_case(case, work, keep_arrays=not args.time_only)
            if args.time_only:
                print(f"{name}: n={case.n} T={case.T} M={case.M} iter_ms={list(res['iter_ms'])} "
                      f"LL={list(res['ll'])}", flush=True)
                with open(os.path.join(args.out, f"ref_time_{name}.txt"), "w") as f:
                    f.write(repr({k: (v.tolist() if isinstance(v, np.ndarray) else v)
                                  for k, v in res.items()}) + "\n")
            else:
                np.savez_compressed(os.path.join(args.out, f"ref_{name}.npz"), **res)
                print(f"{name}: {len(res['ll'])} iterations, LL[-1]={res['ll'][-1]:.12f}, "
                      f"wall {res['wall_s']:.1f}s, newton fallbacks {res['newton_fallbacks']}",
                      flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
