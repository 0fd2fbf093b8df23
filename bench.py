#!/usr/bin/env python
"""Benchmark of the CPU-free Jacobi hot path on B200.

Workload (one "step"): 100 persistent FP64 Jacobi 3d7p sweeps of the 512^3
periodic problem (x faces sin(2 pi y/(ny-1)) sin(2 pi z/(nz-1)), periodic in
y and z), i.e. one solve of that configuration; successive steps continue
from the previous grid, which does not change the work.  Metric: GLUP/s
(interior lattice-point updates per second, 510^3 per sweep).

  value  device-resident throughput: CUDA events on the library's stream
         around K steps (each step = edge preset + one cooperative launch).
  e2e    the same metric through the C ABI with pinned host buffers:
         cfm_jacobi_run_host = H2D of the grid, the sweeps, D2H of the result.
  roofline  16 algorithmic bytes per LUP over the measured launch time,
         against MEASURED_PEAKS.json's copy bandwidth.
  cpu_baseline  the oracle's FP64 sweep loop (C/OpenMP) on the host cores.

  secondary  (one GPU, after the timed regions; --no-secondary skips it) the
         other configurations measured in the same run, each with its own
         CPU baseline from the oracle on the host cores: config 1 (2D 1024^2
         FP64, 1000 sweeps, final-grid L2 norm), config 3 (CG on 128^3
         Poisson to 1e-8: standard, pipelined, FP32 with FP64 reliable
         updates) and config 4 (512^2 variable-coefficient system to 1e-8:
         plain FP64 persistent and pipelined CG, Jacobi-smoothed and learned
         flexible PCG, the network trained first and its time stated).

--gpus N runs N independent replicas (one per GPU, no data exchange; weak
scaling); rank 0 prints the JSON line.  --impl reference times the host
restatement of the reference's single-GPU sweep (the reference ships no CPU
Jacobi of its own) on the host cores with the same metric.

Other workloads (--workload, one JSON line each, same keys):
  jacobi2d   config 1: the 1024^2 FP64 2D problem, 1000 sweeps (on chip).
  jacobi3d_fp32  the same 512^3 problem in FP32 (8 B/LUP) and its error after
             100 sweeps against the FP64 (bit-exact) result.
  cg128      CG on the 128^3 7-point Poisson CSR system to a true relative
             residual of 1e-8: standard, pipelined and FP32-inner/FP64-
             refinement persistent kernels (time to solution, GB/s).
  varcoef512 the 512^2 variable-coefficient system to 1e-8: plain FP64
             persistent CG vs flexible PCG with the Jacobi-smoothed and the
             learned (trained here first, on the 2x-restricted residual)
             preconditioner.
  unet       the preconditioner network: forward (batch 1) at 512^2,
             TFLOP/s against the measured BF16 peak.
  batch256   256 uneven variable-coefficient systems (192 2D, sides
             log-uniform in [64, 512]; 64 3D, sides in [32, 128]) solved to
             1e-8 in one persistent launch (CUDA graph, autotuned plan,
             Jacobi-polynomial PCG) vs one plain persistent CG solve per
             launch; solves/s.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cpu-free-model_b200"))

N = 512
NITER = 100
LUP_PER_SWEEP = (N - 2) ** 3
BYTES_PER_LUP = 16.0  # FP64: one 8-byte read + one 8-byte write per interior point
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "jacobi3d_persistent_512_fp64.md")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--workload", choices=["jacobi3d", "jacobi2d", "jacobi3d_fp32", "cg128", "varcoef512", "fpcg512",
                                           "unet", "unet_train", "batch256", "cpufree"],
                    default="jacobi3d")
    return ap.parse_args()


def peak_bf16(sustained=False):
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["bf16_tflops_sustained" if sustained else "bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def unet_flops(H, W):
    """2 * 9 * Cin * Cout * pixels over the network's convolutions (forward)."""
    layers = [(2, 32, 0), (32, 64, 1), (64, 128, 2), (128, 256, 3), (256, 128, 3), (128, 64, 2),
              (64, 32, 1), (32, 32, 0), (32, 1, 0)]
    return sum(18.0 * ci * co * (H >> l) * (W >> l) for ci, co, l in layers)


def line(metric, value, unit, args, ms, config, higher=True, extra=None, dtype="f64"):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": higher, "scaling": "weak",
         "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": config}
    if extra:
        d.update(extra)
    print(json.dumps(d), flush=True)


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def measure_jacobi2d(steps, warmup, cfm, cpu=True):
    """Config 1: 1024^2 FP64, 1000 sweeps of the reference 2D problem (x
    columns sin(2 pi y/(ny-1)), periodic y), 16 MiB per grid, so it runs on
    chip.  GLUP/s of the resident (PERKS-style) and persistent kernels, the
    final grid's L2 norm, and the oracle's sweep loop as the CPU baseline."""
    import numpy as np
    n2, it = 1024, 1000
    lup = (n2 - 2) ** 2 * it
    peak, kind = peak_hbm()
    res, grid = {}, None
    for impl, name in ((cfm.JACOBI_RESIDENT, "resident"), (cfm.JACOBI_PERSISTENT, "persistent")):
        with cfm.Jacobi(2, n2, n2, 1, cfm.FP64, 1, impl) as j:
            j.load_problem(cfm.PROBLEM_REF)
            j.run(it)
            g = j.download()
            if grid is None:
                grid = g
            same = bool(np.array_equal(g, grid))
            for _ in range(warmup):
                j.run(it)
            ts = [j.run(it).seconds for _ in range(steps)]
        t = statistics.median(ts)
        res[name] = {"ms": t * 1e3, "glups": lup / t * 1e-9, "us_per_sweep": t / it * 1e6,
                     "hbm_equivalent_frac": 16.0 * lup / t * 1e-9 / peak, "same_grid_as_first": same}
    out = {"workload": "jacobi2d5p_1024^2_fp64_1000_sweeps", "impls": res,
           "best": max(res, key=lambda k: res[k]["glups"]),
           "final_l2_norm": float(np.sqrt(np.sum(grid.astype(np.longdouble) ** 2))),
           "timing": "median of steps, CUDA events around one 1000-sweep launch (grid on chip)",
           "peak_hbm_gbs": peak, "peak_kind": kind}
    if cpu:
        oracle = _oracle()
        a = oracle.jacobi2d_init(n2, n2, np.float64)
        t0 = time.perf_counter()
        want = oracle.jacobi2d(a, it)
        tc = time.perf_counter() - t0
        out["matches_oracle_bitexact"] = bool(np.array_equal(grid, want))
        out["cpu_baseline"] = {"value": lup / tc * 1e-9, "unit": "GLUP/s", "cores": oracle.max_threads(),
                               "kind": "port", "sample": "the whole 1000-sweep solve (oracle call, OpenMP)"}
    return out


def workload_jacobi2d(args, cfm):
    r = measure_jacobi2d(args.steps, args.warmup, cfm, cpu=not args.no_cpu_baseline)
    best = r["impls"][r["best"]]
    extra = {"roofline": {"bound": "on-chip (HBM-equivalent bytes)", "achieved": 16.0 * best["glups"],
                          "peak": r["peak_hbm_gbs"], "unit": "GB/s", "frac": best["hbm_equivalent_frac"],
                          "peak_kind": r["peak_kind"]}}
    if "cpu_baseline" in r:
        extra["cpu_baseline"] = r["cpu_baseline"]
    line("Jacobi 2d5p 1024^2 FP64 GLUP/s", best["glups"], "GLUP/s", args, best["ms"], r, extra=extra)


def measure_cg128(steps, warmup, cfm, cpu=True):
    """Config 3: CG on the 128^3 7-point Poisson CSR system to a true
    relative residual of 1e-8, three persistent kernels; the oracle's FP64 CG
    (C/OpenMP) on the host cores as the CPU baseline."""
    rowptr, col, val = cfm.poisson3d(128)
    A = cfm.CSR(rowptr, col, val)
    b = A.spmv(cfm.uniform(0, A.n))
    peak, kind = peak_hbm()
    res = {}
    for impl, name in ((cfm.CG_PERSISTENT, "standard"), (cfm.CG_PERSISTENT_PIPELINED, "pipelined"),
                       (cfm.CG_MIXED, "fp32_cg_fp64_reliable_updates")):
        cg = cfm.CG(A, impl, 20000, 1e-8)
        for _ in range(warmup):
            cg.solve(b)
        ts = []
        for _ in range(steps):
            x, st = cg.solve(b)
            ts.append(st.seconds)
        cg.close()
        t = statistics.median(ts)
        res[name] = {"ms": t * 1e3, "iterations": st.iterations, "refinements": st.refinements,
                     "true_relres": st.residual, "algorithmic_gbs": st.bytes / t * 1e-9,
                     "hbm_frac": st.bytes / t * 1e-9 / peak}
    A.close()
    out = {"workload": "cg_poisson7_128^3_csr_tol1e-8", "n": A.n, "nnz": len(val), "impls": res,
           "best": min(res, key=lambda k: res[k]["ms"]),
           "timing": "median of steps, CUDA events, H2D of b and D2H of x included",
           "peak_hbm_gbs": peak, "peak_kind": kind}
    if cpu:
        oracle = _oracle()
        t0 = time.perf_counter()
        _, _, it, rr = oracle.cg(rowptr, col, val, b, 20000, 1e-8)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": tc * 1e3, "unit": "ms", "cores": oracle.max_threads(), "kind": "port",
                               "iterations": it, "true_relres": rr,
                               "sample": "one whole FP64 CG solve to 1e-8 (oracle call, OpenMP)"}
    return out


def workload_cg128(args, cfm):
    r = measure_cg128(args.steps, args.warmup, cfm, cpu=not args.no_cpu_baseline)
    best = r["impls"][r["best"]]
    extra = {"cpu_baseline": r["cpu_baseline"]} if "cpu_baseline" in r else None
    line("CG 128^3 Poisson CSR time to 1e-8 FP64 true relative residual", best["ms"], "ms", args,
         best["ms"], r, higher=False, extra=extra)


def workload_jacobi3d_fp32(args, cfm):
    """The 512^3 periodic problem in FP32 (8 B/LUP), with its max-abs and
    relative L2 error after 100 sweeps against the FP64 sweep (which is bit
    for bit the reference's)."""
    import numpy as np
    peak, kind = peak_hbm()
    j64 = cfm.Jacobi(3, N, N, N, cfm.FP64, 1, cfm.JACOBI_PERSISTENT)
    j64.load_problem(cfm.PROBLEM_CONFIG)
    j64.run(NITER)
    ref = j64.download()
    j64.close()
    j = cfm.Jacobi(3, N, N, N, cfm.FP32, 1, cfm.JACOBI_PERSISTENT)
    j.load_problem(cfm.PROBLEM_CONFIG)
    best, _ = j.autotune(NITER // 2)
    tuned = cfm.variant_info(best) if best >= 0 else None
    j.load_problem(cfm.PROBLEM_CONFIG)
    j.run(NITER)
    got = j.download().astype(np.float64)
    err = got - ref
    inner = (slice(1, -1),) * 3
    max_abs = float(np.abs(err[inner]).max())
    rel_l2 = float(np.linalg.norm(err[inner]) / np.linalg.norm(ref[inner]))
    del got, err, ref
    for _ in range(args.warmup):
        j.run(NITER)
    secs = []
    for _ in range(args.steps):
        secs.append(j.run(NITER).seconds)
    j.close()
    t = statistics.median(secs)
    glups = NITER * LUP_PER_SWEEP / t / 1e9
    achieved = 8.0 * NITER * LUP_PER_SWEEP / t / 1e9
    line("Jacobi 3d7p 512^3 FP32 GLUP/s", glups, "GLUP/s", args, t * 1e3,
         {"workload": "jacobi3d7p_512^3_fp32_periodic", "niter_per_step": NITER,
          "tuned": None if tuned is None else {"variant": best, "consumer_warps": tuned[0],
                                               "rows_per_warp": tuned[1], "stages": tuned[2],
                                               "sweeps_per_pass": tuned[3]},
          "error_vs_fp64_after_100_sweeps": {"max_abs": max_abs, "rel_l2": rel_l2},
          "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "peak_kind": kind, "bytes_per_lup": 8},
          "timing": "median of steps, CUDA events around one 100-sweep launch"},
         dtype="f32")


def measure_varcoef512(steps, warmup, cfm, cpu=True, variants=((8, 2), (8, 3), (8, 4), (8, 1), (4, 1))):
    """Config 4: the 512^2 variable-coefficient system to 1e-8.  Plain FP64
    persistent and pipelined CG, Jacobi-smoothed FPCG, and learned FPCG (the
    network trained here first; its training time is reported); the oracle's
    plain FP64 CG on the stencil operator as the CPU baseline."""
    N = 512
    k, f = cfm.varcoef_problem((N, N), 0)
    S = cfm.Stencil(k)
    out = {}

    def timed(solver):
        for _ in range(warmup):
            solver()
        ts, st = [], None
        for _ in range(steps):
            x, st = solver()
            ts.append(st.seconds)
        return statistics.median(ts), st

    for impl, name in ((cfm.CG_PERSISTENT, "plain_fp64_persistent_cg"),
                       (cfm.CG_PERSISTENT_PIPELINED, "plain_fp64_pipelined_cg")):
        cg = cfm.CG(S, impl, 50000, 1e-8)
        t, st = timed(lambda: cg.solve(f.ravel()))
        out[name] = {"ms": t * 1e3, "iterations": st.iterations, "true_relres": st.residual}
    fj = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=4)
    t, st = timed(lambda: fj.solve(f))
    out["fpcg_jacobi4"] = {"ms": t * 1e3, "iterations": st.iterations, "true_relres": st.residual,
                           "fallback": st.refinements, "truncation": 1}
    # the learned preconditioner: the U-Net on the 2x-restricted residual
    # (256^2), trained here on plain-CG pairs of 100 fresh 512^2 systems
    net = cfm.UNet(N // 2, N // 2, max_batch=8, seed=7)
    net.set_validation(1000, 1)  # keep the checkpoint fastest on a held-out system (not this one)
    t0 = time.perf_counter()
    info = net.train_varcoef(100, 19, 1000, 16, 8, 1e-3, smooth=4, coarsen=2)
    info["wall_s"] = time.perf_counter() - t0
    info["kept_epoch"], info["validation_ms"] = net.validation()
    for m, per in variants:
        fl = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8, truncation=m, net_period=per)
        t, st = timed(lambda: fl.solve(f))
        out[f"fpcg_learned_m{m}_p{per}"] = {"ms": t * 1e3, "iterations": st.iterations,
                                            "true_relres": st.residual, "fallback": st.refinements,
                                            "truncation": m, "network_every": per}
        fl.close()
    # learned + mixed: the defaults with FP32 Krylov vectors and FP64 reliable updates
    fm = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8, precision=cfm.FP32)
    t, st = timed(lambda: fm.solve(f))
    out["fpcg_learned_mixed_m8_p2"] = {"ms": t * 1e3, "iterations": st.iterations, "true_relres": st.residual,
                                       "fallback": st.refinements, "reliable_updates": fm.reliable_updates(),
                                       "truncation": 8, "network_every": 2, "delta": 0.1}
    fm.close()
    head = out["fpcg_learned_mixed_m8_p2"]  # learned + mixed, the configuration the target names
    head.update({"training": info, "training_pairs": 100 * 20, "network_grid": [N // 2, N // 2],
                 "forward_ms_b1": net.time_forward(1, 20)})
    net.close()
    base = out["plain_fp64_persistent_cg"]["ms"]
    fastest_plain = min(base, out["plain_fp64_pipelined_cg"]["ms"])
    r = {"workload": "varcoef2d_512^2_grf_sigma1_corr16_tol1e-8", "solver": "fpcg_learned_mixed_m8_p2",
         "ms": head["ms"],
         "speedup_vs_plain_persistent_cg": base / head["ms"],
         "speedup_vs_fastest_plain_cg": fastest_plain / head["ms"],
         "speedup_jacobi_only_vs_plain": base / out["fpcg_jacobi4"]["ms"], "solvers": out,
         "learned_fp64_krylov_ms": out["fpcg_learned_m8_p2"]["ms"],
         "precision": "FP32 Krylov vectors with FP64 reliable updates, FP64 dots / alpha / beta / true "
                      "residual; FP32 smoothing; BF16 network (FP32 accumulate)",
         "timing": "median of steps, CUDA events around the whole solve incl. H2D b / D2H x"}
    if cpu:
        oracle = _oracle()
        c = cfm.varcoef_coeffs(k)
        t0 = time.perf_counter()
        _, _, it, _, rr = oracle.krylov_stencil(2, (N, N, 1), c, f.ravel(), 0, 50000, 1e-8)
        tc = time.perf_counter() - t0
        r["cpu_baseline"] = {"value": tc * 1e3, "unit": "ms", "cores": oracle.max_threads(), "kind": "port",
                             "iterations": it, "true_relres": rr,
                             "sample": "one whole plain FP64 CG solve to 1e-8 (oracle call, OpenMP)"}
    return r


def workload_varcoef512(args, cfm):
    r = measure_varcoef512(args.steps, args.warmup, cfm, cpu=not args.no_cpu_baseline)
    extra = {"cpu_baseline": r["cpu_baseline"]} if "cpu_baseline" in r else None
    line("512^2 variable-coefficient time to 1e-8 FP64 true relative residual, learned + mixed FPCG", r["ms"],
         "ms", args, r["ms"], r, higher=False, extra=extra)


def workload_fpcg512(args, cfm):
    """The preconditioner's solver kernels without the network: Jacobi-
    smoothed FPCG (4 FP32 sweeps before and after) on the config-4 512^2
    system to 1e-8, FP64 and mixed Krylov vectors, one kernel per phase and
    the device loop (no training: a quick case for the solver kernels)."""
    N = 512
    k, f = cfm.varcoef_problem((N, N), 0)
    S = cfm.Stencil(k)
    res = {}
    for prec, pname in ((cfm.FP64, "fp64"), (cfm.FP32, "mixed")):
        for loop in (0, 1):
            fp = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=4, precision=prec)
            fp.set_device_loop(loop)
            for _ in range(max(args.warmup, 1)):
                fp.solve(f)
            ts = []
            for _ in range(max(args.steps, 3)):
                x, st = fp.solve(f)
                ts.append(st.seconds)
            fp.close()
            t = statistics.median(ts)
            res[f"{pname}_{'device_loop' if loop else 'kernels'}"] = {
                "ms": t * 1e3, "iterations": st.iterations, "us_per_iteration": t * 1e6 / st.iterations,
                "true_relres": st.residual}
    best = min(res, key=lambda q: res[q]["ms"])
    line("512^2 variable-coefficient time to 1e-8, Jacobi-smoothed FPCG", res[best]["ms"], "ms", args,
         res[best]["ms"], {"workload": "varcoef2d_512^2_fpcg_jacobi4_tol1e-8", "best": best, "solvers": res,
                           "timing": "median of steps, CUDA events around the whole solve incl. H2D b / D2H x"},
         higher=False, dtype="f64")


def secondary(cfm):
    """The other configurations in the default run (rank 0, one GPU): short
    repeats (3 timed after 1 warm-up), each with its CPU baseline."""
    out, t0 = {}, time.perf_counter()
    for name, fn in (("config1_jacobi2d_1024_fp64", lambda: measure_jacobi2d(3, 1, cfm)),
                     ("config3_cg_poisson128", lambda: measure_cg128(3, 1, cfm)),
                     ("config4_varcoef512", lambda: measure_varcoef512(3, 1, cfm, variants=((8, 2),)))):
        t1 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:  # one failing config must not hide the headline
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t1
    v = out.get("config4_varcoef512", {})
    if "ms" in v:
        out["learned_fpcg_vs_plain_fp64_cg"] = v["speedup_vs_plain_persistent_cg"]
        out["learned_fpcg_vs_fastest_plain_cg"] = v["speedup_vs_fastest_plain_cg"]
    out["wall_s"] = time.perf_counter() - t0
    return out


def workload_unet(args, cfm):
    import numpy as np
    N = 512
    net = cfm.UNet(N, N, max_batch=8, seed=1)
    x = np.random.default_rng(0).normal(size=(1, N, N, 2)).astype(np.float32)
    flop = unet_flops(N, N)
    for _ in range(args.warmup):
        net.forward(x)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.forward(x)
    t_host = (time.perf_counter() - t0) / args.steps
    dev = {b: net.time_forward(b, max(args.steps, 5)) * 1e-3 for b in (1, 8)}
    peak, kind = peak_bf16()
    line("U-Net forward 512^2 batch 1, device-resident", flop / dev[1] / 1e12, "TFLOP/s", args,
         dev[1] * 1e3, {"workload": "unet4_32ch_512^2_b1_forward", "gflop_per_apply": flop / 1e9,
                        "batch8_ms": dev[8] * 1e3, "batch8_tflops": 8 * flop / dev[8] / 1e12,
                        "host_call_ms_incl_copies": t_host * 1e3,
                        "peak_bf16_tflops": peak, "peak_kind": kind,
                        "roofline_frac_batch1": flop / dev[1] / 1e12 / peak,
                        "timing": "CUDA events around unet forward passes on device buffers"},
         dtype="bf16")


def workload_unet_train(args, cfm):
    """One training step of the learned preconditioner's network at its
    training shape (256^2, batch 8): forward, backward (data and weight
    gradients on the tensor cores) and Adam, on a scratch network."""
    N, B = 256, 8
    net = cfm.UNet(N, N, max_batch=B, seed=11)
    net.time_train_step(B, max(args.warmup, 1))
    ms = net.time_train_step(B, max(args.steps, 5))
    flop = 3 * B * unet_flops(N, N)  # forward + backward-data + weight gradient
    peak, kind = peak_bf16()
    line("U-Net training step 256^2 batch 8, device-resident", flop / (ms * 1e-3) / 1e12, "TFLOP/s", args,
         ms, {"workload": "unet4_32ch_256^2_b8_train_step", "gflop_per_step": flop / 1e9,
              "peak_bf16_tflops": peak, "peak_kind": kind,
              "roofline_frac": flop / (ms * 1e-3) / 1e12 / peak,
              "timing": "CUDA events around forward + backward + Adam on device buffers"},
         dtype="bf16")


def workload_cpufree(args, cfm):
    """The reference's own 1-GPU comparison: CPU-controlled (a host launch
    per sweep / per CG phase) against CPU-free (one persistent launch), on
    the reference's cases: 2D Jacobi 256^2 FP32 (its launch-bound weak-scaling
    point) and 16384^2 FP32, and CG on its default random tridiagonal matrix
    (n = 20,971,520, b = ones, 1000 iterations, no tolerance exit)."""
    import statistics as stt
    out = {}
    for n2, niter in ((256, 20000), (16384, 200)):
        row = {}
        for impl, name in ((cfm.JACOBI_HOST_LOOP, "host_loop"), (cfm.JACOBI_PERSISTENT, "persistent"),
                           (cfm.JACOBI_RESIDENT, "resident")):
            j = cfm.Jacobi(2, n2, n2, 1, cfm.FP32, 1, impl)
            if impl == cfm.JACOBI_RESIDENT and j.launch_shape()[1] != 1024:
                j.close()
                continue  # does not fit on chip: no resident form at this size
            j.load_problem(cfm.PROBLEM_REF)
            for _ in range(max(args.warmup, 1)):
                j.run(niter)
            ts = [j.run(niter).seconds for _ in range(max(args.steps, 3))]
            t = stt.median(ts)
            row[name] = {"us_per_sweep": t / niter * 1e6, "glups": (n2 - 2) ** 2 * niter / t / 1e9}
            j.close()
        out[f"jacobi2d_{n2}_fp32"] = row
    n = 20971520
    rowptr, col, val = cfm.tridiag(n)
    A = cfm.CSR(rowptr, col, val)
    cgr = {}
    for impl, name in ((cfm.CG_DISCRETE, "cpu_controlled_standard"), (cfm.CG_PERSISTENT, "cpu_free_standard"),
                       (cfm.CG_PERSISTENT_PIPELINED, "cpu_free_pipelined")):
        cg = cfm.CG(A, impl, 1000, 0.0)
        cg.solve(None)
        ts = [cg.solve(None)[1].seconds for _ in range(max(args.steps, 3))]
        cgr[name] = {"s_per_1000_iterations": stt.median(ts)}
        cg.close()
    out["cg_tridiag_20971520"] = cgr
    speed = cgr["cpu_controlled_standard"]["s_per_1000_iterations"] / cgr["cpu_free_standard"]["s_per_1000_iterations"]
    j256 = out["jacobi2d_256_fp32"]
    line("CPU-free over CPU-controlled speedup, CG standard on the reference's tridiagonal matrix", speed, "x",
         args, cgr["cpu_free_standard"]["s_per_1000_iterations"] * 1e3,
         {"workload": "cpufree_vs_cpu_controlled_1gpu", "cases": out,
          "jacobi2d_256_host_loop_over_persistent": j256["host_loop"]["us_per_sweep"] / j256["persistent"]["us_per_sweep"],
          "jacobi2d_256_host_loop_over_resident": j256["host_loop"]["us_per_sweep"] / j256["resident"]["us_per_sweep"],
          "reference_a100": {"jacobi2d_256_us_per_iter_copy_vs_design2": [8.9, 2.4],
                             "cg_tridiag_1000_iter_s_discrete_vs_persistent": [19.99, 10.66]},
          "timing": "CUDA events per call (b and x copies included for CG), median of steps"})


def batch_bytes_per_iteration(dims, n, smooth, word):
    """Algorithmic bytes of one PCG iteration of one batched system: the
    operator pass (c coefficient arrays + p read + s write), the x / r update
    (4 reads, 2 writes), the damped-Jacobi sweeps (first: r, d read, z write;
    each further one: z, r and the c arrays read, z written; <r, z> fused into
    the last) and p = z + beta p (2 reads, 1 write); c = dims + 1."""
    c = dims + 1
    sweeps = 3 + max(0, smooth - 1) * (c + 3)
    return word * n * ((c + 2) + 6 + sweeps + 3)


def workload_batch256(args, cfm):
    import numpy as np
    t0 = time.perf_counter()
    systems = cfm.uneven_systems(192, 64, seed=5)
    gen_s = time.perf_counter() - t0
    peak, kind = peak_hbm()
    B = cfm.Batch(systems)
    smooth = 4
    B.set_solver(smooth=smooth, maxiter=20000, tol=1e-8)
    methods = {}
    for name, prec, delta, word in (("pcg_fp64", cfm.FP64, 0.1, 8),
                                    ("pcg_fp32_fp64_reliable_updates_delta0.1", cfm.FP32, 0.1, 4),
                                    ("pcg_fp32_fp64_reliable_updates_delta0.01", cfm.FP32, 0.01, 4)):
        B.set_precision(prec, 0, delta)
        tune_ms = B.autotune()
        for _ in range(args.warmup):
            B.solve()
        ts = []
        for _ in range(args.steps):
            it, stt, rr, st = B.solve()
            ts.append(st.seconds)
        t = statistics.median(ts)
        nbytes = sum(batch_bytes_per_iteration(k.ndim, k.size, smooth, word) * int(v)
                     for (k, _), v in zip(systems, it))
        methods[name] = {"ms": t * 1e3, "solves_per_s": len(systems) / t,
                         "all_converged": bool((stt == cfm.OK).all()), "max_true_relres": float(rr.max()),
                         "iterations": {"min": int(it.min()), "median": float(np.median(it)),
                                        "max": int(it.max()), "sum": int(it.sum())},
                         "fp64_updates": int(st.refinements),
                         "algorithmic_gbs": nbytes / t * 1e-9, "hbm_frac": nbytes / t * 1e-9 / peak,
                         "autotune_best_ms": tune_ms, "per_system_iterations": [int(v) for v in it]}
    best = min(methods, key=lambda m: methods[m]["ms"])
    t = methods[best]["ms"] * 1e-3
    # one plain persistent FP64 CG solve per launch, same tolerance
    t_plain, it_plain = 0.0, []
    for k, f in systems:
        S = cfm.Stencil(k)
        x, sp = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-8).solve(f.ravel())
        t_plain += sp.seconds
        it_plain.append(sp.iterations)
    n = len(systems)
    learned = batch_learned(args, cfm, systems, methods["pcg_fp32_fp64_reliable_updates_delta0.1"], smooth)
    if learned.get("ms") and learned["ms"] < methods[best]["ms"]:
        best, t = "learned_split", learned["ms"] * 1e-3
    line("256 uneven variable-coefficient systems to 1e-8: aggregate solves/s", n / t, "solves/s", args,
         t * 1e3, {"workload": "batch_192x2d_64..512_64x3d_32..128_varcoef_tol1e-8",
                   "systems": n, "cells": int(sum(k.size for k, _ in systems)),
                   "method": best, "methods": methods, "learned": learned,
                   "iterations_plain": {"min": int(min(it_plain)), "median": float(np.median(it_plain)),
                                        "max": int(max(it_plain))},
                   "plain_one_solve_per_launch_ms": t_plain * 1e3,
                   "speedup_vs_one_plain_solve_per_launch": t_plain / t,
                   "generation_s": gen_s, "peak_hbm_gbs": peak, "peak_kind": kind,
                   "launch": "one cooperative launch in a CUDA graph per step; 4 damped-Jacobi sweeps"})


def batch_learned(args, cfm, systems, poly, smooth, side_min=256):
    """Config 5 with the learned preconditioner: the network of config 4
    (trained here on 100 fresh 512^2 systems, its 256^2 grid x 2) solves the
    2D members of side >= side_min together in one FPCG device loop (each
    member in the 512^2 frame, learned + mixed precision, the network at
    batch up to 64), the other members (smaller 2D, all 3D) run in the
    persistent Jacobi-polynomial mixed-precision kernel; both back to back on
    one stream, timed together."""
    import numpy as np
    N2 = 512
    big = [i for i, (k, _) in enumerate(systems) if k.ndim == 2 and min(k.shape) >= side_min]
    rest = [i for i in range(len(systems)) if i not in big]
    net = cfm.UNet(N2 // 2, N2 // 2, max_batch=64, seed=7)
    net.set_validation(1000, 1)
    t0 = time.perf_counter()
    info = net.train_varcoef(100, 19, 1000, 16, 8, 1e-3, smooth=smooth, coarsen=2)
    info["wall_s"] = time.perf_counter() - t0
    info["kept_epoch"], info["validation_ms"] = net.validation()
    FB = cfm.FPCGBatch([systems[i][0] for i in big], net, maxiter=20000, tol=1e-8, precision=cfm.FP32)
    fb = [systems[i][1] for i in big]
    B = cfm.Batch([systems[i] for i in rest])
    B.set_solver(smooth=smooth, maxiter=20000, tol=1e-8)
    B.set_precision(cfm.FP32, 0, 0.1)
    B.autotune()
    for _ in range(args.warmup):
        FB.solve(fb)
        B.solve()
    ts, tl, tp = [], [], []
    for _ in range(args.steps):
        _, it_l, st_l, rr_l, sl = FB.solve(fb)
        it_p, st_p, rr_p, sp = B.solve()
        tl.append(sl.seconds)
        tp.append(sp.seconds)
        ts.append(sl.seconds + sp.seconds)
    t = statistics.median(ts)
    poly_it = poly["per_system_iterations"]
    it_all = [0] * len(systems)
    for j, i in enumerate(big):
        it_all[i] = int(it_l[j])
    for j, i in enumerate(rest):
        it_all[i] = int(it_p[j])
    out = {"ms": t * 1e3, "solves_per_s": len(systems) / t,
           "learned_members": len(big), "polynomial_members": len(rest), "side_min": side_min,
           "learned_ms": statistics.median(tl), "polynomial_ms": statistics.median(tp),
           "all_converged": bool((st_l == cfm.OK).all() and (st_p == cfm.OK).all()),
           "max_true_relres": float(max(rr_l.max(), rr_p.max())),
           "learned_iterations": [int(v) for v in it_l],
           "same_members_polynomial_iterations": [int(poly_it[i]) for i in big],
           "learned_over_polynomial_iterations": float(np.sum(it_l) / max(1, sum(poly_it[i] for i in big))),
           "reliable_updates_learned": FB.reliable_updates(), "per_system_iterations": it_all,
           "training": info, "network_batch": 64,
           "precision": "learned members: FP32 Krylov vectors + FP64 reliable updates, BF16 network; "
                        "others: FP32 PCG + FP64 reliable updates"}
    out["learned_ms"] *= 1e3
    out["polynomial_ms"] *= 1e3
    FB.close()
    B.close()
    net.close()
    return out


def main_workload(args):
    import torch  # noqa: F401  (device plumbing only)
    import cfm
    {"cg128": workload_cg128, "jacobi2d": workload_jacobi2d, "jacobi3d_fp32": workload_jacobi3d_fp32,
     "varcoef512": workload_varcoef512, "fpcg512": workload_fpcg512,
     "unet": workload_unet, "unet_train": workload_unet_train, "cpufree": workload_cpufree,
     "batch256": workload_batch256}[args.workload](args, cfm)
    return 0


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch():
    """DRAM bytes per persistent launch from the committed ncu summary, if any."""
    try:
        for line in open(TRAFFIC_FILE):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def same_box_copy_gbs(torch):
    """Copy bandwidth of this box, measured like the driver's peak (1 Gi BF16
    elements, b.copy_(a), read + write bytes, best of 10, CUDA events): the
    context for the roofline fraction, whose denominator stays the driver's
    measured peak."""
    a = torch.empty(1 << 30, dtype=torch.bfloat16, device="cuda")
    b = torch.empty_like(a)
    a.fill_(1.0)
    best = 0.0
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * a.numel() * 2 / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_baseline():
    """Oracle FP64 sweep loop on the host cores, sized to ~10 s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    t1 = oracle.jacobi3d_bench(N, 1)
    k = int(max(1, min(60, 10.0 / max(t1, 1e-3))))
    t = oracle.jacobi3d_bench(N, k)
    return {"value": k * LUP_PER_SWEEP / t / 1e9, "unit": "GLUP/s", "cores": oracle.max_threads(),
            "kind": "port",
            "sample": f"{k} FP64 sweeps of the 512^3 periodic problem, sweep loop only (OpenMP)"}


class Ranks:
    """What the replicas share: a barrier and the max over ranks of a time
    (CUDA tensors over NCCL on the GPUs; CPU tensors over gloo in the tests).
    With one rank both are no-ops."""

    def __init__(self, world, device):
        self.world, self.device = world, device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())


def whole_job_rate(world, steps, units_per_step, seconds):
    """Units per second over all replicas: every rank did `steps` steps of
    `units_per_step` units, timed by the slowest rank (`seconds`)."""
    return world * steps * units_per_step / seconds


def run_reference(args, rank):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    sweeps = 1
    for _ in range(args.warmup):
        oracle.jacobi3d_bench(N, sweeps)
    t = 0.0
    for _ in range(args.steps):
        t += oracle.jacobi3d_bench(N, sweeps)
    v = args.steps * sweeps * LUP_PER_SWEEP / t / 1e9
    cores = oracle.max_threads()
    line = {
        "impl": "reference", "metric": "Jacobi 3d7p 512^3 FP64 GLUP/s", "value": v, "unit": "GLUP/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "jacobi3d7p_512^3_fp64_periodic", "nx": N, "ny": N, "nz": N,
                   "sweeps_per_step": sweeps, "impl": "host C/OpenMP restatement of single_gpu()"},
        "cpu_baseline": {"value": v, "unit": "GLUP/s", "cores": cores, "kind": "port",
                         "sample": f"{sweeps} sweep(s) of 512^3 per step"},
        "e2e": {"value": v, "unit": "GLUP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.workload != "jacobi3d":
        return main_workload(args)
    assert args.warmup >= 3, "at least 3 warm-up steps"

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import cfm

    ranks = Ranks(world, "cuda")
    barrier, max_over_ranks = ranks.barrier, ranks.max

    j = cfm.Jacobi(3, N, N, N, cfm.FP64, 1, cfm.JACOBI_PERSISTENT)
    stream = torch.cuda.Stream()
    j.set_stream(stream.cuda_stream)
    j.load_problem(cfm.PROBLEM_CONFIG)
    best, _ = j.autotune(NITER // 2)  # pipeline shape and z-chunk; restores the grid
    tuned = cfm.variant_info(best) if best >= 0 else None
    zchunk = cfm.lib.cfm_jacobi_zchunk(j.h)
    blocks, threads = j.launch_shape()
    time.sleep(1.5)  # let the power state settle after tuning's seconds at full load
    for _ in range(args.warmup):
        j.run(NITER)

    # ---- device-resident timed region
    clocks = Clocks(local)
    time.sleep(0.25)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, kern_s = 0, 0.0
    ev0.record(stream)
    for _ in range(args.steps):
        st = j.run(NITER)
        launches += st.launches
        kern_s += st.seconds
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t_dev = max_over_ranks(ev0.elapsed_time(ev1) * 1e-3)
    kern_s = max_over_ranks(kern_s)

    # ---- end-to-end through the C ABI with pinned host buffers: every step
    # copies its grid in from host memory, sweeps, and copies the result
    # out (cfm_jacobi_run_host).  Three handles with the same tuned shape run
    # on three host threads, so one step's copies overlap another handle's
    # sweeps (a step is ~18 ms in, ~36 ms of sweeps, ~18 ms out: with two
    # handles the copies of one barely fit in the other's sweeps, with three
    # the sweeps run back to back; measured 171 / 311 / 326 / 294 GLUP/s
    # for 1 / 2 / 3 / 4 handles); the timed region spans all steps of all,
    # between two idle points of the device (CUDA events with a synchronize
    # on each side).
    import threading
    os.environ["CFM_J3D_TMA_VARIANT"] = str(best if best >= 0 else 0)
    os.environ["CFM_J3D_ZCHUNK"] = str(zchunk)
    handles = [j] + [cfm.Jacobi(3, N, N, N, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) for _ in range(2)]
    del os.environ["CFM_J3D_TMA_VARIANT"], os.environ["CFM_J3D_ZCHUNK"]
    host_in = torch.from_numpy(j.problem_host(cfm.PROBLEM_CONFIG).reshape(-1)).pin_memory()
    host_out = [torch.empty_like(host_in).pin_memory() for _ in handles]
    last = [None] * len(handles)
    for k, hk in enumerate(handles):  # warm the copy path
        last[k] = hk.run_host(NITER, host_in, host_out[k])
    per_thread = max(4, args.steps // 2)
    e2e_steps = per_thread * len(handles)

    def e2e_worker(k):
        for _ in range(per_thread):
            last[k] = handles[k].run_host(NITER, host_in, host_out[k])

    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    torch.cuda.synchronize()
    workers = [threading.Thread(target=e2e_worker, args=(k,)) for k in range(len(handles))]
    for th in workers:
        th.start()
    for th in workers:
        th.join()
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) * 1e-3)
    h2d, d2h = last[0].h2d_bytes, last[0].d2h_bytes
    e2e_same = all(bool(torch.equal(host_out[0], o)) for o in host_out[1:])
    clk = clocks.stop()
    for hk in handles:
        hk.close()

    lup_step = NITER * LUP_PER_SWEEP
    value = whole_job_rate(world, args.steps, lup_step, t_dev) / 1e9
    e2e_value = whole_job_rate(world, e2e_steps, lup_step, e2e_s) / 1e9
    peak, peak_kind = peak_hbm()
    per_launch_s = kern_s / args.steps
    achieved = BYTES_PER_LUP * lup_step / per_launch_s / 1e9
    traffic = traffic_per_launch()
    line = {
        "metric": "Jacobi 3d7p 512^3 FP64 GLUP/s", "value": value, "unit": "GLUP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "jacobi3d7p_512^3_fp64_periodic", "nx": N, "ny": N, "nz": N,
                   "niter_per_step": NITER, "problem": "config (x faces sin*sin, periodic y,z)",
                   "impl": "persistent cooperative kernel, grid barrier per sweep",
                   "launch": f"{blocks}x{threads}", "parallelism": f"replicas x{world}",
                   "tuned": None if tuned is None else
                   {"variant": best, "consumer_warps": tuned[0], "rows_per_warp": tuned[1], "stages": tuned[2],
                    "sweeps_per_pass": tuned[3], "zchunk": zchunk},
                   "l2": "inputs larger than L2 (two 1.07 GB grids)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": BYTES_PER_LUP * lup_step},
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": "GLUP/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "how": "cfm_jacobi_run_host on 3 handles x 3 host threads (copies of one step overlap "
                       "another's sweeps); CUDA events between idle points",
                "results_equal": e2e_same},
        "gpu_launches": launches,
    }
    if rank == 0 and world == 1:
        box = same_box_copy_gbs(torch)
        line["roofline"]["same_box_copy_gbs"] = box
        line["roofline"]["frac_of_same_box_copy"] = achieved / box
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0 and world == 1 and not args.no_secondary:
        line["secondary"] = secondary(cfm)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
