#!/usr/bin/env python3
"""Benchmark of the blocked SPD solve path for GP kernel matrices.

One step = RBF assembly of the packed kernel matrix from device-resident
inputs and the mixed-precision solve (tensor-core factor whose trailing
updates take FP16 split products of the scaled panel, 3xTF32 TRSM, FP64
diagonal POTRF, FP64 iterative refinement to backward error <= 1e-14), at
N = 131072, d = 16, l = 1, sf2 = 1, sn2 = 1e-2, matrix_bsz = 256 (68.85 GB
packed FP64 matrix, larger than L2, so no flush is needed between steps).
The FP64 factor + solve of the same system is timed in the same run (the
comparison at equal error), with both backward errors.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  `value` is whole-job throughput in solves/s
(N independent replicas under torchrun: the path does not shard).  `e2e` is
the same metric through hs_gp_solve_host (the mixed algorithm of the headline's
split variant) with pinned host buffers.  The reference arm (--impl reference)
times the CPU restatement of the reference's CPU path (RBF assembly, factor,
solve) on a bounded sample and extrapolates it by an exponent fitted in the
same run.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
METRIC = "N=131072 SPD solve time: FP64 vs mixed-prec+IR at equal error; LML+grad time"
WORKLOAD = "c2_n131072"


def load_package():
    import importlib.util
    if "hs_b200" in sys.modules:
        return sys.modules["hs_b200"]
    pkg = ROOT / "heterogeneous-solvers_b200"
    spec = importlib.util.spec_from_file_location("hs_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def bench_config(N, world=1):
    """The workload both arms run: one GP system solved to FP64 accuracy."""
    return {"workload": f"{WORKLOAD}: solve K x = y (RBF kernel matrix assembled from X) to FP64 backward error",
            "N": N, "d": 16, "bsz": 256, "lengthscale": 1.0, "sf2": 1.0, "sn2": 1e-2,
            "l2": "inputs larger than L2 (packed K 68.85 GB at N=131072)", "parallelism": f"replicas x{world}"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=None, help="override N (smaller runs for profiling)")
    ap.add_argument("--cg-iters", type=int, default=20000,
                    help="iteration cap (iMax) of the CG solve to eps = 1e-10 on the benchmark system (0: skip)")
    ap.add_argument("--cpu-sample-n", type=int, default=8192)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison leg")
    ap.add_argument("--tol", type=float, default=1e-14, help="backward-error target of the mixed solve")
    ap.add_argument("--precision", choices=["tf32x3", "bf16x3", "f16x3"], default="f16x3",
                    help="split products of the headline mixed factor's tensor-core updates (the other variant "
                         "is timed as a leg of the same run)")
    ap.add_argument("--lml-n", type=int, default=16384, help="N of the NLML+gradient leg (0: skip)")
    ap.add_argument("--sweep", action="store_true",
                    help="conditioning sweep: mixed vs FP64 solve for sn2 in {1e-1, 1e-3, 1e-6} (one JSON line)")
    ap.add_argument("--lml-steps", type=int, default=3)
    ap.add_argument("--fit", action="store_true",
                    help="hyperparameter fit: L-BFGS on the FP64 NLML + gradient (ARD RBF, d=8) at --fit-n, "
                         "--fit-steps iterations (one JSON line)")
    ap.add_argument("--fit-n", type=int, default=65536,
                    help="N of the L-BFGS configuration (--fit); the default run times one NLML + gradient of both "
                         "forms there (0: skip)")
    ap.add_argument("--fit-steps", type=int, default=30)
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows),
                "power_w_max": max((float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit()), default=None)}


# ------------------------------------------------------------------ CPU baseline
def host_facts():
    """CPU model, logical cores and RAM of this host (from /proc)."""
    model, mem_gb = None, None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemTotal"):
                mem_gb = int(line.split()[1]) / 1024 ** 2
                break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cores": os.cpu_count(), "ram_gb": mem_gb}


def _oracle(threads):
    """The CPU restatement of the reference's CPU path (test infrastructure),
    with OpenMP limited to `threads`."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib
    return oracle_lib


def cpu_solve_sample(n_sample, threads, workload=WORKLOAD):
    """The reference's CPU path (init_gpu_perc=0) on one system of `workload`'s
    configuration at N = n_sample: RBF assembly (MatrixGenerator.cpp:73-162),
    blocked Cholesky factor (Cholesky.cpp:413-493, cpu_opt=2) and forward/back
    solve (TriangularSystemSolver.cpp:15-105).  Returns seconds per phase."""
    import numpy as np
    ol = _oracle(threads)
    hs = load_package()
    wl = __import__("hs_b200.workloads", fromlist=["CONFIGS"])
    cfg = wl.CONFIGS[workload]
    X, y = wl.gp_inputs(n_sample, cfg["d"], cfg["seed"])
    bsz = cfg["bsz"]
    b = np.zeros(hs.padded_size(n_sample, bsz))
    b[:n_sample] = y
    t0 = time.perf_counter()
    K = ol.rbf_assemble(X, bsz, cfg["lengthscale"], cfg["sf2"], cfg["sn2"])
    t1 = time.perf_counter()
    L = ol.cholesky(K, n_sample, bsz)
    ol.triangular_solve(L, b, n_sample, bsz)
    t2 = time.perf_counter()
    return {"assemble_s": t1 - t0, "factor_solve_s": t2 - t1, "total_s": t2 - t0}


def cpu_scaling_fit(threads, sizes=(4096, 8192, 16384)):
    """Times cpu_solve_sample at each size once and returns the growth exponent p
    of the two largest sizes, t(N2) / t(N1) = (N2 / N1)^p, with the samples (and
    the least-squares exponent over all sizes, for reference).  The two largest
    sizes are used because the factor's N^3 term dominates more the larger N is:
    smaller samples fit a lower exponent (cache effects, N^2 terms), which would
    understate the time at the full size."""
    import numpy as np
    samples = {n: cpu_solve_sample(n, threads) for n in sizes}
    ns = np.array(sizes, dtype=float)
    ts = np.array([samples[n]["total_s"] for n in sizes])
    p = float(np.log(ts[-1] / ts[-2]) / np.log(ns[-1] / ns[-2]))
    p_lsq = float(np.polyfit(np.log(ns), np.log(ts), 1)[0])
    return p, dict({str(n): samples[n] for n in sizes}, lsq_exponent_all_sizes=p_lsq)


def cpu_c1_full(threads):
    """The small configuration run in full on the CPU path: N=4096, d=8, l=0.5,
    sn2=1e-2, bsz=128; assembly, factor + solve, and CG to eps=1e-10 with the
    reference's CPU dot product (one chunk per core, VectorOperations.cpp:187-238)."""
    import numpy as np
    ol = _oracle(threads)
    hs = load_package()
    wl = __import__("hs_b200.workloads", fromlist=["CONFIGS"])
    cfg = wl.CONFIGS["c1_n4096"]
    N, bsz = cfg["N"], cfg["bsz"]
    X, y = wl.gp_inputs(N, cfg["d"], cfg["seed"])
    b = np.zeros(hs.padded_size(N, bsz))
    b[:N] = y
    t0 = time.perf_counter()
    K = ol.rbf_assemble(X, bsz, cfg["lengthscale"], cfg["sf2"], cfg["sn2"])
    t1 = time.perf_counter()
    L = ol.cholesky(K, N, bsz)
    x = ol.triangular_solve(L, b, N, bsz)
    t2 = time.perf_counter()
    x_cg, its, dn, d0 = ol.cg(K, b, N, bsz, cfg["eps"], 100000, chunks=threads)
    t3 = time.perf_counter()
    return {"workload": "c1_n4096: N=4096, d=8, l=0.5, sn2=1e-2, bsz=128", "assemble_s": t1 - t0,
            "factor_solve_s": t2 - t1, "cg_s": t3 - t2, "cg_iterations": int(its), "cg_chunks": threads,
            "cg_x_rel_diff_vs_factor": float(np.linalg.norm(x_cg - x) / np.linalg.norm(x))}


def replicas_throughput(torch, dist, t_ms, steps, world, device):
    """Whole-job solves/s of `world` independent replicas, each having timed
    `steps` solves in t_ms: the slowest rank's time (max over ranks, every rank
    gets it) and world * steps / that time.  `device` holds the reduction tensor
    (a GPU for NCCL, the CPU for gloo)."""
    t = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_max_ms = float(t.item())
    return t_max_ms, world * steps / (t_max_ms * 1e-3)


def run_reference_arm(args, rank, world):
    """The reference's CPU path on this host's cores (rank 0 only): each step
    assembles, factors and solves one system of the benchmark's configuration at
    N = --cpu-sample-n, and is extrapolated to the full N by the growth exponent
    of samples at N = 8192 and 16384 timed in the same run."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    N = args.n or 131072
    p, fit_samples = cpu_scaling_fit(threads)
    scale = (N / args.cpu_sample_n) ** p
    for _ in range(args.warmup):
        cpu_solve_sample(args.cpu_sample_n, threads)
    steps = [cpu_solve_sample(args.cpu_sample_n, threads) for _ in range(args.steps)]
    t_sample = sum(s_["total_s"] for s_ in steps) / len(steps)
    t_full = t_sample * scale
    value = 1.0 / t_full
    sample = (f"RBF assembly + FP64 blocked Cholesky factor + forward/back solve at N={args.cpu_sample_n} "
              f"(same d, l, sn2, bsz), {t_sample:.3f} s a step, extrapolated to N={N} by (N/{args.cpu_sample_n})^p "
              f"with p = {p:.3f}, the growth from N = 8192 to 16384 timed in this run (N = 4096 timed too)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_full * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(bench_config(N), implementation="the reference's CPU path (init_gpu_perc=0): RBF "
                                                          "assembly + FP64 blocked Cholesky factor + forward/back "
                                                          "solve"),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample,
                             "host": host_facts(), "sample_seconds_per_step": t_sample, "fitted_exponent": p,
                             "fit_samples": fit_samples, "c1_full": cpu_c1_full(threads)},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def measure_gemm_peak(torch, device, dtype, tf32=False):
    """cuBLAS GEMM 8192^3 through torch.matmul, best of 5, in TFLOP/s (FP64, or
    FP32 inputs on the TF32 tensor-core path when ``tf32``)."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = tf32
    a = torch.randn(8192, 8192, dtype=dtype, device=device)
    b = torch.randn(8192, 8192, dtype=dtype, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


def bench_lml(hs, torch, device, N, steps, precision="f16x3"):
    """NLML + gradient of an ARD RBF GP: X ~ U[0,1]^(N x 8), l_k ~ LogUniform[0.2, 2],
    sf2 = 1, sn2 = 1e-3, y drawn from the GP prior plus noise (a dense FP64
    Cholesky of K through torch draws it at N <= 32768, else y = sin(sum x) + noise;
    not timed).  Times hs_gp_nlml_grad (assembly, FP64 factor, solve, reverse-mode
    Cholesky, gradient contraction) and the same through the mixed-precision factor
    (hs_gp_nlml_grad_mixed), with the mixed results' errors against the FP64 ones."""
    import numpy as np
    d, bsz = 8, 256
    rng = np.random.default_rng(4)
    X = rng.random((N, d))
    ell = np.exp(rng.uniform(np.log(0.2), np.log(2.0), d))
    theta = np.concatenate([np.log(ell), [0.0, np.log(1e-3)]])
    dev = f"cuda:{device}"
    Xd = torch.from_numpy(X).to(dev)
    if N <= 32768:
        Xs = Xd / torch.from_numpy(ell).to(dev)
        K = torch.exp(-0.5 * torch.cdist(Xs, Xs).square()) + 1e-3 * torch.eye(N, dtype=torch.float64, device=dev)
        z = torch.from_numpy(rng.standard_normal(N)).to(dev)
        yd = torch.linalg.cholesky(K) @ z
        del K, Xs
        ydesc = "y ~ GP prior"
    else:
        yd = torch.from_numpy(np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)).to(dev)
        ydesc = "y = sin(sum x) + N(0, 0.1^2)"
    torch.cuda.empty_cache()
    c = hs.Context(device=device, N=N, matrixBlockSize=bsz)
    out = {"workload": f"GP NLML + gradient, ARD RBF, N={N}, d={d}, bsz={bsz}, sn2=1e-3, {ydesc}"}
    for prec in (None, precision):
        hs.gp_nlml_grad(c, Xd, yd, theta, precision=prec)  # warm-up (workspace, kernel loading)
        torch.cuda.synchronize()
        c.reset_profile()
        c.set_profiling(prec is None)
        t0 = time.perf_counter()
        for _ in range(steps):
            nlml, grad, rep = hs.gp_nlml_grad(c, Xd, yd, theta, precision=prec)
        t_ms = (time.perf_counter() - t0) * 1e3 / steps
        c.set_profiling(False)
        row = {"ms_per_call": t_ms, "nlml": nlml, "grad": [float(v) for v in grad],
               "phases_ms": {"assemble+factor(+refine)": rep["factor_ms"], "solve+adjoint": rep["adjoint_ms"],
                             "gradient": rep["grad_ms"]}, "logdet": rep["logdet"], "data_fit": rep["data_fit"]}
        if prec is None:
            adj = c.read_profile("adjoint")
            row["adjoint_dmma_tflops"] = adj["flops"] / (adj["ms"] * 1e-3) / 1e12 if adj["ms"] else None
            row["useful_tflops_whole"] = (N ** 3 / 3 + 2 * N ** 3 / 3) / (t_ms * 1e-3) / 1e12
            out["fp64"] = row
        else:
            row["mixed_report"] = rep["mixed"]
            g64 = np.asarray(out["fp64"]["grad"])
            row["grad_rel_err_vs_fp64"] = float(np.linalg.norm(grad - g64) / np.linalg.norm(g64))
            row["grad_max_component_rel_err_vs_fp64"] = float(np.max(np.abs(grad - g64) / np.abs(g64)))
            row["nlml_abs_diff_vs_fp64"] = abs(nlml - out["fp64"]["nlml"])
            row["logdet_abs_diff_vs_fp64"] = abs(rep["logdet"] - out["fp64"]["logdet"])
            row["data_fit_rel_diff_vs_fp64"] = abs(rep["data_fit"] - out["fp64"]["data_fit"]) / abs(
                out["fp64"]["data_fit"])
            row["speedup_vs_fp64"] = out["fp64"]["ms_per_call"] / t_ms
            out[prec] = row
    c.close()
    return out


def run_fit(hs, torch, device, N, steps, precision=None):
    """Hyperparameter fit of an ARD RBF GP by L-BFGS (hs.fit_hyperparameters: scipy's
    L-BFGS-B over the library's FP64 NLML and analytic gradient): X ~ U[0,1]^(N x 8),
    y = sin(sum_k x_k) + N(0, 0.1^2), theta0 = [log l_k = 0, log sf2 = 0, log sn2 = log 1e-2],
    at most `steps` iterations.  Wall time of the whole fit and of every NLML + gradient."""
    import numpy as np
    d, bsz = 8, 256
    rng = np.random.default_rng(5)
    X = rng.random((N, d))
    y = np.sin(X.sum(axis=1)) + 0.1 * rng.standard_normal(N)
    theta0 = np.concatenate([np.zeros(d), [0.0, np.log(1e-2)]])
    c = hs.Context(device=device, N=N, matrixBlockSize=bsz)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = hs.fit_hyperparameters(c, X, y, theta0, maxiter=steps, precision=precision)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    # both forms' gradients at the fitted theta, against the FP64 one
    _, g64, _ = hs.gp_nlml_grad(c, X, y, res["theta"])
    gm = g64 if precision is None else hs.gp_nlml_grad(c, X, y, res["theta"], precision=precision)[1]
    c.close()
    ev = np.asarray(res["eval_seconds"])
    form = "FP64" if precision is None else f"mixed-precision ({precision} factor, FP64 refinement)"
    return {"workload": f"L-BFGS hyperparameter fit, ARD RBF, N={N}, d={d}, bsz={bsz}, {form} NLML + gradient",
            "grad_at_result_rel_err_vs_fp64": float(np.linalg.norm(gm - g64) / np.linalg.norm(g64)),
            "seconds_per_step": wall / max(1, res["iterations"]),
            "max_iterations": steps, "iterations": res["iterations"], "evaluations": res["evaluations"],
            "fit_seconds": wall, "eval_seconds_median": float(np.median(ev)), "eval_seconds_max": float(ev.max()),
            "nlml_initial": res["nlml_trace"][0], "nlml_final": res["nlml"],
            "theta_final": [float(v) for v in res["theta"]], "message": res["message"]}


def run_sweep(args, hs, torch, ctx, Xd, bd, A, N, cfg, device):
    """Mixed (3xTF32 factor + FP64 refinement / PCG) against FP64 factor + solve on the
    same RBF system for sn2 in {1e-1, 1e-3, 1e-6}: times, backward errors, refinement
    steps and PCG iterations, and the mixed results' error against the FP64 ones."""
    import ctypes
    lib = hs._lib.load()
    nb, bsz = ctx.blockCountXY, cfg["bsz"]

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    def k_fro():
        blocks = A.view(-1, bsz * bsz)
        diag_ids = torch.tensor([hs.block_id(k, k, nb) for k in range(nb)], device=A.device)
        sq = (blocks * blocks).sum(dim=1)
        return float(torch.sqrt(2.0 * sq.sum() - sq[diag_ids].sum()).item())

    out = []
    for sn2 in (1e-1, 1e-3, 1e-6):
        def assemble():
            hs.MatrixGenerator.assemble(ctx, A, Xd, cfg["lengthscale"], cfg["sf2"], sn2)

        def bwd(x):
            assemble()
            r = torch.empty_like(bd)
            hs.MatrixVectorOperations.matrixVectorBlock(ctx, A, x, r, 0, 0, nb, nb, nb)
            return torch.linalg.norm(r - bd).item() / (k_fro() * torch.linalg.norm(x).item())

        row = {"sn2": sn2}
        xm = torch.empty_like(bd)
        rep = hs._lib.MixedReport()
        assemble()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = lib.hs_mixed_solve(ctx.handle, P(A), P(bd), P(xm), hs.PRECISIONS[args.precision], args.tol, 30,
                                ctypes.byref(rep))
        e1.record()
        torch.cuda.synchronize()
        row["mixed"] = {f: getattr(rep, f) for f, _ in hs._lib.MixedReport._fields_ if f != "reserved"}
        row["mixed"]["status"] = hs._lib.STATUS_NAMES.get(int(st), int(st))
        row["mixed"]["ms"] = e0.elapsed_time(e1)
        row["mixed"]["backward_error_host_check"] = bwd(xm) if st == 0 else None
        x64 = torch.empty_like(bd)
        info = ctypes.c_int64()
        assemble()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        st64 = lib.hs_cholesky_factor(ctx.handle, P(A), ctypes.byref(info))
        x64.copy_(bd)
        if st64 == 0:
            lib.hs_cholesky_solve(ctx.handle, P(A), P(x64))
        f1.record()
        torch.cuda.synchronize()
        row["fp64"] = {"status": hs._lib.STATUS_NAMES.get(int(st64), int(st64)), "ms": f0.elapsed_time(f1)}
        if st64 == 0:
            ld64 = hs.cholesky_logdet(ctx, A)
            row["fp64"]["logdet"] = ld64
            row["fp64"]["backward_error"] = bwd(x64)
            if st == 0:
                row["mixed_x_rel_err_vs_fp64"] = float((torch.linalg.norm(xm - x64) / torch.linalg.norm(x64)).item())
                row["mixed_logdet_rel_err_vs_fp64"] = abs(rep.logdet - ld64) / abs(ld64)
                row["speedup_mixed_vs_fp64"] = row["fp64"]["ms"] / row["mixed"]["ms"]
        out.append(row)
    return out


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    hs = load_package()
    wl = __import__("hs_b200.workloads", fromlist=["CONFIGS"])
    device = local_rank
    torch.cuda.set_device(device)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", device))

    if args.fit:
        fits = {"fp64": run_fit(hs, torch, device, args.fit_n, args.fit_steps)}
        fits[args.precision] = run_fit(hs, torch, device, args.fit_n, args.fit_steps, precision=args.precision)
        m, f = fits[args.precision], fits["fp64"]
        cmp = {"speedup_per_step": f["seconds_per_step"] / m["seconds_per_step"],
               "speedup_whole_fit": f["fit_seconds"] / m["fit_seconds"],
               "nlml_final_diff": m["nlml_final"] - f["nlml_final"],
               "theta_final_max_abs_diff": float(max(abs(a - b) for a, b in zip(m["theta_final"], f["theta_final"])))}
        if rank == 0:
            print(json.dumps({"metric": METRIC, "mode": "hyperparameter fit", "n_gpus": world, "data": "synthetic",
                              "fit": fits, "mixed_vs_fp64": cmp}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    cfg = dict(wl.CONFIGS[WORKLOAD])
    N = args.n or cfg["N"]
    bsz, d = cfg["bsz"], cfg["d"]
    X, y = wl.gp_inputs(N, d, cfg["seed"] + rank)
    dev = f"cuda:{device}"
    ctx = hs.Context(device=device)
    ctx.set_problem(N, bsz)
    nb = ctx.blockCountXY
    n_pad = hs.padded_size(N, bsz)
    Xd = torch.from_numpy(X).to(dev)
    bd = torch.zeros(n_pad, dtype=torch.float64, device=dev)
    bd[:N] = torch.from_numpy(y).to(dev)
    A = torch.empty(hs.packed_size(N, bsz), dtype=torch.float64, device=dev)
    xd = torch.empty_like(bd)
    lib = hs._lib.load()

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    info = ctypes.c_int64()
    mrep = hs._lib.MixedReport()

    def assemble():
        hs.MatrixGenerator.assemble(ctx, A, Xd, cfg["lengthscale"], cfg["sf2"], cfg["sn2"])

    def step_mixed():
        assemble()
        hs._lib.check(lib.hs_mixed_solve(ctx.handle, P(A), P(bd), P(xd), hs.PRECISIONS[args.precision], args.tol,
                                         30, ctypes.byref(mrep)))

    def step_fp64(x_out):
        assemble()
        hs._lib.check(lib.hs_cholesky_factor(ctx.handle, P(A), ctypes.byref(info)))
        x_out.copy_(bd)
        hs._lib.check(lib.hs_cholesky_solve(ctx.handle, P(A), P(x_out)))

    def k_fro():
        blocks = A.view(-1, bsz * bsz)
        diag_ids = torch.tensor([hs.block_id(k, k, nb) for k in range(nb)], device=A.device)
        sq_all = (blocks * blocks).sum(dim=1)
        return float(torch.sqrt(2.0 * sq_all.sum() - sq_all[diag_ids].sum()).item())

    def backward_error(x):
        """||y - K x|| / (||K||_F ||x||) with K re-assembled in A."""
        assemble()
        r = torch.empty_like(bd)
        hs.MatrixVectorOperations.matrixVectorBlock(ctx, A, x, r, 0, 0, nb, nb, nb)
        res = torch.linalg.norm(r - bd).item()
        return res / (k_fro() * torch.linalg.norm(x).item())

    for _ in range(args.warmup):
        step_mixed()
    torch.cuda.synchronize()
    if args.sweep:
        rows = run_sweep(args, hs, torch, ctx, Xd, bd, A, N, cfg, device)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "mode": "conditioning sweep", "n_gpus": world,
                              "config": dict(bench_config(N, world), sn2="sweep"), "sweep": rows}), flush=True)
        ctx.close()
        return
    tf32_peak = measure_gemm_peak(torch, device, torch.float32, tf32=True)

    # ---------------- timed region: mixed-precision solve (device-resident inputs)
    sampler = ClockSampler(device)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.reset_profile()
    ctx.set_profiling(True)
    launches0 = ctx.launch_count()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step_mixed()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = ctx.launch_count() - launches0
    ctx.set_profiling(False)
    t_ms = e0.elapsed_time(e1)
    kernels = ("update", "update_side", "potrf", "trsm", "assemble", "trsv", "colupd", "symv", "vector")
    prof = {k: ctx.read_profile(k) for k in kernels}
    t_max_ms, value = replicas_throughput(torch, dist, t_ms, args.steps, world, dev)
    if world > 1:
        dist.barrier()
    ms_per_step = t_max_ms / args.steps
    mixed_report = {f: getattr(mrep, f) for f, _ in hs._lib.MixedReport._fields_ if f != "reserved"}
    x_mixed = xd.clone()
    bwd_mixed = backward_error(x_mixed)

    # ---------------- the same step with the look-ahead by one diagonal block only (the
    # trailing-update launches then have every SM to themselves): step time, and the
    # update kernel's rate per launch on the whole GPU, against the timed default
    ahead = None
    if not args.no_fp64:
        ctx.set_mixed_lookahead(0, 0)
        torch.cuda.synchronize()
        ctx.reset_profile()
        ctx.set_profiling(True)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        step_mixed()
        a1.record()
        torch.cuda.synchronize()
        ctx.set_profiling(False)
        ctx.set_mixed_lookahead()
        pa = ctx.read_profile("update")
        ahead = {"one_block_lookahead_ms_per_step": a0.elapsed_time(a1),
                 "group_lookahead_ms_per_step": ms_per_step,
                 "one_block_lookahead_update_tflops": pa["flops"] / (pa["ms"] * 1e-3) / 1e12 if pa["ms"] else None,
                 "same_x": bool(torch.equal(xd, x_mixed))}

    # ---------------- the other split variant of the mixed form on the same system
    other = {"f16x3": "bf16x3", "bf16x3": "f16x3", "tf32x3": "f16x3"}[args.precision]
    alt = None
    if not args.no_fp64:
        orep = hs._lib.MixedReport()
        xo = torch.empty_like(bd)

        def step_other():
            assemble()
            hs._lib.check(lib.hs_mixed_solve(ctx.handle, P(A), P(bd), P(xo), hs.PRECISIONS[other], args.tol, 30,
                                             ctypes.byref(orep)))

        step_other()  # warm-up (kernel loading)
        torch.cuda.synchronize()
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        o0.record()
        step_other()
        o1.record()
        torch.cuda.synchronize()
        alt = {"precision": other, "ms_per_step": o0.elapsed_time(o1),
               "report": {f: getattr(orep, f) for f, _ in hs._lib.MixedReport._fields_ if f != "reserved"},
               "backward_error": backward_error(xo)}
        del xo

    # ---------------- FP64 factor + solve on the same system (the comparison at equal error)
    fp64 = None
    if not args.no_fp64:
        x64 = torch.empty_like(bd)
        # load the FP64 kernels on a small system, then time one full step
        ctx_s = hs.Context(device=device, N=4096, matrixBlockSize=bsz)
        As = torch.empty(hs.packed_size(4096, bsz), dtype=torch.float64, device=dev)
        hs.MatrixGenerator.assemble(ctx_s, As, Xd[:4096], cfg["lengthscale"], cfg["sf2"], cfg["sn2"])
        lib.hs_cholesky_factor(ctx_s.handle, P(As), ctypes.byref(info))
        ctx_s.close()
        del As
        torch.cuda.synchronize()
        ctx.reset_profile()
        ctx.set_profiling(True)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        step_fp64(x64)
        f1.record()
        torch.cuda.synchronize()
        ctx.set_profiling(False)
        prof64 = {k: ctx.read_profile(k) for k in ("update", "potrf", "trsm", "trsv", "colupd", "assemble")}
        upd64 = prof64["update"]
        fp64_ms = f0.elapsed_time(f1)
        logdet64 = hs.cholesky_logdet(ctx, A)
        bwd64 = backward_error(x64)
        dgemm = measure_gemm_peak(torch, device, torch.float64)
        fac = (N ** 3 / 3) / (fp64_ms * 1e-3) / 1e12
        upd_tf = upd64["flops"] / (upd64["ms"] * 1e-3) / 1e12 if upd64["ms"] else None
        fp64 = {"ms_per_step": fp64_ms, "solves_per_s": 1e3 / fp64_ms, "backward_error": bwd64,
                "factor_tflops_whole": fac, "update_dmma_tflops": upd_tf,
                "dgemm_peak_tflops": dgemm,
                "dgemm_peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul, FP64) measured in this run, best of 5",
                "factor_frac_of_dgemm": fac / dgemm, "update_frac_of_dgemm": upd_tf / dgemm if upd_tf else None,
                "phases_ms": {k: v["ms"] for k, v in prof64.items() if v["launches"]},
                "phases_tflops": {k: v["flops"] / (v["ms"] * 1e-3) / 1e12 for k, v in prof64.items()
                                  if v["launches"] and v["ms"] and k in ("update", "potrf", "trsm")},
                "speedup_mixed_vs_fp64": fp64_ms / ms_per_step}
        fp64["mixed_x_rel_diff"] = float((torch.linalg.norm(x_mixed - x64) / torch.linalg.norm(x64)).item())
        if alt is not None:
            alt["speedup_vs_fp64"] = fp64_ms / alt["ms_per_step"]
        fp64["mixed_logdet_rel_diff"] = abs(mixed_report["logdet"] - logdet64) / abs(logdet64)
        fp64["logdet"] = logdet64

    # ---------------- CG on the same system to eps = 1e-10 (CG.cpp:38-163), against the FP64 solve
    cg_info = None
    if args.cg_iters > 0:
        assemble()
        x_cg = torch.empty_like(bd)
        it, dn, d0 = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        ctx.reset_profile()
        ctx.set_profiling(True)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        st = lib.hs_cg_solve(ctx.handle, P(A), P(bd), P(x_cg), cfg["eps"], args.cg_iters, ctypes.byref(it),
                             ctypes.byref(dn), ctypes.byref(d0))
        c1.record()
        torch.cuda.synchronize()
        ctx.set_profiling(False)
        symv = ctx.read_profile("symv")
        cg_ms = c0.elapsed_time(c1)
        r_cg = torch.empty_like(bd)
        hs.MatrixVectorOperations.matrixVectorBlock(ctx, A, x_cg, r_cg, 0, 0, nb, nb, nb)
        cg_info = {"epsilon": cfg["eps"], "iMax": args.cg_iters, "status": hs._lib.STATUS_NAMES.get(int(st), int(st)),
                   "iterations": it.value, "ms": cg_ms, "ms_per_iteration": cg_ms / max(1, it.value),
                   "rel_residual": (dn.value / d0.value) ** 0.5 if d0.value else None,
                   "true_rel_residual": (torch.linalg.norm(r_cg - bd) / torch.linalg.norm(bd)).item(),
                   "matvecs": symv["launches"], "matvec_ms": symv["ms"] / max(1, symv["launches"]),
                   "matvec_gbs": symv["bytes"] / (symv["ms"] * 1e-3) / 1e9 if symv["ms"] else None,
                   "matvec_frac_of_hbm": None}
        if fp64 is not None:
            cg_info["x_rel_diff_vs_fp64_solve"] = float((torch.linalg.norm(x_cg - x64) / torch.linalg.norm(x64)).item())
        del x_cg, r_cg
    if fp64 is not None:
        del x64

    # ---------------- e2e through the host-buffer API (mixed precision, algorithm 2)
    e2e = None
    if not args.no_e2e:
        del A
        torch.cuda.empty_cache()
        Xh = torch.from_numpy(X).pin_memory()
        yh = torch.from_numpy(y).pin_memory()
        xh = torch.empty(N, dtype=torch.float64).pin_memory()
        kw = dict(algorithm=f"mixed_{args.precision}", epsilon=args.tol, iMax=30, out=xh)
        hs.gp_solve_host(ctx, Xh, yh, cfg["lengthscale"], cfg["sf2"], cfg["sn2"], **kw)  # warm-up
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _, rep = hs.gp_solve_host(ctx, Xh, yh, cfg["lengthscale"], cfg["sf2"], cfg["sn2"], **kw)
        torch.cuda.synchronize()
        _, e2e_value = replicas_throughput(torch, dist, (time.perf_counter() - t0) * 1e3, args.steps, world, dev)
        e2e = {"value": e2e_value, "unit": "solves/s",
               "h2d_bytes_per_step": int(X.nbytes + y.nbytes), "d2h_bytes_per_step": int(N * 8),
               "report_ms": {"assemble+h2d": rep.assemble_ms, "factor+refine": rep.factor_ms,
                             "total": rep.total_ms}}

    # ---------------- GP NLML + gradient (ARD, d = 8): FP64 and mixed-precision forms, at
    # N = --lml-n and at the L-BFGS configuration's N = --fit-n (the main system's
    # buffers are released first)
    lml = None
    if args.lml_n > 0 or args.fit_n > 0:
        lib.hs_ctx_release_buffers(ctx.handle)
        torch.cuda.empty_cache()
        lml = {}
        if args.lml_n > 0:
            lml[str(args.lml_n)] = bench_lml(hs, torch, ctx.device, args.lml_n, args.lml_steps)
        if args.fit_n > 0 and args.fit_n != args.lml_n:
            lml[str(args.fit_n)] = bench_lml(hs, torch, ctx.device, args.fit_n, 1)

    # ---------------- roofline of the dominant kernel (tensor-core trailing update)
    upd = prof["update"]
    useful = upd["flops"] / (upd["ms"] * 1e-3) / 1e12 if upd["ms"] else None
    traffic = None
    tfile = ROOT / "profiles" / "update_tc_traffic.json"
    if tfile.exists() and upd["launches"]:
        tj = json.loads(tfile.read_text())
        traffic = tj["dram_bytes_per_flop"] * upd["flops"] / upd["launches"]
    peaks = {}
    pf = ROOT / "MEASURED_PEAKS.json"
    if pf.exists():
        peaks = json.loads(pf.read_text())
    if cg_info and peaks.get("hbm_gbs") and cg_info["matvec_gbs"]:
        cg_info["matvec_frac_of_hbm"] = cg_info["matvec_gbs"] / peaks["hbm_gbs"]

    if args.precision == "tf32x3":
        peak3, peak_src, issued_key = tf32_peak / 3.0, (
            "cuBLAS TF32 GEMM 8192^3 measured in this run, divided by the 3 TF32 products of one split FP32 "
            "product (TF32 is absent from MEASURED_PEAKS.json)"), "issued_tf32_tflops"
    else:
        # FP16 and BF16 products run at the same tensor-core rate (kind::f16)
        bf = peaks.get("bf16_tflops_sustained") or 1400.0
        name = "BF16" if args.precision == "bf16x3" else "FP16"
        peak3, peak_src, issued_key = bf / 3.0, (
            ("MEASURED_PEAKS.json bf16_tflops_sustained" if peaks.get("bf16_tflops_sustained") else
             "fallback 1.4 PFLOP/s sustained bf16") + f", divided by the 3 {name} products of one split product"), \
            f"issued_{args.precision[:-2]}_tflops"
    roof = {"bound": "tensor", "achieved": useful, "peak": peak3 if useful else None, "unit": "TFLOP/s",
            "frac": useful / peak3 if useful else None, "traffic": traffic,
            "kernel": f"tc_update_kernel<256, {args.precision}> (split-product SYRK+GEMM trailing update, tcgen05, "
                      "persistent)",
            "launches": "main-stream launches; while the trailing matrix is large, 16 of the SMs run the next "
                        "panel group beside each update launch and then join it",
            "peak_source": peak_src, "tf32_gemm_peak": tf32_peak, issued_key: 3 * useful if useful else None}

    if ahead and ahead["one_block_lookahead_update_tflops"]:
        roof["frac_all_sms_one_block_lookahead"] = ahead["one_block_lookahead_update_tflops"] / peak3

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        p, fit_samples = cpu_scaling_fit(threads)
        t_s = fit_samples[str(args.cpu_sample_n)]["total_s"] if str(args.cpu_sample_n) in fit_samples else \
            cpu_solve_sample(args.cpu_sample_n, threads)["total_s"]
        t_full = t_s * (N / args.cpu_sample_n) ** p
        cpu = {"value": 1.0 / t_full, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"RBF assembly + FP64 factor + solve at N={args.cpu_sample_n} ({t_s:.3f} s), extrapolated "
                         f"to N={N} by (N/{args.cpu_sample_n})^p, p = {p:.3f} the growth from N = 8192 to 16384 in this run",
               "host": host_facts(), "fitted_exponent": p, "fit_samples": fit_samples}

    if rank == 0:
        phases = {k: {"launches": v["launches"], "ms_per_step": v["ms"] / args.steps,
                      "tflops": v["flops"] / (v["ms"] * 1e-3) / 1e12 if v["ms"] else None}
                  for k, v in prof.items() if v["launches"]}
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"tf32x3": "f32 (3xTF32 tensor-core factor) + f64 refinement",
                      "bf16x3": "f32 (BF16-split tensor-core updates, 3xTF32 TRSM) + f64 refinement",
                      "f16x3": "f32 (scaled FP16-split tensor-core updates, 3xTF32 TRSM) + f64 refinement",
                      }[args.precision],
            "data": f"synthetic: X~U[0,1]^({N}x{d}) seed {cfg['seed']}+rank, y=sin(sum_k x_k)+N(0,0.1^2)",
            "config": dict(bench_config(N, world), implementation=(
                "RBF assembly + mixed-precision Cholesky (" +
                {"tf32x3": "3xTF32 tensor-core TRSM/SYRK/GEMM",
                 "bf16x3": "BF16-split tensor-core SYRK/GEMM, 3xTF32 tensor-core TRSM",
                 "f16x3": "FP16-split (panel scaled by a power of two) tensor-core SYRK/GEMM, 3xTF32 tensor-core "
                          "TRSM"}[args.precision] +
                f", FP64 POTRF) + FP64 iterative refinement / preconditioned CG to backward error <= {args.tol:g}")),
            "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "phases": phases, "mixed": mixed_report, "backward_error": bwd_mixed, "fp64": fp64,
            "precision": args.precision, "other_split_variant": alt, "lml_grad": lml, "cg": cg_info,
            "lookahead": ahead,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
