"""Command line of the reference's `main.cpp` (src/main.cpp:37-249) over this
library: the same flag names, defaults (src/utility/Configuration.hpp:21-56),
errors and outputs.

    python heterogeneous-solvers_b200/cli.py --path_A A.txt --path_b b.txt --algorithm cholesky
    python heterogeneous-solvers_b200/cli.py --gp_input x.txt --gp_output y.txt --size 4096 \\
        --algorithm cg --eps 1e-10 --write_result true
    python heterogeneous-solvers_b200/cli.py --gp_input x.txt --gp_output y.txt --gp_test t.txt \\
        --size 4096 --test_size 100 --gpr true --algorithm cholesky

Outputs, as the reference writes them: `x_result.txt` in the working directory
(`--write_result`), the factor as `./A_chol_result` (`--write_matrix`, cholesky),
`metrics.json` in `<output>/<YYYY_MM_DD__HH_MM_SS>/` (cg, cholesky), and
"Average error of Ax - b: ..." on stdout (`--check_result`, generated matrices).
`--algorithm mixed` (no reference counterpart) runs the mixed-precision solve.
The flags of the reference's CPU/GPU split, load balancing and energy sampling
(mode, update_int, init_gpu_perc, cpu_lb_factor, block_update_th, wg_size_*,
gpu_opt, cpu_opt, enableHWS, track_chol_solve) are accepted and have no effect:
one GPU owns every block row.
"""
import argparse
import json
import os
import sys
import time
from pathlib import Path

_TRUE = {"true", "1", "yes", "on"}


def _bool(v):
    if isinstance(v, bool):
        return v
    return str(v).strip().lower() in _TRUE


def parse_args(argv):
    ap = argparse.ArgumentParser(prog="cli.py", description="Heterogeneous Conjugate Gradients (one-GPU B200 form)")
    for name in ("path_A", "path_b", "output", "gp_input", "gp_output", "gp_test", "mode", "algorithm"):
        ap.add_argument(f"--{name}", type=str)
    for name in ("matrix_bsz", "wg_size_vec", "wg_size_sp", "i_max", "update_int", "gpu_opt", "cpu_opt"):
        ap.add_argument(f"--{name}", type=int)
    for name in ("eps", "init_gpu_perc", "cpu_lb_factor"):
        ap.add_argument(f"--{name}", type=float)
    for name in ("block_update_th", "size", "test_size"):
        ap.add_argument(f"--{name}", type=int)
    for name in ("write_result", "write_matrix", "enableHWS", "print_verbose", "check_result", "track_chol_solve",
                 "gpr"):
        ap.add_argument(f"--{name}", type=_bool, nargs="?", const=True)
    a = ap.parse_args(argv)
    conf = {  # Configuration.hpp:21-56 defaults
        "matrixBlockSize": 128, "workGroupSizeVector": 128, "workGroupSizeFinalScalarProduct": 512, "iMax": 100000,
        "epsilon": 1.0e-6, "updateInterval": 10, "initialProportionGPU": 0.5, "outputPath": "./output",
        "writeResult": False, "writeMatrix": False, "mode": "static", "N": 0, "N_test": 0, "runtimeLBFactorCPU": 1.2,
        "blockUpdateThreshold": 1, "enableHWS": False, "algorithm": "cg", "gpuOptimizationLevel": 3,
        "cpuOptimizationLevel": 2, "printVerbose": False, "checkResult": False, "trackCholeskySolveStep": True,
    }
    conf["performGPR"] = bool(a.gpr)
    if conf["performGPR"] and not (a.gp_input and a.gp_output and a.gp_test):
        raise RuntimeError("Not all required arguments for GPR provided")
    conf["generateMatrix"] = False
    if a.path_A and a.path_b:
        conf["path_A"], conf["path_b"] = a.path_A, a.path_b
    elif a.gp_input and a.gp_output:
        conf["path_gp_input"], conf["path_gp_output"] = a.gp_input, a.gp_output
        conf["generateMatrix"] = True
        if a.size is not None:
            conf["N"] = a.size
        if a.test_size is not None:
            conf["N_test"] = a.test_size
        if a.gp_test:
            conf["path_gp_test"] = a.gp_test
    else:
        raise RuntimeError("No path to .txt file for matrix A specified and no path to input data for matrix "
                           "generation specified")
    pairs = [("algorithm", "algorithm"), ("output", "outputPath"), ("mode", "mode"), ("matrix_bsz", "matrixBlockSize"),
             ("wg_size_vec", "workGroupSizeVector"), ("wg_size_sp", "workGroupSizeFinalScalarProduct"),
             ("i_max", "iMax"), ("eps", "epsilon"), ("update_int", "updateInterval"),
             ("init_gpu_perc", "initialProportionGPU"), ("write_result", "writeResult"),
             ("write_matrix", "writeMatrix"), ("cpu_lb_factor", "runtimeLBFactorCPU"),
             ("block_update_th", "blockUpdateThreshold"), ("enableHWS", "enableHWS"),
             ("gpu_opt", "gpuOptimizationLevel"), ("cpu_opt", "cpuOptimizationLevel"),
             ("print_verbose", "printVerbose"), ("check_result", "checkResult"),
             ("track_chol_solve", "trackCholeskySolveStep")]
    for flag, key in pairs:
        v = getattr(a, flag)
        if v is not None:
            conf[key] = v
    conf["workGroupSize"] = conf["matrixBlockSize"]
    if conf["mode"] not in ("static", "runtime", "power"):
        raise RuntimeError(f"Invalid mode selected: '{conf['mode']}' --> must be 'static', 'runtime' or 'power'")
    if conf["algorithm"] not in ("cg", "cholesky", "mixed"):
        raise RuntimeError(f"Invalid algorithm: {conf['algorithm']}")
    return conf


def metrics_json(conf, gpu_name, times, block_count):
    """The reference's metrics.json layout (MetricsTracker.cpp:152-300); the
    power, utilisation and load-balancing series it samples with hws are empty."""
    cfg = {"algorithm": conf["algorithm"], "GPU": gpu_name, "N": conf["N"], "FP_type": "FP_64",
           "matrixBlockSize": conf["matrixBlockSize"], "workGroupSize": conf["workGroupSize"],
           "workGroupSizeVector": conf["workGroupSizeVector"],
           "workGroupSizeFinalScalarProduct": conf["workGroupSizeFinalScalarProduct"], "iMax": conf["iMax"],
           "epsilon": conf["epsilon"], "updateInterval": conf["updateInterval"],
           "initialProportionGPU": conf["initialProportionGPU"], "runtimeLBFactorCPU": conf["runtimeLBFactorCPU"],
           "blockUpdateThreshold": conf["blockUpdateThreshold"],
           "gpuOptimizationLevel": conf["gpuOptimizationLevel"],
           "cpuOptimizationLevel": conf["cpuOptimizationLevel"], "enableHWS": int(conf["enableHWS"]),
           "cpuBind": os.environ.get("OMP_PROC_BIND", ""), "ompCores": os.environ.get("OMP_NUM_THREADS", ""),
           "mode": conf["mode"]}
    rt = {"iterationTimes": times.get("iterationTimes", []), "memoryInitTime": times.get("memoryInitTime", 0.0),
          "resultCopyTime": times.get("resultCopyTime", 0.0), "totalTime": times.get("totalTime", 0.0),
          "choleskySolveStepTime": times.get("choleskySolveStepTime", 0.0), "averageUtilization_GPU": [],
          "averageUtilization_CPU": [], "powerDraw_GPU": [], "powerDraw_CPU": [], "blockCounts_GPU": [block_count],
          "blockCounts_CPU": [0]}
    if conf["algorithm"] == "cg":
        for k in ("matrixVectorTimes_GPU", "matrixVectorTimes_CPU", "times_q", "times_alpha", "times_x", "times_r",
                  "times_delta", "times_d", "memcopy_d"):
            rt[k] = times.get(k, [])
    else:
        for k in ("shiftTimes", "choleskyDiagonalBlockTimes", "copyTimes", "triangularSolveTimes_GPU",
                  "triangularSolveTimes_CPU", "triangularSolveTimes_total", "matrixMatrixDiagonalTimes_GPU",
                  "matrixMatrixDiagonalTimes_CPU", "matrixMatrixDiagonalTimes_total", "matrixMatrixTimes_GPU",
                  "matrixMatrixTimes_CPU", "matrixMatrixTimes_total"):
            rt[k] = times.get(k, [])
    return {"configuration": cfg, "runtime-metrics": rt}


def _write_metrics(conf, gpu_name, times, block_count):
    stamp = time.strftime("%Y_%m_%d__%H_%M_%S", time.localtime())
    d = Path(conf["outputPath"]) / stamp
    d.mkdir(parents=True, exist_ok=True)
    (d / "metrics.json").write_text(json.dumps(metrics_json(conf, gpu_name, times, block_count), indent=1) + "\n")
    return d / "metrics.json"


def main(argv=None):
    conf = parse_args(sys.argv[1:] if argv is None else argv)
    import importlib.util

    pkg_dir = Path(__file__).resolve().parent
    if "hs_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("hs_b200", pkg_dir / "__init__.py",
                                                      submodule_search_locations=[str(pkg_dir)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["hs_b200"] = mod
        spec.loader.exec_module(mod)
    hs = sys.modules["hs_b200"]
    import numpy as np
    import torch

    print("Using FP64 double precision")
    gpu_name = torch.cuda.get_device_name(0)
    print(f"GPU: {gpu_name}")
    bsz = conf["matrixBlockSize"]
    ctx = hs.Context(device=0)
    if conf["generateMatrix"]:
        N = conf["N"]
        ys = np.loadtxt(conf["path_gp_output"], dtype=np.float64, ndmin=1)
        if ys.size < N:
            raise RuntimeError("Not enough data available!")
        b = hs.RightHandSide(N, bsz)
        b.rightHandSideData[:N] = torch.from_numpy(ys[:N])
        A = hs.MatrixGenerator.generateSPDMatrix(ctx, conf["path_gp_input"], N, bsz)
    else:
        b = hs.MatrixParser.parseRightHandSide(conf["path_b"], bsz)
        A = hs.MatrixParser.parseSymmetricMatrix(conf["path_A"], bsz)
        conf["N"] = A.N
    ctx.set_problem(A.N, bsz)
    print("-- starting with computation")
    t0 = time.perf_counter()
    times = {}
    if conf["performGPR"]:
        gp = hs.GaussianProcess(A, b, conf["path_gp_input"], conf["path_gp_test"], ctx,
                                algorithm="cg" if conf["algorithm"] == "cg" else "cholesky",
                                N_test=conf["N_test"] or None)
        result = gp.start()
        if conf["writeResult"]:
            hs.UtilityFunctions.writeResult(".", result)
        return result
    if conf["algorithm"] == "cg":
        cg = hs.CG(A, b, ctx).solveHeterogeneous(epsilon=conf["epsilon"], iMax=conf["iMax"])
        times["totalTime"] = (time.perf_counter() - t0) * 1e3
        _write_metrics(conf, gpu_name, times, A.blockCountXY)
        x = cg.x
        if conf["writeResult"]:
            hs.UtilityFunctions.writeResult(".", x)
        if conf["printVerbose"]:
            print(f"CG iterations: {cg.iterations}")
    elif conf["algorithm"] == "cholesky":
        chol = hs.Cholesky(A, ctx).solve_heterogeneous()
        solve_ms = hs.TriangularSystemSolver(A, chol.A_gpu, b, ctx).solve()
        times["totalTime"] = (time.perf_counter() - t0) * 1e3
        times["choleskySolveStepTime"] = solve_ms
        if conf["writeMatrix"]:
            hs.MatrixParser.writeFullMatrix("./A_chol_result", A)
        _write_metrics(conf, gpu_name, times, A.blockCountXY)
        x = b.rightHandSideData
        if conf["writeResult"]:
            hs.UtilityFunctions.writeResult(".", x)
    else:
        solver = hs.MixedPrecisionSolver(A, ctx)
        x = solver.solve(b, tol=1e-14).cpu()
        if conf["writeResult"]:
            hs.UtilityFunctions.writeResult(".", x)
    if conf["checkResult"] and conf["generateMatrix"]:
        # UtilityFunctions.cpp:70-90: mean |A_new x - b_new| over N with A regenerated
        print("Checking result")
        A_new = hs.MatrixGenerator.generateSPDMatrix(ctx, conf["path_gp_input"], conf["N"], bsz)
        xd = torch.as_tensor(np.asarray(x, dtype=np.float64)).to("cuda:0")
        r = torch.empty_like(xd)
        nb = A_new.blockCountXY
        hs.MatrixVectorOperations.matrixVectorBlock(ctx, A_new.matrixData, xd, r, 0, 0, nb, nb, nb)
        yb = torch.zeros_like(xd)
        yb[:conf["N"]] = torch.from_numpy(np.loadtxt(conf["path_gp_output"], ndmin=1)[:conf["N"]]).cuda()
        error = float(torch.abs(yb - r).sum().item()) / conf["N"]
        print(f"Average error of Ax - b: {error}")
    ctx.close()
    return x


if __name__ == "__main__":
    main()
