"""Benchmark: solve time to relative residual 1e-10 on the 1.01M-DOF cantilever.

Workload (one "step" = one full solve): the 3D linear-elastic cantilever
1.0 x 0.2 x 0.2 m, 200 x 40 x 40 linear hexahedra (n = 1,008,600 equations,
78.8M CSR entries), E = 210 GPa, nu = 0.3, clamped at x = 0, 1 MPa traction
in -z on the x = 1 face, 2x2x2 Gauss points.  The mesh is generated; the
stiffness matrix is assembled on the GPU (untimed set-up), then each step
solves K u = f from u = 0 with the mixed-precision refined PCG (FP32 inner
iteration, FP64 reliable updates) to ||f - K u|| / ||f|| < 1e-10.

Reported (one JSON line on rank 0):
  value         mixed solve time (ms), CUDA events on the solve's stream,
                matrix and vectors resident in HBM; max over ranks
  fp64          the plain FP64 Jacobi-PCG drop-in on the same system
  e2e           the drop-in C-ABI call sgpu_scr_cg_prec with host (pinned)
                SCR arrays: upload, device format build, solve, download
  roofline      the FP32 SpMV of the mixed iteration (its dominant kernel)
  cpu_baseline  SIFEL's own symcomprow::cg_prec (compiled reference) on a
                bounded sample of iterations of the same system, scaled to
                the full solve

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank solves its own replica (the single system
has no independent parts to shard without a per-iteration exchange).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ssf_b200 import _lib as L  # noqa: E402
from ssf_b200 import decks  # noqa: E402

WORKLOADS = {
    # name: (nx, ny, nz)
    "cantilever_200x40x40": (200, 40, 40),
    "cantilever_100x20x20": (100, 20, 20),
    "cantilever_20x4x4": (20, 4, 4),
}
METRIC = "solve time to relative residual 1e-10, mixed-precision refined PCG (FP64 PCG beside it)"
TOL = 1.0e-10
# Iterations SIFEL's own Jacobi-PCG (symcomprow::cg_prec, SCR storage,
# (r.r)/(f.f) < 1e-20) takes on each workload, from full runs of the compiled
# reference (tests/golden/reference_iterations.json, made by
# tests/golden/make_golden.py).
GOLDEN_ITERS = os.path.join(ROOT, "tests", "golden", "reference_iterations.json")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        import datetime
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank


def dist_max(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_from_profiles(kernel_key: str):
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(p) as fh:
            return json.load(fh).get(kernel_key)
    except (OSError, ValueError):
        return None


def reference_iterations(workload: str):
    try:
        with open(GOLDEN_ITERS) as fh:
            return int(json.load(fh)[workload]["iterations"])
    except (OSError, KeyError, ValueError):
        return None


# ----------------------------------------------------------------------------
# CPU leg: SIFEL's own solver (compiled from the reference sources)
# ----------------------------------------------------------------------------

def cpu_reference_time(adr, ci, a, f, workload, sample_iters=20, repeats=1):
    """Time symcomprow::cg_prec of the compiled reference on `sample_iters`
    iterations; scale to the full solve.  Returns (ms_full, info)."""
    from oracle import oracle as O  # test infrastructure: the CPU baseline leg only
    if not O.ref_available():
        return None, {"kind": "reference", "error": "oracle/_ref not built"}
    full_iters = reference_iterations(workload)
    best = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.ref_scr_cg_prec(adr, ci, a, f, ni=sample_iters, res=1e-20)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    per_iter = best / (sample_iters + 1)  # + the initial product / setup pass
    ms_full = per_iter * ((full_iters or 0) + 1) * 1e3
    return ms_full, {
        "per_iter_ms": per_iter * 1e3,
        "sample": f"{sample_iters} Jacobi-PCG iterations of SIFEL's symcomprow::cg_prec on the same "
                  f"{len(f)}-equation system, scaled to the {full_iters} iterations of the full reference solve",
        "full_iterations": full_iters,
    }


# ----------------------------------------------------------------------------
# the GPU arm
# ----------------------------------------------------------------------------

def run_ours(args, ws, rank):
    import torch
    from ssf_b200 import mefel
    dev = torch.device("cuda", torch.cuda.current_device())
    nx, ny, nz = WORKLOADS[args.workload]
    mesh = decks.cantilever_hex(nx, ny, nz)
    f_host = mefel.mefel_right_hand_side(mesh)
    K = mefel.stiffness_matrix(mesh)
    n = K.n
    nnz = K.nnz()
    log(f"[rank {rank}] assembled n={n} nnz={nnz} {K.assembly}")
    stream = torch.cuda.Stream()
    L.check(L.lib().sgpu_matrix_set_stream(K.h, C.c_void_p(stream.cuda_stream)))
    f_d = torch.from_numpy(f_host).to(dev)
    x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    lib = L.lib()

    def solve(mode):
        info = L.SolveInfo()
        ani, ares = C.c_int64(-1), C.c_double(0.0)
        st = lib.sgpu_matrix_pcg_d(K.h, C.c_void_p(x_d.data_ptr()), C.c_void_p(f_d.data_ptr()), 200000,
                                   TOL * TOL if mode == L.FP64 else TOL, 1e-30, 0,
                                   L.CRIT_SCR_PREC if mode == L.FP64 else L.CRIT_TRUE, 1, mode,
                                   C.byref(ani), C.byref(ares), C.byref(info))
        L.check(st)
        return info

    def timed(mode, steps, warmup):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                solve(mode)
            torch.cuda.synchronize()
            barrier(ws)
            torch.cuda.synchronize()
            l0 = L.kernel_launches()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            infos = []
            e0.record(stream)
            for _ in range(steps):
                infos.append(solve(mode))
            e1.record(stream)
            torch.cuda.synchronize()
            barrier(ws)
            launches = L.kernel_launches() - l0
        ms = e0.elapsed_time(e1) / steps
        return dist_max(ms, ws), infos, launches

    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    ms_mixed, inf_mixed, launches = timed(L.MIXED, args.steps, args.warmup)
    clk = clocks.stop()
    ms_fp64, inf_fp64, _ = timed(L.FP64, max(2, args.steps // 2), 1)
    im, i64 = inf_mixed[-1], inf_fp64[-1]
    log(f"[rank {rank}] mixed {ms_mixed:.2f} ms {im.as_dict()}")
    log(f"[rank {rank}] fp64  {ms_fp64:.2f} ms {i64.as_dict()}")

    # roofline of the dominant kernel: the FP32 SpMV of the mixed iteration
    def spmv_time(prec, reps=50):
        bytes_, fmt, var = C.c_double(), C.c_int32(), C.c_int32()
        L.check(lib.sgpu_matrix_spmv_plan(K.h, prec, C.byref(bytes_), C.byref(fmt), C.byref(var)))
        dt = torch.float32 if prec == 32 else torch.float64
        xv = torch.ones(n, dtype=dt, device=dev)
        yv = torch.empty(n, dtype=dt, device=dev)
        fn = lib.sgpu_matrix_mxv32_d if prec == 32 else lib.sgpu_matrix_mxv_d
        with torch.cuda.stream(stream):
            for _ in range(5):
                L.check(fn(K.h, C.c_void_p(xv.data_ptr()), C.c_void_p(yv.data_ptr())))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                L.check(fn(K.h, C.c_void_p(xv.data_ptr()), C.c_void_p(yv.data_ptr())))
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        return ms, bytes_.value, fmt.value, var.value

    peak, peak_kind = measured_peak()
    ms32, b32, fmt32, var32 = spmv_time(32)
    ms64, b64, fmt64, var64 = spmv_time(64)
    csr64_bytes = nnz * 12.0 + (n + 1) * 4.0 + 2.0 * n * 8.0
    fmt_name = {0: "csr", 3: "bsr3"}
    kern32 = f"spmv_fp32_{fmt_name[fmt32]}"
    traffic = traffic_from_profiles(f"{kern32}:{args.workload}")
    ach = b32 / (ms32 * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": traffic, "kernel": kern32,
                "bytes_per_launch": b32, "ms_per_launch": round(ms32, 5),
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else
                "fallback 6650 GB/s"}
    spmv64 = {"kernel": f"spmv_fp64_{fmt_name[fmt64]}", "ms_per_launch": round(ms64, 5),
              "bytes_per_launch": b64, "achieved_gbs": round(b64 / (ms64 * 1e-3) / 1e9, 1),
              "frac": round(b64 / (ms64 * 1e-3) / 1e9 / peak, 4),
              "csr_fp64_equiv_gbs": round(csr64_bytes / (ms64 * 1e-3) / 1e9, 1)}

    # e2e: the drop-in call with host (pinned) SCR arrays
    adr_h, ci_h, a_h = K.download(symmetric=1)
    K.close()
    pin = lambda arr: torch.from_numpy(arr).pin_memory().numpy()  # noqa: E731
    adr_p, ci_p, a_p, f_p = pin(adr_h), pin(ci_h), pin(a_h), pin(f_host)
    x_p = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    e2e_ms = []
    for rep in range(2):
        info = L.SolveInfo()
        ani, ares = C.c_int64(-1), C.c_double(0.0)
        t0 = time.perf_counter()
        st = lib.sgpu_scr_cg_prec(n, adr_p, ci_p, a_p, x_p, f_p, 200000, TOL * TOL, C.byref(ani), C.byref(ares),
                                  1e-30, 0, L.MIXED, C.byref(info))
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        L.check(st)
    e2e_v = dist_max(min(e2e_ms), ws)
    h2d = adr_h.nbytes + ci_h.nbytes + a_h.nbytes + f_host.nbytes
    d2h = x_p.nbytes

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        ms_cpu, cinfo = cpu_reference_time(adr_h, ci_h, a_h, f_host, args.workload,
                                           sample_iters=args.cpu_sample_iters)
        if ms_cpu is not None:
            cpu = {"value": round(ms_cpu, 1), "unit": "ms", "cores": 1, "kind": "reference",
                   "sample": cinfo["sample"], "per_iter_ms": round(cinfo["per_iter_ms"], 3)}
        else:
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": cinfo.get("error")}
    out = {
        "metric": METRIC,
        "value": round(ms_mixed, 3),
        "unit": "ms",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_mixed, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 refinement",
        "data": "synthetic (generated mesh, GPU-assembled stiffness)",
        "config": {"workload": args.workload, "n_equations": n, "nnz_full": nnz, "tolerance": TOL,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "inputs larger than L2 (matrix >= 0.6 GB vs 126 MB)"},
        "mixed": {"solve_ms": round(ms_mixed, 3), "iterations": im.iterations, "refinements": im.refinements,
                  "true_relres": im.true_relres},
        "fp64": {"solve_ms": round(ms_fp64, 3), "iterations": i64.iterations, "true_relres": i64.true_relres,
                 "speedup_mixed_vs_fp64": round(ms_fp64 / ms_mixed, 3)},
        "spmv_fp64": spmv64,
        "roofline": roofline,
        "e2e": {"value": round(e2e_v, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "sgpu_scr_cg_prec (host SCR arrays, mixed mode)"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------
# the reference arm: SIFEL's own CPU solver on the same workload
# ----------------------------------------------------------------------------

def run_reference(args, ws, rank):
    if rank != 0:
        return
    from oracle import oracle as O  # the compiled reference and its assembly restatement
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (compiled SIFEL) not built"}))
        return
    nx, ny, nz = WORKLOADS[args.workload]
    mesh = decks.cantilever_hex(nx, ny, nz)
    adr, ci, a = O.assemble(mesh, sym=True)
    f = O.load_vector(mesh)
    full = reference_iterations(args.workload)
    samples = []
    for i in range(args.warmup + args.steps):
        ms, info = cpu_reference_time(adr, ci, a, f, args.workload, sample_iters=args.cpu_sample_iters)
        if i >= args.warmup:
            samples.append(ms)
    v = statistics.mean(samples)
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 1),
        "unit": "ms",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(v, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (generated mesh)",
        "config": {"workload": args.workload, "n_equations": int(len(f)), "tolerance": TOL,
                   "solver": "SIFEL symcomprow::cg_prec (Jacobi PCG, SCR), compiled from the reference sources"},
        "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": 1, "kind": "reference",
                         "sample": info["sample"]},
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_iterations": full,
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cantilever_200x40x40", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample-iters", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3")
        args.warmup = 3
    ws, rank = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
