"""Benchmark: solve time to relative residual 1e-10 on the 1.01M-DOF cantilever.

Workload (one "step" = one full solve): the 3D linear-elastic cantilever
1.0 x 0.2 x 0.2 m, 200 x 40 x 40 linear hexahedra (n = 1,008,600 equations,
78.8M CSR entries), E = 210 GPa, nu = 0.3, clamped at x = 0, 1 MPa traction
in -z on the x = 1 face, 2x2x2 Gauss points.  The mesh is generated; the
stiffness matrix is assembled on the GPU (untimed set-up), then each step
solves K u = f from u = 0 to relative residual 1e-10.  Four GPU forms:

  fp64       the reference's iteration (Jacobi-PCG, symcomprow::cg_prec, its
             criterion (r.r)/(f.f) < 1e-20), all FP64 -- the drop-in;
  mixed      FP32 inner Jacobi-PCG on the scaled matrix with FP64 reliable
             updates (falls back to FP64 when the FP32 iteration stagnates);
  agg_mixed  FP64 flexible CG, preconditioned by one FP32 W-cycle of the
             aggregation multilevel preconditioner (GEFEL's precondtype
             boss = 101); every step rebuilds the hierarchy, so set-up is in
             the timed region;
  agg_fp64   the same with an FP64 W-cycle (isolates what FP32 buys).

Stopping tests: fp64 keeps the reference's (r.r)/(f.f) < 1e-20 on the
recurrence residual; the other forms stop on the true FP64 residual
||f - K x|| / ||f|| < 1e-10.  Every form reports its status, true residual
and its solution's error against the reference's own FP64 solution.

Reported (one JSON line on rank 0):
  value         time per step (ms) of the fastest form that met its
                criterion, CUDA events on the solve's stream, matrix and
                vectors resident in HBM; max over ranks; every form's time,
                iterations, residuals and errors beside it
  e2e           the same form through the C ABI with host (pinned) arrays,
                median of `steps` calls: sgpu_scr_cg_prec (drop-in for
                symcomprow::cg_prec) for the Jacobi forms, sgpu_matrix_create +
                sgpu_matrix_set_rigid_body_modes + sgpu_matrix_pcg for the
                aggregation forms
  roofline      the dominant kernel of the timed form (its FP64 SpMV)
  cpu_baseline  SIFEL's own symcomprow::cg_prec (compiled reference) on a
                bounded sample of iterations of the same system, scaled to
                the full solve; beside it one complete reference solve (its
                own assembly), run in a spawned process while the GPU arm
                runs, whose solution is the FP64 reference the errors use
  vs_reference_jacobi  the FP64 Jacobi form against that complete solve
                (the same algorithm on both sides)

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--forms all|fp64|mixed|agg_mixed|agg_fp64|jacobi]

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
import threading
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
# the other benchmark configurations, one JSON line each when asked for
EXTRA = ("cantilever_100x20x20_64rhs", "heat_cube_128_50steps", "plates_512", "deck_cantilever_200x40x40",
         "deck_heat_cube_128_50steps")
METRIC = "solve time to relative residual 1e-10 (fastest GPU form; mixed and FP64 forms all reported)"
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

    INTERVAL_MS = 50

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.p = None
        self.lines = []
        self.reader = None
        self.first = 0

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line)

    def start(self):
        """Starts the sampler and returns once it has taken its first sample
        (at most 2 s), so that the samples after that one cover the region."""
        self.lines = []
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
            return
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        t0 = time.time()
        while not self.lines and self.p.poll() is None and time.time() - t0 < 2.0:
            time.sleep(0.005)
        self.first = len(self.lines)  # samples taken before the region

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.p.kill()
            self.p.wait()
        self.reader.join(timeout=10)
        # the samples of the region; the one before it only when the region
        # ended before the next sample
        lines = self.lines[self.first:] or self.lines
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
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


def workload_config(workload: str, n: int, nnz: int, ws: int) -> dict:
    """The config object of both arms' lines (identical for the same run)."""
    return {"workload": workload, "n_equations": int(n), "nnz_full": int(nnz), "tolerance": TOL,
            "parallelism": f"replicas x{ws}" if ws > 1 else "one system",
            "l2": ("inputs larger than L2 (matrix >= 0.6 GB vs 126 MB)" if nnz * 12 > 126e6
                   else "inputs smaller than L2 (parity-size workload)")}


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


def _reference_full_solve(nx, ny, nz, out_path, q):
    """Child process (spawned): SIFEL's own assembly and Jacobi-PCG
    (symcomprow::cg_prec, compiled reference) of the whole workload to
    (r.r)/(f.f) < 1e-20; writes the solution to out_path and puts the timings
    on q.  Runs beside the GPU arm: it is both the measured full CPU solve and
    the FP64 solution the GPU forms' errors are taken against."""
    try:
        from oracle import oracle as O
        if not O.ref_available():
            q.put({"error": "oracle/_ref not built"})
            return
        mesh = decks.cantilever_hex(nx, ny, nz)
        t0 = time.perf_counter()
        adr, ci, a = O.assemble(mesh, sym=True)
        f = O.load_vector(mesh)
        t1 = time.perf_counter()
        x, ani, ares = O.ref_scr_cg_prec(adr, ci, a, f, ni=200000, res=TOL * TOL)
        t2 = time.perf_counter()
        np.save(out_path, x)
        q.put({"assemble_ms": (t1 - t0) * 1e3, "solve_ms": (t2 - t1) * 1e3, "iterations": int(ani),
               "ares": float(ares)})
    except Exception as e:  # noqa: BLE001  (reported, never fatal to the GPU arm)
        q.put({"error": repr(e)})


class ReferenceSolution:
    """The background full reference solve of the CPU baseline leg."""

    def __init__(self, workload):
        import multiprocessing as mp
        import tempfile
        self.path = os.path.join(tempfile.mkdtemp(prefix="sifel_ref_"), "u_ref.npy")
        ctx = mp.get_context("spawn")  # never fork a process that holds a CUDA context
        self.q = ctx.Queue()
        self.p = ctx.Process(target=_reference_full_solve, args=(*WORKLOADS[workload], self.path, self.q),
                             daemon=True)
        self.p.start()

    def result(self, timeout=900):
        import queue
        try:
            info = self.q.get(timeout=timeout)
        except queue.Empty:
            info = {"error": f"no result within {timeout} s"}
        self.p.join(timeout=30)
        if self.p.is_alive():
            self.p.terminate()
        u = None
        if "error" not in info and os.path.exists(self.path):
            u = np.load(self.path)
            os.remove(self.path)
        return u, info


# ----------------------------------------------------------------------------
# the GPU arm
# ----------------------------------------------------------------------------

FORMS = {
    # name: (preconditioner, arithmetic)
    "fp64": (1, 0),
    "mixed": (1, 1),
    "agg_mixed": (101, 1),
    "agg_fp64": (101, 0),
}
FORM_SETS = {"all": ["fp64", "mixed", "agg_mixed", "agg_fp64"], "jacobi": ["fp64", "mixed"],
             "fp64": ["fp64"], "mixed": ["mixed"], "agg_mixed": ["agg_mixed"], "agg_fp64": ["agg_fp64"]}
CRITERION = {"fp64": "(r.r)/(f.f) < 1e-20 on the recurrence residual (symcomprow::cg_prec)",
             "mixed": "||f - K x|| / ||f|| < 1e-10, recomputed in FP64",
             "agg_mixed": "||f - K x|| / ||f|| < 1e-10, recomputed in FP64",
             "agg_fp64": "||f - K x|| / ||f|| < 1e-10, recomputed in FP64"}
DTYPE = {"fp64": "f64", "mixed": "f32 inner PCG / f64 refinement",
         "agg_mixed": "f64 iteration / f32 multilevel preconditioner", "agg_fp64": "f64"}


def run_ours(args, ws, rank):
    # the CPU baseline's full reference solve runs beside the GPU arm (rank 0,
    # one rank only); started before the first CUDA call
    ref_job = ReferenceSolution(args.workload) if (rank == 0 and ws == 1 and not args.no_cpu) else None
    import torch
    from ssf_b200 import mefel
    dev = torch.device("cuda", torch.cuda.current_device())
    nx, ny, nz = WORKLOADS[args.workload]
    mesh = decks.cantilever_hex(nx, ny, nz)
    f_host = mefel.mefel_right_hand_side(mesh)
    rbm = mefel.rigid_body_modes(mesh)
    rbm_cols = np.ascontiguousarray(rbm.T)
    # a small assembly first loads the assembly kernels (lazy module loading),
    # and a first assembly of the workload takes the device memory the
    # assembly needs (cudaMalloc on first use, cached afterwards), so that the
    # assembly kept below is timed in steady state; the first one is reported
    with mefel.stiffness_matrix(decks.cantilever_hex(4, 2, 2)) as Kw:
        first_call = dict(Kw.assembly)
    with mefel.stiffness_matrix(mesh) as Kw:
        first_full = dict(Kw.assembly)
    K = mefel.stiffness_matrix(mesh)
    n = K.n
    nnz = K.nnz()
    assembly = {"pattern_ms": round(K.assembly["pattern_ms"], 3), "integrate_ms": round(K.assembly["integrate_ms"], 3),
                "colours": K.assembly.get("colours"),
                "first_call_4x2x2_ms": round(first_call["pattern_ms"] + first_call["integrate_ms"], 3),
                "first_full_pattern_ms": round(first_full["pattern_ms"], 3),
                "first_full_integrate_ms": round(first_full["integrate_ms"], 3)}
    # the integration's roofline on algorithmic bytes: per element its 8
    # nodes' coordinates and 24 code numbers, per CSR entry one read and one
    # write of its value (the element scatter's read-modify-write)
    asm_bytes = mesh.ne * (8 * 3 * 8 + 24 * 4) + nnz * 8 * 2
    asm_peak, _ = measured_peak()
    asm_gbs = asm_bytes / (K.assembly["integrate_ms"] * 1e-3) / 1e9
    assembly["roofline"] = {"bound": "hbm", "algorithmic_bytes": int(asm_bytes), "achieved": round(asm_gbs, 1),
                            "peak": asm_peak, "unit": "GB/s", "frac": round(asm_gbs / asm_peak, 4)}
    log(f"[rank {rank}] assembled n={n} nnz={nnz} {K.assembly}")
    stream = torch.cuda.Stream()
    L.check(L.lib().sgpu_matrix_set_stream(K.h, C.c_void_p(stream.cuda_stream)))
    K.set_nullspace(rbm)
    f_d = torch.from_numpy(f_host).to(dev)
    x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    lib = L.lib()

    def crit_args(form):
        # FP64 Jacobi (the drop-in): the reference's criterion, (r.r)/(f.f) <
        # 1e-20 on the recurrence residual.  Mixed Jacobi and both aggregation
        # forms: the true FP64 residual ||f - K x|| / ||f|| < 1e-10 (the
        # recurrence stop is confirmed on the recomputed residual).  Every
        # form's true residual is reported.
        if form == "fp64":
            return TOL * TOL, L.CRIT_SCR_PREC
        return TOL, L.CRIT_TRUE

    def solve(form):
        prec, mode = FORMS[form]
        if prec == L.PREC_AGG:
            L.check(lib.sgpu_matrix_precond_clear(K.h))  # set-up inside the step
        info = L.SolveInfo()
        ani, ares = C.c_int64(-1), C.c_double(0.0)
        res, crit = crit_args(form)
        st = lib.sgpu_matrix_pcg_d(K.h, C.c_void_p(x_d.data_ptr()), C.c_void_p(f_d.data_ptr()), 200000,
                                   res, 1e-30, 0, crit, prec, mode, C.byref(ani), C.byref(ares), C.byref(info))
        L.check(st, (L.OK, L.NOT_CONVERGED))
        info.status = st
        return info

    def timed(form, steps, warmup):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                solve(form)
            torch.cuda.synchronize()
            barrier(ws)
            torch.cuda.synchronize()
            l0 = L.kernel_launches()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            infos = []
            e0.record(stream)
            for _ in range(steps):
                infos.append(solve(form))
            e1.record(stream)
            torch.cuda.synchronize()
            barrier(ws)
            launches = L.kernel_launches() - l0
        ms = e0.elapsed_time(e1) / steps
        if args.profile_step:
            # one more step, untimed, inside a profiler range (ncu
            # --profile-from-start off captures exactly its launches)
            with torch.cuda.stream(stream):
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
                solve(form)
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
        return dist_max(ms, ws), infos, launches

    forms = FORM_SETS[args.forms]
    # every form timed the same way (warm-up, K steps, CUDA events, clocks
    # sampled during its timed region); the fastest is the line's value
    clocks = Clocks(torch.cuda.current_device())
    timed_all = {}
    x_of = {}
    for form in forms:
        clocks.start()
        ms_f, inf_f, launches_f = timed(form, args.steps, args.warmup)
        timed_all[form] = (ms_f, inf_f, launches_f, clocks.stop())
        x_of[form] = x_d.cpu().numpy()  # the last timed step's solution
    # the line's value: the fastest form that met 1e-10 on its own criterion
    ok_forms = [k for k in timed_all if timed_all[k][1][-1].status == L.OK] or list(timed_all)
    best = min(ok_forms, key=lambda k: timed_all[k][0])
    ms_best, inf_best, launches, clk = timed_all[best]
    results = {form: (v[0], v[1][-1]) for form, v in timed_all.items()}
    forms_out = {}
    for form, (ms, inf) in results.items():
        d = {"ms_per_step": round(ms, 3), "iterations": inf.iterations, "true_relres": inf.true_relres,
             "status": L.STATUS_NAMES[inf.status], "criterion": CRITERION[form], "dtype": DTYPE[form]}
        if FORMS[form][0] == L.PREC_AGG:
            d.update({"precond_setup_ms": round(inf.precond_setup_ms, 3), "solve_ms": round(inf.solve_ms, 3),
                      "levels": inf.precond_levels, "coarsest_equations": inf.precond_coarse_n})
        if form == "mixed":
            d.update({"refinements": inf.refinements, "fell_back_to_fp64": bool(inf.fallback)})
        if form == "fp64":
            d["reference_iterations"] = reference_iterations(args.workload)
        forms_out[form] = d
        log(f"[rank {rank}] {form:9s} {ms:9.3f} ms {inf.as_dict()}")
    if "fp64" in results:
        for form in results:
            forms_out[form]["speedup_vs_fp64"] = round(results["fp64"][0] / results[form][0], 3)
    if "agg_fp64" in results and "agg_mixed" in results:
        forms_out["agg_mixed"]["speedup_vs_agg_fp64"] = round(results["agg_fp64"][0] / results["agg_mixed"][0], 3)

    # roofline of the dominant kernel: the FP64 SpMV (the iteration's SpMV for
    # the FP64 forms, the outer flexible CG's SpMV of the aggregation forms);
    # the FP32 SpMV beside it
    def spmv_time(prec, reps=50):
        """Average launch time of the tuned SpMV kernel alone (CUDA events)."""
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
    var_of = {64: var64, 32: var32}

    def spmv_record(prec, ms, b, fmt):
        kern = f"spmv_fp{prec}_{fmt_name[fmt]}"
        ach = b / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": traffic_from_profiles(f"{kern}:{args.workload}"),
                "kernel": kern, "variant": var_of[prec], "bytes_per_launch": b, "ms_per_launch": round(ms, 5),
                "peak_source": (f"{peak_kind} hbm_gbs, MEASURED_PEAKS.json" if peak_kind == "measured"
                                else "fallback 6650 GB/s")}

    rec64 = spmv_record(64, ms64, b64, fmt64)
    rec64["csr_fp64_equiv_gbs"] = round(csr64_bytes / (ms64 * 1e-3) / 1e9, 1)
    rec32 = spmv_record(32, ms32, b32, fmt32)
    roofline = rec32 if best == "mixed" else rec64
    spmv_other = rec64 if best == "mixed" else rec32

    if args.no_e2e:
        K.close()
        print(json.dumps({"profile_run": True, "value": round(ms_best, 3), "form": best}), flush=True)
        return
    # e2e: the same form through the C ABI with host (pinned) arrays
    adr_h, ci_h, a_h = K.download(symmetric=1)
    K.close()
    pin = lambda arr: torch.from_numpy(arr).pin_memory().numpy()  # noqa: E731
    adr_p, ci_p, a_p, f_p = pin(adr_h), pin(ci_h), pin(a_h), pin(f_host)
    # the near-null space from the nodes, formed on the device (as the SIFEL binding does from Gtm)
    xyz_p = pin(np.ascontiguousarray(mesh.coords, dtype=np.float64))
    cn_p = pin(np.ascontiguousarray(mesh.code_numbers(), dtype=np.int64))
    x_p = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    prec_b, mode_b = FORMS[best]
    res_b, crit_b = crit_args(best)
    e2e_ms = []
    for rep in range(args.steps + 1):  # the first call is a warm-up
        info = L.SolveInfo()
        ani, ares = C.c_int64(-1), C.c_double(0.0)
        t0 = time.perf_counter()
        if prec_b == L.PREC_AGG:
            h = C.c_void_p()
            L.check(lib.sgpu_matrix_create(n, adr_p, ci_p, a_p, 1, C.byref(h)))
            L.check(lib.sgpu_matrix_set_rigid_body_modes(h, xyz_p.shape[0], cn_p.shape[1], xyz_p.ctypes.data,
                                                         cn_p.ctypes.data))
            st = lib.sgpu_matrix_pcg(h, x_p, f_p, 200000, res_b, 1e-30, 0, crit_b, prec_b, mode_b,
                                     C.byref(ani), C.byref(ares), C.byref(info))
            lib.sgpu_matrix_destroy(h)
        else:
            st = lib.sgpu_scr_cg_prec(n, adr_p, ci_p, a_p, x_p, f_p, 200000, TOL * TOL, C.byref(ani), C.byref(ares),
                                      1e-30, 0, mode_b, C.byref(info))
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        L.check(st, (L.OK, L.NOT_CONVERGED))
    e2e_v = dist_max(statistics.median(e2e_ms[1:]), ws)
    h2d = adr_h.nbytes + ci_h.nbytes + a_h.nbytes + f_host.nbytes + \
        (xyz_p.nbytes + cn_p.nbytes if prec_b == L.PREC_AGG else 0)
    d2h = x_p.nbytes

    cpu = None
    like_for_like = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        ms_cpu, cinfo = cpu_reference_time(adr_h, ci_h, a_h, f_host, args.workload,
                                           sample_iters=args.cpu_sample_iters)
        if ms_cpu is not None:
            cpu = {"value": round(ms_cpu, 1), "unit": "ms", "cores": 1, "kind": "reference",
                   "sample": cinfo["sample"], "per_iter_ms": round(cinfo["per_iter_ms"], 3)}
        else:
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": cinfo.get("error")}
    # the full reference solve that ran beside the GPU arm: its time, and every
    # form's solution error against it (the FP64 reference solution)
    if ref_job is not None:
        u_ref, rinfo = ref_job.result()
        if cpu is not None:
            cpu["full_solve"] = {k: (round(v, 1) if isinstance(v, float) else v) for k, v in rinfo.items()}
            cpu["full_solve"]["note"] = ("one complete symcomprow::cg_prec solve of the same system (its own "
                                         "assembly, 1 core), measured while the GPU arm ran")
        if u_ref is not None:
            nrm = float(np.linalg.norm(u_ref))
            for form, xf in x_of.items():
                forms_out[form]["err_vs_fp64_reference"] = float(np.linalg.norm(xf - u_ref) / nrm)
        else:
            for form in x_of:
                forms_out[form]["err_vs_fp64_reference"] = None
        if "fp64" in timed_all and "solve_ms" in rinfo:
            like_for_like = {"form": "fp64", "gpu_ms": round(timed_all["fp64"][0], 3),
                             "reference_ms": round(rinfo["solve_ms"], 1),
                             "reference_iterations": rinfo.get("iterations"),
                             "gpu_iterations": timed_all["fp64"][1][-1].iterations,
                             "ratio": round(rinfo["solve_ms"] / timed_all["fp64"][0], 1),
                             "note": "the same Jacobi-PCG algorithm on both sides; the headline form "
                                     "changes the algorithm"}
    out = {
        "metric": METRIC,
        "value": round(ms_best, 3),
        "unit": "ms",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_best, 3),
        "form": best,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": DTYPE[best],
        "data": "synthetic (generated mesh, GPU-assembled stiffness)",
        "config": workload_config(args.workload, n, nnz, ws),
        "forms": forms_out,
        "assembly": assembly,
        "vs_reference_jacobi": like_for_like,
        "spmv_other": spmv_other,
        "roofline": roofline,
        "e2e": {"value": round(e2e_v, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": ("sgpu_matrix_create + sgpu_matrix_set_rigid_body_modes + sgpu_matrix_pcg (host arrays)"
                         if prec_b == L.PREC_AGG else
                         "sgpu_scr_cg_prec, the drop-in for symcomprow::cg_prec (host SCR arrays)")},
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------
# the other configurations: many load cases, transient conduction, plate batch
# ----------------------------------------------------------------------------

def _timed_calls(fn, steps, warmup, ws):
    """Wall-clock of synchronous library calls bracketed by device syncs and
    CUDA events on the current stream (the calls finish their own streams
    before returning); max over ranks."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    l0 = L.kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    outs = [fn() for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    barrier(ws)
    return dist_max(e0.elapsed_time(e1) / steps, ws), outs, L.kernel_launches() - l0


def run_extra(args, ws, rank):
    import torch
    from ssf_b200 import gefel, mefel
    from oracle import oracle as O  # CPU baseline leg only
    torch.cuda.set_device(torch.cuda.current_device())
    peak, peak_kind = measured_peak()
    out = {"n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated meshes)", "unit": "ms"}
    clocks = Clocks(torch.cuda.current_device())
    if args.workload == "cantilever_100x20x20_64rhs":
        from ssf_b200 import shard
        mesh = decks.cantilever_top_loads(decks.cantilever_hex(100, 20, 20), 64, seed=1234)
        K = mefel.stiffness_matrix(mesh)
        cases = shard.partition(np.ones(64), ws)[rank]  # independent load cases: no exchange
        F = np.stack([mefel.mefel_right_hand_side(mesh, lc) for lc in cases], axis=1)
        # the load cases in the reference's layout (column blocks of n), in pinned host memory
        Fc = torch.from_numpy(np.ascontiguousarray(F.T)).pin_memory().numpy()
        Xc_pin = torch.zeros(Fc.shape, dtype=torch.float64).pin_memory().numpy()
        K.set_nullspace(mefel.rigid_body_modes(mesh))
        multi_forms = {"jacobi_fp64": ("jacobi", "fp64"), "agg_mixed": ("agg", "mixed"), "agg_fp64": ("agg", "fp64")}
        timings = {}
        clk = None
        for name, (prec, mode) in multi_forms.items():
            if prec == "agg":
                K.precond_clear()  # the first timed-region call builds the hierarchy (untimed warm-up does too)

            def step(prec=prec, mode=mode):
                if prec == "agg":
                    K.precond_clear()  # set-up inside every step
                return gefel.pcg_multi_blocks(K, Fc, res=1e-20, prec=prec, mode=mode, Xc=Xc_pin)
            if name == "agg_mixed":
                clocks.start()
            ms_f, outs_f, launches_f = _timed_calls(step, args.steps, args.warmup, ws)
            if name == "agg_mixed":
                clk = clocks.stop()
            X_f, res_f = outs_f[-1]
            timings[name] = (ms_f, launches_f, res_f)
        best = min(timings, key=lambda k: timings[k][0])
        ms, launches, res = timings[best]
        # the same 64 cases one after the other (the reference's order), device-resident matrix
        t0 = time.perf_counter()
        seq_its = []
        for c in range(F.shape[1]):
            _, r = K.pcg(F[:, c], res=1e-20, crit="scr", prec=1, mode="fp64")
            seq_its.append(r.info["iterations"])
        torch.cuda.synchronize()
        seq_ms = (time.perf_counter() - t0) * 1e3
        n = K.n
        adr_h, ci_h, a_h = K.download(symmetric=1)
        K.close()
        per_it = None
        if rank == 0 and O.ref_available():
            t0 = time.perf_counter()
            O.ref_scr_cg_prec(adr_h, ci_h, a_h, F[:, 0], ni=20, res=1e-20)
            per_it = (time.perf_counter() - t0) / 21
        forms_out = {}
        for name, (ms_f, _, res_f) in timings.items():
            its_f = [r.info["iterations"] for r in res_f]
            forms_out[name] = {"ms_per_step": round(ms_f, 3), "iterations_max": int(max(its_f)),
                               "device_solve_ms": round(res_f[0].info["solve_ms"], 3),
                               "all_converged": all(r.status == L.OK for r in res_f),
                               "speedup_vs_sequential_fp64": round(seq_ms / ms_f, 2)}
            if name.startswith("agg"):
                forms_out[name]["precond_setup_ms"] = round(res_f[0].info["precond_setup_ms"], 3)
        out.update({"metric": "64 load cases to (r.r)/(f.f) < 1e-20 each, all in one batched solve (fastest form; "
                              "each step: pinned host load cases in, set-up, solve, solutions out)",
                    "value": round(ms, 3), "ms_per_step": round(ms, 3), "form": best,
                    "dtype": {"jacobi_fp64": "f64", "agg_mixed": "f64 iteration / f32 multilevel preconditioner",
                              "agg_fp64": "f64"}[best],
                    "scaling": "strong",
                    "config": {"workload": args.workload, "n_equations": n, "load_cases": 64,
                               "parallelism": "single GPU" if ws == 1 else f"load cases sharded over {ws} GPUs"},
                    "forms": forms_out,
                    "sequential_fp64": {"solve_ms": round(seq_ms, 3), "iterations_total": int(sum(seq_its))},
                    "gpu_launches": int(launches), "clocks": clk})
        if per_it is not None:
            out["cpu_baseline"] = {"value": round(per_it * 1e3 * (sum(seq_its)), 1), "unit": "ms", "cores": 1,
                                   "kind": "reference",
                                   "sample": "20 iterations of SIFEL's symcomprow::cg_prec on load case 0, scaled to "
                                             f"the {int(sum(seq_its))} iterations of the 64 sequential solves"}
    elif args.workload == "heat_cube_128_50steps":
        mesh = decks.heat_cube(128, seed=1234)
        Kt = mefel.conductivity_matrix(mesh)
        Ct = mefel.capacity_matrix(mesh, rho=np.ones(mesh.ne))
        rhs = mefel.trfel_lift(Kt, mesh.meta["prescribed"][:, 0])
        n = Kt.n
        st_holder = {}

        def run(prec, mode):
            d = np.zeros(n)
            v = np.zeros(n)
            its = np.zeros(50, dtype=np.int64)
            info = L.SolveInfo()
            rc = L.lib().sgpu_transient_dform(Kt.h, Ct.h, rhs, d, v, 10.0, 1.0, 50, 100000, 1e-20, 1e-30, 1, prec, mode,
                                              its.ctypes.data, C.byref(info))
            L.check(rc)
            st_holder[(prec, mode)] = (its, info.as_dict())
            return d
        heat_forms = {"fp64": (L.PREC_JACOBI, L.FP64), "mixed": (L.PREC_JACOBI, L.MIXED),
                      "agg_mixed": (L.PREC_AGG, L.MIXED), "agg_fp64": (L.PREC_AGG, L.FP64)}
        timings = {}
        clk = None
        for name, (prec, mode) in heat_forms.items():
            if name == "fp64":
                clocks.start()
            ms_f, outs, launches_f = _timed_calls(lambda: run(prec, mode), args.steps, max(1, args.warmup // 3), ws)
            if name == "fp64":
                clk = clocks.stop()
            timings[name] = (ms_f, launches_f)
        best = min(timings, key=lambda k: timings[k][0])
        ms, launches = timings[best]
        its, binfo = st_holder[heat_forms[best]]
        forms_out = {}
        for name, (prec, mode) in heat_forms.items():
            its_f, inf_f = st_holder[(prec, mode)]
            forms_out[name] = {"ms_per_step": round(timings[name][0], 3), "iterations_total": int(its_f.sum()),
                               "device_solve_ms": round(inf_f["solve_ms"], 3), "true_relres_last": inf_f["true_relres"],
                               "precond_setup_ms": round(inf_f["precond_setup_ms"], 3),
                               "speedup_vs_fp64": round(timings["fp64"][0] / timings[name][0], 3)}
        out.update({"metric": "50 implicit-Euler steps of (C + dt K) T = f, each to (r.r)/(f.f) < 1e-20, K and C "
                              "assembled on the GPU (fastest form; every form reported)",
                    "value": round(ms, 3), "ms_per_step": round(ms, 3), "form": best,
                    "config": {"workload": args.workload, "n_equations": n, "elements": int(mesh.ne), "dt_s": 10.0,
                               "parallelism": "single GPU" if ws == 1 else f"replicas x{ws}"},
                    "forms": forms_out,
                    "iterations_total": int(its.sum()), "iterations_per_step": [int(i) for i in its[:5]] + ["..."],
                    "assembly": Kt.assembly, "gpu_launches": int(launches), "clocks": clk})
        Kt.close()
        Ct.close()
        if rank == 0 and ws == 1 and not args.no_cpu:
            t0 = time.perf_counter()
            adr, ci, ka = O.assemble(mesh, sym=True, kind="hex8t_k")
            _, _, ca = O.assemble(mesh, sym=True, kind="hex8t_c")
            t_asm = time.perf_counter() - t0
            d, v, sits = O.trfel_steps(mesh, 1, 10.0, iv=1, ni=100000)
            t_step = time.perf_counter() - t0 - t_asm
            # the reference integrates K and C (and the lifting) again in every step
            est = 50 * (1.5 * t_asm + t_step) * 1e3
            out["cpu_baseline"] = {"value": round(est, 1), "unit": "ms", "cores": 1, "kind": "port",
                                   "sample": "the oracle's K and C integration and one step on this mesh, scaled "
                                             "to 50 steps that each integrate K, C and the lifting again as "
                                             "the reference does"}
    elif args.workload == "deck_cantilever_200x40x40":
        # SIFEL's whole linear-statics run from its input file: read the
        # positional deck, number the DOFs, assemble K, solve, solution back
        import tempfile
        mesh = decks.cantilever_hex(200, 40, 40)
        tdir = tempfile.mkdtemp(prefix="sgpu_deck_")
        path = os.path.join(tdir, "cantilever_200x40x40.in")
        decks.write_mefel_deck(mesh, path)  # res 1e-20 on (r.r)/(f.f), SCR, diagonal preconditioner
        deck_bytes = os.path.getsize(path)
        state = {}
        timings = {}
        clk = None
        for name, (prec, mode) in {"agg_mixed": ("agg", "mixed"), "jacobi_fp64": (None, "fp64")}.items():
            def run(prec=prec, mode=mode, name=name):
                X, res, info = mefel.solve_deck(path, prec=prec, mode=mode)
                state[name] = (res, info)
                return X
            if name == "agg_mixed":
                clocks.start()
            ms_f, outs, launches_f = _timed_calls(run, args.steps, args.warmup, ws)
            if name == "agg_mixed":
                clk = clocks.stop()
            timings[name] = (ms_f, launches_f)
        best = min(timings, key=lambda k: timings[k][0])
        ms, launches = timings[best]
        forms_out = {}
        for name, (ms_f, _) in timings.items():
            res, info = state[name]
            forms_out[name] = {"ms_per_step": round(ms_f, 3), "parse_ms": round(info["parse_ms"], 3),
                               "pattern_ms": round(info["assembly"]["pattern_ms"], 3),
                               "integrate_ms": round(info["assembly"]["integrate_ms"], 3),
                               "precond_setup_ms": round(res[0].info.get("precond_setup_ms", 0.0), 3),
                               "device_solve_ms": round(res[0].info["solve_ms"], 3),
                               "iterations": int(res[0].info["iterations"]),
                               "true_relres": res[0].info["true_relres"],
                               "converged": all(r.status == L.OK for r in res)}
        out.update({"metric": "SIFEL linear-statics run from its input deck to relative residual 1e-10: read the "
                              "34 MB positional deck, DOF numbering, assembly, solve, solution on the host "
                              "(fastest form, wall clock)",
                    "value": round(ms, 3), "ms_per_step": round(ms, 3), "form": best,
                    "dtype": {"jacobi_fp64": "f64", "agg_mixed": "f64 iteration / f32 multilevel preconditioner"}[best],
                    "scaling": "weak",
                    "config": {"workload": args.workload, "n_equations": int(mesh.ndof), "deck_bytes": deck_bytes,
                               "parallelism": "single GPU" if ws == 1 else f"{ws} independent replicas",
                               "host_threads": os.cpu_count()},
                    "forms": forms_out, "gpu_launches": int(launches), "clocks": clk})
        if rank == 0 and ws == 1 and not args.no_cpu and O.ref_available():
            # the reference's own front end on the same file: mefel_init and
            # stiffness_matrix timed live by the harness, the solve by a
            # 20-iteration sample of its cg_prec scaled to its full count
            with tempfile.TemporaryDirectory() as od:
                subprocess.run([os.path.join(ROOT, "oracle", "_ref", "mefel_dump"), path, od, "nosolve"],
                               check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                dd = O.read_dump(od)
            meta, adr, ci, a, f = dd["meta"], dd["K_adr"], dd["K_ci"], dd["K_a"], dd["f"]
            ms_solve, cinfo = cpu_reference_time(adr, ci, a, f, "cantilever_200x40x40",
                                                 sample_iters=args.cpu_sample_iters)
            del dd, adr, ci, a
            t_front = (float(meta["t_init"]) + float(meta["t_stiffness"]) + float(meta["t_rhs"])) * 1e3
            out["cpu_baseline"] = {"value": round(t_front + ms_solve, 1), "unit": "ms", "cores": 1,
                                   "kind": "reference",
                                   "sample": f"SIFEL's mefel_init + stiffness_matrix + right-hand side on this deck "
                                             f"timed live ({t_front:.0f} ms), plus " + cinfo["sample"],
                                   "front_end_ms": round(t_front, 1), "solve_ms": round(ms_solve, 1)}
        import shutil
        shutil.rmtree(tdir, ignore_errors=True)  # the deck and the reference's log beside it
    elif args.workload == "deck_heat_cube_128_50steps":
        # SIFEL's whole transient heat run from its input file: read the
        # 370 MB TRFEL deck (2.1M element and material records), assemble K
        # and C, lift, 50 implicit-Euler steps, temperatures on the host
        import shutil
        import tempfile
        mesh = decks.heat_cube(128, seed=1234)
        tdir = tempfile.mkdtemp(prefix="sgpu_deck_")
        path = os.path.join(tdir, "heat_cube_128.in")
        decks.write_trfel_deck(mesh, path, dt=10.0, nsteps=50)
        deck_bytes = os.path.getsize(path)
        state = {}
        timings = {}
        clk = None
        for name, (prec, mode) in {"jacobi_fp64": ("jacobi", "fp64"), "agg_mixed": ("agg", "mixed")}.items():
            def run(prec=prec, mode=mode, name=name):
                d, v, its, info = mefel.solve_trfel_deck(path, prec=prec, mode=mode)
                state[name] = (its, info)
                return d
            if name == "jacobi_fp64":
                clocks.start()
            ms_f, outs, launches_f = _timed_calls(run, args.steps, args.warmup, ws)
            if name == "jacobi_fp64":
                clk = clocks.stop()
            timings[name] = (ms_f, launches_f)
        best = min(timings, key=lambda k: timings[k][0])
        ms, launches = timings[best]
        forms_out = {}
        for name, (ms_f, _) in timings.items():
            its, info = state[name]
            forms_out[name] = {"ms_per_step": round(ms_f, 3), "parse_ms": round(info["parse_ms"], 3),
                               "pattern_ms": round(info["assembly"]["pattern_ms"], 3),
                               "integrate_ms": round(info["assembly"]["integrate_ms"], 3),
                               "device_solve_ms": round(info["solve"]["solve_ms"], 3),
                               "iterations_total": int(its.sum()), "steps": int(info["nsteps"])}
        out.update({"metric": "SIFEL transient heat run from its input deck: read the 370 MB TRFEL deck, "
                              "assemble K and C, lift, 50 implicit-Euler steps each to (r.r)/(f.f) < 1e-20, "
                              "temperatures on the host (fastest form, wall clock)",
                    "value": round(ms, 3), "ms_per_step": round(ms, 3), "form": best,
                    "dtype": {"jacobi_fp64": "f64", "agg_mixed": "f64 iteration / f32 multilevel preconditioner"}[best],
                    "scaling": "weak",
                    "config": {"workload": args.workload, "n_equations": int(mesh.ndof), "elements": int(mesh.ne),
                               "deck_bytes": deck_bytes, "dt_s": 10.0, "steps": 50,
                               "parallelism": "single GPU" if ws == 1 else f"{ws} independent replicas",
                               "host_threads": os.cpu_count()},
                    "forms": forms_out, "gpu_launches": int(launches), "clocks": clk})
        shutil.rmtree(tdir, ignore_errors=True)
        if rank == 0 and ws == 1 and not args.no_cpu and O.ref_available():
            # the reference's trfel_init + K + C on a 64^3 deck of the same
            # kind (1/8 of the elements), timed live and scaled by elements;
            # its 50 steps from the oracle's one-step sample as in the
            # heat_cube_128_50steps line
            small = decks.heat_cube(64, seed=1234)
            with tempfile.TemporaryDirectory() as od:
                sp = os.path.join(od, "h64.in")
                decks.write_trfel_deck(small, sp, dt=10.0, nsteps=1)
                subprocess.run([os.path.join(ROOT, "oracle", "_ref", "trfel_dump"), sp, od, "nosolve"],
                               check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                meta = O.read_dump(od)["meta"]
            scale = mesh.ne / small.ne
            t_front = (float(meta["t_init"]) + float(meta["t_conductivity"]) + float(meta["t_capacity"])) * 1e3 * scale
            t0 = time.perf_counter()
            O.trfel_steps(small, 1, 10.0, iv=1, ni=100000)
            t_step = (time.perf_counter() - t0) * 1e3 * scale * 2.0  # one step; iterations grow ~2x at 128^3
            out["cpu_baseline"] = {"value": round(t_front + 50 * t_step, 1), "unit": "ms", "cores": 1,
                                   "kind": "port",
                                   "sample": "SIFEL's trfel_init + conductivity and capacity matrices on a 64^3 deck "
                                             "timed live and scaled by elements (8x), plus 50 steps from one "
                                             "oracle step on 64^3 scaled by elements and 2x iterations",
                                   "front_end_ms": round(t_front, 1)}
    else:  # plates_512
        from ssf_b200 import shard
        all_plates = decks.plate_batch(512, seed=0)
        mine = shard.partition([shard.plate_weight(p) for p in all_plates], ws)[rank]  # no exchange
        plates = [all_plates[k] for k in mine]
        nd = sum(p.ndof for p in all_plates)
        state = {}

        plate_forms = {"jacobi_fp64": ("jacobi", "fp64"), "agg_mixed": ("agg", "mixed"), "agg_fp64": ("agg", "fp64")}
        timings = {}
        clk = None
        for name, (prec, mode) in plate_forms.items():
            def run(prec=prec, mode=mode, name=name):
                xs, o = mefel.solve_batch(plates, res=1e-20, zero=1e-300, tune=state.get("tune", True),
                                          prec=prec, mode=mode)
                if prec == "jacobi":
                    state["tune"] = False
                state[name] = o
                return xs
            if name == "jacobi_fp64":
                clocks.start()
            ms_f, outs, launches_f = _timed_calls(run, args.steps, args.warmup, ws)
            if name == "jacobi_fp64":
                clk = clocks.stop()
            timings[name] = (ms_f, launches_f)
        def device_ms(of):  # assembly + set-up + solve on the device clock
            asm = of["assembly"]
            return asm["pattern_ms"] + asm["integrate_ms"] + of["info"].get("precond_setup_ms", 0.0) + \
                of["info"]["solve_ms"]
        best = min(timings, key=lambda k: device_ms(state[k]))
        ms_host, launches = timings[best]
        o = state[best]
        ms = device_ms(o)
        forms_out = {}
        for name in plate_forms:
            of = state[name]
            forms_out[name] = {"device_ms": round(device_ms(of), 3), "host_to_host_ms": round(timings[name][0], 3),
                               "device_solve_ms": round(of["info"]["solve_ms"], 3),
                               "precond_setup_ms": round(of["info"].get("precond_setup_ms", 0.0), 3),
                               "iterations_max": int(of["iterations"].max()),
                               "iterations_total": int(of["iterations"].sum()),
                               "all_converged": bool((of["status"] == 0).all()),
                               "speedup_vs_jacobi_fp64": round(device_ms(state["jacobi_fp64"]) / device_ms(of), 3)}
        out.update({"metric": "512 uneven plane-stress plates assembled and solved together on the device (each to "
                              "(r.r)/(f.f) < 1e-20): assembly + set-up + solve, device clock (fastest form; every "
                              "form reported, host mesh to host solution beside it)",
                    "value": round(ms, 3), "ms_per_step": round(ms, 3), "form": best,
                    "host_to_host_ms": round(ms_host, 3),
                    "dtype": {"jacobi_fp64": "f64", "agg_mixed": "f64 iteration / f32 multilevel preconditioner",
                              "agg_fp64": "f64"}[best],
                    "scaling": "strong",
                    "config": {"workload": args.workload, "plates": 512, "n_equations": int(nd),
                               "parallelism": "single GPU" if ws == 1 else f"plates sharded over {ws} GPUs",
                               "zero": "1e-300 (the reference's 1e-30 absolute |d.p| test stops these "
                                       "unit-traction plates before 1e-10)"},
                    "forms": forms_out, "assembly": o["assembly"],
                    "iterations_max": int(o["iterations"].max()), "iterations_total": int(o["iterations"].sum()),
                    "all_converged": bool((o["status"] == 0).all()),
                    "tuned": {"lanes_per_row": state["jacobi_fp64"]["info"]["spmv_variant"],
                              "segment_rows": state["jacobi_fp64"]["info"]["tile_rows"]},
                    "gpu_launches": int(launches), "clocks": clk})
        if rank == 0 and ws == 1 and not args.no_cpu and O.ref_available():
            # sample: 8 plates spread over the size range, reference solve timed, scaled by nnz x iterations
            order = np.argsort([p.ndof for p in plates])
            pick = order[np.linspace(0, len(order) - 1, 8).astype(int)]
            t_s, work_s = 0.0, 0.0
            for k in pick:
                adr, ci, a = O.assemble(plates[k], sym=True)
                f = O.load_vector(plates[k])
                t0 = time.perf_counter()
                O.ref_scr_cg_prec(adr, ci, a, f, ni=200000, res=1e-20, zero=1e-300)
                t_s += time.perf_counter() - t0
                work_s += plates[k].ndof * float(o["iterations"][k])
            work_all = float(sum(p.ndof * float(o["iterations"][k]) for k, p in enumerate(plates)))
            out["cpu_baseline"] = {"value": round(t_s * work_all / work_s * 1e3, 1),
                                   "unit": "ms", "cores": 1, "kind": "reference",
                                   "sample": "SIFEL's symcomprow::cg_prec on 8 of the 512 plates (sizes spread), "
                                             "scaled by equations x iterations to the whole batch "
                                             "(solve only)"}
    if rank == 0:
        print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------
# the reference arm: SIFEL's own CPU solver on the same workload
# ----------------------------------------------------------------------------

def run_reference(args, ws, rank):
    """SIFEL's own CPU path on the same workload: assembly by the oracle's
    restatement (bit-exact with the reference's), then the compiled
    reference's symcomprow::cg_prec.  Each timed step is a bounded sample of
    the solve (the first cpu_sample_iters iterations); one complete solve to
    (r.r)/(f.f) < 1e-20 is measured after them and is the line's value (the
    sample steps scaled to the full iteration count are reported beside it)."""
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
    n = int(len(f))
    nnz_full = int(2 * adr[-1] - n)
    step_ms, scaled = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ms_full, info = cpu_reference_time(adr, ci, a, f, args.workload, sample_iters=args.cpu_sample_iters)
        dt = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            step_ms.append(dt)
            scaled.append(ms_full)
    t0 = time.perf_counter()
    _, ani, _ = O.ref_scr_cg_prec(adr, ci, a, f, ni=200000, res=TOL * TOL)
    full_ms = (time.perf_counter() - t0) * 1e3
    extrapolated = statistics.mean(scaled)
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(full_ms, 1),
        "unit": "ms",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(statistics.mean(step_ms), 1),
        "step": f"each timed step is a bounded sample: the first {args.cpu_sample_iters} iterations of the "
                "solve; the value is the complete solve measured once after the steps",
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (generated mesh)",
        "config": workload_config(args.workload, n, nnz_full, ws),
        "solver": "SIFEL symcomprow::cg_prec (Jacobi PCG, SCR), compiled from the reference sources",
        "cpu_baseline": {"value": round(full_ms, 1), "unit": "ms", "cores": 1, "kind": "reference",
                         "sample": f"one complete solve ({ani} iterations, measured); the {args.steps} timed "
                                   f"steps of {args.cpu_sample_iters} iterations scaled to it give "
                                   f"{extrapolated:.1f} ms"},
        "e2e": {"value": round(full_ms, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_iterations": int(ani),
        "extrapolated_ms": round(extrapolated, 1),
        "extrapolated_vs_measured": round(extrapolated / full_ms, 4),
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cantilever_200x40x40", choices=sorted(WORKLOADS) + list(EXTRA))
    ap.add_argument("--cpu-sample-iters", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--forms", default="all", choices=sorted(FORM_SETS),
                    help="GPU forms to run (profiling runs time one form only)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the e2e and CPU legs (profiling runs)")
    ap.add_argument("--profile-step", action="store_true",
                    help="after each form's timed steps, one untimed step inside a profiler range "
                         "(for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3")
        args.warmup = 3
    ws, rank = dist_setup()
    try:
        if args.workload in EXTRA:
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "workload": args.workload,
                                      "unavailable": "the reference arm is timed on the default workload; "
                                                     "this line's cpu_baseline carries the CPU estimate"}))
            else:
                run_extra(args, ws, rank)
        elif args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
