"""Benchmark: seconds per frequency (assemble + solve) of the dense VIE path.

Workload (N=1 default): the plain FP64 method at scale -- synthetic sphere,
cube [-1,1]^3 cut into 12^3 cells x 6 tetrahedra, radially mapped (10,368
tetrahedra, N = 19,872 SWG unknowns, 6.3 GB complex128 matrix), anisotropic
permittivity [[4,.5,0],[.5,6,0],[0,0,9]] + 0.1i, omega = 1, three plane-wave
right-hand sides (x-pol along +z, y-pol along +z, z-pol along +x).

One step = one frequency: assemble the VIE matrix on the device, LU-factor
it, assemble the 3 RHS and solve.  The frequency-independent near-field
precompute runs once per mesh before timing and is reported separately
("precompute_s"), as the reference amortises its FIBBI cache.

value: device time of K steps (CUDA events on the library stream, barrier +
synchronize on both sides, max over ranks) / steps.  The 6.3 GB matrix is far
larger than L2, so no flush is needed.
e2e: the same per-frequency work through the host-buffer C-ABI calls
(bg_assemble, bg_rhs_planewave -> host, bg_lu_factor, bg_lu_solve with host
RHS in / solution out), host-side wall time including the copies.

--impl reference times the CPU restatement of the reference path (oracle
port, OpenMP over all host cores for assembly, LAPACK zgetrf via OpenBLAS) on
bounded samples of the same workload and extrapolates to the full size.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "buff-em_b200"))

METRIC = "sec/frequency (assemble+solve), N=19k & 58k: mixed/learned vs FP64, err<=1e-8"
TENSOR = [[4, 0.5, 0], [0.5, 6, 0], [0, 0, 9]]
WAVES = [([1, 0, 0], [0, 0, 1]), ([0, 1, 0], [0, 0, 1]), ([0, 0, 1], [1, 0, 0])]
OMEGA = 1.0


def eps_tensor():
    return np.array(TENSOR, complex) + 0.1j * np.eye(3)


def mesh_path(n):
    import meshgen
    d = os.path.join(tempfile.gettempdir(), "buffem_bench_meshes")
    return meshgen.cached_sphere(d, n)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for k, nm in enumerate(names):
                    if s[5 + k].lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ peaks
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def zgemm_peak_tflops():
    """FP64 tensor reference: cuBLAS ZGEMM (torch complex128 matmul) 8192^3,
    best of 5, CUDA events -- the measured denominator of the FP64 roofline."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    b = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 8.0 * n ** 3 / best / 1e12


def gemm_kernel_bench(n, reps=5):
    """Library complex GEMM (C -= A B, DMMA f64) on one n^3 problem, CUDA events
    on the library stream, best of reps; cuBLAS ZGEMM on the same shape beside it."""
    import torch
    import buffem
    L = buffem.lib()
    stream = torch.cuda.ExternalStream(L.bg_stream())
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(n, n, dtype=torch.complex128, device="cuda", generator=g)
    B = torch.randn(n, n, dtype=torch.complex128, device="cuda", generator=g)
    C = torch.zeros(n, n, dtype=torch.complex128, device="cuda")
    # column-major views: the library sees the storage of X.T as column-major X
    best = 1e30
    for i in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        buffem.zgemm_sub_device(n, n, n, A.data_ptr(), n, B.data_ptr(), n, C.data_ptr(), n)
        e1.record(stream)
        buffem.synchronize()
        if i:
            best = min(best, e0.elapsed_time(e1) / 1e3)
    ours = 8.0 * n ** 3 / best / 1e12
    # check one column against torch (column-major: C = -(B^T A^T)^T ... use transposes)
    ref = -(B.T @ A.T).T if False else None
    cub = zgemm_peak_tflops()
    return {"kernel": "k_zgemm_sub", "shape": [n, n, n], "tflops": ours, "ms": best * 1e3,
            "cublas_zgemm_tflops": cub, "frac_of_cublas": ours / cub}


# ------------------------------------------------------------------ GPU arm
def run_gpu(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import buffem

    torch.cuda.set_device(local_rank)
    n = args.n
    G = buffem.SWGGeometry(meshfiles=mesh_path(n),
                           materials=buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=eps_tensor()),
                           singular_order=args.order)
    N = G.TotalBFs
    t0 = time.perf_counter()
    G.precompute()
    buffem.synchronize()
    precompute_s = time.perf_counter() - t0
    M = G.AllocateVIEMatrix()
    L = buffem.lib()
    stream = torch.cuda.ExternalStream(L.bg_stream())
    nrhs = len(WAVES)
    dB = torch.zeros((nrhs, N), dtype=torch.complex128, device="cuda")  # column-major N x nrhs
    E0s = [np.ascontiguousarray(np.array(e, complex)) for e, _ in WAVES]
    nhs = [np.ascontiguousarray(np.array(k, float)) for _, k in WAVES]

    def step():
        buffem._check(L.bg_assemble(G.h, OMEGA, 0.0, M.h))
        buffem._check(L.bg_lu_factor(M.h))
        for i in range(nrhs):
            buffem._check(L.bg_rhs_planewave_device(G.h, OMEGA, 0.0, buffem._ptr(E0s[i]), buffem._ptr(nhs[i]),
                                                    buffem.C.c_void_p(dB[i].data_ptr())))
        buffem._check(L.bg_lu_solve_device(M.h, buffem.C.c_void_p(dB.data_ptr()), N, nrhs))

    for _ in range(args.warmup):
        step()
    buffem.synchronize()

    # phase breakdown of one untimed step (events on the library stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        buffem._check(L.bg_assemble(G.h, OMEGA, 0.0, M.h))
        ev[1].record(stream)
        buffem._check(L.bg_lu_factor(M.h))
        ev[2].record(stream)
        for i in range(nrhs):
            buffem._check(L.bg_rhs_planewave_device(G.h, OMEGA, 0.0, buffem._ptr(E0s[i]), buffem._ptr(nhs[i]),
                                                    buffem.C.c_void_p(dB[i].data_ptr())))
        buffem._check(L.bg_lu_solve_device(M.h, buffem.C.c_void_p(dB.data_ptr()), N, nrhs))
        ev[3].record(stream)
    buffem.synchronize()
    phases = {"assemble_s": ev[0].elapsed_time(ev[1]) / 1e3, "lu_s": ev[1].elapsed_time(ev[2]) / 1e3,
              "rhs_solve_s": ev[2].elapsed_time(ev[3]) / 1e3}

    # ---------------- timed region (device): plain FP64 path
    clocks = ClockSampler(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    buffem.synchronize()
    clocks.start()
    launches0 = buffem.launch_count()
    buffem.profile_begin()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    buffem.synchronize()
    torch.cuda.synchronize()
    prof = buffem.profile_read()
    buffem.profile_end()
    launches_fp64 = buffem.launch_count() - launches0
    elapsed_fp64 = e0.elapsed_time(e1) / 1e3
    x_fp64 = dB.clone()

    # ---------------- precision form: FP64 assembly -> complex64 copy ->
    # tcgen05 TF32 LU -> FP64-refined solve
    F = G.AllocateVIEMatrix(buffem.BG_C64)
    stats = np.zeros(3)

    def step_mixed():
        buffem._check(L.bg_assemble(G.h, OMEGA, 0.0, M.h))
        buffem._check(L.bg_matrix_convert(M.h, F.h))
        buffem._check(L.bg_lu_factor(F.h))
        for i in range(nrhs):
            buffem._check(L.bg_rhs_planewave_device(G.h, OMEGA, 0.0, buffem._ptr(E0s[i]), buffem._ptr(nhs[i]),
                                                    buffem.C.c_void_p(dB[i].data_ptr())))
        buffem._check(L.bg_lu_solve_refined_device(M.h, F.h, buffem.C.c_void_p(dB.data_ptr()), N, nrhs,
                                                   args.refine_tol, 60, buffem._ptr(stats)))

    for _ in range(args.warmup):
        step_mixed()
    buffem.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    ev[0].record(stream)
    buffem._check(L.bg_assemble(G.h, OMEGA, 0.0, M.h))
    ev[1].record(stream)
    buffem._check(L.bg_matrix_convert(M.h, F.h))
    buffem._check(L.bg_lu_factor(F.h))
    ev[2].record(stream)
    for i in range(nrhs):
        buffem._check(L.bg_rhs_planewave_device(G.h, OMEGA, 0.0, buffem._ptr(E0s[i]), buffem._ptr(nhs[i]),
                                                buffem.C.c_void_p(dB[i].data_ptr())))
    ev[3].record(stream)
    buffem._check(L.bg_lu_solve_refined_device(M.h, F.h, buffem.C.c_void_p(dB.data_ptr()), N, nrhs,
                                               args.refine_tol, 60, buffem._ptr(stats)))
    ev[4].record(stream)
    buffem.synchronize()
    phases_mixed = {"assemble_s": ev[0].elapsed_time(ev[1]) / 1e3, "convert_lu_s": ev[1].elapsed_time(ev[2]) / 1e3,
                    "rhs_s": ev[2].elapsed_time(ev[3]) / 1e3, "refined_solve_s": ev[3].elapsed_time(ev[4]) / 1e3,
                    "refine_sweeps": int(stats[0]), "final_rel_residual": float(stats[1]),
                    "first_rel_residual": float(stats[2])}
    launches1 = buffem.launch_count()
    buffem.profile_begin()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        step_mixed()
    e3.record(stream)
    buffem.synchronize()
    torch.cuda.synchronize()
    prof_mixed = buffem.profile_read()
    buffem.profile_end()
    launches_mixed = buffem.launch_count() - launches1
    clk = clocks.stop()
    elapsed_mixed = e2.elapsed_time(e3) / 1e3
    err = float(torch.linalg.norm(dB - x_fp64) / torch.linalg.norm(x_fp64))
    if world > 1:
        t = torch.tensor([elapsed_fp64, elapsed_mixed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_fp64, elapsed_mixed = float(t[0].item()), float(t[1].item())
        dist.barrier()
    launches = launches_mixed

    # ---------------- e2e through host buffers (precision form)
    hostB = np.zeros((N, nrhs), complex, order="F")
    rhs_h = np.zeros(N, complex)
    times = []
    for _ in range(0 if args.lean else max(1, args.steps)):
        buffem.synchronize()
        t0 = time.perf_counter()
        buffem._check(L.bg_assemble(G.h, OMEGA, 0.0, M.h))
        buffem._check(L.bg_matrix_convert(M.h, F.h))
        buffem._check(L.bg_lu_factor(F.h))
        for i in range(nrhs):
            buffem._check(L.bg_rhs_planewave(G.h, OMEGA, 0.0, buffem._ptr(E0s[i]), buffem._ptr(nhs[i]),
                                             buffem._ptr(rhs_h)))
            hostB[:, i] = rhs_h
        buffem._check(L.bg_lu_solve_refined(M.h, F.h, buffem._ptr(hostB), nrhs, args.refine_tol, 60,
                                            buffem._ptr(stats)))
        times.append(time.perf_counter() - t0)
    e2e_s = max(times) if times else None
    if world > 1 and e2e_s is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    del F
    return dict(N=N, elapsed=elapsed_mixed, elapsed_fp64=elapsed_fp64, phases=phases, phases_mixed=phases_mixed,
                prof=prof, prof_mixed=prof_mixed, launches=launches, launches_fp64=launches_fp64, clocks=clk,
                precompute_s=precompute_s, e2e_s=e2e_s, nrhs=nrhs, err_vs_fp64=err)



# ------------------------------------------------------------------ CPU arm
def cpu_sample(n, order, nrow_sample=48, lu_n=3000, threads=None):
    """Oracle port on the host: warm-cache assembly of a uniform row sample and
    LAPACK zgetrf at a smaller order, extrapolated to the full workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import scipy.linalg as sl
    G = oracle.Geometry(mesh_path(n), oracle.material(kind=oracle.MAT_CONST_TENSOR, tensor=eps_tensor()),
                        nang=order)
    N = G.N
    t0 = time.perf_counter()
    G.cache_build()
    t_cache = time.perf_counter() - t0
    rows = np.linspace(0, N - 1, nrow_sample).astype(np.int32)
    t0 = time.perf_counter()
    G.assemble_rows(complex(OMEGA), rows)
    t_rows = time.perf_counter() - t0
    t_asm = t_rows * N / nrow_sample
    rng = np.random.default_rng(0)
    A = rng.normal(size=(lu_n, lu_n)) + 1j * rng.normal(size=(lu_n, lu_n))
    t0 = time.perf_counter()
    lu = sl.lu_factor(A, overwrite_a=True, check_finite=False)
    t_lu_s = time.perf_counter() - t0
    t_lu = t_lu_s * (N / lu_n) ** 3
    B = rng.normal(size=(lu_n, 3)) + 1j * rng.normal(size=(lu_n, 3))
    t0 = time.perf_counter()
    sl.lu_solve(lu, B, check_finite=False)
    t_sv = (time.perf_counter() - t0) * (N / lu_n) ** 2
    total = t_asm + t_lu + t_sv
    sample = (f"warm-cache oracle assembly of {nrow_sample} of {N} rows (x{N / nrow_sample:.0f}) + "
              f"OpenBLAS zgetrf/zgetrs at N={lu_n} scaled by (N/{lu_n})^3 and ^2; "
              f"near-field cache build {t_cache:.1f}s excluded like the precompute")
    return dict(value=total, assemble=t_asm, lu=t_lu, solve=t_sv, cache=t_cache, sample=sample,
                cores=oracle.lib().or_num_threads())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=12, help="cells per cube edge (12 -> N=19,872)")
    ap.add_argument("--order", type=int, default=10, help="singular-rule order")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lean", action="store_true",
                    help="timed steps only (no e2e pass, CPU baseline or peak measurement): profiler runs")
    ap.add_argument("--kernel", default=None, choices=["gemm"],
                    help="time the LU trailing-update GEMM alone on an M=N=K problem")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--refine-tol", type=float, default=1e-12,
                    help="relative residual target of the FP64 refinement (precision form)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup

    if args.kernel == "gemm":
        print(json.dumps(gemm_kernel_bench(args.size)), flush=True)
        return
    if args.lean:
        args.no_cpu_baseline = True

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": f"plain FP64: sphere {args.n}^3 cells x 6 tets, anisotropic eps tensor, 3 plane-wave RHS",
              "n_cells": args.n, "omega": OMEGA, "rhs": 3, "singular_order": args.order,
              "parallelism": f"replicas x{world} (independent frequencies)",
              "l2": "matrix (16 N^2 bytes) >> 126 MB L2; no flush needed"}

    if args.impl == "reference":
        if rank != 0:
            return
        r = cpu_sample(args.n, args.order)
        N = 12 * args.n ** 3 - 6 * args.n ** 2
        config["N"] = N
        vals = [r["value"]]
        for _ in range(max(0, args.steps - 1)):
            vals.append(cpu_sample(args.n, args.order)["value"])
        v = statistics.median(vals)
        line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "s", "cores": r["cores"], "kind": "port", "sample": r["sample"]},
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "breakdown": {k: r[k] for k in ("assemble", "lu", "solve", "cache")}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    res = run_gpu(args, rank, world, local_rank)
    N = res["N"]
    config["N"] = N
    config["paths"] = "value: precision form (FP64 assembly, complex64 tcgen05/TF32 LU, FP64-refined solve); " \
                      "fp64: plain path (FP64 assembly, DMMA LU, FP64 solve)"
    value = res["elapsed"] / args.steps / world    # whole-job seconds per frequency
    value_fp64 = res["elapsed_fp64"] / args.steps / world
    gemm = res["prof"]["lu_gemm"]
    achieved = gemm["flops"] / (gemm["ms"] / 1e3) / 1e12 if gemm["ms"] > 0 else None
    gm = res["prof_mixed"]["lu_gemm"]
    achieved_tc = gm["flops"] / (gm["ms"] / 1e3) / 1e12 if gm["ms"] > 0 else None
    peak = None
    peak_src = None
    if rank == 0 and not args.lean:
        try:
            peak = zgemm_peak_tflops()
            peak_src = "measured in-run: cuBLAS ZGEMM 8192^3 (torch complex128 matmul), best of 5"
        except Exception as e:  # pragma: no cover
            peak_src = f"unavailable: {e}"
    mp = measured_peaks()
    bf16 = mp.get("bf16_tflops")
    total_ms = sum(v["ms"] for v in res["prof"].values())
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["elapsed"] / args.steps * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128 (complex64 TF32 tensor-core LU + FP64 refinement)",
            "data": "synthetic", "config": config,
            "fp64_path": {"value": value_fp64, "unit": "s", "phases": res["phases"],
                          "speedup_of_precision_form": value_fp64 / value, "gpu_launches": res["launches_fp64"]},
            "precision_form": {"phases": res["phases_mixed"], "err_vs_fp64_lu": res["err_vs_fp64"]},
            "precompute_s": res["precompute_s"],
            "roofline": {"bound": "tensor", "kernel": "k_zgemm_sub (FP64 path LU trailing update, DMMA f64)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if (achieved and peak) else None, "traffic": None,
                         "peak_source": peak_src,
                         "algorithmic": "8*M*N*K flops per launch (4M complex product)",
                         "gemm_share_of_profiled_ms": gemm["ms"] / total_ms if total_ms else None,
                         "lu_flops_rate_tflops": (8 / 3 * N ** 3) / res["phases"]["lu_s"] / 1e12,
                         "precision_form_gemm": {"kernel": "k_cgemm_tf32 (tcgen05 kind::tf32)",
                                                 "achieved": achieved_tc, "unit": "TFLOP/s",
                                                 "peak_bf16_dense_measured": bf16,
                                                 "frac_of_bf16_peak": (achieved_tc / bf16) if (achieved_tc and bf16) else None}},
            "kernel_classes": res["prof"], "kernel_classes_precision_form": res["prof_mixed"],
            "e2e": {"value": res["e2e_s"] / world if res["e2e_s"] else None, "unit": "s",
                    "h2d_bytes_per_step": 16 * N * res["nrhs"],
                    "d2h_bytes_per_step": 2 * 16 * N * res["nrhs"]},
            "gpu_launches": res["launches"], "clocks": res["clocks"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_sample(args.n, args.order)
        line["cpu_baseline"] = {"value": r["value"], "unit": "s", "cores": r["cores"], "kind": "port",
                                "sample": r["sample"],
                                "breakdown": {k: r[k] for k in ("assemble", "lu", "solve", "cache")}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
