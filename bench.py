"""Benchmark: seconds per frequency (assemble + solve) of the dense VIE path.

Headline workload (N=1 default, the learned form): synthetic sphere, cube
[-1,1]^3 cut into 17^3 cells x 6 tetrahedra, radially mapped (29,478
tetrahedra, N = 57,222 SWG unknowns: 52 GB complex128 matrix plus a 26 GB
complex64 copy), eps = 6 + 0.5i, omega = 1, three plane-wave right-hand sides
(x-pol along +z, y-pol along +z, z-pol along +x).

One step = one frequency.
  value (mixed + learned): assemble the complex128 matrix, copy it to
    complex64, predict the near-field approximate inverse with the graph
    network (shipped weights), assemble the RHS, solve by GMRES(80) on the
    complex64 copy with FP64 refinement against the complex128 matrix to a
    1e-10 relative residual, LU fallback if 1000 Krylov steps do not reach it.
  fp64_path: assemble, FP64 LU (DMMA tensor cores), FP64 solve -- the plain
    path and the reference answer: the learned answer's error is measured against it.
The same two paths plus the precision form (complex64 tcgen05 LU + FP64
refinement) also run on the 12^3-cell sphere (N = 19,872) with the
anisotropic tensor [[4,.5,0],[.5,6,0],[0,0,9]] + 0.1i ("secondary").  The
frequency-independent near-field precompute runs once per mesh before timing
("precompute_s"), as the reference amortises its FIBBI cache.

Also beside the headline: "learned_form.omega_sweep" runs the learned step
at omega = 0.5, 2 and 3 on the same sphere (the workload's frequency range
is [0.5, 3]) with Jacobi's step count beside it, and "jittered_n19872" the
12^3-cell sphere with jittered vertices -- the precision-form configuration
(+-0.05 h, Janus eps 4+0.2i / 12+1i) and the graph network's held-out check
(+-0.1 h, eps 6+0.5i) -- through the FP64, precision and learned paths.

Beside the headline (--no-extras skips them): "get_fields" times
GetFields for 4096 far and 4096 near points on the N = 57,222 sphere, and
"neq_flux" the buff-neq flux chain (dressed Rytov matrix, EMT flux columns)
per frequency for the N = 19,872 sphere.

value: device time of K steps (CUDA events on the library stream, barrier +
synchronize on both sides, max over ranks) / steps.  The matrices are far
larger than the 126 MB L2, so no flush is needed.
e2e: the learned step through the host-buffer C-ABI calls (RHS assembled to
host memory, solution copied back), host wall time including the copies,
mean over K steps (max over ranks).

--impl reference times the CPU restatement of the reference path (oracle
port: OpenMP assembly over all host cores, LAPACK zgetrf/zgetrs via OpenBLAS)
on bounded samples of the headline workload, extrapolated to the full size
(CpuModel): each step times a seeded 1 % sample of the assembly rows; the
LU is fitted from zgetrf timings at several N; a whole frequency of the
N = 19,872 sphere is run once as the calibration point.  ms_per_step is the
measured sample time, value the extrapolated seconds per frequency
("extrapolated": true).
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
EPS_LEARNED = 6 + 0.5j
WAVES = [([1, 0, 0], [0, 0, 1]), ([0, 1, 0], [0, 0, 1]), ([0, 0, 1], [1, 0, 0])]
OMEGA = 1.0
GMRES = dict(tol=1e-10, restart=80, maxit=1000, inner_tol=1e-5)
# ncu --set full capture of k_gm_matvec_sym_c64 (one launch, N = 5,760,
# profiles/gmres_matvec_c64_n5760.md): dram__bytes_read.sum + dram__bytes_write.sum
MATVEC_NCU_N, MATVEC_NCU_BYTES = 5760, 138.911232e6 + 5.009664e6


def eps_tensor():
    return np.array(TENSOR, complex) + 0.1j * np.eye(3)


def mesh_path(n, jitter=0.0, seed=0):
    import meshgen
    d = os.path.join(tempfile.gettempdir(), "buffem_bench_meshes")
    return meshgen.cached_sphere(d, n, 1.0, jitter, seed)


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


_ZGEMM_PEAK = []


def zgemm_peak_tflops():
    """FP64 tensor reference: cuBLAS ZGEMM (torch complex128 matmul) 8192^3,
    best of 5, CUDA events -- the measured denominator of the FP64 roofline
    (measured once per run)."""
    if _ZGEMM_PEAK:
        return _ZGEMM_PEAK[0]
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
    _ZGEMM_PEAK.append(8.0 * n ** 3 / best / 1e12)
    return _ZGEMM_PEAK[0]


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


def cgemm_kernel_bench(n, reps=5, shape=None):
    """Library complex64 GEMM (C -= A B on the tcgen05 TF32 tensor cores) on
    one n^3 (or M x N x K) problem, CUDA events on the library stream, best
    of reps."""
    import torch
    import buffem
    L = buffem.lib()
    stream = torch.cuda.ExternalStream(L.bg_stream())
    M, Nc, K = shape if shape else (n, n, n)
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(K, M, dtype=torch.complex64, device="cuda", generator=g)      # column-major M x K
    B = torch.randn(Nc, K, dtype=torch.complex64, device="cuda", generator=g)     # column-major K x N
    C = torch.zeros(Nc, M, dtype=torch.complex64, device="cuda")
    best = 1e30
    for i in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        buffem.cgemm_sub_device(M, Nc, K, A.data_ptr(), M, B.data_ptr(), K, C.data_ptr(), M)
        e1.record(stream)
        buffem.synchronize()
        if i:
            best = min(best, e0.elapsed_time(e1) / 1e3)
    tf = 8.0 * M * Nc * K / best / 1e12
    mp = measured_peaks().get("bf16_tflops")
    return {"kernel": "k_cgemm_tf32 (+ k_expand_a)", "shape": [M, Nc, K], "tflops": tf, "ms": best * 1e3,
            "tf32_peak_tflops": mp / 2 if mp else None, "peak_source": "half the measured dense BF16 burst rate",
            "frac_of_tf32_peak": tf / (mp / 2) if mp else None}


# ------------------------------------------------------------------ GPU arm
class Case:
    """One mesh/material on the device with the library's C-ABI handles."""

    def __init__(self, n, material, order, jitter=0.0, seed=0):
        import buffem
        self.buffem = buffem
        self.L = buffem.lib()
        self.G = buffem.SWGGeometry(meshfiles=mesh_path(n, jitter, seed), materials=material, singular_order=order)
        self.N = self.G.TotalBFs
        t0 = time.perf_counter()
        self.G.precompute()
        buffem.synchronize()
        self.precompute_s = time.perf_counter() - t0
        self.M = self.G.AllocateVIEMatrix()
        self.F = None
        self.E0s = [np.ascontiguousarray(np.array(e, complex)) for e, _ in WAVES]
        self.nhs = [np.ascontiguousarray(np.array(k, float)) for _, k in WAVES]
        self.nrhs = len(WAVES)

    def rhs_device(self, dB, w=OMEGA):
        b = self.buffem
        for i in range(self.nrhs):
            b._check(self.L.bg_rhs_planewave_device(self.G.h, w, 0.0, b._ptr(self.E0s[i]), b._ptr(self.nhs[i]),
                                                    b.C.c_void_p(dB[i].data_ptr())))

    def step_fp64(self, dB, w=OMEGA):
        b = self.buffem
        b._check(self.L.bg_assemble(self.G.h, w, 0.0, self.M.h))
        b._check(self.L.bg_lu_factor(self.M.h))
        self.rhs_device(dB, w)
        b._check(self.L.bg_lu_solve_device(self.M.h, b.C.c_void_p(dB.data_ptr()), self.N, self.nrhs))

    def ensure_c64(self):
        if self.F is None:
            self.F = self.G.AllocateVIEMatrix(self.buffem.BG_C64)

    def step_precision(self, dB, stats, tol=1e-12, w=OMEGA):
        b = self.buffem
        self.ensure_c64()
        b._check(self.L.bg_assemble_with_copy(self.G.h, w, 0.0, self.M.h, self.F.h))
        b._check(self.L.bg_lu_factor(self.F.h))
        self.rhs_device(dB, w)
        b._check(self.L.bg_lu_solve_refined_device(self.M.h, self.F.h, b.C.c_void_p(dB.data_ptr()), self.N,
                                                   self.nrhs, tol, 60, b._ptr(stats)))

    def step_learned(self, dB, net, stats, w=OMEGA, jacobi=False):
        b = self.buffem
        self.ensure_c64()
        b._check(self.L.bg_assemble_with_copy(self.G.h, w, 0.0, self.M.h, self.F.h))
        P = b.Preconditioner.jacobi(self.M) if jacobi else b.Preconditioner.learned(self.G, self.M, w, net)
        self.rhs_device(dB, w)
        b._check(self.L.bg_gmres_solve_lu_fallback_device(
            self.M.h, self.F.h, P.h, b.C.c_void_p(dB.data_ptr()), self.N, self.nrhs, GMRES["tol"],
            GMRES["restart"], GMRES["maxit"], GMRES["inner_tol"], b._ptr(stats)))
        del P

    def step_learned_host(self, hostB, rhs_h, net, stats):
        """Same work through host buffers: RHS to host, solve with host in/out."""
        b = self.buffem
        self.ensure_c64()
        b._check(self.L.bg_assemble_with_copy(self.G.h, OMEGA, 0.0, self.M.h, self.F.h))
        P = b.Preconditioner.learned(self.G, self.M, OMEGA, net)
        for i in range(self.nrhs):
            b._check(self.L.bg_rhs_planewave(self.G.h, OMEGA, 0.0, b._ptr(self.E0s[i]), b._ptr(self.nhs[i]),
                                             b._ptr(rhs_h)))
            hostB[:, i] = rhs_h
        b._check(self.L.bg_gmres_solve_lu_fallback(self.M.h, self.F.h, P.h, b._ptr(hostB), self.nrhs,
                                                   GMRES["tol"], GMRES["restart"], GMRES["maxit"],
                                                   GMRES["inner_tol"], b._ptr(stats)))
        del P

    def free(self):
        self.F = None
        self.M = None
        self.G = None


def max_over_ranks(t, world, device="cuda"):
    """The largest of the ranks' values (all_reduce MAX over the process
    group; every rank gets it); with one rank, t itself."""
    if world <= 1:
        return t
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def whole_job_seconds_per_frequency(t_max, steps, world):
    """Replicas: each of the world ranks runs `steps` independent frequencies
    in t_max seconds (the slowest rank), so the whole job processes
    steps * world frequencies in that time."""
    return t_max / (steps * world)


def timed(stream, fn, steps, warmup, world):
    """Device seconds of `steps` calls after `warmup` untimed ones (CUDA events
    on the library stream, barrier + synchronize on both sides, max over ranks)."""
    import torch
    import torch.distributed as dist
    import buffem
    for _ in range(warmup):
        fn()
    buffem.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    buffem.synchronize()
    torch.cuda.synchronize()
    return max_over_ranks(e0.elapsed_time(e1) / 1e3, world)


def rel_err(x, ref):
    import torch
    return float(torch.linalg.norm(x - ref) / torch.linalg.norm(ref))


def batch_geometries(seed=2026, count=8):
    """Two-sphere geometries of the batching workload: radii U[0.5, 1.5],
    surface gap U[0.2, 1] along z, cells per edge n1, n2 in 2..10 redrawn until
    1k <= N1 + N2 <= 12k, eps(x) = 3 + 1.5 exp(-|x - c|^2) + 0.1i about each
    sphere's own centre c."""
    import buffem
    import meshgen
    rng = np.random.default_rng(seed)
    d = os.path.join(tempfile.gettempdir(), "buffem_bench_meshes")
    F = lambda n: 12 * n ** 3 - 6 * n ** 2
    out = []
    for _ in range(count):
        r1, r2 = rng.uniform(0.5, 1.5, 2)
        gap = rng.uniform(0.2, 1.0)
        while True:
            n1, n2 = rng.integers(2, 11, 2)
            if 1000 <= F(n1) + F(n2) <= 12000:
                break
        z2 = r1 + gap + r2
        mats = [buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, width=1.0, center=(0, 0, 0)),
                buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, width=1.0, center=(0, 0, z2))]
        G = buffem.SWGGeometry(meshfiles=[meshgen.cached_sphere(d, int(n1), float(r1)),
                                          meshgen.cached_sphere(d, int(n2), float(r2))],
                               materials=mats, displacements=[[0, 0, 0], [0, 0, z2]])
        out.append((G, dict(r1=float(r1), r2=float(r2), gap=float(gap), n1=int(n1), n2=int(n2), N=G.TotalBFs)))
    return out


def run_batching(nomega=64):
    """Batching form: 8 geometries x 64 log-spaced omega in [0.01, 10] through
    bg_batch_sweep, and the same kind of job one at a time through the plain
    calls (two frequencies per geometry) for comparison."""
    import torch
    import buffem
    geo = batch_geometries()
    omegas = np.logspace(-2, 1, nomega)
    wave = buffem.PlaneWave([1, 0, 0], [0, 0, 1])
    for G, _ in geo:
        G.precompute()
    buffem.synchronize()
    pabs, st = buffem.BatchSweep([g for g, _ in geo], omegas, wave, max_streams=8)
    seq = []
    for G, meta in geo:
        ts = []
        for w in (omegas[10], omegas[40]):
            buffem.synchronize()
            t0 = time.perf_counter()
            M = G.AssembleVIEMatrix(w)
            M.LUFactorize()
            x = G.AssembleRHSVector(w, wave)
            M.LUSolve(x)
            G.GetPFTMatrix(x, w, wave, method=buffem.BG_PFT_OVERLAP)
            ts.append(time.perf_counter() - t0)
            del M
        seq.append(min(ts))
    Ns = [m["N"] for _, m in geo]
    seq_total = sum(t * nomega for t in seq)
    # roofline: the jobs' LU flops (8/3 N^3 real flops of a complex LU) over
    # the sweep's time, against the measured FP64 tensor rate (cuBLAS ZGEMM)
    lu_flops = sum(8.0 / 3.0 * float(n) ** 3 for n in Ns) * nomega
    zpk = zgemm_peak_tflops()
    achieved = lu_flops / float(st[0]) / 1e12
    tiles = ("64x64", "128x64", "64x128")
    tuning = [{"N": Ns[i], "panel_rows": int(st[4 + 4 * i]), "slots": int(st[5 + 4 * i]),
               "gemm_tile": tiles[int(st[7 + 4 * i])]} for i in range(len(geo))]
    torch.cuda.empty_cache()
    return {"jobs": int(st[1]), "seconds": float(st[0]), "s_per_job": float(st[0] / st[1]),
            "graphs": bool(st[2]), "capture_fell_back": bool(st[3]), "geometries": [m for _, m in geo],
            "tuning": tuning, "one_by_one_estimate_s": seq_total,
            "speedup_vs_one_by_one": seq_total / float(st[0]),
            "one_by_one_note": "plain host-API calls per job (assemble, LU, RHS, solve, overlap PFT), best of 2 "
                               "frequencies per geometry x 64",
            "pabs_finite": bool(np.all(np.isfinite(pabs))),
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": zpk, "unit": "TFLOP/s",
                         "frac": achieved / zpk if zpk else None,
                         "algorithmic": "8/3 N^3 FP64 flops per job (the complex LU; assembly, solve and power "
                                        "not counted) summed over the 8 geometries x omegas, over the sweep's time",
                         "peak_source": "cuBLAS ZGEMM 8192^3 measured in this run"}}


FIELD_FLOPS_PER_POINT = 156   # FP64 adds/multiplies of one quadrature point (FMA = 2), no sincos/rsqrt


def run_fields(stream, n=17, npts=4096, steps=3):
    """GetFields on the headline sphere (N = 57,222): npts far points (4-point
    rule for every basis function) and npts near points (both rules), for
    seeded random currents already on the device."""
    import ctypes as C
    import torch
    import buffem
    G = buffem.SWGGeometry(meshfiles=mesh_path(n), materials=buffem.Material(eps=EPS_LEARNED))
    N, NT = G.TotalBFs, 6 * n ** 3
    rng = np.random.default_rng(11)
    J = torch.tensor(rng.normal(size=N) + 1j * rng.normal(size=N), dtype=torch.complex128, device="cuda")
    L = buffem.lib()
    out = {"N": N, "tets": NT, "points": npts}
    for label, rmin, rmax in (("far", 5.0, 50.0), ("near", 1.02, 2.0)):
        d = rng.normal(size=(npts, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        X = torch.tensor(d * rng.uniform(rmin, rmax, size=(npts, 1)), dtype=torch.float64, device="cuda")
        F = torch.zeros((npts, 6), dtype=torch.complex128, device="cuda")
        fn = lambda: buffem._check(L.bg_get_fields_device(G.h, OMEGA, 0.0, C.c_void_p(J.data_ptr()), None, None,
                                                          npts, C.c_void_p(X.data_ptr()), C.c_void_p(F.data_ptr())))
        t = timed(stream, fn, steps, 2, 1) / steps
        out[label] = {"ms": t * 1e3, "radius": [rmin, rmax], "tet_point_pairs_per_s": npts * NT / t}
        if label == "far":
            evals = 4.0 * npts * NT
            out[label]["quadrature_points_per_s"] = evals / t
            out[label]["fp64_tflops"] = evals * FIELD_FLOPS_PER_POINT / t / 1e12
    del G
    return out


def small_case(kind, n):
    """Profiler-sized runs of the GetFields and buff-neq kernels (wall time)."""
    import ctypes as C
    import torch
    import buffem
    G = buffem.SWGGeometry(meshfiles=mesh_path(n), materials=buffem.Material(eps=EPS_LEARNED))
    N = G.TotalBFs
    t0 = time.perf_counter()
    if kind == "fields":
        rng = np.random.default_rng(1)
        J = torch.tensor(rng.normal(size=N) + 1j * rng.normal(size=N), dtype=torch.complex128, device="cuda")
        P = 2048
        d = rng.normal(size=(P, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        X = torch.tensor(d * rng.uniform(5, 50, size=(P, 1)), dtype=torch.float64, device="cuda")
        F = torch.zeros((P, 6), dtype=torch.complex128, device="cuda")
        for _ in range(2):
            buffem._check(buffem.lib().bg_get_fields_device(G.h, OMEGA, 0.0, C.c_void_p(J.data_ptr()), None, None,
                                                            P, C.c_void_p(X.data_ptr()), C.c_void_p(F.data_ptr())))
        res = {"points": P, "checksum": float(F.abs().sum())}
    else:
        G.precompute()
        neq = buffem.NEQ(G)
        neq.GetFlux(0.3)
        F = neq.GetFlux(0.31)
        res = {"prad": float(F[0, 0, 1])}
    res.update({"kind": kind, "N": N, "wall_s": time.perf_counter() - t0})
    return res


def precision_case(n, order):
    """Profiler-sized run of the precision form: the --n-cell sphere with the
    anisotropic tensor eps, one warm-up step, then one step inside an NVTX
    range 'prec' (for ncu --nvtx-include "prec/"), timed with CUDA events,
    with its kernel classes."""
    import torch
    import buffem
    L = buffem.lib()
    stream = torch.cuda.ExternalStream(L.bg_stream())
    sc = Case(n, buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=eps_tensor()), order)
    dB = torch.zeros((sc.nrhs, sc.N), dtype=torch.complex128, device="cuda")
    st = np.zeros(3)
    sc.step_precision(dB, st)
    buffem.synchronize()
    buffem.profile_begin()
    torch.cuda.nvtx.range_push("prec")
    t = timed(stream, lambda: sc.step_precision(dB, st), 1, 0, 1)
    torch.cuda.nvtx.range_pop()
    pm = buffem.profile_read()
    buffem.profile_end()
    return {"kind": "precision", "N": sc.N, "step_s": t, "refinement_sweeps": int(st[0]),
            "kernel_ms": {k: round(v["ms"], 2) for k, v in pm.items() if v["launches"]},
            "launches": {k: v["launches"] for k, v in pm.items() if v["launches"]}}


def neq_flops(N):
    """FP64 flops of one frequency of the flux chain for one object: S^-1 G,
    S^-1 (V S^-1 G), LU of W, S^-1 R S^-1 (dense block), two N-column solves."""
    return (8 + 8 + 8.0 / 3 + 8 + 8 + 8) * float(N) ** 3


def run_neq(stream, n=12, steps=2):
    """buff-neq flux chain for one sphere (N = 19,872 at n = 12): set-up (S^-1)
    once, then GetFlux at distinct frequencies (each refactors W)."""
    import buffem
    G = buffem.SWGGeometry(meshfiles=mesh_path(n), materials=buffem.Material(eps=EPS_LEARNED))
    N = G.TotalBFs
    G.precompute()
    buffem.synchronize()
    t0 = time.perf_counter()
    neq = buffem.NEQ(G)
    t_setup = time.perf_counter() - t0
    k = [0]

    def fn():
        k[0] += 1
        neq.GetFlux(0.3 + 0.01 * k[0])
    t = timed(stream, fn, steps, 1, 1) / steps
    F = neq.GetFlux(0.3)
    del neq
    return {"N": N, "setup_s": t_setup, "s_per_frequency": t, "flops_per_frequency": neq_flops(N),
            "fp64_tflops": neq_flops(N) / t / 1e12, "prad_at_0.3": float(F[0, 0, 1]),
            "pabs_plus_prad": float(F[0, 0, 0] + F[0, 0, 1]),
            "note": "one object, EMT flux columns; W factored once per frequency"}


def run_gpu(args, rank, world, local_rank):
    import torch
    import buffem

    torch.cuda.set_device(local_rank)
    L = buffem.lib()
    stream = torch.cuda.ExternalStream(L.bg_stream())
    net = buffem.GNN.load()
    out = {}

    # ---------------- headline: learned form at N = 57,222
    case = Case(args.n, buffem.Material(eps=EPS_LEARNED), args.order)
    N = case.N
    dB = torch.zeros((case.nrhs, N), dtype=torch.complex128, device="cuda")   # column-major N x nrhs
    x_fp64 = None
    t_fp64 = None
    prof_fp64 = None
    if args.fp64_steps > 0:
        for _ in range(args.fp64_warmup):   # outside the class profile: it covers the timed steps only
            case.step_fp64(dB)
        buffem.profile_begin()
        t_fp64 = timed(stream, lambda: case.step_fp64(dB), args.fp64_steps, 0, world)
        prof_fp64 = buffem.profile_read()
        buffem.profile_end()
        x_fp64 = dB.clone()
    stats = np.zeros(4)
    clocks = ClockSampler(local_rank)
    for _ in range(args.warmup):
        case.step_learned(dB, net, stats)
    buffem.synchronize()
    clocks.start()
    launches0 = buffem.launch_count()
    buffem.profile_begin()
    t_learned = timed(stream, lambda: case.step_learned(dB, net, stats), args.steps, 0, world)
    prof = buffem.profile_read()
    buffem.profile_end()
    launches = buffem.launch_count() - launches0
    clk = clocks.stop()
    learned = {"steps_per_frequency": int(stats[0]), "final_rel_residual": float(stats[1]),
               "refinement_sweeps": int(stats[2]), "lu_fallback": bool(stats[3]), "gmres": buffem.GMRESLastInfo()}
    # phase breakdown of one more (untimed) step, events on the library stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    ev[0].record(stream)
    buffem._check(L.bg_assemble_with_copy(case.G.h, OMEGA, 0.0, case.M.h, case.F.h))   # + complex64 copy
    ev[1].record(stream)
    P = buffem.Preconditioner.learned(case.G, case.M, OMEGA, net)
    ev[2].record(stream)
    case.rhs_device(dB)
    ev[3].record(stream)
    buffem._check(L.bg_gmres_solve_lu_fallback_device(case.M.h, case.F.h, P.h, buffem.C.c_void_p(dB.data_ptr()),
                                                      N, case.nrhs, GMRES["tol"], GMRES["restart"], GMRES["maxit"],
                                                      GMRES["inner_tol"], buffem._ptr(stats)))
    ev[4].record(stream)
    buffem.synchronize()
    rho_smax = P.bound()
    del P
    learned["phases_s"] = {k: ev[i].elapsed_time(ev[i + 1]) / 1e3 for i, k in
                           enumerate(("assemble_with_c64_copy", "gnn_precond", "rhs", "gmres_solve"))}
    learned["precond_bound"] = {"rho_K1": rho_smax[0], "smax": rho_smax[1]}
    if x_fp64 is not None:
        learned["err_vs_fp64_lu"] = rel_err(dB, x_fp64)
    # the same solve preconditioned by Jacobi: what the network gains
    P = buffem.Preconditioner.jacobi(case.M)
    js = np.zeros(4)
    case.rhs_device(dB)
    buffem._check(L.bg_assemble_with_copy(case.G.h, OMEGA, 0.0, case.M.h, case.F.h))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    buffem._check(L.bg_gmres_solve_lu_fallback_device(case.M.h, case.F.h, P.h, buffem.C.c_void_p(dB.data_ptr()),
                                                      N, case.nrhs, GMRES["tol"], GMRES["restart"], GMRES["maxit"],
                                                      GMRES["inner_tol"], buffem._ptr(js)))
    e1.record(stream)
    buffem.synchronize()
    learned["jacobi_same_solve"] = {"steps": int(js[0]), "solve_s": e0.elapsed_time(e1) / 1e3,
                                    "lu_fallback": bool(js[3])}
    del P
    # the learned form across the frequency range of the workload (omega in
    # [0.5, 3]; the headline runs omega = 1): steps, fallback and device time
    # of one whole step each, beside Jacobi's steps at the same omega
    if not args.lean:
        sweep = []
        for w in (0.5, 2.0, 3.0):
            st = np.zeros(4)
            t = timed(stream, lambda: case.step_learned(dB, net, st, w=w), 1, 0, world)
            info = buffem.GMRESLastInfo()
            sj = np.zeros(4)
            tj = timed(stream, lambda: case.step_learned(dB, net, sj, w=w, jacobi=True), 1, 0, world)
            sweep.append({"omega": w, "step_s": t, "steps": int(st[0]), "final_rel_residual": float(st[1]),
                          "lu_fallback": bool(st[3]), "switched_to_jacobi": info["switched_to_jacobi"],
                          "stopped_early": info["stopped_early"], "longest_cycle": info["longest_cycle"],
                          "jacobi_steps": int(sj[0]), "jacobi_step_s": tj, "jacobi_lu_fallback": bool(sj[3])})
        learned["omega_sweep"] = sweep
    # e2e through host buffers
    hostB = np.zeros((N, case.nrhs), complex, order="F")
    rhs_h = np.zeros(N, complex)
    times = []
    for _ in range(0 if args.lean else max(1, args.steps)):
        buffem.synchronize()
        t0 = time.perf_counter()
        case.step_learned_host(hostB, rhs_h, net, stats)
        times.append(time.perf_counter() - t0)
    e2e_s = sum(times) / len(times) if times else None     # mean over the K steps, as value
    if e2e_s is not None:
        e2e_s = max_over_ranks(e2e_s, world)
    out.update(N=N, nrhs=case.nrhs, t_learned=t_learned, t_fp64=t_fp64, prof=prof, prof_fp64=prof_fp64,
               launches=launches, clocks=clk, learned=learned, precompute_s=case.precompute_s, e2e_s=e2e_s)
    case.free()
    del dB, x_fp64
    torch.cuda.empty_cache()

    # ---------------- secondary: N = 19,872 anisotropic sphere, all three paths
    if args.n_small > 0 and not args.lean:
        sc = Case(args.n_small, buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=eps_tensor()), args.order)
        dB = torch.zeros((sc.nrhs, sc.N), dtype=torch.complex128, device="cuda")
        sec = {"N": sc.N, "precompute_s": sc.precompute_s}
        sc.step_fp64(dB)   # warm-up, outside the class profile
        buffem.profile_begin()
        t = timed(stream, lambda: sc.step_fp64(dB), 2, 0, world)
        pf = buffem.profile_read()
        buffem.profile_end()
        ref = dB.clone()
        sec["fp64_path_s"] = t / 2
        sec["fp64_lu_tflops"] = pf["lu_gemm"]["flops"] / (pf["lu_gemm"]["ms"] / 1e3) / 1e12 if pf["lu_gemm"]["ms"] else None
        st = np.zeros(3)
        sc.step_precision(dB, st)   # warm-up, outside the class profile
        buffem.profile_begin()
        t = timed(stream, lambda: sc.step_precision(dB, st), 2, 0, world)
        pm = buffem.profile_read()
        buffem.profile_end()
        sec["precision_form_s"] = t / 2
        sec["precision_form_err_vs_fp64_lu"] = rel_err(dB, ref)
        sec["precision_form_gemm_tflops"] = pm["lu_gemm"]["flops"] / (pm["lu_gemm"]["ms"] / 1e3) / 1e12 if pm["lu_gemm"]["ms"] else None
        sec["precision_form_kernel_ms_per_step"] = {k: v["ms"] / 2 for k, v in pm.items() if v["launches"]}
        # roofline of the precision form's LU: the TF32 trailing updates
        # against the TF32 tensor rate (half the measured dense BF16 burst),
        # and the factorisation's 8/3 N^3 flops over all its LU kernels
        mp = measured_peaks().get("bf16_tflops")
        lu_ms = sum(pm[c]["ms"] for c in ("lu_gemm", "lu_panel", "lu_laswp", "trsm_leaf")) / 2
        lu_tf = 8.0 / 3.0 * float(sc.N) ** 3 / (lu_ms / 1e3) / 1e12 if lu_ms else None
        gtf = sec["precision_form_gemm_tflops"]
        sec["precision_form_roofline"] = {
            "bound": "tensor", "kernel": "k_cgemm_tf32 (tcgen05 kind::tf32, complex64 trailing updates)",
            "achieved": gtf, "peak": mp / 2 if mp else None, "unit": "TFLOP/s",
            "frac": gtf / (mp / 2) if (mp and gtf) else None,
            "algorithmic": "8 M N K real flops per complex64 GEMM call, summed over the factorisation, over the "
                           "calls' CUDA-event time",
            "peak_source": "half the measured dense BF16 burst of MEASURED_PEAKS.json (of measured)",
            "lu_step": {"flops": 8.0 / 3.0 * float(sc.N) ** 3, "lu_kernels_ms": lu_ms, "achieved_tflops": lu_tf,
                        "frac_of_tf32": lu_tf / (mp / 2) if (mp and lu_tf) else None,
                        "note": "the panels, TRSM leaves and interchanges are latency-bound; the GEMMs are not"}}
        sec["fp64_kernel_ms_per_step"] = {k: v["ms"] / 2 for k, v in pf.items() if v["launches"]}
        st4 = np.zeros(4)
        t = timed(stream, lambda: sc.step_learned(dB, net, st4), 2, 1, world)
        sec["learned_s"] = t / 2
        sec["learned_err_vs_fp64_lu"] = rel_err(dB, ref)
        sec["learned_steps"] = int(st4[0])
        sec["learned_lu_fallback"] = bool(st4[3])
        out["secondary"] = sec
        sc.free()
        del dB, ref
        torch.cuda.empty_cache()
        out["jittered_n19872"] = run_jittered(args, stream, net, world)
    return out


def run_jittered(args, stream, net, world):
    """The 12^3-cell sphere with jittered vertices: (a) the precision-form
    configuration (+-0.05 h, seed 2, Janus eps = 4+0.2i for z > 0, 12+1i
    below), precision form and learned form against the FP64 path; (b) the
    graph network's held-out training check (+-0.1 h, seed 4254, eps 6+0.5i),
    learned form against Jacobi.  omega = 1, three plane waves."""
    import torch
    import buffem
    res = {}
    cases = (("janus_jitter0.05", buffem.Material(kind=buffem.BG_MAT_JANUS_Z, eps=4 + 0.2j, eps2=12 + 1j), 0.05, 2),
             ("eps6_jitter0.1", buffem.Material(eps=EPS_LEARNED), 0.1, 4242 + 12))
    for name, mat, jit, seed in cases:
        sc = Case(args.n_small, mat, args.order, jitter=jit, seed=seed)
        dB = torch.zeros((sc.nrhs, sc.N), dtype=torch.complex128, device="cuda")
        r = {"N": sc.N, "jitter": jit, "seed": seed, "precompute_s": sc.precompute_s}
        r["fp64_path_s"] = timed(stream, lambda: sc.step_fp64(dB), 1, 1, world)
        ref = dB.clone()
        st = np.zeros(3)
        r["precision_form_s"] = timed(stream, lambda: sc.step_precision(dB, st), 1, 1, world)
        r["precision_form_err_vs_fp64_lu"] = rel_err(dB, ref)
        r["precision_form_refinement_sweeps"] = int(st[0])
        st4 = np.zeros(4)
        r["learned_s"] = timed(stream, lambda: sc.step_learned(dB, net, st4), 1, 1, world)
        r["learned_gmres"] = buffem.GMRESLastInfo()
        r["learned_err_vs_fp64_lu"] = rel_err(dB, ref)
        r["learned_steps"] = int(st4[0])
        r["learned_lu_fallback"] = bool(st4[3])
        sj = np.zeros(4)
        r["jacobi_s"] = timed(stream, lambda: sc.step_learned(dB, net, sj, jacobi=True), 1, 0, world)
        r["jacobi_steps"] = int(sj[0])
        r["jacobi_lu_fallback"] = bool(sj[3])
        res[name] = r
        sc.free()
        del dB, ref
        torch.cuda.empty_cache()
    return res


# ------------------------------------------------------------------ CPU arm
# The CPU restatement of the reference path (oracle port: OpenMP assembly on
# all host cores, OpenBLAS zgetrf/zgetrs through scipy) cannot run a whole
# frequency of the headline workload inside a bench step (about 9 minutes
# on 16 cores), so it is measured in parts and extrapolated:
#   assembly: a seeded sample of 1 % of the rows, the upper-triangle entries
#     b >= a that the reference computes (AssembleGBlock, VIEMatrix.cc:365-426,
#     the lower triangle is the symmetric fill), scaled by all entries
#     N (N + 1) / 2 over the entries of the sampled rows;
#   LU and solve: zgetrf + zgetrs (3 right-hand sides) timed at several N and
#     fitted by a N^3 + b N^2 and c N^2.
# Each step times one row sample; the LU fit is measured once before the
# steps.  The near-field cache of the sampled rows is built before timing
# (the reference's FIBBI cache, amortised like the GPU's precompute; the
# singular rule used to fill it does not change the per-frequency work, so
# the fixed order-6 rule keeps its build short).  With calibrate=True a whole
# frequency of the 12^3-cell sphere (N = 19,872) is also run and timed --
# full assembly, zgetrf and zgetrs of that matrix -- beside the model's
# prediction for it; its factorisation is one of the LU fit points.

def _cpu_random_matrix(N, rng):
    A = np.empty((N, N), np.complex128, order="F")
    A.real = rng.random((N, N))
    A.imag = rng.random((N, N))
    return A


def _cpu_time_lu(A, nrhs=3, rng=None):
    import scipy.linalg as sl
    rng = rng or np.random.default_rng(0)
    N = A.shape[0]
    t0 = time.perf_counter()
    lu = sl.lu_factor(A, overwrite_a=True, check_finite=False)
    t_f = time.perf_counter() - t0
    B = rng.random((N, nrhs)) + 1j * rng.random((N, nrhs))
    t0 = time.perf_counter()
    sl.lu_solve(lu, B, check_finite=False)
    return t_f, time.perf_counter() - t0


class CpuModel:
    """Extrapolation model of one frequency of the oracle port at size n."""

    def __init__(self, n, fit_ns=(5760, 11400), calibrate=False, row_frac=0.01, seed=0, cal_n=12):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        self.oracle = oracle
        self.cores = oracle.lib().or_num_threads()
        rng = np.random.default_rng(seed)
        self.lu_points = []
        for N in fit_ns:
            self.lu_points.append((N,) + _cpu_time_lu(_cpu_random_matrix(N, rng), rng=rng))
        self.calibration = None
        if calibrate:
            self.calibration = self._calibrate(cal_n, row_frac, rng)
        self._fit()
        self.G = oracle.Geometry(mesh_path(n), oracle.material(eps=EPS_LEARNED), nang=6)
        self.N = self.G.N
        self.rows = self._rows(self.N, row_frac, rng)
        t0 = time.perf_counter()
        self.G.cache_build(self.rows)
        self.t_cache = time.perf_counter() - t0

    @staticmethod
    def _rows(N, frac, rng):
        return np.sort(rng.choice(N, max(32, int(math.ceil(frac * N))), replace=False)).astype(np.int32)

    @staticmethod
    def _entry_scale(N, rows):
        return N * (N + 1) / 2.0 / float(np.sum(N - rows.astype(np.float64)))

    def _fit(self):
        self.lu_points.sort(key=lambda p: p[0])
        Ns = np.array([p[0] for p in self.lu_points], float)
        tf = np.array([p[1] for p in self.lu_points])
        ts = np.array([p[2] for p in self.lu_points])
        X = np.stack([Ns ** 3, Ns ** 2], 1)
        coef, *_ = np.linalg.lstsq(X, tf, rcond=None)
        if coef[0] <= 0 or coef[1] < 0 or len(Ns) < 3:   # a N^3 through the largest point instead
            coef = np.array([tf[-1] / Ns[-1] ** 3, 0.0])
        self.lu_coef = coef
        self.sv_coef = float(ts[-1] / Ns[-1] ** 2)
        self.lu_residuals = [float((X[i] @ coef) / tf[i] - 1) for i in range(len(Ns))]

    def lu_seconds(self, N):
        return float(self.lu_coef[0] * N ** 3 + self.lu_coef[1] * N ** 2), float(self.sv_coef * N ** 2)

    def _calibrate(self, n, row_frac, rng):
        G = self.oracle.Geometry(mesh_path(n), self.oracle.material(eps=EPS_LEARNED), nang=6)
        N = G.N
        rows = self._rows(N, row_frac, rng)
        G.cache_build()
        t0 = time.perf_counter()
        G.assemble_rows(complex(OMEGA), rows)
        t_rows = time.perf_counter() - t0
        t0 = time.perf_counter()
        A = G.assemble(complex(OMEGA))
        t_asm = time.perf_counter() - t0
        A = np.asfortranarray(A)
        t_f, t_s = _cpu_time_lu(A, rng=rng)
        del A
        self.lu_points.append((N, t_f, t_s))
        return {"N": N, "n_cells": n, "measured_s": t_asm + t_f + t_s,
                "measured": {"assemble": t_asm, "lu": t_f, "solve": t_s},
                "predicted_assemble_s": t_rows * self._entry_scale(N, rows), "rows": int(len(rows))}

    def step(self):
        """One timed sample: the row sample's assembly; returns (seconds
        measured, extrapolated seconds per frequency, parts)."""
        t0 = time.perf_counter()
        self.G.assemble_rows(complex(OMEGA), self.rows)
        t_rows = time.perf_counter() - t0
        t_asm = t_rows * self._entry_scale(self.N, self.rows)
        t_lu, t_sv = self.lu_seconds(self.N)
        return t_rows, t_asm + t_lu + t_sv, {"assemble": t_asm, "lu": t_lu, "solve": t_sv}

    def describe(self):
        d = {"rows": int(len(self.rows)), "row_fraction": len(self.rows) / self.N,
             "entry_scale": self._entry_scale(self.N, self.rows),
             "lu_fit": {"points": [{"N": p[0], "zgetrf_s": p[1], "zgetrs_3rhs_s": p[2]} for p in self.lu_points],
                        "a_N3_plus_b_N2": [float(c) for c in self.lu_coef], "solve_c_N2": self.sv_coef,
                        "relative_residuals": self.lu_residuals},
             "near_cache_build_s_excluded": self.t_cache}
        if self.calibration:
            c = dict(self.calibration)
            lu, sv = self.lu_seconds(c["N"])
            c["predicted_s"] = c["predicted_assemble_s"] + lu + sv
            c["predicted_over_measured"] = c["predicted_s"] / c["measured_s"]
            d["calibration"] = c
        return d

    def sample_text(self):
        pts = ", ".join(str(p[0]) for p in self.lu_points)
        return (f"sphere {round((self.N / 12) ** (1 / 3))}^3 cells, N={self.N}, eps={EPS_LEARNED}, omega={OMEGA}: "
                f"oracle assembly of a seeded {len(self.rows)}-row sample ({100 * len(self.rows) / self.N:.1f} % of "
                f"rows, upper-triangle entries, scaled x{self._entry_scale(self.N, self.rows):.0f}) timed per step; "
                f"OpenBLAS zgetrf + zgetrs (3 RHS) timed at N = {pts} and fitted a N^3 + b N^2; near-field cache "
                f"build excluded like the GPU precompute; extrapolated to the full frequency")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=17, help="cells per cube edge of the headline sphere (17 -> N=57,222)")
    ap.add_argument("--n-small", type=int, default=12, help="secondary sphere (12 -> N=19,872); 0 skips it")
    ap.add_argument("--fp64-steps", type=int, default=1, help="timed steps of the FP64 path at the headline size")
    ap.add_argument("--fp64-warmup", type=int, default=1)
    ap.add_argument("--order", type=int, default=10, help="singular-rule order")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching-form sweep (8 geometries x 64 omega)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the GetFields and buff-neq flux measurements")
    ap.add_argument("--lean", action="store_true",
                    help="headline learned steps only (no FP64 arm, e2e, secondary, CPU baseline): profiler runs")
    ap.add_argument("--kernel", default=None, choices=["gemm", "cgemm", "fields", "neq", "precision"],
                    help="one small case for profilers: gemm = the LU trailing-update GEMM on an M=N=K=--size "
                         "problem (complex128, DMMA); cgemm = the same on the complex64 tcgen05 GEMM of the "
                         "precision form; fields = two GetFields calls, 2048 far points on the --size-cell "
                         "sphere; neq = two buff-neq flux frequencies on the --size-cell sphere; precision = "
                         "one precision-form step (complex64 LU + FP64 refinement) on the --n-cell sphere")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--shape", default=None, help="M,N,K for --kernel cgemm (default: --size cubed)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup

    if args.kernel == "gemm":
        print(json.dumps(gemm_kernel_bench(args.size)), flush=True)
        return
    if args.kernel == "cgemm":
        shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else None
        print(json.dumps(cgemm_kernel_bench(args.size, shape=shape)), flush=True)
        return
    if args.kernel in ("fields", "neq"):
        print(json.dumps(small_case(args.kernel, args.size)), flush=True)
        return
    if args.kernel == "precision":
        print(json.dumps(precision_case(args.n, args.order)), flush=True)
        return
    if args.lean:
        args.no_cpu_baseline = True
        args.fp64_steps = 0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    N_head = 12 * args.n ** 3 - 6 * args.n ** 2
    config = {"workload": f"learned form: sphere {args.n}^3 cells x 6 tets (N={N_head}), eps={EPS_LEARNED}, "
                          f"omega={OMEGA}, 3 plane-wave RHS; mixed-precision GMRES(80) + graph-network "
                          f"near-field preconditioner, LU fallback; vs plain FP64 assemble+LU+solve",
              "N": N_head, "n_cells": args.n, "omega": OMEGA, "rhs": 3, "singular_order": args.order,
              "gmres": GMRES, "parallelism": f"replicas x{world} (independent frequencies)",
              "l2": "matrices (8-16 N^2 bytes) >> 126 MB L2; no flush needed"}

    if args.impl == "reference":
        if rank != 0:
            return
        model = CpuModel(args.n, fit_ns=(5760, 11400), calibrate=True)
        for _ in range(args.warmup):
            model.step()
        meas, vals, parts = [], [], None
        for _ in range(max(1, args.steps)):
            t, v, parts = model.step()
            meas.append(t)
            vals.append(v)
        v = statistics.median(vals)
        line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": statistics.mean(meas) * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": config,
                "impl": "reference", "extrapolated": True,
                "timing_note": "ms_per_step is the measured time of one step's sample (1 % of the assembly rows); "
                               "value is the whole frequency extrapolated from it and from the LU fit",
                "cpu_baseline": {"value": v, "unit": "s", "cores": model.cores, "kind": "port",
                                 "sample": model.sample_text()},
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "breakdown": parts, "spread": {"min": min(vals), "max": max(vals)},
                "extrapolation": model.describe()}
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
    value = whole_job_seconds_per_frequency(res["t_learned"], args.steps, world)
    prof = res["prof"]
    mp = measured_peaks()
    hbm = mp.get("hbm_gbs")
    mv = prof["gmres_matvec"]
    far = prof["assemble_far"]
    total_ms = sum(v["ms"] for v in prof.values())
    mv_gbs = mv["flops"] / (mv["ms"] / 1e3) / 1e9 if mv["ms"] > 0 else None
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["t_learned"] / args.steps * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "c128 assembly; c64 Krylov matrix-vector products with FP64 refinement",
            "data": "synthetic", "config": config,
            "learned_form": res["learned"],
            "kernel_classes": prof, "precompute_s": res["precompute_s"],
            "roofline": {"bound": "hbm", "kernel": "k_gm_matvec_sym_c64 (+ k_gm_matvec_sum): GMRES matrix-vector "
                                                   "products on the complex64 matrix",
                         "achieved": mv_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": (mv_gbs / hbm) if (mv_gbs and hbm) else None,
                         "traffic": MATVEC_NCU_BYTES * (N / MATVEC_NCU_N) ** 2,
                         "traffic_source": f"ncu dram read+write of one launch at N={MATVEC_NCU_N} "
                                           f"({MATVEC_NCU_BYTES:.4g} B), scaled by N^2",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm else "unavailable",
                         "algorithmic": "4 N^2 + 1024 N bytes per product: the upper-triangle 256x256 tiles of the "
                                        "symmetric complex64 matrix, read once for all 3 right-hand sides ("
                                        "16 N^2 for the complex128 residual products)",
                         "share_of_profiled_ms": mv["ms"] / total_ms if total_ms else None,
                         "assemble_far_share_of_profiled_ms": far["ms"] / total_ms if total_ms else None},
            "e2e": {"value": whole_job_seconds_per_frequency(res["e2e_s"], 1, world) if res["e2e_s"] else None,
                    "unit": "s",
                    "h2d_bytes_per_step": 16 * N * res["nrhs"],
                    "d2h_bytes_per_step": 2 * 16 * N * res["nrhs"]},
            "gpu_launches": res["launches"] // max(1, args.steps), "clocks": res["clocks"]}
    if res["t_fp64"] is not None:
        v64 = whole_job_seconds_per_frequency(res["t_fp64"], args.fp64_steps, world)
        pf = res["prof_fp64"]
        line["fp64_path"] = {"value": v64, "unit": "s", "steps": args.fp64_steps, "warmup": args.fp64_warmup,
                             "speedup_of_learned_form": v64 / value,
                             "lu_gemm_tflops": pf["lu_gemm"]["flops"] / (pf["lu_gemm"]["ms"] / 1e3) / 1e12
                             if pf["lu_gemm"]["ms"] else None,
                             "kernel_classes": pf}
    if "secondary" in res:
        line["secondary_n19872"] = res["secondary"]
    if "jittered_n19872" in res:
        line["jittered_n19872"] = res["jittered_n19872"]
    if not args.lean and not args.no_batch:
        line["batching_form"] = run_batching()
    if not args.lean and not args.no_extras and world == 1:
        import torch
        import buffem
        stream = torch.cuda.ExternalStream(buffem.lib().bg_stream())
        zpk = zgemm_peak_tflops()
        gf = run_fields(stream)
        gf["roofline"] = {"bound": "fp64", "kernel": "k_fields", "achieved": gf["far"]["fp64_tflops"], "peak": zpk,
                          "unit": "TFLOP/s", "frac": gf["far"]["fp64_tflops"] / zpk,
                          "peak_source": "cuBLAS ZGEMM 8192^3 measured here (FP64 tensor rate; the FP64 "
                                         "CUDA-core peak is the same nominal 40 TFLOP/s on B200)",
                          "algorithmic": f"{FIELD_FLOPS_PER_POINT} flops per quadrature point, 4 points per "
                                         "(point, tetrahedron) pair in the far case; sincos and rsqrt not counted"}
        line["get_fields"] = gf
        nq = run_neq(stream)
        nq["roofline"] = {"bound": "tensor", "achieved": nq["fp64_tflops"], "peak": zpk, "unit": "TFLOP/s",
                          "frac": nq["fp64_tflops"] / zpk, "peak_source": "cuBLAS ZGEMM 8192^3 measured here"}
        line["neq_flux"] = nq
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model = CpuModel(args.n, fit_ns=(5760, 11400))
        t, v, parts = model.step()
        line["cpu_baseline"] = {"value": v, "unit": "s", "cores": model.cores, "kind": "port",
                                "extrapolated": True, "sample": model.sample_text(),
                                "sample_s": t, "breakdown": parts, "extrapolation": model.describe()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
