#!/usr/bin/env python3
"""Benchmark of the B200 sparse hot path (one JSON line on rank 0).

Headline: FP64 CSR SpMV (segmented-sum form) throughput in GB/s on the
irregular-row workload -- 4,000,000 rows, power-law row lengths (exponent
2.1, clipped to [1, 20000]), uniform sorted columns, N(0,1) values,
x ~ U[-1,1] seed 0 -- with algorithmic bytes per SpMV
  nnz*(8 + 4) + (n+1)*4 + n*8 (x) + n*8 (y).
A step is one SpMV over the whole matrix.  The matrix (~0.4 GB) is larger
than L2, so no L2 flush is done between steps; x (32 MB) may stay in L2.

Also reported (N == 1 only): the same SpMV on the 2D/3D Laplacians, the
IC(0)-PCG time to a 1e-10 true residual on the RCM-ordered 128^3 3D
Laplacian in FP64 vs mixed precision, the reference's OpenMP CPU path timed
on this host, and clocks sampled during the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (torchrun, one rank per GPU) every rank runs its own replica of
the workload (the solve path does not shard; weak scaling) and the time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV GB/s vs ~8 TB/s HBM; IC(0)-PCG time to 1e-10 resid, mixed vs FP64"
WORKLOAD = "powerlaw_spmv_fp64_segsum"


def spmv_bytes(n, nnz, vbytes=8, xbytes=8, beta=False):
    return nnz * (vbytes + 4) + (n + 1) * 4 + n * xbytes + n * xbytes * (2 if beta else 1)


def workload_config(n, nnz, byt):
    """The workload's description, identical in both arms (arm-specific
    notes such as the parallelism go outside it)."""
    return {"workload": WORKLOAD, "rows": n, "nnz": nnz, "bytes_per_step": byt,
            "row_lengths": "ceil(Pareto(2.1)) clipped to [1, 20000]",
            "l2": "inputs larger than L2 (matrix %.2f GB); no flush" % (byt / 1e9)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel_key):
    """Per-launch DRAM bytes recorded from an ncu capture, if committed."""
    f = ROOT / "profiles" / "traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel_key:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML in a thread."""

    def __init__(self, index=0, period=0.002):
        self.period, self.samples, self.reasons = period, [], set()
        self.ok = False
        try:
            import pynvml as N
            N.nvmlInit()
            self.N = N
            self.h = N.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None
        self._stop = threading.Event()

    def _run(self):
        N = self.N
        names = {
            "gpu_idle": N.nvmlClocksEventReasonGpuIdle,
            "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap,
            "hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
            "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
            "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
            "hw_power_brake": N.nvmlClocksEventReasonHwPowerBrakeSlowdown,
        }
        while not self._stop.is_set():
            try:
                self.samples.append(N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM))
                r = N.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, v in names.items():
                    if r & v:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "samples": len(self.samples)}


def powerlaw_workload():
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.powerlaw(4_000_000, seed=0)
    x = gen.uniform_vector(n, 0)
    return n, ai, aj, av, x


def cpu_reference_spmv(n, ai, aj, av, x, budget_s=10.0, max_reps=100):
    """The reference's own SegSumSPMV (compiled in place, oracle/_ref) with
    all host threads: median seconds per SpMV over a bounded sample."""
    import oracle
    rf = oracle.ref()
    kind = "reference"
    if rf is None:
        raise RuntimeError("oracle/_ref/libla_ref.so is missing (build() compiles it)")
    P = oracle.ptr
    T = rf.la_ref_max_threads()
    h = rf.la_ref_segsum_create(T, n, 0, P(ai), P(aj), P(av))
    y = np.zeros(n)
    rf.la_ref_segsum_apply(h, n, 0, P(ai), P(aj), P(av), P(x), P(y), 1.0, 0.0)  # warm
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_reps and (time.perf_counter() < t_end or len(times) < 3):
        t0 = time.perf_counter()
        rf.la_ref_segsum_apply(h, n, 0, P(ai), P(aj), P(av), P(x), P(y), 1.0, 0.0)
        times.append(time.perf_counter() - t0)
    rf.la_ref_segsum_destroy(h)
    return statistics.median(times), T, len(times), kind


def run_reference(args, rank, world):
    """--impl reference: the reference's OpenMP SegSumSPMV on the host."""
    if rank != 0:
        return
    n, ai, aj, av, x = powerlaw_workload()
    nnz = int(ai[-1])
    byt = spmv_bytes(n, nnz)
    import oracle
    rf = oracle.ref()
    P = oracle.ptr
    T = rf.la_ref_max_threads()
    h = rf.la_ref_segsum_create(T, n, 0, P(ai), P(aj), P(av))
    y = np.zeros(n)
    for _ in range(args.warmup):
        rf.la_ref_segsum_apply(h, n, 0, P(ai), P(aj), P(av), P(x), P(y), 1.0, 0.0)
    steps = args.steps if args.steps_given else 30
    t0 = time.perf_counter()
    for _ in range(steps):
        rf.la_ref_segsum_apply(h, n, 0, P(ai), P(aj), P(av), P(x), P(y), 1.0, 0.0)
    dt = time.perf_counter() - t0
    rf.la_ref_segsum_destroy(h)
    v = steps * byt / dt / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, nnz, byt), "parallelism": f"host OpenMP x{T}",
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": T, "kind": "reference",
                         "sample": f"{steps} full SegSumSPMV calls on the same matrix"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def max_over_ranks(pg, seconds, device):
    """The largest of every rank's time (each rank passes its own); the job's
    time for a replica run.  pg is torch.distributed or None (one rank)."""
    if pg is None:
        return seconds
    import torch
    tt = torch.tensor([seconds], dtype=torch.float64, device=device)
    pg.all_reduce(tt, op=pg.ReduceOp.MAX)
    return float(tt.item())


def replica_value(world, steps, bytes_per_step, seconds):
    """Whole-job GB/s of `world` replicas that each ran `steps` steps of
    `bytes_per_step` within `seconds` (the max over ranks)."""
    return world * steps * bytes_per_step / seconds / 1e9


def time_device_spmv(la, torch, plan, xd, yd, steps, warmup, alpha=1.0, beta=0.0):
    for _ in range(warmup):
        plan(xd, yd, alpha, beta)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        plan(xd, yd, alpha, beta)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def extras(la, torch, peak):
    """Single-GPU extras: Laplacian SpMV rooflines and the PCG comparisons."""
    from linearalgebra_b200 import gen
    out = {"spmv": [], "pcg": None}
    for label, t in (("C1_lap2d_512", gen.laplacian_2d(512)), ("C3_lap3d_128", gen.laplacian_3d(128))):
        n, ai, aj, av = t
        nnz = int(ai[-1])
        A = la.CSR(n, n, 0, ai, aj, av, keep_f32=True)
        x = gen.uniform_vector(n, 0)
        for kind, kid in (("segsum", la.api.LA_SPMV_SEGSUM), ("albus", la.api.LA_SPMV_ALBUS)):
            plan = la.SPMV(A, kid)
            for dt, tdt, vb in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
                xd = torch.as_tensor(x).to("cuda", tdt)
                yd = torch.empty(n, dtype=tdt, device="cuda")
                # flush L2 between reps for the L2-resident 2D case
                flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
                times = []
                for _ in range(60):
                    flush.fill_(1)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    plan(xd, yd)
                    e1.record()
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1) / 1e3)
                # the event clock ticks in ~2 us steps here: the mean over many
                # calls resolves a ~50 us kernel better than any one sample
                t = statistics.fmean(times[5:])
                del flush
                # back to back, as a solver calls it (the headline's method): the
                # launch latency of one call hides behind the previous call
                tb = time_device_spmv(la, torch, plan, xd, yd, 200, 5) / 200
                b = spmv_bytes(n, nnz, vb, vb)
                out["spmv"].append({"config": label, "form": kind, "dtype": dt, "n": n, "nnz": nnz,
                                    "layout": plan.layout(),
                                    "bytes": b, "us": t * 1e6, "GB/s": b / t / 1e9,
                                    "frac_of_measured_hbm": b / t / 1e9 / peak,
                                    "frac_of_8TBs": b / t / 8e12,
                                    "l2": "flushed before each call; one call per event pair",
                                    "us_back_to_back": tb * 1e6, "GB/s_back_to_back": b / tb / 1e9,
                                    "frac_of_measured_hbm_back_to_back": b / tb / 1e9 / peak,
                                    "back_to_back_l2": ("inputs larger than the 126 MB L2" if b > 126e6
                                                        else "fits in L2: not an HBM figure")})
    # IC(0)-PCG, FP64 vs mixed: the RCM-ordered 128^3 Laplacian (C3) and the
    # 192^3 anisotropic diffusion (C5, mixed precision at scale)
    out["pcg"], mats = pcg_case(la, torch, "C3_lap3d_128_rcm", gen.laplacian_3d(128))
    out["pcg_c5"], mats_c5 = pcg_case(la, torch, "C5_aniso7_192_rcm", gen.aniso7(192, seed=0))
    out["adjoint_c4"] = adjoint_case(la, torch, peak)
    try:
        out["ingest"] = ingest_case(la)
    except Exception as e:  # reported, never silently replaced
        out["ingest"] = {"error": str(e)}
    return out, {"pcg": mats, "pcg_c5": mats_c5}


def adjoint_case(la, torch, peak):
    """Differentiation configuration: SPD 27-point stencil on a 96^3 grid, FP64;
    L = 1/2 ||u - u*||^2 with u = A^-1 b.  Times the forward IC(0)-PCG, the
    adjoint solve with dL/dvalues (la_pcg_adjoint), and the SpMV adjoints --
    transpose SpMV (dL/dx) and the sampled outer product over the pattern
    (dL/dvalues) -- each to 1e-10.  Gradient parity (finite differences on 64
    entries, FP64 CPU gradient) is tests/test_gpu_adjoint.py's job."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.stencil27(96, seed=0)
    nnz = int(ai[-1])
    t0 = time.perf_counter()
    ua, uj, uv = la.SplitTriangle("U", n, 0, ai, aj, av)
    f = la.FactorPlan("ic0", n, 0, ua, uj).factor(uv)  # IC(0) on the GPU
    A = la.CSR(n, n, 0, ai, aj, av)
    s = la.PCG(A, ua, uj, f)
    plan = la.SPMV(A)
    setup_s = time.perf_counter() - t0
    t1 = time.perf_counter()
    f_host = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
    icc0_host_s = time.perf_counter() - t1
    icc0_identical = bool(np.array_equal(f, f_host))
    rng = np.random.default_rng(0)
    us = torch.as_tensor(rng.standard_normal(n)).cuda()
    b = torch.as_tensor(rng.standard_normal(n)).cuda()
    u = torch.empty_like(b)
    db = torch.empty_like(b)
    dv = torch.empty(nnz, dtype=torch.float64, device="cuda")
    dx = torch.empty_like(b)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    fwd_ms, rf = timed(lambda: s.solve(b, u, rtol=1e-10), 3)
    g = u - us
    adj_ms, ra = timed(lambda: s.adjoint(g, u, db, dv, rtol=1e-10), 3)
    tr_ms, _ = timed(lambda: plan.transpose(g, dx), 50)
    sd_ms, _ = timed(lambda: plan.sddmm(g, u, dv), 50)
    spmv_b = spmv_bytes(n, nnz)
    sddmm_b = nnz * 12 + n * 8 * 2 + (n + 1) * 4
    _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
    t_ai, t_aj, t_av = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
    ts = la.OptimizedTriangularSolve("L").analysis(n, 0, t_ai, t_aj, t_av, d)
    return {"config": "C4_stencil27_96_fp64", "n": n, "nnz": nnz, "rtol": 1e-10,
            "setup_s": setup_s, "icc0_host_s": icc0_host_s,
            "icc0_device_bit_identical": icc0_identical, "levels": ts.levels()[0],
            "trsv_schedule": list(ts.schedule()),
            "forward_pcg": {"iterations": rf.iterations, "ms": fwd_ms,
                            "rel_residual": rf.rel_residual},
            "adjoint_pcg_and_dvalues": {"iterations": ra.iterations, "ms": adj_ms,
                                        "rel_residual": ra.rel_residual},
            "spmv_transpose": {"us": tr_ms * 1e3, "GB/s": spmv_b / (tr_ms * 1e-3) / 1e9,
                               "frac_of_measured_hbm": spmv_b / (tr_ms * 1e-3) / 1e9 / peak},
            "sddmm_pattern": {"us": sd_ms * 1e3, "GB/s": sddmm_b / (sd_ms * 1e-3) / 1e9,
                              "frac_of_measured_hbm": sddmm_b / (sd_ms * 1e-3) / 1e9 / peak},
            "timing": "back to back after one warm-up call; inputs larger than L2 except x/g"}


def ingest_case(la):
    """Ingest (utils/utils.h:23-91): the 128^3 Laplacian's 14.6M entries,
    shuffled, written in ReadFromBinaryCOO's layout (base 1), read into a
    device CSR by ReadFromBinaryCSR's drop-in -- against the reference's own
    ReadFromBinaryCSR (compiled in place) on the host; the CSRs compared."""
    import tempfile
    import oracle
    from linearalgebra_b200 import gen
    n, ai, aj, av = gen.laplacian_3d(128)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(ai))
    order = np.random.default_rng(0).permutation(len(aj))
    rec = np.zeros(len(aj), np.dtype([("v", "<f8"), ("c", "<i4"), ("r", "<i4")]))
    rec["r"], rec["c"], rec["v"] = rows[order] + 1, aj[order] + 1, av[order]
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "lap3d_128.bin"
        with open(path, "wb") as f:
            f.write(np.int64(len(rec)).tobytes())
            f.write(rec.tobytes())
        la.ReadFromBinaryCSR(path, 1)  # warm
        t0 = time.perf_counter()
        A = la.ReadFromBinaryCSR(path, 1)
        t_dev = time.perf_counter() - t0
        out = {"config": "lap3d_128 shuffled, 14,581,760 entries, base 1",
               "file_bytes": path.stat().st_size, "device_csr_s": t_dev}
        rf = oracle.ref()
        if rf is not None:
            P = oracle.ptr
            m_, n_ = np.zeros(1, np.int32), np.zeros(1, np.int32)
            rai, raj, rav = np.zeros(n + 1, np.int32), np.zeros(len(aj), np.int32), np.zeros(len(aj))
            t0 = time.perf_counter()
            rf.la_ref_read_binary_csr(str(path).encode(), 1, P(rai), P(raj), P(rav), P(m_), P(n_))
            out["reference_host_s"] = time.perf_counter() - t0
            g = A.host
            out["identical_to_reference"] = bool(np.array_equal(g[0], rai) and
                                                 np.array_equal(g[1], raj) and
                                                 np.array_equal(g[2], rav))
    return out


def pcg_iteration_bytes(n, nnz, nnz_tri, vb):
    """Algorithmic bytes of one PCG iteration with values and vectors of vb
    bytes: SpMV + two triangular solves (strict triangle, row pointers,
    execution map, diagonal, b, x) + about ten n-vector reads/writes."""
    spmv = spmv_bytes(n, nnz, vb, vb)
    trsv = nnz_tri * (vb + 4) + (n + 1) * 4 + n * 4 + 3 * n * vb
    return spmv + 2 * trsv + 10 * n * 8


def pcg_case(la, torch, label, matrix):
    """FP64 vs mixed IC(0)-PCG to 1e-10 on an RCM-ordered SPD matrix."""
    from linearalgebra_b200 import gen
    n, ai, aj, av = matrix
    br = {}
    t0 = time.perf_counter()

    def lap(key, t=[t0]):
        now = time.perf_counter()
        br[key] = now - t[0]
        t[0] = now

    # the setup path: RCM ordered on the GPU, permutation and the upper
    # triangle on the host's threads, IC(0) on the GPU (its plan built there,
    # one numeric pass, host arrays in and out), CSR upload, both solvers'
    # analyses
    iperm, perm = la.SerialCM(n, 0, ai, aj, device=True)
    lap("rcm_device")
    b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
    lap("permute")
    ua, uj, uv = la.SplitTriangle("U", n, 0, b_ai, b_aj, b_av)
    lap("upper_triangle")
    fp = la.FactorPlan("ic0", n, 0, ua, uj)
    lap("icc0_device_plan")
    f = fp.factor(uv)
    lap("icc0_device_numeric")
    A = la.CSR(n, n, 0, b_ai, b_aj, b_av, keep_f32=True)
    lap("csr_upload")
    s64 = la.PCG(A, ua, uj, f)
    lap("pcg_create_fp64")
    s32 = la.PCG(A, ua, uj, f, mixed=True)
    lap("pcg_create_mixed")
    setup_keys = ("rcm_device", "permute", "upper_triangle", "icc0_device_plan",
                  "icc0_device_numeric", "csr_upload", "pcg_create_fp64", "pcg_create_mixed")
    setup_s = sum(br[k] for k in setup_keys)
    # the same steps once more in this process: the first pass pays first-use
    # costs (a fresh box's first large allocations) that vary from run to run
    t1 = time.perf_counter()
    ip2, pm2 = la.SerialCM(n, 0, ai, aj, device=True)
    c_ai, c_aj, c_av = la.Permute(n, 0, ai, aj, av, ip2, pm2)
    u2 = la.SplitTriangle("U", n, 0, c_ai, c_aj, c_av)
    f2 = la.FactorPlan("ic0", n, 0, u2[0], u2[1]).factor(u2[2])
    A2 = la.CSR(n, n, 0, c_ai, c_aj, c_av, keep_f32=True)
    s64b = la.PCG(A2, u2[0], u2[1], f2)
    s32b = la.PCG(A2, u2[0], u2[1], f2, mixed=True)
    br["setup_repeat_s"] = time.perf_counter() - t1
    del s64b, s32b, A2, f2, u2, c_ai, c_aj, c_av
    # beside it: the host's RCM and IC(0) (same ordering, same factor bit for
    # bit), the device numeric pass on device arrays, the L factor's level
    # sets on the host and on the GPU
    t1 = time.perf_counter()
    ip_h, pm_h = la.SerialCM(n, 0, ai, aj)
    br["rcm_host"] = time.perf_counter() - t1
    br["rcm_identical"] = bool(np.array_equal(ip_h, iperm) and np.array_equal(pm_h, perm))
    t1 = time.perf_counter()
    f_host = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
    br["icc0_host"] = time.perf_counter() - t1
    br["icc0_device_bit_identical"] = bool(np.array_equal(f, f_host))
    uv_d = torch.as_tensor(uv).cuda()
    f_d = torch.empty_like(uv_d)
    fp.factor(uv_d, out=f_d)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    fp.factor(uv_d, out=f_d)
    br["icc0_device_numeric_device_arrays"] = time.perf_counter() - t1
    del uv_d, f_d
    br["icc0_levels"] = fp.levels()
    del fp
    bvec = gen.uniform_vector(n, 0)
    bd = torch.as_tensor(bvec).to("cuda")
    x64 = torch.empty(n, dtype=torch.float64, device="cuda")
    x32 = torch.empty(n, dtype=torch.float64, device="cuda")
    s64.solve(bd, x64, maxit=20000)  # warm-up
    s32.solve(bd, x32, maxit=20000)
    r64 = s64.solve(bd, x64, maxit=20000)
    r32 = s32.solve(bd, x32, maxit=20000)
    err = float(torch.linalg.norm(x32 - x64) / torch.linalg.norm(x64))
    nnz = int(ai[-1])
    nnz_tri = (nnz - n) // 2
    _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
    t_ai, t_aj, t_av = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
    t1 = time.perf_counter()
    lh = la.TopologicalSort2("L", n, 0, t_ai, t_aj)
    br["levels_host"] = time.perf_counter() - t1
    t1 = time.perf_counter()
    ld = la.TopologicalSort2("L", n, 0, t_ai, t_aj, device=True)
    br["levels_device"] = time.perf_counter() - t1
    br["levels_identical"] = bool(lh[0] == ld[0] and np.array_equal(lh[1], ld[1])
                                  and np.array_equal(lh[2], ld[2]))
    sched = {}
    for name, dt in (("fp64", np.float64), ("fp32", np.float32)):
        ts = la.OptimizedTriangularSolve("L", dtype=dt).analysis(n, 0, t_ai, t_aj, t_av, d)
        sched[name] = list(ts.schedule())
        levels = ts.levels()[0]
    b64 = pcg_iteration_bytes(n, nnz, nnz_tri, 8)
    b32 = pcg_iteration_bytes(n, nnz, nnz_tri, 4)
    res = {"config": label, "n": n, "nnz": nnz, "rtol": 1e-10, "levels": levels,
           "setup_s": setup_s, "setup_steps": list(setup_keys), "setup_breakdown_s": br,
           "fp64": {"iterations": r64.iterations, "ms": r64.solve_ms,
                    "rel_residual": r64.rel_residual,
                    "GB/s_algorithmic": b64 * r64.iterations / (r64.solve_ms * 1e-3) / 1e9},
           "mixed": {"inner_iterations": r32.iterations, "outer": r32.outer_iterations,
                     "ms": r32.solve_ms, "rel_residual": r32.rel_residual,
                     "rel_err_vs_fp64": err,
                     "GB/s_algorithmic": b32 * r32.iterations / (r32.solve_ms * 1e-3) / 1e9},
           "speedup_mixed_vs_fp64": r64.solve_ms / r32.solve_ms,
           "trsv_schedules": sched}
    return res, (b_ai, b_aj, b_av, ua, uj, f, bvec, r64, x64.cpu().numpy(), x32.cpu().numpy())


def cpu_pcg(mats):
    import oracle
    rf = oracle.ref()
    b_ai, b_aj, b_av, ua, uj, f, bvec, r64, x64, x32 = mats
    n = len(b_ai) - 1
    P = oracle.ptr
    T = rf.la_ref_max_threads()
    h = rf.la_ref_pcg_create(T, n, 0, P(b_ai), P(b_aj), P(b_av), P(ua), P(uj), P(f))
    x = np.zeros(n)
    rel = np.zeros(1)
    t0 = time.perf_counter()
    it = rf.la_ref_pcg_solve(h, P(bvec), P(x), 1e-10, 5000, P(rel))
    dt = time.perf_counter() - t0
    rf.la_ref_pcg_destroy(h)
    xn = float(np.linalg.norm(x))
    return {"kind": "reference kernels (ParallelSPMV + OptimizedTriangularSolve<Barrier>) "
                    "composed into PCG; MKL PCG driver absent",
            "cores": T, "iterations": it, "s": dt, "rel_residual": float(rel[0]),
            "gpu_fp64_iterations": r64.iterations,
            "rel_diff_gpu_fp64_vs_cpu": float(np.linalg.norm(x64 - x)) / xn,
            "rel_diff_gpu_mixed_vs_cpu": float(np.linalg.norm(x32 - x)) / xn}


def run_case(case):
    """A small, fixed workload for profiling: builds one configuration and
    launches its kernel 3 times (the first is a warm-up)."""
    import torch
    import linearalgebra_b200 as la
    from linearalgebra_b200 import gen
    if case.startswith("spmv"):
        n, ai, aj, av = (gen.powerlaw(4_000_000, seed=0) if case == "spmv-powerlaw"
                         else gen.laplacian_3d(128))
        A = la.CSR(n, n, 0, ai, aj, av)
        P = la.SPMV(A, la.api.LA_SPMV_SEGSUM)
        x = torch.as_tensor(gen.uniform_vector(n, 0)).cuda()
        y = torch.empty_like(x)
        for _ in range(3):
            P(x, y)
    elif case == "adjoint-c4":
        # the SpMV adjoints on the 96^3 27-point stencil: transpose SpMV and
        # the sampled outer product over the pattern
        n, ai, aj, av = gen.stencil27(96, seed=0)
        P = la.SPMV(la.CSR(n, n, 0, ai, aj, av))
        g = torch.as_tensor(gen.uniform_vector(n, 1)).cuda()
        x = torch.as_tensor(gen.uniform_vector(n, 2)).cuda()
        out = torch.empty_like(x)
        dv = torch.empty(int(ai[-1]), dtype=torch.float64, device="cuda")
        for _ in range(3):
            P.transpose(g, out)
            P.sddmm(g, x, dv)
    elif case in ("factor-c3", "levels-c3"):
        # IC(0) of the RCM-ordered 128^3 Laplacian on the GPU, or the level
        # sets of its L factor on the GPU
        n, ai, aj, av = gen.laplacian_3d(128)
        iperm, perm = la.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = la.SplitTriangle("U", n, 0, b_ai, b_aj, b_av)
        if case == "factor-c3":
            fp = la.FactorPlan("ic0", n, 0, ua, uj)
            for _ in range(3):
                fp.factor(uv)
        else:
            f = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
            _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
            t_ai, t_aj, _ = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
            for _ in range(3):
                la.TopologicalSort2("L", n, 0, t_ai, t_aj, device=True)
    elif case == "factor-c4":
        # IC(0) of the 96^3 27-point stencil (natural order) on the GPU: the
        # warp-per-row numeric pass
        n, ai, aj, av = gen.stencil27(96, seed=0)
        ua, uj, uv = la.SplitTriangle("U", n, 0, ai, aj, av)
        fp = la.FactorPlan("ic0", n, 0, ua, uj)
        for _ in range(3):
            fp.factor(uv)
    elif case == "pcg-mixed-c3":
        # mixed-precision IC(0)-PCG on the RCM-ordered 128^3 Laplacian, 30
        # iterations (FP32 copy of A, the solvers' analysis with its device
        # partition stage, two reliable updates)
        n, ai, aj, av = gen.laplacian_3d(128)
        iperm, perm = la.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
        f = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
        A = la.CSR(n, n, 0, b_ai, b_aj, b_av, keep_f32=True)
        s = la.PCG(A, ua, uj, f, mixed=True)
        b = torch.as_tensor(gen.uniform_vector(n, 0)).cuda()
        x = torch.empty_like(b)
        s.solve(b, x, rtol=1e-10, maxit=30, allow_not_converged=True)
    elif case == "rcm-c3":
        # reverse Cuthill-McKee of the 128^3 Laplacian ordered on the GPU
        n, ai, aj, av = gen.laplacian_3d(128)
        for _ in range(2):
            la.SerialCM(n, 0, ai, aj, device=True)
    elif case == "icplan-c3":
        # the IC(0) plan of the RCM-ordered 128^3 Laplacian built on the GPU
        n, ai, aj, av = gen.laplacian_3d(128)
        iperm, perm = la.SerialCM(n, 0, ai, aj, device=True)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = la.SplitTriangle("U", n, 0, b_ai, b_aj, b_av)
        for _ in range(2):
            la.FactorPlan("ic0", n, 0, ua, uj)
    elif case == "ingest":
        # 16M shuffled COO entries (4M x 4M) sorted into a device CSR
        rng = np.random.default_rng(0)
        k, m = 16_000_000, 4_000_000
        rows, cols = rng.integers(0, m, k), rng.integers(0, m, k)
        vals = rng.standard_normal(k)
        for _ in range(2):
            la.csr_from_coo(m, m, 0, rows, cols, vals)
    elif case == "noalloc-c3":
        # the allocation-free SpMV on the 128^3 Laplacian
        n, ai, aj, av = gen.laplacian_3d(128)
        dev_ = lambda a, t: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", t)
        ai_d, aj_d, av_d = dev_(ai, torch.int32), dev_(aj, torch.int32), dev_(av, torch.float64)
        x = dev_(gen.uniform_vector(n, 0), torch.float64)
        y = torch.empty_like(x)
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for _ in range(3):
            la.lib().la_spmv_noalloc(la.api.LA_SPMV_SEGSUM, n, int(ai[-1]), 0,
                                     C.c_void_p(ai_d.data_ptr()), C.c_void_p(aj_d.data_ptr()),
                                     C.c_void_p(av_d.data_ptr()), 1.0, C.c_void_p(x.data_ptr()),
                                     0.0, C.c_void_p(y.data_ptr()), st)
    elif case == "trsv-c5":
        # FP64 lower solve of the RCM-ordered 192^3 anisotropic IC(0) factor:
        # the partitioned kernel with its x values in a shared-memory ring
        n, ai, aj, av = gen.aniso7(192, seed=0)
        iperm, perm = la.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
        f = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
        _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
        t_ai, t_aj, t_av = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
        ts = la.OptimizedTriangularSolve("L").analysis(n, 0, t_ai, t_aj, t_av, d)
        b = torch.as_tensor(gen.uniform_vector(n, 0)).cuda()
        x = torch.empty_like(b)
        for _ in range(3):
            ts(b, x)
        print("schedule", ts.schedule())
    elif case == "trsv-c5-f32":
        # FP32 lower solve of the RCM-ordered 192^3 anisotropic IC(0) factor:
        # the partitioned kernel with second-row register sets
        n, ai, aj, av = gen.aniso7(192, seed=0)
        iperm, perm = la.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
        f = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
        _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
        t_ai, t_aj, t_av = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
        ts = la.OptimizedTriangularSolve("L", dtype=np.float32).analysis(n, 0, t_ai, t_aj,
                                                                        t_av, d)
        b = torch.as_tensor(gen.uniform_vector(n, 0)).to("cuda", torch.float32)
        x = torch.empty_like(b)
        for _ in range(3):
            ts(b, x)
        print("schedule", ts.schedule())
    else:
        n, ai, aj, av = gen.laplacian_3d(128)
        iperm, perm = la.SerialCM(n, 0, ai, aj)
        b_ai, b_aj, b_av = la.Permute(n, 0, ai, aj, av, iperm, perm)
        ua, uj, uv = gen.upper_with_diag(n, b_ai, b_aj, b_av)
        f = la.ICCLevelNumeric0(n, 0, ua, uj, uv)
        b = torch.as_tensor(gen.uniform_vector(n, 0)).cuda()
        x = torch.empty_like(b)
        if case == "trsv-lap3d":
            _, d, (s_ai, s_aj, s_av) = la.SplitLDU(n, 0, ua, uj, f)
            t_ai, t_aj, t_av = la.Transpose(n, n, 0, s_ai, s_aj, s_av)
            ts = la.OptimizedTriangularSolve("L").analysis(n, 0, t_ai, t_aj, t_av, d)
            for _ in range(3):
                ts(b, x)
        else:
            A = la.CSR(n, n, 0, b_ai, b_aj, b_av)
            s = la.PCG(A, ua, uj, f)
            s.solve(b, x, rtol=1e-10, maxit=5, allow_not_converged=True)
    torch.cuda.synchronize()
    print(f"case {case} done")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu-pcg", action="store_true")
    ap.add_argument("--case", default=None,
                    choices=["spmv-powerlaw", "spmv-lap3d", "trsv-lap3d", "trsv-c5", "trsv-c5-f32",
                             "pcg-lap3d", "adjoint-c4", "factor-c3", "levels-c3", "ingest",
                             "noalloc-c3", "rcm-c3", "icplan-c3", "factor-c4", "pcg-mixed-c3"],
                    help="run one kernel workload a few times and exit (for ncu)")
    args = ap.parse_args()
    args.steps_given = args.steps is not None
    if args.steps is None:
        args.steps = 1000
    args.warmup = max(args.warmup, 3)
    if args.case:
        run_case(args.case)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    import linearalgebra_b200 as la

    peak, peak_kind = measured_peak()
    n, ai, aj, av, x = powerlaw_workload()
    nnz = int(ai[-1])
    byt = spmv_bytes(n, nnz)
    A = la.CSR(n, n, 0, ai, aj, av)
    plan = la.SPMV(A, la.api.LA_SPMV_SEGSUM)
    xd = torch.as_tensor(x).to("cuda")
    yd = torch.empty(n, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        plan(xd, yd)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with sampler:
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            plan(xd, yd)
        e1.record()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
    t = max_over_ranks(pg, e0.elapsed_time(e1) / 1e3, "cuda")
    value = replica_value(world, args.steps, byt, t)
    launch_s = t / args.steps

    # the matrix's own bound for the tile pass (la_spmv_ceiling): its columns
    # and values streamed, with and without the random x gather, back to back
    ceiling = {}
    for key, gather in (("stream_us", False), ("stream_and_gather_us", True)):
        sink = torch.zeros(1, dtype=torch.float64, device="cuda")
        for _ in range(3):
            plan.ceiling(xd, gather, sink)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        for _ in range(100):
            plan.ceiling(xd, gather, sink)
        c1.record()
        torch.cuda.synchronize()
        ceiling[key] = c0.elapsed_time(c1) / 100 * 1e3
    ceiling["matrix_bytes_streamed"] = (nnz // 1024) * 1024 * 12
    ceiling["headline_over_gather_ceiling"] = ceiling["stream_and_gather_us"] / (launch_s * 1e6)

    # end to end through the reference-facing host-pointer call: pinned host
    # x in, y out, every step
    hx = torch.as_tensor(x).pin_memory()
    hy = torch.empty(n, dtype=torch.float64).pin_memory()
    hxn, hyn = hx.numpy(), hy.numpy()
    e2e_steps = max(10, min(args.steps, 200))
    for _ in range(3):
        plan(hxn, hyn)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plan(hxn, hyn)
    te = max_over_ranks(pg, time.perf_counter() - t0, "cuda")
    e2e = replica_value(world, e2e_steps, byt, te)
    ok = np.allclose(hyn, yd.cpu().numpy(), rtol=1e-12, atol=1e-12)

    result = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator standing in for the reference's "
                "downloaded matrices)",
        "config": workload_config(n, nnz, byt),
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "roofline": {"bound": "hbm", "achieved": byt / launch_s / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": byt / launch_s / 1e9 / peak,
                     "peak_kind": peak_kind,
                     "kernel": "spmv_tile_kernel<SegSum, f64> + spmv_merge_kernel (one step)",
                     "traffic": profiled_traffic("spmv_tile_kernel_segsum_f64_powerlaw4M"),
                     "traffic_source": "DRAM bytes per launch from a stored ncu capture of "
                                       "this workload (profiles/traffic.txt), not this run"},
        "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": n * 8,
                "d2h_bytes_per_step": n * 8, "steps": e2e_steps,
                "api": "SPMV.__call__ host arrays -> la_spmv_host", "matches_device": bool(ok)},
        "gather_ceiling": ceiling,
        "gpu_launches": 2 * args.steps,
        "clocks": sampler.summary(),
    }
    if rank == 0 and world == 1:
        try:
            sec, T, reps, kind = cpu_reference_spmv(n, ai, aj, av, x)
            result["cpu_baseline"] = {"value": byt / sec / 1e9, "unit": "GB/s", "cores": T,
                                      "kind": kind,
                                      "sample": f"{reps} full SegSumSPMV calls (median)"}
        except Exception as ex:  # reported, never silently replaced
            result["cpu_baseline"] = {"value": None, "unit": "GB/s", "cores": None,
                                      "kind": "reference", "sample": f"failed: {ex}"}
        if not args.no_extras:
            ex, mats = extras(la, torch, peak)
            result["extras"] = ex
            if not args.no_cpu_pcg:
                for key, m in mats.items():
                    try:
                        ex[key]["cpu_reference"] = cpu_pcg(m)
                    except Exception as e:
                        ex[key]["cpu_reference"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
