#!/usr/bin/env python
"""Benchmark: GInteractions/s of BAEMM's boundary-operator apply on B200.

Workload (one "step" = one operator apply): the large-block apply -- torus
with major radius 1.0 and minor radius 0.4 on a 160 x 480 parametric grid,
2 triangles per quad (76800 vertices, 153600 triangles); 64 right-hand sides
= 4 wavenumbers {2, 4, 8, 16} x 16 complex64 vertex vectors, re/im iid N(0,1)
(seed 0); single- plus double-layer operator of the mixed indirect BIE
(coefficients per chunk: mass 0, SL -i kappa, DL 1, adjoint DL 0) with the
singular SL diagonal.  Interactions per apply I = N_t * N_s * wave_count.

  value  device time of the apply (AvOp, dense kernel, AvOp^T epilogue) with
         inputs resident in HBM, L2 flushed (256 MiB write) before every step;
         default arithmetic: the compensated tensor-core form (TF32 hi+lo
         operands, FP32 accumulation); --mode fp32 is the plain SIMT form
  compare  the plain FP32 apply timed the same way, and both forms' relative
         error against the FP64 apply of the same inputs (Frobenius norm)
  e2e    the same apply through the host-pointer C ABI call
         (baemm_apply_boundary_operators_c) from pinned host memory,
         host->device and device->host copies inside the timed region

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode tc|fp32|fp64] [--shard]
  python bench.py --impl reference ...   # the reference's own kernel on the host cores

Multi-GPU (torchrun, one process per GPU): independent replicas of the same
workload per rank (the operator apply does not exchange data); value = all
ranks' interactions / the max over ranks of the timed device time.  --shard:
one apply per step split by target rows over the ranks, shards summed by an
NCCL all-reduce (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GInteractions/s per operator apply"
UNIT = "GInteractions/s"
WORKLOAD = "torus R1.0 r0.4 160x480 grid (76800 V, 153600 T), 64 RHS = kappa {2,4,8,16} x 16, SL+DL apply"
KAPPA = np.array([2.0, 4.0, 8.0, 16.0])
WCS = 16
WC = 64


def coefficients(kappa):
    return np.array([[0.0, -1j * k, 1.0, 0.0] for k in kappa], np.complex128)


def build_workload(seed=0, small=False):
    """The torus workload; small=True is the 80 x 240 grid (38400 triangles)
    used only for ncu captures of the same kernels."""
    from baemm_b200 import meshes
    coords, tris = meshes.torus(1.0, 0.4, 80, 240) if small else meshes.torus(1.0, 0.4, 160, 480)
    rng = np.random.default_rng(seed)
    B = (rng.standard_normal((coords.shape[0], WC)) + 1j * rng.standard_normal((coords.shape[0], WC)))
    return coords, tris, B.astype(np.complex64)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0),
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", 1400.0), "source": "of measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "of fallback"}


KERNEL_SOURCE = {"tc": "tc.cu", "fp32": "dense.cu", "fp64": "dense.cu"}


def source_sha16(mode):
    """Content hash of the source file of this mode's dense kernel."""
    import hashlib
    p = os.path.join(ROOT, "baemm_b200", "csrc", KERNEL_SOURCE[mode])
    return hashlib.sha256(open(p, "rb").read()).hexdigest()[:16]


def load_traffic(mode):
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
    the dense kernel on this workload, from the committed ncu summary
    (profiles/traffic_torus.json), with the content hash of the kernel source
    it was captured on: `stale` when the source has changed since."""
    p = os.path.join(ROOT, "profiles", "traffic_torus.json")
    if not os.path.exists(p):
        return None, None
    try:
        rec = json.load(open(p)).get(mode)
    except Exception:
        return None, None
    if not isinstance(rec, dict) or "bytes" not in rec:
        return None, None
    now = source_sha16(mode)
    src = {"from": "profiles/traffic_torus.json (ncu, one launch)", "captured_on_source_sha16": rec.get("source_sha16"),
           "current_source_sha16": now, "stale": rec.get("source_sha16") != now}
    return int(rec["bytes"]), src


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
REASON_BITS = {
    0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
    0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
    0x100: "display_clock_setting",
}


class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the first sample before the timed region starts: nvidia-smi's start-up
            # (NVML initialisation on a fresh machine) must not fall inside it
            t0 = time.time()
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 15.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], 0
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 4:
                continue
            try:
                s, m = float(parts[0]), float(parts[1])
                r = int(parts[3], 16) if parts[3].startswith("0x") else int(parts[3])
            except ValueError:
                continue
            sm.append(s)
            mx.append(m)
            if s > 0.5 * m:    # under load
                reasons |= r
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = [n for b, n in REASON_BITS.items() if reasons & b and n != "gpu_idle"]
        loaded = [s for s, m in zip(sm, mx) if s > 0.5 * m] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": float(max(mx)), "reasons": names,
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's own kernel on the host (CPU baseline and --impl reference)
# ---------------------------------------------------------------------------
REF_FLAGS = ("g++ -O3 -march=x86-64-v3 -ffast-math -fopenmp (the counterpart of the reference's "
             "-cl-fast-relaxed-math, Helmholtz_OpenCL.hpp:77)")


class ReferenceRows:
    """The reference BoundaryOperatorKernel.cl (compiled as C++ with fast math,
    oracle/_ref/libbaemm_refcl_fast.so) on contiguous blocks of target rows
    against all sources, OpenMP over rows on every host core.  Cost is
    separable per target row, so a block's rows/s projects exactly to the full
    apply; AvOp / AvOp^T (O(N wc)) are left out of the sample."""

    def __init__(self, coords, tris, B_vertex, threads=0):
        from oracle import oracle as O
        self.O = O
        orc = O.Oracle(coords, tris, np.eye(3), precision=32, threads=threads)
        mid, nrm, area, _ = orc.geometry()
        self.mid, self.nrm = mid, nrm
        self.n = tris.shape[0]
        # B_tri = AvOp B (PL -> PC), as the reference does before the kernel
        self.Btri = ((area / 3.0)[:, None] * B_vertex[tris].sum(axis=1)).astype(np.complex64)
        self.cs = O.scaled_coefficients(coefficients(KAPPA))
        self.threads = threads
        self.cores = int(threads or O.reflib(fast=True).refcl_max_threads())
        self.next_row = 0

    def run(self, rows):
        """Time one block of `rows` target rows (the next block, wrapping around); seconds."""
        r0 = self.next_row if self.next_row + rows <= self.n else 0
        self.next_row = r0 + rows
        t0 = time.perf_counter()
        self.O.ref_boundary(self.mid, self.nrm, self.Btri, KAPPA, self.cs, WCS, r0, r0 + rows, self.threads,
                            fast=True)
        return time.perf_counter() - t0

    def rows_for(self, seconds):
        """Rows whose block takes about `seconds` (from a short calibration run)."""
        rows = max(self.cores, 8)
        dt = self.run(rows)
        while dt < 0.25 * seconds and rows < self.n:   # short runs are dominated by start-up
            rows = int(min(self.n, rows * 4))
            dt = self.run(rows)
        return int(min(self.n, max(self.cores, rows * seconds / max(dt, 1e-3))))

    def rate(self, rows, dt):
        return rows * self.n * WC / dt / 1e9

    def sample_text(self, rows):
        return (f"reference BoundaryOperatorKernel.cl (oracle/_ref, compiled as C++: {REF_FLAGS}) on {rows} "
                f"contiguous target rows x all {self.n} sources x 64 RHS per step, OpenMP over rows; projected "
                f"per interaction to the full apply (cost is separable per target row); AvOp/AvOp^T (O(N wc)) "
                f"not in the sample")


def reference_rows_rate(coords, tris, B_vertex, target_seconds=15.0, threads=0):
    """GInteractions/s of the reference kernel on one sample of about
    `target_seconds` (the GPU line's cpu_baseline)."""
    from oracle import oracle as O
    if not O.ref_available(fast=True):
        return None
    R = ReferenceRows(coords, tris, B_vertex, threads)
    rows = R.rows_for(target_seconds)
    dt = R.run(rows)
    return {"value": R.rate(rows, dt), "unit": UNIT, "cores": R.cores, "kind": "reference", "seconds": dt,
            "rows": rows, "projected": True, "sample": R.sample_text(rows)}


def run_reference_arm(args, rank, world):
    """--impl reference: rank 0 alone times the reference kernel on the host
    cores; `warmup` untimed and `steps` timed samples of the same size (about
    BAEMM_REF_SECONDS, default 4 s, each), every step a different block of
    target rows."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    if not O.ref_available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbaemm_refcl_fast.so not built "
                                                              "(oracle/build_ref.sh needs the reference tree)"}))
        return 0
    coords, tris, B = build_workload(small=args.small)
    R = ReferenceRows(coords, tris, B)
    rows = R.rows_for(float(os.environ.get("BAEMM_REF_SECONDS", "4")))
    for _ in range(args.warmup):
        R.run(rows)
    dts = [R.run(rows) for _ in range(args.steps)]
    v = R.rate(rows * args.steps, float(np.sum(dts)))
    n = tris.shape[0]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": n * n * WC / (v * 1e9) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "projected": True, "rows_sampled_per_step": rows,
        "sample_ms_per_step": float(np.mean(dts)) * 1e3,
        "config": {"workload": WORKLOAD if not args.small else "SMALL torus 80x240 (profiling only)",
                   "interactions_per_step": n * n * WC, "parallelism": "host cores", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": R.cores, "kind": "reference", "projected": True,
                         "sample": R.sample_text(rows)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# replicas across ranks
# ---------------------------------------------------------------------------
def max_over_ranks(x: float, dist, device) -> float:
    """The largest `x` over all ranks (the job takes as long as its slowest
    replica); `dist` None means a single process."""
    if not dist:
        return float(x)
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, interactions_per_step: int, steps: int, total_ms: float) -> float:
    """GInteractions/s of the whole job: every rank applies the same workload
    `steps` times (weak scaling) in at most `total_ms`."""
    return world * interactions_per_step * steps / (total_ms * 1e-3) / 1e9


def roofline_model(n_targets, n_sources, n_k, inter, mode, peaks, clk_mhz, n_sm, kernel_ms):
    """Roofline model of one dense launch (algorithmic work per launch):
    W = 8 I contraction FLOPs, G = N_t N_s n_k kernel evaluations (2 MUFU sincos
    + 20 FLOPs each) and N_t N_s rsqrt;
    plain FP32 form T* = (W + 20 G) / P_fp32, FP64 form T* = (W + 20 G) / P_fp64,
    tensor-core form T* = max(W / P_tf32, (2 G + N_t N_s) / P_mufu, 20 G / P_fp32).
    Each term comes with its work and rate, so achieved = work / t and
    frac = achieved / rate = term / t."""
    G = float(n_targets) * n_sources * n_k
    f_hz = (clk_mhz or 1965.0) * 1e6
    p_fp32 = n_sm * 128 * 2 * f_hz               # FFMA: 128 lanes/SM/clk
    p_fp64 = n_sm * 64 * 2 * f_hz                # DFMA: 64 lanes/SM/clk
    p_mufu = n_sm * 16 * f_hz                    # MUFU: 16 lanes/SM/clk
    p_tf32 = peaks["bf16_tflops"] * 1e12 / 2.0   # dense TF32 = half the measured dense BF16 rate
    W = 8.0 * inter
    work = {"tensor_tf32": (W, p_tf32, "TFLOP/s"),
            "mufu": (2 * G + float(n_targets) * n_sources, p_mufu, "Top/s (MUFU sin, cos, rsqrt)"),
            "fp32": (20.0 * G, p_fp32, "TFLOP/s")}
    if mode == "fp32":
        work = {"fp32": (W + 20.0 * G, p_fp32, "TFLOP/s")}
    elif mode == "fp64":
        work = {"fp64": (W + 20.0 * G, p_fp64, "TFLOP/s")}
    terms = {k + "_ms": w / r * 1e3 for k, (w, r, _) in work.items()}
    limiter = max(terms, key=terms.get)
    t_star = terms[limiter]
    w, r, unit = work[limiter[:-3]]
    return {"T_star_ms": t_star, "limiter": limiter, "terms_ms": terms, "frac": t_star / kernel_ms,
            "achieved": w / (kernel_ms * 1e-3) / 1e12, "peak": r / 1e12, "unit": unit,
            "clock_mhz": clk_mhz or 1965.0,
            "peaks": "P_fp32 = SMs x 256 FLOP/clk, P_fp64 = SMs x 128 FLOP/clk, P_mufu = SMs x 16/clk at the "
                     "sampled SM clock; P_tf32 = measured dense BF16 / 2"}


# ---------------------------------------------------------------------------
# the CUDA arm
# ---------------------------------------------------------------------------
def run_gpu_arm(args, rank, world, local_rank):
    import torch
    from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    coords, tris, B = build_workload(seed=0, small=args.small)
    nv, nt = coords.shape[0], tris.shape[0]
    inter = nt * nt * WC
    H = Helmholtz_CUDA(coords, tris, np.eye(3), device=local_rank)
    mode = {"fp32": APPLY_FP32, "fp64": APPLY_FP64, "tc": APPLY_TC}[args.mode]
    H.SetApplyMode(mode)
    kap, coeff = KAPPA, coefficients(KAPPA)
    stream = torch.cuda.Stream()
    H.SetStream(stream.cuda_stream)
    H.SetProfiling(True)
    Bd = torch.from_numpy(B).cuda()
    Cd = torch.zeros_like(Bd)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    H.LoadBoundaryOperators_PL(kap, coeff, WC, WCS)
    # the library's autotuner picks the kernel shape of the timed form and of the plain FP32 form it is
    # compared with (both tuned, so the comparison is against the best plain variant)
    tuned = {}
    if args.shape:
        # a fixed tensor-core shape (profiling runs: the tuner's timing would be distorted under a profiler)
        from baemm_b200 import _capi as _cp
        gw, ch, seg = (int(x) for x in args.shape.split(","))
        H.SetTuning(_cp.TUNE_TC_GEN_WARPS, gw)
        H.SetTuning(_cp.TUNE_TC_CHUNKS, ch)
        H.SetTuning(_cp.TUNE_TC_SEGMENT, seg)
        tuned["fixed_shape"] = {"tc_gen_warps": gw, "tc_chunks": ch, "tc_segment": seg}
    elif not args.no_tune and args.mode in ("tc", "fp32"):
        from baemm_b200 import APPLY_FP32 as _F32, APPLY_TC as _TC
        for name, m in (("fp32", _F32), ("tc", _TC)):
            if name == "tc" and args.mode != "tc":
                continue
            r = H.Autotune(m, repeats=2)
            tuned[name] = {k: r[k] for k in ("dense_variant", "tc_gen_warps", "tc_chunks", "tc_segment", "candidates",
                                             "best_ms", "cached")}
        H.SetApplyMode(mode)
    S = None
    if args.shard:
        # one apply split by target rows over the ranks, shards summed by an all-reduce
        from baemm_b200.sharded import ShardedBoundaryApply
        S = ShardedBoundaryApply(H)
    inter_kernel = (S.r1 - S.r0) * nt * WC if S is not None else inter   # this rank's dense-kernel interactions

    def step():
        if S is not None:
            S(1.0, Bd, 0.0, Cd)
        else:
            H.ApplyBoundaryOperators_PL(1.0, Bd, 0.0, Cd)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1.0)
            step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = H.KernelLaunchCount()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dense_ms, phase_ms = [], []
    with ClockSampler(torch.cuda.current_device()) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))
                ev[k][0].record(stream)
                step()
                ev[k][1].record(stream)
                phase_ms.append(H.LastApplyTimes())
                dense_ms.append(phase_ms[-1][1])
        torch.cuda.synchronize()
    launches = H.KernelLaunchCount() - launches0 - 0  # library kernels only (flush is torch's)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(float(np.sum(step_ms)), dist, "cuda")
    jobs = 1 if S is not None else world   # sharded: one apply per step for the whole job; replicas: one per rank
    value = whole_job_rate(jobs, inter, args.steps, total_ms)

    # ---- e2e through the host-pointer C ABI (pinned host buffers) -----------------
    Bp = torch.from_numpy(B).pin_memory()
    Cp = torch.zeros(B.shape, dtype=torch.complex64).pin_memory()
    Bh, Ch = Bp.numpy(), Cp.numpy()
    H.SetStream(None)

    def e2e_step():
        if S is not None:   # host blocks through the sharded apply (copies on torch's stream)
            Bd.copy_(Bp, non_blocking=True)
            S(1.0, Bd, 0.0, Cd)
            Cp.copy_(Cd, non_blocking=True)
            torch.cuda.synchronize()
        else:
            H.ApplyBoundaryOperators_PL(1.0, Bh, 0.0, Ch)   # H2D, apply, D2H, synchronised

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = max_over_ranks(float(np.sum(e2e_ms)), dist, "cuda")
    e2e_value = whole_job_rate(jobs, inter, args.steps, e2e_total)
    # ---- plain FP32 form and accuracy against the FP64 apply (rank 0, untimed for value) ----
    compare = None
    if rank == 0 and not args.no_compare and S is None:
        H.SetStream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            C_mode = Cd.clone()
            H.SetApplyMode(APPLY_FP64)
            Bz = Bd.to(torch.complex128)
            Cz = torch.zeros_like(Bz)
            H.ApplyBoundaryOperators_PL(1.0, Bz, 0.0, Cz)
            fp64_ms = H.LastApplyTimes()[1]
            H.SetApplyMode(APPLY_FP32)
            Cp = torch.zeros_like(Bd)
            plain_ms = []
            for k in range(2):
                flush.fill_(float(k))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                H.ApplyBoundaryOperators_PL(1.0, Bd, 0.0, Cp)
                e1.record(stream)
                plain_ms.append((e0, e1))
        torch.cuda.synchronize()
        H.SetApplyMode(mode)
        ref = Cz.cpu().numpy()
        nref = float(np.linalg.norm(ref))
        err = {args.mode: float(np.linalg.norm(C_mode.cpu().numpy().astype(np.complex128) - ref) / nref),
               "fp32": float(np.linalg.norm(Cp.cpu().numpy().astype(np.complex128) - ref) / nref)}
        p_ms = float(np.mean([a.elapsed_time(b) for a, b in plain_ms]))
        compare = {"plain_fp32_ms_per_step": p_ms, "speedup_vs_plain_fp32": p_ms / (total_ms / args.steps),
                   "rel_err_vs_fp64": err, "fp64_dense_ms": fp64_ms,
                   "note": "relative Frobenius error of the apply output against the FP64 apply of the same inputs"}
    H.UnloadBoundaryOperators_PL()

    if rank != 0:
        H.close()
        return 0
    peaks = load_peaks()
    dense_avg = float(np.mean(dense_ms))
    flops = 8.0 * inter_kernel
    achieved = flops / (dense_avg * 1e-3) / 1e12
    traffic, traffic_src = (load_traffic(args.mode) if not args.kappa else
                            (None, "captured on the default wavenumbers only"))
    kernel_name = {"tc": "boundary_tc_kernel", "fp32": "boundary_dense_kernel", "fp64": "boundary_dense_kernel<double>"}[args.mode]
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = reference_rows_rate(coords, tris, B, target_seconds=float(os.environ.get("BAEMM_REF_SECONDS", "12")))
    cs = clk.summary()
    clk_mhz = cs.get("sm_mhz") or None
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    n_tgt = (S.r1 - S.r0) if S is not None else nt
    model = roofline_model(n_tgt, nt, len(KAPPA), inter_kernel, args.mode, peaks, clk_mhz, n_sm, dense_avg)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if S is not None else "weak", "vs_baseline": None, "dtype": args.mode,
        "data": "synthetic",
        "config": {"workload": WORKLOAD if not args.small else "SMALL torus 80x240 (profiling only)", "interactions_per_step": inter, "wave_count": WC,
                   "wave_chunk_size": WCS, "kappa": KAPPA.tolist(), "apply_mode": args.mode,
                   "parallelism": (f"target rows x{world} + all-reduce" if S is not None else
                                   f"replicas x{world}" if world > 1 else "single GPU"),
                   "l2": "flushed (256 MiB write) before every timed step",
                   "autotuned": tuned or None},
        "roofline": {"bound": model["limiter"][:-3], "kernel": kernel_name, "achieved": model["achieved"],
                     "peak": model["peak"], "unit": model["unit"], "frac": model["frac"],
                     "peak_source": ("nominal SM pipe rates at the sampled clock" if model["limiter"] != "tensor_tf32_ms"
                                     else peaks["source"] + " (dense bf16 burst / 2)"),
                     "algorithmic": "the limiting term of the dense kernel's model (below) per launch; "
                                    "N_t = this rank's target rows",
                     "dense_kernel_ms": dense_avg, "traffic": traffic, "traffic_source": traffic_src,
                     "algorithmic_bytes": int(nt * WC * 8 * 2 + ((nt + 15) // 16) * 384),
                     "model": model},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(B.nbytes),
                "d2h_bytes_per_step": int(B.nbytes), "ms_per_step": e2e_total / args.steps},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    # HBM-bound sparse steps of the apply (device times of the same steps):
    #   AvOp:     reads AvOp (3 int32 + a3 per triangle) and the vertex block, writes B_tri;
    #   epilogue: reads the AvOp^T CSR, a3, diag, C_tri and B_tri (SL diagonal), writes the vertex block.
    cb = 8 if args.mode != "fp64" else 16            # bytes per complex of the internal blocks
    nnz = 3 * nt
    avop_bytes = nt * 16 + nv * WC * B.itemsize + nt * WC * cb
    epi_bytes = (nv + 1) * 4 + nnz * 4 + nt * 8 + 2 * nt * WC * cb + nv * WC * B.itemsize
    if S is None:
        ph = np.mean(np.array(phase_ms), axis=0)
        line["sparse_steps"] = {
            name: {"ms": float(ms), "algorithmic_bytes": int(nb), "GB_s": nb / (ms * 1e-3) / 1e9,
                   "frac_of_hbm_peak": nb / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                   "peak_source": peaks["source"] + " (copy bandwidth)"}
            for name, ms, nb in (("avop", ph[0], avop_bytes), ("avopT_epilogue", ph[2], epi_bytes))}
    if args.mode == "tc":
        # the tensor pipe beside the limiter: algorithmic contraction FLOPs (8 I, counted once) and the
        # FLOPs the compensated products issue (Ahi [Bhi | Blo] + Alo Bhi: 3 x 8 I) against dense TF32
        p_tf32 = peaks["bf16_tflops"] / 2.0
        line["roofline"]["tensor_pipe"] = {
            "algorithmic_TFLOP_s": achieved, "issued_TFLOP_s": 3.0 * achieved, "peak_tf32_TFLOP_s": p_tf32,
            "frac_issued": 3.0 * achieved / p_tf32, "peak_source": peaks["source"] + " (dense bf16 burst / 2)"}
    if compare is not None:
        # the comparison forms against their own bounds (plain FP32: the FMA pipe over its step time,
        # FP64: the DFMA pipe over its dense-kernel time), so the speed-up is read against kernels
        # whose distance from their rooflines is stated
        for key, form, ms in (("plain_fp32_model", "fp32", compare["plain_fp32_ms_per_step"]),
                              ("fp64_model", "fp64", compare["fp64_dense_ms"])):
            if ms and ms > 0:
                mm = roofline_model(n_tgt, nt, len(KAPPA), inter_kernel, form, peaks, clk_mhz, n_sm, ms)
                compare[key] = {"T_star_ms": mm["T_star_ms"], "frac": mm["frac"], "limiter": mm["limiter"]}
        line["compare"] = compare
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": cpu["kind"],
                                "projected": True, "sample": cpu["sample"]}
    H.close()
    if world == 1 and S is None and args.extras and not args.small:
        # the other configurations, compact (not part of value): the scattering solve and a serving sample
        res, apply, ntri = solve_runs(6, ("fp64", "fp32", "tc", "tc_ir"), with_apply_ms=False)
        kry = res.pop("krylov_steps")
        line["solve_icosphere6"] = {
            "workload": SOLVE_WORKLOAD, "triangles": ntri,
            "runs": {k: {q: v[q] for q in ("seconds", "gmres_iterations", "refinement_steps",
                                           "far_field_rel_err_vs_fp64", "phi_rel_err_vs_fp64")}
                     for k, v in res.items()},
            "krylov_steps": kry}
        line["serving_sample"] = dict(serve_runs(args.serve_sample, slots=6, seed=0), requests=args.serve_sample,
                                      workload="perturbed-icosphere scattering solves, levels 4-6, kappa U[1,10], "
                                               "1-64 plane waves, GMRES 1e-6, far field at 128 directions; "
                                               "Poisson arrivals at 80 % of capacity for the latencies")
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the near-field workload (--workload nearfield): not the headline line
# ---------------------------------------------------------------------------
NF_WORKLOAD = ("torus R1.0 r0.4 160x480 grid (76800 V, 153600 T), 64 RHS = kappa {2,4,8,16} x 16, SL+DL potential "
               "(ApplyNearFieldOperators_PL) at 153600 seeded points in [-1.6,1.6]^2 x [-0.6,0.6], at least 0.05 "
               "from the surface")


def nearfield_points(small=False):
    """Seeded evaluation points around the torus (small: 38400, with the small torus)."""
    from baemm_b200 import meshes
    return meshes.points_off_torus(38400 if small else 153600, seed=0)


def reference_nearfield_rate(coords, tris, B_vertex, pts, target_seconds=10.0, threads=0):
    """GInteractions/s of the reference NearFieldOperatorKernel.cl (compiled as
    C++, oracle/_ref) on a contiguous block of points against all sources
    (cost is separable per point)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    orc = O.Oracle(coords, tris, np.eye(3), precision=32, threads=threads)
    mid, nrm, area, _ = orc.geometry()
    n = tris.shape[0]
    Btri = ((area / 3.0)[:, None] * B_vertex[tris].sum(axis=1)).astype(np.complex64)
    cs = O.scaled_coefficients(coefficients(KAPPA))
    nthreads = threads or O.reflib().refcl_max_threads()
    rows = max(nthreads, 8)
    t0 = time.perf_counter()
    O.ref_nearfield(mid, nrm, Btri, pts[:rows], KAPPA, cs, WCS, threads=threads)
    dt = time.perf_counter() - t0
    rows2 = int(min(pts.shape[0] - rows, max(rows, rows * target_seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    O.ref_nearfield(mid, nrm, Btri, pts[rows:rows + rows2], KAPPA, cs, WCS, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": rows2 * n * WC / dt / 1e9, "unit": UNIT, "cores": int(nthreads), "kind": "reference",
            "sample": f"reference NearFieldOperatorKernel.cl (oracle/_ref, compiled as C++) on {rows2} points x "
                      f"all {n} sources x 64 RHS, OpenMP over points; scaled per interaction"}


def run_nearfield_workload(args):
    """ApplyNearFieldOperators_PL (ApplyNearFieldOperators.hpp:56-122) on the
    torus: device-resident blocks, CUDA-event times over `steps` evaluations
    after `warmup` (L2 flushed before each), for the tensor-core, plain FP32
    and FP64 arithmetic; errors against the FP64 evaluation; the end-to-end
    rate through the host-pointer C ABI; the reference kernel on the host."""
    import torch
    from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA
    coords, tris, B = build_workload(seed=0, small=args.small)
    pts = nearfield_points(args.small)
    nt, m = tris.shape[0], pts.shape[0]
    inter = m * nt * WC
    H = Helmholtz_CUDA(coords, tris, np.eye(3))
    H.LoadParameters(KAPPA, coefficients(KAPPA), WC, WCS)
    stream = torch.cuda.Stream()
    H.SetStream(stream.cuda_stream)
    H.SetProfiling(True)
    Bd = torch.from_numpy(B).cuda()
    Pd = torch.from_numpy(pts).cuda()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(mode, steps, warmup):
        H.SetApplyMode(mode)
        Bm = Bd.to(torch.complex128) if mode == APPLY_FP64 else Bd
        Cd = torch.zeros((m, WC), dtype=Bm.dtype, device="cuda")
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                flush.fill_(1.0)
                H.ApplyNearFieldOperators_PL(1.0, Bm, 0.0, Cd, Pd)
        torch.cuda.synchronize()
        evs, kern = [], []
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(float(k))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                H.ApplyNearFieldOperators_PL(1.0, Bm, 0.0, Cd, Pd)
                e1.record(stream)
                evs.append((e0, e1))
                kern.append(H.LastApplyTimes()[1])
        torch.cuda.synchronize()
        return (Cd.cpu().numpy().astype(np.complex128), float(np.mean([a.elapsed_time(b) for a, b in evs])),
                float(np.mean(kern)))

    launches0 = H.KernelLaunchCount()
    with ClockSampler(torch.cuda.current_device()) as clk:
        C_tc, ms_tc, k_tc = timed(APPLY_TC, args.steps, args.warmup)
    launches = H.KernelLaunchCount() - launches0
    C_32, ms_32, k_32 = timed(APPLY_FP32, 2, 1)
    C_64, ms_64, k_64 = timed(APPLY_FP64, 1, 1)
    nref = float(np.linalg.norm(C_64))
    err = lambda C: float(np.linalg.norm(C - C_64) / nref)
    # end to end through the host-pointer C ABI (pinned host blocks, copies inside)
    H.SetStream(None)
    H.SetApplyMode(APPLY_TC)
    Bh = torch.from_numpy(B).pin_memory().numpy()
    Ch = torch.zeros((m, WC), dtype=torch.complex64).pin_memory().numpy()
    P32 = pts.astype(np.float32)
    H.ApplyNearFieldOperators_PL(1.0, Bh, 0.0, Ch, P32)
    e2e = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        H.ApplyNearFieldOperators_PL(1.0, Bh, 0.0, Ch, P32)
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = float(np.mean(e2e))
    peaks = load_peaks()
    cs = clk.summary()
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    model = roofline_model(m, nt, len(KAPPA), inter, "tc", peaks, cs.get("sm_mhz") or None, n_sm, k_tc)
    rate = lambda ms: inter / (ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        cpu = reference_nearfield_rate(coords, tris, B, pts, float(os.environ.get("BAEMM_REF_SECONDS", "10")))
    line = {"metric": "GInteractions/s per near-field evaluation", "value": rate(ms_tc), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_tc, "higher_is_better": True,
            "dtype": "tc", "data": "synthetic",
            "config": {"workload": NF_WORKLOAD if not args.small else "SMALL torus 80x240, 38400 points (profiling)",
                       "points": m, "interactions_per_step": inter, "wave_count": WC,
                       "l2": "flushed (256 MiB write) before every timed step"},
            "runs": {"tc": {"ms": ms_tc, "kernel_ms": k_tc, "GInteractions_per_s": rate(ms_tc),
                            "rel_err_vs_fp64": err(C_tc)},
                     "fp32": {"ms": ms_32, "kernel_ms": k_32, "GInteractions_per_s": rate(ms_32),
                              "rel_err_vs_fp64": err(C_32)},
                     "fp64": {"ms": ms_64, "kernel_ms": k_64, "GInteractions_per_s": rate(ms_64)}},
            "speedup_tc_vs_fp32": ms_32 / ms_tc,
            "roofline": {"kernel": "boundary_tc_kernel (targets = points)", "model": model},
            "e2e": {"value": rate(e2e_ms), "unit": UNIT, "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(B.nbytes + P32.nbytes), "d2h_bytes_per_step": int(m * WC * 8)},
            "gpu_launches": int(launches), "clocks": cs}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    H.close()
    return 0


# ---------------------------------------------------------------------------
# the scattering-solve workload (--workload solve): not the headline line
# ---------------------------------------------------------------------------
SOLVE_WORKLOAD = ("unit icosphere level 6 (40962 V, 81920 T), kappa {4, 8} x 16 plane waves (Fibonacci "
                  "directions), far field at 256 Fibonacci directions, mixed indirect BIE, GMRES(30) + CG M^-1")


def solve_runs(level=6, modes=("fp64", "fp32", "tc", "tc_ir"), with_apply_ms=True):
    """FarField (FarField.hpp:28-144) on the scattering-solve configuration
    (icosphere `level`, kappa {4, 8} x 16 Fibonacci plane waves, far field at
    256 Fibonacci directions) in the given arithmetic forms: plain FP32 apply
    to residual 1e-6, compensated tensor-core apply to 1e-6, the tensor-core
    apply inside FP64 iterative refinement to 1e-10, and the FP64 path to
    1e-10; wall time of one warm solve each, GMRES iterations, and the errors
    of the far field and of the boundary density phi against the FP64 solve
    (the FP64 device path is held to 1e-11 of the FP64 oracle by the tests at
    smaller sizes).  Returns (runs, apply_ms, triangles)."""
    import torch
    from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA, WaveType, meshes
    coords, tris = meshes.icosphere(level)
    meas = meshes.fibonacci_sphere(256)
    inc = meshes.fibonacci_sphere(16)
    kap = np.array([4.0, 8.0])
    H = Helmholtz_CUDA(coords, tris, meas)

    # the weak incident wave of FarField, scaled by 4 pi (the boundary-density errors are relative)
    wave = np.zeros((coords.shape[0], 32), complex)
    H.CreateIncidentWave_PL(1.0, inc, 0.0, wave, kap, [[0, -4 * np.pi, 0, 0]] * 2, 32, 16)

    def solve(mode, gmres_tol, ir_steps=0, inner=1e-5):
        H.SetApplyMode(mode)
        H.SetRefinement(ir_steps, inner)
        F = np.zeros((meas.shape[0], 32), complex)
        H.FarField(kap, inc, F, WaveType.Plane, 1e-10, gmres_tol)   # warm (buffers, set-up)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        H.FarField(kap, inc, F, WaveType.Plane, 1e-10, gmres_tol)
        dt = time.perf_counter() - t0
        st = H.LastSolveStats()
        # the boundary density phi of the same solve (not timed)
        phi = np.zeros_like(wave)
        H.BoundaryPotential(kap, np.zeros((2, 4), complex), wave, phi, 16, 1e-10, gmres_tol)
        H.SetRefinement(0)
        H.SetApplyMode(APPLY_FP32)
        return F, dt, st, phi

    def apply_ms(mode):
        """One boundary apply of the solve's operator (BIE coefficients, 32
        right-hand sides), CUDA events, minimum of 3 after a warm-up."""
        dt = torch.complex128 if mode == APPLY_FP64 else torch.complex64
        coeff = np.array([[0.5, -1j * k, 1, 0] for k in kap], np.complex128)
        rng = np.random.default_rng(0)
        B = torch.from_numpy(rng.standard_normal((coords.shape[0], 32)) +
                             1j * rng.standard_normal((coords.shape[0], 32))).to(dt).cuda()
        C = torch.zeros_like(B)
        H.LoadBoundaryOperators_PL(kap, coeff, 32, 16)
        H.SetApplyMode(mode)
        try:
            ts = []
            for _ in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C)
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
        finally:
            H.SetApplyMode(APPLY_FP32)
            H.UnloadBoundaryOperators_PL()
        return min(ts[1:])

    known = {"fp64": ("fp64_tol1e-10", APPLY_FP64, 1e-10, 0), "fp32": ("fp32_tol1e-6", APPLY_FP32, 1e-6, 0),
             "tc": ("tc_tol1e-6", APPLY_TC, 1e-6, 0), "tc_ir": ("tc_fp64ir_tol1e-10", APPLY_TC, 1e-10, 8)}
    bad = [m for m in modes if m not in known]
    if bad:
        raise SystemExit(f"--solve-modes: unknown {bad}; choose from {sorted(known)}")
    runs = {}
    for m in modes:
        name, mode, tol, ir = known[m]
        runs[name] = solve(mode, tol, ir_steps=ir, inner=1e-5)
    F64, phi64 = (runs["fp64_tol1e-10"][0], runs["fp64_tol1e-10"][3]) if "fp64" in modes else (None, None)

    def rel(x, ref):
        return float(np.linalg.norm(x - ref) / np.linalg.norm(ref)) if ref is not None else None

    res = {}
    for name, (F, dt, st, phi) in runs.items():
        res[name] = {"seconds": dt, "solves_per_s": 1.0 / dt, "gmres_iterations": st["gmres_iterations"],
                     "refinement_steps": st["refinement_steps"],
                     "gmres_relative_residual": st["gmres_relative_residual"],
                     "far_field_rel_err_vs_fp64": rel(F, F64), "phi_rel_err_vs_fp64": rel(phi, phi64)}
    apply = ({name.split("_")[0]: apply_ms(mode) for m in ("tc", "fp32", "fp64") if m in modes
              for name, mode, _, _ in [known[m]]} if with_apply_ms else {})
    # the Krylov-vector kernels of these solves (32 complex columns, basis of 12 = the iterations the
    # tensor-core solve takes), against the measured copy bandwidth
    peaks = load_peaks()
    kry = H.ProfileKrylov(32, 20, 12)
    for v in kry.values():
        v["frac_of_hbm_peak"] = v["GB_s"] / peaks["hbm_gbs"] if v["GB_s"] else None
    kry["note"] = ("algorithmic bytes per launch / CUDA-event time per launch; the 21 MB vectors stay in the 126 MB L2 "
                   "between kernels, so rates above the HBM peak are possible; peak " + peaks["source"] +
                   " copy bandwidth")
    res["krylov_steps"] = kry
    H.close()
    return res, apply, int(tris.shape[0])


def run_solve_workload(args):
    modes = [m.strip() for m in args.solve_modes.split(",") if m.strip()]
    res, apply, nt = solve_runs(args.solve_level, modes)
    kry = res.pop("krylov_steps")
    head = "tc_fp64ir_tol1e-10" if "tc_fp64ir_tol1e-10" in res else next(iter(res))
    line = {"metric": "scattering solves/s (FarField)", "value": res[head]["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": SOLVE_WORKLOAD if args.solve_level == 6 else f"icosphere level {args.solve_level}",
                       "triangles": nt, "wave_count": 32, "meas_count": 256, "value_run": head},
            "runs": res, "apply_ms": apply, "krylov_steps": kry}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the serving workload (--workload serve): not the headline line
# ---------------------------------------------------------------------------
def serve_runs(n_requests, slots=6, seed=0, seq_sample=0, seq_tc=True, latency=True, levels=(4, 5, 6),
               pack_wait_us=None):
    """Stream of scattering-solve requests (icosphere levels `levels` (4-6) radially
    perturbed by a random degree-8 spherical-harmonic field of amplitude 0.1,
    kappa ~ U[1, 10], 1-64 plane waves, GMRES to 1e-6, far field at 128
    directions).  Runs over the same requests:
      sequential_plain_fp32  the plain FP32 apply, one request at a time (the baseline);
      sequential_tc          the tensor-core apply with graph replay, one request at a
                             time (the same arithmetic as the server: the server's own
                             gain over it is the batching);
      capacity               the serving loop as configured by default (slots of resident
                             contexts on their own streams, memory-budget admission,
                             tensor-core apply, CUDA-graph replay) with every request queued
                             at once: solves/s is its throughput (capacity_with_packing: the
                             same with the slots' applies packed into shared launches);
      latency                the serving loop with Poisson arrivals at 80 % of that
                             capacity: p50 / p99 of finish - arrival.
    The far fields of the served runs are compared with the sequential ones."""
    from baemm_b200 import APPLY_FP32, APPLY_TC, meshes
    from baemm_b200.serving import SolveServer, make_stream, summarize
    from baemm_b200.serving import SolveRequest
    meas = meshes.fibonacci_sphere(128)
    reqs = make_stream(n_requests, rate=0.0, levels=tuple(levels), seed=seed)
    # warm-up: one request per problem shape (mesh level x padded right-hand sides), so the
    # autotuner's choices and the device buffers exist before any timing
    warm = []
    for level in levels:
        coords_w, tris_w = meshes.icosphere(level)
        for nrhs in (16, 32, 64):
            d = meshes.fibonacci_sphere(nrhs)
            warm.append(SolveRequest(len(warm) + 1000000, coords_w, tris_w, 3.0, d, mesh_key=("warm", level)))

    def at_once():
        for r in reqs:
            r.arrival = 0.0
        return reqs

    n_seq = len(reqs) if seq_sample <= 0 else min(seq_sample, len(reqs))

    def sequential(mode, graphs):
        with SolveServer(meas, slots=1, apply_mode=mode, graphs=graphs) as seq:
            seq.run(warm, realtime=False)
            t0 = time.perf_counter()
            out = seq.run(at_once()[:n_seq], realtime=False)
            return out, time.perf_counter() - t0

    base, t_seq = sequential(APPLY_FP32, False)
    res = {"sequential_plain_fp32": {"solves_per_s": n_seq / t_seq, "seconds": t_seq, "requests": n_seq,
                                     "note": "the first requests of the same stream" if n_seq < len(reqs) else "all"}}
    if seq_tc:
        _, t_tc = sequential(APPLY_TC, True)
        res["sequential_tc"] = {"solves_per_s": n_seq / t_tc, "seconds": t_tc, "requests": n_seq}
    # the server with packing (the slots' GMRES applies share launches), for the packing's own effect
    pkw = {} if pack_wait_us is None else {"pack_wait_us": pack_wait_us}
    with SolveServer(meas, slots=slots, apply_mode=APPLY_TC, graphs=True, pack=True, **pkw) as srvp:
        srvp.run(warm, realtime=False)
        p0 = srvp.pack_stats()
        t0 = time.perf_counter()
        packed = srvp.run(at_once(), realtime=False)
        t_p = time.perf_counter() - t0
        p1 = srvp.pack_stats()
        launches, probs = p1["launches"] - p0["launches"], p1["problems"] - p0["problems"]
        res["capacity_with_packing"] = {"solves_per_s": len(reqs) / t_p, "packed_launches": launches,
                                        "packed_problems": probs,
                                        "problems_per_packed_launch": probs / launches if launches else None}
    served = [packed]
    # the server as configured by default (packing off: each slot launches its own applies on its stream)
    with SolveServer(meas, slots=slots, apply_mode=APPLY_TC, graphs=True) as srv:
        srv.run(warm, realtime=False)
        t0 = time.perf_counter()
        cap = srv.run(at_once(), realtime=False)
        t_cap = time.perf_counter() - t0
        thr_served = len(reqs) / t_cap
        res["capacity"] = {"solves_per_s": thr_served, "seconds": t_cap,
                           "peak_concurrent": srv.scheduler.peak_running,
                           "converged": int(sum(r.converged for r in cap.values())), "requests": len(reqs)}
        served.append(cap)
        if latency:
            rate = 0.8 * thr_served
            rng = np.random.default_rng(seed + 1)
            t = 0.0
            for r in reqs:
                t += rng.exponential(1.0 / rate)
                r.arrival = t
            lat = srv.run(reqs, realtime=True)
            s_lat = summarize(lat)
            res["latency_at_80pct_load"] = {"arrival_rate_per_s": rate, "p50_s": s_lat["p50_latency_s"],
                                            "p99_s": s_lat["p99_latency_s"], "mean_s": s_lat["mean_latency_s"],
                                            "solves_per_s": s_lat["solves_per_s"]}
            served.append(lat)
    res["speedup_vs_sequential_plain"] = thr_served / res["sequential_plain_fp32"]["solves_per_s"]
    res["speedup_of_packing"] = res["capacity_with_packing"]["solves_per_s"] / thr_served
    if seq_tc:
        res["speedup_vs_sequential_tc"] = thr_served / res["sequential_tc"]["solves_per_s"]
    res["max_far_field_rel_diff_served_vs_sequential"] = max(
        max(float(np.linalg.norm(run[k].far_field - base[k].far_field) /
                  max(np.linalg.norm(base[k].far_field), 1e-300)) for k in base) for run in served)
    return res


def run_serve_workload(args):
    levels = tuple(int(v) for v in args.serve_levels.split(","))
    res = serve_runs(args.requests, args.slots, args.serve_seed, args.seq_sample, levels=levels,
                     pack_wait_us=args.pack_wait_us)
    line = {"metric": "served solves/s (scattering, FarField)", "value": res["capacity"]["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": f"perturbed-icosphere scattering solves, levels {','.join(map(str, levels))}, "
                                   "kappa U[1,10], 1-64 plane waves, GMRES 1e-6, far field at 128 directions",
                       "requests": args.requests, "slots": args.slots, "seed": args.serve_seed}}
    line.update(res)
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the Gauss-Newton workload (--workload gauss-newton): not the headline line
# ---------------------------------------------------------------------------
def run_sizes_workload(args):
    """The boundary apply's dense stage against mesh size (not the headline
    line): icosphere levels 3-7 (1280 to 327680 triangles), 64 RHS = kappa
    {2, 4, 8, 16} x 16, SL + DL of the mixed BIE; the tensor-core and the
    plain FP32 form, each autotuned for the size first.  Dense-kernel time =
    median of 5 applies after one (CUDA events of the library's profiling;
    L2 not flushed: the smaller meshes are L2-resident, as they are inside a
    solve)."""
    from baemm_b200 import APPLY_FP32, APPLY_TC, Helmholtz_CUDA, meshes
    import torch
    levels = [int(v) for v in args.size_levels.split(",")]
    rows = []
    for level in levels:
        coords, tris = meshes.icosphere(level)
        nt = int(tris.shape[0])
        H = Helmholtz_CUDA(coords, tris, np.eye(3))
        H.SetProfiling(True)
        H.LoadBoundaryOperators_PL(KAPPA, coefficients(KAPPA), WC, WCS)
        rng = np.random.default_rng(0)
        B = (rng.standard_normal((coords.shape[0], WC)) + 1j * rng.standard_normal((coords.shape[0], WC))).astype(
            np.complex64)
        Bd = torch.from_numpy(B).cuda()
        Cd = torch.zeros_like(Bd)
        row = {"level": level, "triangles": nt, "interactions": nt * nt * WC}
        for name, mode in (("tc", APPLY_TC), ("fp32", APPLY_FP32)):
            H.SetApplyMode(mode)
            tr = H.Autotune(mode, repeats=2)
            ts = []
            for _ in range(6):
                H.ApplyBoundaryOperators_PL(1.0, Bd, 0.0, Cd)
                ts.append(H.LastApplyTimes()[1])
            ms = float(np.median(ts[1:]))
            row[name] = {"dense_ms": ms, "GInteractions_s": nt * nt * WC / (ms * 1e-3) / 1e9,
                         "tuned": {k: tr[k] for k in ("dense_variant", "tc_gen_warps", "tc_chunks", "tc_segment")}}
        row["speedup_tc_vs_fp32"] = row["fp32"]["dense_ms"] / row["tc"]["dense_ms"]
        rows.append(row)
        H.close()
    line = {"metric": "dense-stage GInteractions/s vs mesh size", "unit": "GInteractions/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "icosphere levels " + ",".join(map(str, levels)) + ", 64 RHS = kappa {2,4,8,16} x "
                                   "16, SL+DL of the mixed BIE, each form autotuned per size"},
            "sizes": rows}
    print(json.dumps(line), flush=True)
    return 0


def run_gn_workload(args):
    """One Gauss-Newton shape step (GaussNewtonSolve, FarField.hpp:457-604) on
    the configuration: initial shape the icosphere level 5 (10242 V, 20480 T),
    synthetic far-field data from a target shape perturbed by a degree-6
    spherical-harmonic field of amplitude 0.05, 2 wavenumbers {2, 4} x 32
    Fibonacci plane-wave directions, 128 far-field directions.  The right-hand
    side is the adjoint derivative of the far-field residual; the system
    (regpar M + DF* DF) X = B is solved by CG (outer tolerance 1e-8) with
    M = regpar x mass and the lumped-mass preconditioner (the reference's
    tangent-point metric lives in an unvendored library).  Runs: plain FP32,
    tensor-core, tensor-core inside FP64 iterative refinement, FP64; error of X
    against the FP64 run."""
    from baemm_b200 import APPLY_FP32, APPLY_FP64, APPLY_TC, Helmholtz_CUDA, WaveType, meshes
    coords, tris = meshes.icosphere(args.gn_level)
    tcoords, ttris = meshes.sh_perturbed_sphere(args.gn_level, 6, 0.05, seed=5)
    meas = meshes.fibonacci_sphere(128)
    inc = meshes.fibonacci_sphere(32)
    kap = np.array([2.0, 4.0])
    wc = 64
    regpar = 0.1
    with Helmholtz_CUDA(tcoords, ttris, meas) as T:
        T.SetApplyMode(APPLY_FP64)
        F_data = np.zeros((meas.shape[0], wc), complex)
        T.FarField(kap, inc, F_data, WaveType.Plane, 1e-12, 1e-12)
    H = Helmholtz_CUDA(coords, tris, meas)
    H.gmres_max_restarts = 10     # caps the outer CG at 30 x 10 iterations (and the inner GMRES at 10 cycles)
    nv = coords.shape[0]

    def Mop(x, y):
        H.MassDot(regpar, x, 0.0, y)

    def Pop(x, y):
        H.ApplyLumpedMassInverse(x, y)
        y /= regpar

    def step(mode, ir_steps=0):
        H.SetApplyMode(mode)
        H.SetRefinement(ir_steps, 1e-6)
        t0 = time.perf_counter()
        F0 = np.zeros((meas.shape[0], wc), complex)
        H.FarField(kap, inc, F0, WaveType.Plane, 1e-12, 1e-10)
        du = np.zeros((nv, wc), complex)
        H.Derivative_FF_Helper(kap, inc, du, WaveType.Plane, 1e-12, 1e-10)
        B = np.zeros((nv, 3))
        H.AdjointDerivative_FF(kap, inc, F0 - F_data, B, du, WaveType.Plane, 1e-12, 1e-10)
        X = np.zeros((nv, 3))
        ok = H.GaussNewtonSolve(kap, inc, Mop, Pop, 1.0, B, 0.0, X, du, WaveType.Plane, 1e-12, 1e-10, 1e-8,
                                solver=1)
        dt = time.perf_counter() - t0
        st = H.LastSolveStats()
        H.SetRefinement(0)
        H.SetApplyMode(APPLY_FP32)
        return X, dt, bool(ok), int(st["gmres_iterations"]), float(st["gmres_relative_residual"])

    r64 = step(APPLY_FP64)
    X64 = r64[0]
    runs = {"fp64": r64, "fp32": step(APPLY_FP32), "tc": step(APPLY_TC), "tc_fp64ir": step(APPLY_TC, ir_steps=6)}
    n64 = float(np.linalg.norm(X64))
    res = {k: {"seconds": v[1], "converged": v[2], "cg_iterations": v[3], "cg_relative_residual": v[4],
               "rel_err_vs_fp64": float(np.linalg.norm(v[0] - X64) / n64)}
           for k, v in runs.items()}
    line = {"metric": "Gauss-Newton shape step (s)", "value": res["tc_fp64ir"]["seconds"], "unit": "s",
            "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": f"icosphere level {args.gn_level} ({nv} V, {tris.shape[0]} T), kappa {{2,4}} x 32 "
                                   "plane waves, 128 far-field directions, CG to 1e-8 on regpar M + DF*DF, regpar 0.1",
                       "wave_count": wc},
            "runs": res,
            "note": "each run: far field, du/dn, adjoint-derivative gradient, GaussNewtonSolve (wall time)"}
    print(json.dumps(line), flush=True)
    H.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--mode", default="tc", choices=["fp32", "tc", "fp64"],
                    help="apply arithmetic: plain FP32, compensated tensor-core (default), FP64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain-FP32 and FP64 comparison applies")
    ap.add_argument("--workload", default="apply", choices=["apply", "nearfield", "solve", "serve", "gauss-newton", "apply-sizes"],
                    help="apply: the headline operator-apply line; solve: the scattering-solve configuration; "
                         "serve: the request stream through the serving loop")
    ap.add_argument("--requests", type=int, default=100, help="requests of --workload serve")
    ap.add_argument("--no-tune", action="store_true", help="time the default kernel shapes (no autotuning)")
    ap.add_argument("--shape", default="", help="fixed tensor-core shape 'gen_warps,chunks,segment' (no autotuning)")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="default apply line without the solve and serving keys")
    ap.add_argument("--serve-sample", type=int, default=48, help="requests of the default line's serving sample")
    ap.add_argument("--slots", type=int, default=6, help="serving slots of --workload serve")
    ap.add_argument("--serve-seed", type=int, default=0)
    ap.add_argument("--serve-levels", default="4,5,6", help="icosphere levels of --workload serve's stream")
    ap.add_argument("--pack-wait-us", type=int, default=None,
                    help="the packer's wait for partners in --workload serve (default: the server's)")
    ap.add_argument("--seq-sample", type=int, default=0,
                    help="--workload serve: run the sequential baseline on the first N requests only (0: all)")
    ap.add_argument("--gn-level", type=int, default=5, help="icosphere level of --workload gauss-newton")
    ap.add_argument("--size-levels", default="3,4,5,6,7", help="icosphere levels of --workload apply-sizes")
    ap.add_argument("--solve-level", type=int, default=6, help="icosphere level of --workload solve")
    ap.add_argument("--solve-modes", default="fp64,fp32,tc,tc_ir",
                    help="--workload solve: the runs to make (fp64 is the error reference; without it the errors "
                         "are null)")
    ap.add_argument("--small", action="store_true", help="38400-triangle torus (profiling captures only)")
    ap.add_argument("--kappa", default="",
                    help="--workload apply: wavenumbers of the 64 RHS, comma-separated, each over 64 / count columns "
                         "(default 2,4,8,16 x 16; e.g. 8 = one wavenumber x 64, whose column groups share the "
                         "tensor-core form's kernel entries)")
    ap.add_argument("--shard", action="store_true",
                    help="split each apply by target rows over the ranks (strong scaling; default: replicas)")
    args = ap.parse_args(argv)
    if args.kappa:
        global KAPPA, WCS, WORKLOAD
        kap = [float(x) for x in args.kappa.split(",")]
        if WC % len(kap) or (WC // len(kap)) % 16:
            ap.error("--kappa: 64 / count must be a multiple of 16 (1, 2 or 4 wavenumbers)")
        KAPPA, WCS = np.array(kap), WC // len(kap)
        WORKLOAD = WORKLOAD.replace("kappa {2,4,8,16} x 16",
                                    "kappa {%s} x %d" % (",".join("%g" % k for k in kap), WCS))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.workload == "nearfield":
        return run_nearfield_workload(args) if rank == 0 else 0
    if args.workload == "solve":
        return run_solve_workload(args) if rank == 0 else 0
    if args.workload == "serve":
        return run_serve_workload(args) if rank == 0 else 0
    if args.workload == "gauss-newton":
        return run_gn_workload(args) if rank == 0 else 0
    if args.workload == "apply-sizes":
        return run_sizes_workload(args) if rank == 0 else 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
