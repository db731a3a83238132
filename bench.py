#!/usr/bin/env python
"""Benchmark: VUMPS on the spinful Hubbard chain (Jordan-Wigner, t=1, U=4, mu=2,
d=4, w=6), unit cell N=2, bond dimension D=1024, ComplexF64 states.

A step is one VUMPS iteration (localupdate eigensolves + regauge!, gauge_step!,
environment rebuild, Galerkin error and energy) on device-resident data.  The
state starts from seeded random site tensors (PCG64 seed 3), canonicalised, and
is advanced by W untimed warm-up iterations before K timed ones.  Inputs (the
2 x 64 MiB site tensors and 2 x 96 MiB environments per side) exceed nothing in
L2-resident terms: every Heff GEMM streams >100 MB operands, so no L2 flush is
needed between iterations.

One JSON line on rank 0 (see the keys below).  ``--impl reference`` times the
CPU oracle (the NumPy restatement of the reference, which is not runnable here:
no Julia) on a bounded sample of the same workload.  With ``--gpus N > 1`` the
job runs N independent replicas (the path does not shard; no collective).
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

WORKLOAD = dict(workload="vumps_hubbard_jw", model="Fermi-Hubbard JW t=1 U=4 mu=2 (d=4, w=6)", N=2, D=1024,
                seed=3, dtype="complex128")
METRIC = "VUMPS iterations/s (Hubbard JW, N=2, D=1024)"
UNIT = "iter/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="split", choices=["fp64", "split"],
                   help="split: int8-sliced tensor-core Heff/transfer GEMMs with FP64 gauge, Krylov and "
                        "residual (the mixed-precision form); fp64: the plain FP64 pipeline")
    p.add_argument("--nslices", type=int, default=0, help="int8 slices (0 = adaptive to the solver tolerance)")
    p.add_argument("--D", type=int, default=WORKLOAD["D"])
    p.add_argument("--mode", default="vumps", choices=["vumps", "heff", "converge", "tdvp", "batch", "kernels"],
                   help="vumps: one VUMPS iteration per step; heff: one AC Heff apply per step; "
                        "converge: VUMPS to convergence in FP64 and split precision from the same start; "
                        "tdvp: TFIM quench, TDVP in FP64 and split precision from one ground state; "
                        "batch: 64 TFIM instances of uneven D by batched VUMPS, with dE/dh checks")
    p.add_argument("--tdvp-steps", type=int, default=200)
    p.add_argument("--mpo-steps", type=int, default=20,
                   help="tdvp mode: steps of the W^II MPO side run (mult with VOMPS at bond D)")
    p.add_argument("--instances", type=int, default=64)
    p.add_argument("--threads", type=int, default=16)
    p.add_argument("--no-seq", action="store_true")
    p.add_argument("--model", default="hubbard", choices=["tfim", "xxz", "hubbard"])
    p.add_argument("--N", type=int, default=None)
    p.add_argument("--h", type=float, default=1.0, help="TFIM field")
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--maxiter", type=int, default=200)
    p.add_argument("--seed", type=int, default=None)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-full", action="store_true",
                   help="cpu_baseline from a whole oracle VUMPS iteration (minutes at D=1024) instead of a sample")
    p.add_argument("--fp64-steps", type=int, default=None,
                   help="iterations of the plain FP64 arm timed beside the split run (default: --steps; 0 = skip)")
    p.add_argument("--ref-steps", type=int, default=1,
                   help="whole oracle VUMPS iterations timed by --impl reference (each is minutes of CPU work)")
    a = p.parse_args()
    if a.fp64_steps is None:
        a.fp64_steps = a.steps
    return a


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, v):
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return v


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # a timed iteration that overlapped nvidia-smi's start-up ran about 0.6 s
            # long; wait for its first sample, so the start-up is over before the timed
            # region begins (bounded: 10 s)
            t0 = time.time()
            while not self.samples and self.proc.poll() is None and time.time() - t0 < 10.0:
                time.sleep(0.02)
            self.samples.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            if len(s) >= 9:
                for k, nm in enumerate(names):
                    if s[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_reference_tflops():
    """cuBLAS ZGEMM throughput on this GPU (the FP64 ceiling the plain method is compared with)."""
    import torch
    a = torch.randn(4096, 1024, dtype=torch.complex128, device="cuda")
    b = torch.randn(1024, 4096, dtype=torch.complex128, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        a @ b
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    return 8.0 * 4096 * 4096 * 1024 / (ms / 1e3) / 1e12


# DRAM bytes per k_gemm_i8 launch: the mean of the two launches of one AC Heff apply at
# Hubbard D=1024, 4 slices, 128 x 128 tiles (GL x: 189 MB read + 369 MB written; T2 GR:
# 616 MB read + 62 MB written), from one ncu capture
# (profiles/k_gemm_i8_ac_heff_hubbard_d1024_traffic.md).  The algorithmic bytes of the same
# two launches are 538 MB and 520 MB.
GEMM_I8_TRAFFIC_PER_LAUNCH = 0.5 * (188907008 + 368586240 + 616073728 + 61922048)
GEMM_I8_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, mean of the 2 k_gemm_i8 launches of "
                          "one AC Heff apply (Hubbard D=1024, 4 slices; bench.py --mode heff --nslices 4); the timed "
                          "region mixes these with the smaller C-Heff and push launches")


def ac_flops(D, d, w):
    # F_AC = 16 w d D^3 + 8 w^2 d^2 D^2 (algorithmic, complex MAC = 8 flops)
    return 16.0 * w * d * D ** 3 + 8.0 * w * w * d * d * D ** 2


def vumps_prep(ctx, D, N, seed):
    """Seeded start of the benchmark workload on the device: random site tensors
    (PCG64 ``seed``), canonicalised (CanonicalIMPS(As)), environments built, then the
    prelude of find_groundstate(::VUMPS) (Galerkin error and recalculate!)."""
    import infinitempsalgorithms_b200 as imps
    H = imps.SparseIMPO([imps.hubbard_hamiltonian().Ws[0]] * N)
    As = imps.random_site_tensors([4] * N, D, seed)
    psi = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
    envs = imps.DMRGCache(psi, H)
    eps = imps.calc_galerkin(psi, H, envs)
    imps.recalculate(envs, psi, H, tol=imps.updatetol(imps.Defaults.alg_environments(), 0, eps)["tol"])
    return H, psi, envs, eps


def timed_iterations(ctx, H, psi, envs, eps, k, stream, it0=0):
    """k VUMPS iterations (imps_vumps_iter) from outer index it0 + 1, each bracketed
    by CUDA events on the library's stream.  Returns (total ms, per-iteration ms,
    per-iteration infos, eps)."""
    import torch
    import ctypes as C
    from infinitempsalgorithms_b200 import _lib as L
    lib, Hh = ctx.lib, H.handle(ctx)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
    infos = []
    torch.cuda.synchronize()
    ev[0].record(stream)
    for i in range(k):
        info = L.VumpsInfo()
        L.check(lib.imps_vumps_iter(envs.h, Hh, psi.h, it0 + i + 1, eps, C.byref(info)), ctx.h)
        ev[i + 1].record(stream)
        eps = info.galerkin
        infos.append(info)
    torch.cuda.synchronize()
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(k)]
    return ev[0].elapsed_time(ev[k]), per, infos, eps


def run_ours(args, world, rank, local):
    import torch
    import infinitempsalgorithms_b200 as imps
    from infinitempsalgorithms_b200 import _lib as L
    import ctypes as C

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    ctx = imps.Context(local)
    ctx.set_stream(stream.cuda_stream)
    if args.precision == "split":
        ctx.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices)
    lib = ctx.lib
    D, N = args.D, WORKLOAD["N"]
    t0 = time.time()
    H, psi, envs, eps0 = vumps_prep(ctx, D, N, WORKLOAD["seed"] + 1000 * rank)
    prep_s = time.time() - t0
    Hh = H.handle(ctx)
    # the warmed-up run restarts from this seeded start: the timed window is the
    # first K iterations of find_groundstate(::VUMPS), the window the CPU
    # reference arm times too
    snap0 = snapshot(ctx, psi, envs)
    timed_iterations(ctx, H, psi, envs, eps0, args.warmup, stream)
    restore(ctx, psi, envs, snap0)
    barrier(world)
    clocks = Clocks(local)
    clocks.start()
    # inside the timed region only the dominant GEMM class is timed (pooled CUDA events
    # around its launches on this stream), so the profiler adds almost nothing
    gem_key = "gemm_split" if args.precision == "split" else "zgemm_fp64"
    ctx.profile_classes([gem_key])
    ctx.profile(True)
    ctx.profile_reset()
    c0 = ctx.counters()
    torch.cuda.nvtx.range_push("vumps_timed")
    ms, per_ms, infos, eps = timed_iterations(ctx, H, psi, envs, eps0, args.steps, stream)
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    c1 = ctx.counters()
    gem_dump = ctx.profile_dump()
    ctx.profile_classes(None)
    ctx.profile_reset()
    # one more iteration, outside the timed region, with every kernel class timed
    timed_iterations(ctx, H, psi, envs, eps, 1, stream, it0=args.steps)
    dump = ctx.profile_dump()
    ctx.profile(False)
    prof = {}
    for name, (n, kms, work) in dump.items():
        base = name.split("@")[0]
        a = prof.get(base, (0, 0.0, 0.0))
        prof[base] = (a[0] + n, a[1] + kms, a[2] + work)
    gsum = [0, 0.0, 0.0]
    for name, (n, kms, work) in gem_dump.items():
        gsum[0] += n
        gsum[1] += kms
        gsum[2] += work
    barrier(world)
    ms_max = allmax(world, ms)
    value = args.steps * world / (ms_max / 1e3)
    launches = c1["kernels"] - c0["kernels"]
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c128 (int8-split Heff/transfer GEMMs, FP64 elsewhere)",
        "data": "synthetic (seeded PCG64 random MPS, no dataset)",
        "config": dict(WORKLOAD, D=D, precision=args.precision,
                       nslices=args.nslices if args.precision == "split" else None,
                       window=f"VUMPS iterations 1..{args.steps} from the seeded canonical start "
                              f"(warm-up: iterations 1..{args.warmup}, then the start is restored)",
                       parallelism=f"replicas{world}" if world > 1 else "single",
                       l2="inputs > L2 (>100 MB operands per GEMM); no flush"),
        "gpu_launches": int(launches),
        "iter_ms": [round(x, 2) for x in per_ms],
        "galerkin_trace": [i.galerkin for i in infos],
        "galerkin": infos[-1].galerkin, "energy_per_site": infos[-1].energy_re / N,
        "ac_matvecs": int(sum(i.ac_matvecs for i in infos)), "c_matvecs": int(sum(i.c_matvecs for i in infos)),
        "gauge_iters": [int(i.gauge_iters) for i in infos],
        "prep_s": prep_s,
        "op_counts_per_iter": iter_counts(c0, c1, args.steps, D),
        "profiled_iteration_ms": {k: round(v[1], 3) for k, v in prof.items()},
        "profiled_iteration_ms_by_site": {k: round(v[1], 1)
                                          for k, v in sorted(dump.items(), key=lambda kv: -kv[1][1])[:16]},
    }
    n_g, ms_g = gsum[0], gsum[1]
    if n_g:
        pk, pk_kind = peaks()
        if args.precision == "split":
            alg = c1["split_alg_flops"] - c0["split_alg_flops"]
            exe = c1["split_exec_ops"] - c0["split_exec_ops"]
            nl = c1["split_launches"] - c0["split_launches"]
            peak = 2.0 * pk["bf16_tflops"]
            achieved = alg / (ms_g / 1e3) / 1e12
            result["roofline"] = {
                "bound": "tensor", "kernel": "k_gemm_i8 (int8-split complex GEMM)",
                "achieved": achieved, "unit": "TFLOP/s",
                "achieved_meaning": "algorithmic FP64-accurate complex GEMM flops (8 M N K per launch) / event time",
                "peak": peak, "peak_kind": f"int8 dense tensor = 2 x {pk_kind} bf16 dense ({pk['bf16_tflops']} TFLOP/s)",
                "frac": achieved / peak,
                "executed_tops": exe / (ms_g / 1e3) / 1e12, "frac_executed": exe / (ms_g / 1e3) / 1e12 / peak,
                "launches": n_g, "launches_counted": nl, "avg_launch_ms": ms_g / n_g,
                "alg_flops_per_launch": alg / max(nl, 1), "exec_ops_per_launch": exe / max(nl, 1),
                "traffic": GEMM_I8_TRAFFIC_PER_LAUNCH, "traffic_source": GEMM_I8_TRAFFIC_SOURCE,
                "share_of_step": ms_g / ms}
        else:
            flops = gsum[2]
            achieved = flops / (ms_g / 1e3) / 1e12
            ref = fp64_reference_tflops()
            result["roofline"] = {"bound": "fp64-tensor", "kernel": "k_zgemm_dmma (FP64 complex GEMM)",
                                  "achieved": achieved, "unit": "TFLOP/s", "peak": ref,
                                  "peak_kind": "FP64: cuBLAS ZGEMM (torch complex128 matmul 4096x4096x1024) "
                                               "measured in this run",
                                  "frac": achieved / ref, "launches": n_g, "avg_launch_ms": ms_g / n_g,
                                  "traffic": None, "share_of_step": ms_g / ms}
    result["clocks"] = clk
    # the plain FP64 method on the same GPU, same seeded start, same iteration window
    if args.precision == "split" and args.fp64_steps > 0:
        k64 = min(args.fp64_steps, args.steps)
        c64 = imps.Context(local)
        c64.set_stream(stream.cuda_stream)
        psi64 = imps.CanonicalIMPS(c64, [4] * N, [D] * N)
        envs64 = imps.DMRGCache(psi64, H, build=False)
        # one untimed FP64 iteration first (buffers of the FP64 context, its kernels)
        restore(c64, psi64, envs64, snap0)
        timed_iterations(c64, H, psi64, envs64, eps0, 1, stream)
        restore(c64, psi64, envs64, snap0)
        ms64, per64, inf64, _ = timed_iterations(c64, H, psi64, envs64, eps0, k64, stream)
        ms_s = sum(per_ms[:k64])
        result["fp64"] = {
            "value": k64 / (ms64 / 1e3), "unit": UNIT, "steps": k64, "ms_per_step": ms64 / k64,
            "iter_ms": [round(x, 2) for x in per64], "galerkin_trace": [i.galerkin for i in inf64],
            "energy_per_site": inf64[-1].energy_re / N, "ac_matvecs": int(sum(i.ac_matvecs for i in inf64)),
            "c_matvecs": int(sum(i.c_matvecs for i in inf64))}
        result["speedup_vs_fp64"] = ms64 / ms_s
        result["speedup_vs_fp64_window"] = f"iterations 1..{k64} of both runs"
        result["delta_e_vs_fp64"] = abs(infos[k64 - 1].energy_re / N - inf64[-1].energy_re / N)
        result["delta_galerkin_vs_fp64"] = abs(infos[k64 - 1].galerkin - inf64[-1].galerkin)
        c64.close()
    # Heff matvec throughput on the final state (device-resident, AC site 1)
    nrep = 10
    x = torch.zeros(D * 4 * D, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    x.copy_(torch.randn(D * 4 * D, dtype=torch.complex128, device="cuda"))
    for _ in range(2):
        L.check(lib.imps_ac_apply_dev(envs.h, Hh, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), ctx.h)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nrep):
        L.check(lib.imps_ac_apply_dev(envs.h, Hh, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), ctx.h)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_ac = e0.elapsed_time(e1) / nrep
    result["heff_matvecs_per_s"] = 1e3 / ms_ac
    result["heff_ms"] = ms_ac
    result["heff_tflops"] = ac_flops(D, 4, 6) / (ms_ac / 1e3) / 1e12
    if not args.no_e2e:
        restore(ctx, psi, envs, snap0)
        result["e2e"] = run_e2e(args, ctx, psi, envs, H, 0, eps0, world)
    return result, ctx, psi, envs, H, snap0, eps0


def run_heff(args, world, rank, local):
    """AC effective-Hamiltonian matvecs/s at the workload's D (site 1, random
    environments of the right shape): the dominant operation of every solver."""
    import torch
    import ctypes as C
    import infinitempsalgorithms_b200 as imps
    from infinitempsalgorithms_b200 import _lib as L
    torch.cuda.set_device(local)
    ctx = imps.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    if args.precision == "split":
        ctx.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices if args.nslices > 0 else 5)
    D = args.D
    H = imps.hubbard_hamiltonian()
    d, w = 4, 6
    psi = imps.CanonicalIMPS(ctx, [d], [D])
    envs = imps.DMRGCache(psi, H, build=False)
    rng = np.random.default_rng(rank)
    envs.set_leftenv(1, rng.standard_normal((D, w, D)) + 1j * rng.standard_normal((D, w, D)))
    envs.set_rightenv(1, rng.standard_normal((D, w, D)) + 1j * rng.standard_normal((D, w, D)))
    x = torch.randn(D * d * D, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    Hh = H.handle(ctx)

    def apply():
        L.check(ctx.lib.imps_ac_apply_dev(envs.h, Hh, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), ctx.h)
    for _ in range(args.warmup):
        apply()
    torch.cuda.synchronize()
    barrier(world)
    ctx.profile(True)
    ctx.profile_reset()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        apply()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = allmax(world, e0.elapsed_time(e1))
    prof = {k: ctx.profile_get(k) for k in ("zgemm_fp64", "gemm_split", "level_mix", "split_slice")}
    return {"metric": f"AC Heff matvecs/s (Hubbard JW, D={D})", "value": args.steps * world / (ms / 1e3),
            "unit": "matvec/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "tflops_alg": ac_flops(D, d, w) * args.steps / (ms / 1e3) / 1e12,
            "config": {"workload": "ac_heff_hubbard_jw", "D": D, "precision": args.precision,
                       "nslices": args.nslices if args.precision == "split" else None},
            "kernel_ms": {k: round(v[1] / args.steps, 3) for k, v in prof.items()}}


def run_kernels(args, world, rank, local):
    """The FP64 building blocks around the GEMM engines at the workload's sizes (d = 4):
    QRpos of the (4 D) x D site matrix of the gauge fix and one restart cycle of the AC
    Lanczos eigensolve of the Hubbard model (its Gram-Schmidt passes).  Kernel-class times
    from CUDA events on the context stream (the library's profiler), after one untimed
    repetition of each."""
    import torch
    import infinitempsalgorithms_b200 as imps
    torch.cuda.set_device(local)
    ctx = imps.Context(local)
    D = args.D
    rng = np.random.default_rng(7)
    M = np.asfortranarray(rng.standard_normal((4 * D, D)) + 1j * rng.standard_normal((4 * D, D)))
    imps.qrpos(M, ctx=ctx)
    ctx.synchronize()
    ctx.profile(True)
    ctx.profile_reset()
    reps = max(1, args.steps)
    for _ in range(reps):
        Q, R = imps.qrpos(M, ctx=ctx)
    ctx.synchronize()
    qr = ctx.profile_get("qr")
    zg = ctx.profile_get("zgemm_fp64")
    qs = ctx.profile_get("qr_small")
    ctx.profile(False)
    qerr = float(np.linalg.norm(Q @ R - M) / np.linalg.norm(M))
    H = imps.hubbard_hamiltonian()
    psi = imps.CanonicalIMPS(ctx, [4], [D])
    envs = imps.DMRGCache(psi, H, build=False)
    GL = rng.standard_normal((D, 6, D)) + 1j * rng.standard_normal((D, 6, D))
    GR = rng.standard_normal((D, 6, D)) + 1j * rng.standard_normal((D, 6, D))
    envs.set_leftenv(1, GL + GL.conj().transpose(2, 1, 0))
    envs.set_rightenv(1, GR + GR.conj().transpose(2, 1, 0))
    x0 = np.asfortranarray(rng.standard_normal((D, 4, D)) + 1j * rng.standard_normal((D, 4, D)))
    hac = imps.AC_hamiltonian(1, psi, H, psi, envs)
    alg = dict(tol=1e-9, krylovdim=30, maxiter=1, eager=False)
    imps.fixedpoint(hac, x0, "SR", alg)
    ctx.synchronize()
    ctx.profile(True)
    ctx.profile_reset()
    imps.fixedpoint(hac, x0, "SR", alg)
    ctx.synchronize()
    # the eigensolve tags its kernel classes with the call site ("orth@eig_ac")
    orth = [0, 0.0, 0.0]
    for k, v in ctx.profile_dump().items():
        if k.split("@")[0] == "orth":
            orth = [orth[i] + v[i] for i in range(3)]
    ctx.profile(False)
    n = D * 4 * D
    return {"metric": f"QRpos and Gram-Schmidt kernel times (d=4, D={D})", "unit": "ms",
            "config": {"workload": "fp64_blocks", "D": D, "qr_shape": [4 * D, D], "krylovdim": 30},
            "qrpos_ms": qr[1] / reps, "qrpos_tflops": qr[2] / reps / (qr[1] / reps / 1e3) / 1e12 if qr[1] else None,
            "qrpos_inner_gemm_ms": zg[1] / reps, "qrpos_small_update_ms": qs[1] / reps,
            "qrpos_rel_residual": qerr,
            "gram_schmidt": {"projections": orth[0], "ms": orth[1],
                             "min_bytes": orth[2], "vector_bytes": 16 * n,
                             "gbs_min_bytes": orth[2] / (orth[1] / 1e3) / 1e9 if orth[1] else None}}


def run_converge(args, world, rank, local):
    """find_groundstate(VUMPS) to Galerkin <= tol in FP64 and in split precision from
    the same seeded state; reports iterations, wall time, Galerkin error and |delta e|."""
    import torch
    import infinitempsalgorithms_b200 as imps
    from infinitempsalgorithms_b200 import _lib as L
    torch.cuda.set_device(local)
    models = {"tfim": (lambda: imps.tfim_hamiltonian(h=args.h), 2, 1),
              "xxz": (imps.heisenberg_hamiltonian, 2, 2),
              "hubbard": (imps.hubbard_hamiltonian, 4, 2)}
    mk, d, N0 = models[args.model]
    N = args.N or N0
    H = imps.SparseIMPO([mk().Ws[0]] * N)
    seed = args.seed if args.seed is not None else {"tfim": 1, "xxz": 2, "hubbard": 3}[args.model]
    As = imps.random_site_tensors([d] * N, args.D, seed)
    out = {}
    traces = {}
    for prec in ("fp64", "split"):
        ctx = imps.Context(local)
        if prec == "split":
            ctx.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices)
        psi0 = imps.CanonicalIMPS.from_sites(As, ctx=ctx)
        trace = []        # (iteration, seconds since the start, energy per site)
        excl = [0.0]      # time spent evaluating the traced energies, left out of the clock

        def record(it, psi, H_, envs, trace=trace, excl=excl):
            torch.cuda.synchronize()
            t = time.perf_counter()
            e_it = imps.expectationvalue(psi, H_, envs).real / N
            torch.cuda.synchronize()
            trace.append((it, t - t0 - excl[0], e_it))
            excl[0] += time.perf_counter() - t
            return psi, envs

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        psi, envs, info = imps.find_groundstate(psi0, H, imps.VUMPS(D=args.D, maxiter=args.maxiter, tol=args.tol,
                                                                    finalize=record))
        e = imps.expectationvalue(psi, H, envs).real / N
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0 - excl[0]
        # galerkin of iteration it is losses[it] (losses[0]: the start state)
        traces[prec] = [(it, ts, et, info.losses[it]) for it, ts, et in trace]
        out[prec] = {"iterations": info.niter, "converged": bool(info.converged), "galerkin": info.itererr,
                     "energy_per_site": e, "wall_s": dt, "s_per_iter": dt / max(info.niter, 1)}
        if rank == 0:
            # each arm as soon as it ends, so that a run cut short still reports the first
            print(json.dumps({"arm": prec, **out[prec], "trace": traces[prec]}), file=sys.stderr, flush=True)
        ctx.close()

    def time_to(tr, g):
        return next((ts for it, ts, et, gal in tr if gal <= g), None)

    thresholds = [1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8]
    reach = {f"{g:.0e}": {"fp64_s": time_to(traces["fp64"], g), "split_s": time_to(traces["split"], g)}
             for g in thresholds}
    for v in reach.values():
        v["speedup"] = (v["fp64_s"] / v["split_s"]) if (v["fp64_s"] and v["split_s"]) else None
    common = min(len(traces["fp64"]), len(traces["split"]))
    de_iter = [abs(traces["split"][i][2] - traces["fp64"][i][2]) for i in range(common)]
    res = {"metric": f"VUMPS to convergence ({args.model}, N={N}, D={args.D}, tol={args.tol})",
           "config": {"model": args.model, "N": N, "D": args.D, "seed": seed, "tol": args.tol,
                      "maxiter": args.maxiter, "h": args.h if args.model == "tfim" else None,
                      "nslices": args.nslices or "adaptive"},
           "fp64": out["fp64"], "split": out["split"],
           "delta_e": abs(out["split"]["energy_per_site"] - out["fp64"]["energy_per_site"]),
           "wall_speedup": out["fp64"]["wall_s"] / out["split"]["wall_s"],
           "time_to_galerkin": reach,
           "delta_e_same_iteration": {"first": de_iter[:5], "last": de_iter[-5:], "max_last10": max(de_iter[-10:])
                                      if de_iter else None},
           "galerkin_trace": {"fp64": [t[3] for t in traces["fp64"]], "split": [t[3] for t in traces["split"]]},
           "energy_trace": {"fp64": [t[2] for t in traces["fp64"]], "split": [t[2] for t in traces["split"]]},
           "time_trace": {"fp64": [round(t[1], 3) for t in traces["fp64"]],
                          "split": [round(t[1], 3) for t in traces["split"]]}}
    if args.model == "hubbard":
        res["lieb_wu_e0"] = -2.5737293679
    if args.model == "tfim":
        import math as _m
        from scipy.integrate import quad
        e0 = -quad(lambda k: _m.sqrt(1 + args.h ** 2 - 2 * args.h * _m.cos(k)), 0, _m.pi)[0] / _m.pi
        res["exact_e0"] = e0
        res["fp64_err_vs_exact"] = abs(out["fp64"]["energy_per_site"] - e0)
    return res


def run_tdvp(args, world, rank, local):
    """TDVP quench: FP64 VUMPS ground state of the TFIM at J=1, h=0.5 (bond D, seed 4),
    then single-site TDVP under h=1.5 with dt = -0.01i for --tdvp-steps steps, once in
    FP64 and once in split precision from the same ground state.  Reports TDVP
    steps/s of each, <sigma_x>(t) and <sigma_z>(t) of both, the largest
    difference between them, and each run's energy drift |E(t) - E(0)|."""
    import torch
    import infinitempsalgorithms_b200 as imps
    from infinitempsalgorithms_b200 import _lib as L
    torch.cuda.set_device(local)
    J, h0, h1, dt = 1.0, 0.5, 1.5, -0.01j
    D = args.D
    H0, H1 = imps.tfim_hamiltonian(J, h0), imps.tfim_hamiltonian(J, h1)
    sx, sz = imps.sigma("x"), imps.sigma("z")
    ctx = imps.Context(local)
    t0 = time.perf_counter()
    psi0 = imps.CanonicalIMPS.from_sites(imps.random_site_tensors([2], D, 4), ctx=ctx)
    gs, genvs, ginfo = imps.find_groundstate(psi0, H0, imps.VUMPS(D=D, maxiter=args.maxiter, tol=args.tol))
    gs_s = time.perf_counter() - t0
    snap = {f: gs.get(f, 0) for f in (L.IMPS_AL, L.IMPS_AR, L.IMPS_C, L.IMPS_AC)}
    e_gs = imps.expectationvalue(gs, H0, genvs).real
    ctx.close()
    runs = {}
    for prec in ("fp64", "split"):
        c = imps.Context(local)
        if prec == "split":
            c.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices)
        psi = imps.CanonicalIMPS(c, [2], [D])
        for f, a in snap.items():
            psi.set(f, 0, a)
        envs = imps.DMRGCache(psi, H1)
        E0 = imps.expectationvalue(psi, H1, envs).real
        xs, zs, es = [imps.expectationvalue(psi, (1, sx)).real], [imps.expectationvalue(psi, (1, sz)).real], [E0]
        t_steps = 0.0
        for k in range(args.tdvp_steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            psi, envs = imps.timestep(psi, H1, dt, imps.TDVP(), envs)
            c.synchronize()
            t_steps += time.perf_counter() - t1
            xs.append(imps.expectationvalue(psi, (1, sx)).real)
            zs.append(imps.expectationvalue(psi, (1, sz)).real)
            es.append(imps.expectationvalue(psi, H1, envs).real)
        runs[prec] = {"steps_per_s": args.tdvp_steps / t_steps, "s_per_step": t_steps / args.tdvp_steps,
                      "energy_drift_max": float(np.max(np.abs(np.array(es) - E0))), "sx": xs, "sz": zs}
        c.close()
    # side run: the same quench by the W^II time-evolution MPO applied with mult(W, psi, VOMPS(D))
    side = None
    if args.mpo_steps > 0:
        c = imps.Context(local)
        psi = imps.CanonicalIMPS(c, [2], [D])
        for f, a in snap.items():
            psi.set(f, 0, a)
        W = imps.timeevompo(H1, dt, "WII")
        xs_m = [imps.expectationvalue(psi, (1, sx)).real]
        t_m, iters = 0.0, []
        for k in range(args.mpo_steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            psi, _, minfo = imps.mult(W, psi, imps.VOMPS(D=D, maxiter=50, tol=args.tol))
            c.synchronize()
            t_m += time.perf_counter() - t1
            iters.append(minfo.niter)
            xs_m.append(imps.expectationvalue(psi, (1, sx)).real)
        ref = runs["fp64"]["sx"][:args.mpo_steps + 1]
        side = {"mpo": "timeevompo(H(h=1.5), -0.01i, WII)", "steps": args.mpo_steps,
                "steps_per_s": args.mpo_steps / t_m, "vomps_iterations": iters,
                "max_abs_dsx_vs_tdvp_fp64": float(np.max(np.abs(np.array(xs_m) - np.array(ref)))),
                "sx": [round(v, 12) for v in xs_m]}
        c.close()
    dsx = float(np.max(np.abs(np.array(runs["split"]["sx"]) - np.array(runs["fp64"]["sx"]))))
    dsz = float(np.max(np.abs(np.array(runs["split"]["sz"]) - np.array(runs["fp64"]["sz"]))))
    every = max(1, args.tdvp_steps // 20)
    for prec in runs:
        runs[prec]["sx"] = [round(v, 12) for v in runs[prec]["sx"][::every]]
        runs[prec]["sz"] = [round(v, 12) for v in runs[prec]["sz"][::every]]
    return {"metric": f"TDVP steps/s (TFIM quench h=0.5->1.5, D={D}, dt=0.01)", "value": runs["split"]["steps_per_s"],
            "unit": "step/s", "higher_is_better": True, "n_gpus": world,
            "config": {"workload": "tdvp_quench_tfim", "J": J, "h0": h0, "h1": h1, "dt": "-0.01i", "D": D,
                       "steps": args.tdvp_steps, "seed": 4, "gs_tol": args.tol, "nslices": args.nslices or "adaptive"},
            "ground_state": {"iterations": ginfo.niter, "galerkin": ginfo.itererr, "energy_per_site": e_gs,
                             "wall_s": gs_s},
            "fp64": runs["fp64"], "split": runs["split"], "max_abs_dsx": dsx, "max_abs_dsz": dsz,
            "sample_every_steps": every, "mpo_side_run": side}


def run_batch(args, world, rank, local):
    """Batched VUMPS over 64 TFIM instances (J=1, h ~ U[0.5, 1.5] and D from
    {32, 64, 128, 256, 512}, both drawn with seed 5; instance k starts from random
    site tensors with seed 1000 + k), split precision, each instance on its own
    context and stream.  Reports aggregate VUMPS iterations/s and the wall time to
    solve all of them, the same instances solved one after another on one stream,
    energies against the exact TFIM energy, and dE/dh from the adjoint contraction
    against Hellmann-Feynman (all instances) and central differences of converged
    energies (the four smallest instances, FP64, Galerkin 1e-10, dh = 1e-5)."""
    import torch
    import math as _m
    from scipy.integrate import quad
    import infinitempsalgorithms_b200 as imps
    from infinitempsalgorithms_b200 import _lib as L
    torch.cuda.set_device(local)
    rng = np.random.default_rng(5)
    n = args.instances
    hs = rng.uniform(0.5, 1.5, n)
    Ds = rng.choice([32, 64, 128, 256, 512], n)
    Hs = [imps.tfim_hamiltonian(1.0, float(h)) for h in hs]
    As = [imps.random_site_tensors([2], int(D), 1000 + k) for k, D in enumerate(Ds)]
    alg = imps.VUMPS(maxiter=args.maxiter, tol=args.tol)

    def e0(h):
        return -quad(lambda k: _m.sqrt(1 + h * h - 2 * h * _m.cos(k)), 0, _m.pi)[0] / _m.pi

    def make(ctxs):
        return [imps.CanonicalIMPS.from_sites(As[k], ctx=ctxs[k]) for k in range(n)]
    res = {}
    # concurrent: one context (stream) per instance
    ctxs = [imps.Context(local) for _ in range(n)]
    for c in ctxs:
        c.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices)
    psi0s = make(ctxs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = imps.find_groundstate_batch(psi0s, Hs, alg, nthreads=args.threads)
    torch.cuda.synchronize()
    wall_b = time.perf_counter() - t0
    iters_b = sum(o[2].niter for o in out)
    es = [imps.expectationvalue(o[0], Hs[k], o[1]).real for k, o in enumerate(out)]
    dW = [[(imps.tfim_hamiltonian(1.0, float(h) + 1e-3).Ws[0] - imps.tfim_hamiltonian(1.0, float(h) - 1e-3).Ws[0])
           / 2e-3] for h in hs]
    grads = [imps.coupling_gradient(o[0], Hs[k], dW[k], o[1]).real for k, o in enumerate(out)]
    hf = [-imps.expectationvalue(o[0], (1, imps.sigma("z"))).real for o in out]
    res["batched"] = {"wall_s": wall_b, "iterations": int(iters_b), "iter_per_s": iters_b / wall_b,
                      "converged": int(sum(o[2].converged for o in out)),
                      "max_galerkin": float(max(o[2].itererr for o in out))}
    for c in ctxs:
        c.close()
    # the same instances one after another on one stream
    if not args.no_seq:
        c1 = imps.Context(local)
        c1.set_precision(L.IMPS_PREC_SPLIT_I8, args.nslices)
        t0 = time.perf_counter()
        its = 0
        for k in range(n):
            p0 = imps.CanonicalIMPS.from_sites(As[k], ctx=c1)
            _, _, inf = imps.find_groundstate(p0, Hs[k], alg)
            its += inf.niter
        c1.synchronize()
        wall_s = time.perf_counter() - t0
        res["sequential"] = {"wall_s": wall_s, "iterations": its, "iter_per_s": its / wall_s}
        c1.close()
    # central differences of converged FP64 energies for the four smallest instances
    fd = []
    small = [int(k) for k in np.argsort(Ds, kind="stable")[:4]]
    c2 = imps.Context(local)
    # Galerkin 1e-10 leaves energy errors near 1e-20 (quadratic), far below the
    # central-difference resolution at dh = 1e-5
    tight = imps.VUMPS(maxiter=100, tol=1e-10)
    for k in small:
        p0 = imps.CanonicalIMPS.from_sites(As[k], ctx=c2)
        g0, genv, _ = imps.find_groundstate(p0, Hs[k], tight)
        dh = 1e-5
        vals = []
        for sgn in (1, -1):
            Hk = imps.tfim_hamiltonian(1.0, float(hs[k]) + sgn * dh)
            pk, ek, _ = imps.find_groundstate(g0, Hk, tight)
            vals.append(imps.expectationvalue(pk, Hk, ek).real)
        gk = imps.coupling_gradient(g0, Hs[k], dW[k], genv).real
        fd.append({"instance": k, "D": int(Ds[k]), "h": float(hs[k]), "adjoint": gk,
                   "central_difference": (vals[0] - vals[1]) / (2 * dh)})
    c2.close()
    value = res["batched"]["iter_per_s"]
    return {"metric": f"batched VUMPS iterations/s ({n} TFIM instances, D in 32..512)", "value": value,
            "unit": "iter/s", "higher_is_better": True, "n_gpus": world,
            "config": {"workload": "vumps_tfim_batch", "instances": n, "h": "U[0.5,1.5] seed 5",
                       "D": "from {32,64,128,256,512} seed 5", "tol": args.tol, "maxiter": args.maxiter,
                       "threads": args.threads, "precision": "split", "nslices": args.nslices or "adaptive"},
            **res,
            "max_abs_e_minus_exact": float(max(abs(es[k] - e0(float(hs[k]))) for k in range(n))),
            "max_abs_grad_minus_hellmann_feynman": float(max(abs(grads[k] - hf[k]) for k in range(n))),
            "fd_check": fd,
            "max_abs_grad_minus_fd": float(max(abs(f["adjoint"] - f["central_difference"]) for f in fd))}


def snapshot(ctx, psi, envs):
    """Host copies of the state tensors and the environments (used to replay iterations)."""
    from infinitempsalgorithms_b200 import _lib as L
    st = {(f, l): psi.get(f, l) for l in range(psi.N) for f in (L.IMPS_AL, L.IMPS_AR, L.IMPS_C, L.IMPS_AC)}
    ev = {}
    for l in range(psi.N):
        for side in (0, 1):
            a = envs.leftenv(l + 1) if side == 0 else envs.rightenv(l + 1)
            ev[(side, l)] = np.asfortranarray(a)
    return st, ev


def restore(ctx, psi, envs, snap):
    from infinitempsalgorithms_b200 import _lib as L
    st, ev = snap
    for (f, l), a in st.items():
        psi.set(f, l, a)
    for (side, l), a in ev.items():
        L.check(ctx.lib.imps_envs_set(envs.h, side, l, a.ctypes.data_as(L.DP)), ctx.h)


def run_e2e(args, ctx, psi, envs, H, it, eps, world):
    """Same metric through the C ABI with host buffers, replaying the timed
    iterations from the warmed-up snapshot: each step uploads the state
    (AL/AR/C/AC of both sites) from pinned host memory, runs imps_vumps_iter,
    and downloads the new state and the energy."""
    import torch
    import ctypes as C
    from infinitempsalgorithms_b200 import _lib as L
    lib = ctx.lib
    N = psi.N
    fields = [(f, l) for l in range(N) for f in (L.IMPS_AL, L.IMPS_AR, L.IMPS_C, L.IMPS_AC)]
    host = {}
    for f, l in fields:
        shp = psi._shape(f, l)
        t = torch.empty(int(np.prod(shp)), dtype=torch.complex128, pin_memory=True)
        a = t.numpy()
        L.check(lib.imps_state_get(psi.h, f, l, a.ctypes.data_as(L.DP)), ctx.h)
        host[(f, l)] = (t, a)
    h2d = sum(a.nbytes for _, a in host.values())
    Hh = H.handle(ctx)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        it += 1
        for (f, l), (_, a) in host.items():
            L.check(lib.imps_state_set(psi.h, f, l, a.ctypes.data_as(L.DP)), ctx.h)
        info = L.VumpsInfo()
        L.check(lib.imps_vumps_iter(envs.h, Hh, psi.h, it, eps, C.byref(info)), ctx.h)
        eps = info.galerkin
        for (f, l), (_, a) in host.items():
            L.check(lib.imps_state_get(psi.h, f, l, a.ctypes.data_as(L.DP)), ctx.h)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    dt = allmax(world, dt)
    return {"value": args.steps * world / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(h2d + 16)}


# ---------------------------------------------------------------------------
# CPU timings of the oracle (the reference is Julia and cannot run here)
# ---------------------------------------------------------------------------
def cpu_threads():
    """BLAS threads the oracle's NumPy actually uses (OpenBLAS defaults to every host core)."""
    try:
        from threadpoolctl import threadpool_info
        n = [i["num_threads"] for i in threadpool_info() if i.get("user_api") == "blas"]
        if n:
            return int(max(n))
    except Exception:
        pass
    return os.cpu_count() or 1


def iter_counts(c0, c1, steps, D, d=4, w=6):
    """Per-iteration operation counts from the library's counters over the timed steps."""
    ac = (c1["ac_apply"] - c0["ac_apply"]) / steps
    cc = (c1["c_apply"] - c0["c_apply"]) / steps
    gf = (c1["gemm_flops"] - c0["gemm_flops"]) / steps
    other = max(0.0, gf - ac * 16.0 * w * d * D ** 3 - cc * 16.0 * w * D ** 3)
    return {"ac": ac, "c": cc, "qr": (c1["qr"] - c0["qr"]) / steps,
            "qr_flops": (c1["qr_flops"] - c0["qr_flops"]) / steps, "other_gemm_flops": other}


def oracle_from_snapshot(snap, N):
    """Oracle objects holding a device snapshot's state and environments."""
    import oracle as O
    from infinitempsalgorithms_b200 import _lib as L
    st, ev = snap
    f = {k: [np.asfortranarray(st[(k, l)]) for l in range(N)] for k in (L.IMPS_AL, L.IMPS_AR, L.IMPS_C, L.IMPS_AC)}
    opsi = O.CanonicalIMPS(f[L.IMPS_AL], f[L.IMPS_AR], f[L.IMPS_C], f[L.IMPS_AC])
    oenvs = O.DMRGCache([ev[(0, l)] for l in range(N)], [ev[(1, l)] for l in range(N)])
    return opsi, oenvs


def oracle_iterations(opsi, oH, oenvs, eps, k, D):
    """k real VUMPS iterations of the oracle (iterations 1..k of find_groundstate),
    each timed on the host clock; returns the per-iteration seconds and the final
    Galerkin error."""
    import oracle as O
    alg = O.VUMPS(D=D)
    secs = []
    for it in range(1, k + 1):
        t = time.perf_counter()
        opsi, oenvs, eps = O.vumps_iteration(opsi, oH, oenvs, alg, it, eps)
        secs.append(time.perf_counter() - t)
    return secs, eps


def oracle_sample(opsi, oH, oenvs, counts, D, reps=2):
    """A bounded sample of the oracle's VUMPS iteration (about half a minute of CPU work):
    ``reps`` AC and C Heff applies, one Gram-Schmidt projection against a 15-vector basis
    of the AC size, one QRpos of the (4 D) x D site matrix and one (D x 4 D) x D complex
    product, each timed on the host clock, scaled by this run's per-iteration operation
    counts (AC / C applies, one projection per apply, QRs, the remaining GEMM flops)."""
    import oracle as O
    N = len(opsi)
    GL, GR, W = oenvs.lefts[0], oenvs.rights[0], oH[0]
    t = time.perf_counter()
    for _ in range(reps):
        O.ac_apply(GL, W, GR, opsi.AC[0])
    t_ac = (time.perf_counter() - t) / reps
    GLc = oenvs.lefts[1 % N]
    t = time.perf_counter()
    for _ in range(reps):
        O.c_apply(GLc, GR, opsi.C[0])
    t_c = (time.perf_counter() - t) / reps
    n = opsi.AC[0].size
    basis = O.imps_oracle._KBasis(n, 16)
    rng = np.random.default_rng(0)
    for _ in range(15):
        v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        v, _ = O.imps_oracle._cgs2(basis, v / np.linalg.norm(v))
        basis.append(v / np.linalg.norm(v))
    w = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    t = time.perf_counter()
    O.imps_oracle._cgs2(basis, w)
    t_gs = time.perf_counter() - t
    M = np.asfortranarray(opsi.AC[0].reshape((-1, opsi.AC[0].shape[2]), order="F"))
    t = time.perf_counter()
    O.qrpos(M)
    t_qr = time.perf_counter() - t
    t = time.perf_counter()
    X = M @ opsi.C[0]
    t_mm = time.perf_counter() - t
    gemm_rate = 8.0 * M.shape[0] * M.shape[1] * opsi.C[0].shape[1] / t_mm
    sec = (counts["ac"] * (t_ac + t_gs) + counts["c"] * (t_c + t_gs) + counts["qr"] * t_qr
           + counts["other_gemm_flops"] / gemm_rate)
    del X
    sample = (f"oracle (NumPy/OpenBLAS, {cpu_threads()} threads) op times at D={D} from the GPU run's start state: "
              f"AC apply {t_ac:.2f} s, C apply {t_c:.2f} s, Gram-Schmidt projection (15 vectors) {t_gs:.2f} s, "
              f"QRpos {M.shape[0]}x{M.shape[1]} {t_qr:.2f} s, ZGEMM {gemm_rate / 1e9:.0f} GFLOP/s; scaled by this "
              f"run's per-iteration counts ({counts['ac']:.0f} AC, {counts['c']:.0f} C, {counts['qr']:.0f} QR, "
              f"{counts['other_gemm_flops'] / 1e12:.1f} TFLOP other GEMM) to {sec:.0f} s per iteration; "
              f"`--cpu-full` times a whole oracle iteration instead")
    return sec, sample


def run_reference(args, world, rank):
    """The reference arm: the CPU oracle (NumPy/OpenBLAS restatement of the
    reference's VUMPS; Julia is absent) on the same seeded workload.  Preparation
    (canonicalising the seeded site tensors, building the environments and the
    find_groundstate prelude) is untimed; then ``min(steps, --ref-steps)`` whole
    VUMPS iterations, iterations 1.. of the run, are timed on the host clock."""
    if rank != 0:
        return None
    import oracle as O
    D, N = args.D, WORKLOAD["N"]
    k = max(1, min(args.steps, args.ref_steps))
    t0 = time.perf_counter()
    oH = O.SchurMPO([O.hubbard_hamiltonian().Ws[0]] * N)
    opsi = O.canonical_from_sites(O.random_site_tensors([4] * N, D, WORKLOAD["seed"]))
    oenvs = O.build_envs(opsi, oH)
    eps = O.calc_galerkin(opsi, oH, oenvs)
    ae = O.updatetol(O.alg_environments(), 0, eps)
    oenvs = O.build_envs(opsi, oH, tol=ae["tol"], maxiter=ae["maxiter"], init=oenvs)
    prep = time.perf_counter() - t0
    secs, eps_k = oracle_iterations(opsi, oH, oenvs, eps, k, D)
    sec = float(np.sum(secs))
    value = k / sec
    sample = (f"whole VUMPS iterations 1..{k} of the oracle (NumPy/OpenBLAS, {cpu_threads()} threads) from the "
              f"seeded canonical start (untimed preparation {prep:.0f} s: canonicalisation, environments); "
              f"{args.steps} steps requested, {k} timed: one D={D} iteration is minutes of CPU work")
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": k, "steps_requested": args.steps,
            "warmup": 0, "ms_per_step": sec * 1e3 / k, "iter_s": [round(x, 2) for x in secs],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded PCG64 random MPS, no dataset)", "impl": "reference",
            "config": dict(WORKLOAD, D=D, window=f"VUMPS iterations 1..{k} from the seeded canonical start"),
            "galerkin": eps_k, "prep_s": prep,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu_threads(), "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        res = run_reference(args, world, rank)
        if rank == 0:
            print(json.dumps(res))
        return
    if args.mode == "converge":
        res = run_converge(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if args.mode == "batch":
        res = run_batch(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if args.mode == "tdvp":
        res = run_tdvp(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if args.mode == "kernels":
        res = run_kernels(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if args.mode == "heff":
        res = run_heff(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    res, ctx, psi, envs, H, snap0, eps0 = run_ours(args, world, rank, local)
    if rank == 0 and world == 1 and not args.no_cpu:
        # the oracle's first VUMPS iteration from the very state (and environments)
        # the GPU's timed window starts from: a whole iteration, measured
        import oracle as O
        opsi, oenvs = oracle_from_snapshot(snap0, WORKLOAD["N"])
        oH = O.SchurMPO([O.hubbard_hamiltonian().Ws[0]] * WORKLOAD["N"])
        if args.cpu_full:
            secs, _ = oracle_iterations(opsi, oH, oenvs, eps0, 1, args.D)
            sec, sample = secs[0], (f"VUMPS iteration 1 of the oracle (NumPy/OpenBLAS) at D={args.D} from the "
                                    f"GPU run's seeded canonical start, timed on the host clock ({secs[0]:.1f} s)")
        else:
            sec, sample = oracle_sample(opsi, oH, oenvs, res["op_counts_per_iter"], args.D)
        res["cpu_baseline"] = {"value": 1.0 / sec, "unit": UNIT, "cores": cpu_threads(), "kind": "port",
                               "sample": sample}
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
