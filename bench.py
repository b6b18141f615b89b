"""Benchmark of the CCSD ground-state iteration on B200 (one JSON line on rank 0).

Workload: the synthetic Cholesky-factored CCSD system o=32, v=320, N_J=1200
(seeded generator in et_b200/synthetic.py), MP2 start, quasi-Newton + DIIS(8).
A step is one ground-state iteration: T1-transformed Cholesky vectors, T1 Fock
matrix, energy, Omega, quasi-Newton update and DIIS extrapolation, in mixed
precision refining toward the benchmark's |dE| <= 1e-8 Eh target.

value = seconds per iteration (device time by CUDA events, max over ranks; lower
is better).  "tflops" gives the contraction flops the window performed and eT's
flop count of the same iterations; "e2e" times eT's per-iteration calls through
the C ABI with host buffers; the FP64 GPU paths, the other benchmark
configurations (EOM block Davidson, adjoint check, uneven batch) and the CPU
baseline at the same shape are reported beside it.  Multi-GPU runs are
independent replicas (one system per rank, no collective on the data path).

--impl reference times the CPU restatement of eT's algorithm (oracle/et_cpu.py:
batched A2, numpy/OpenBLAS + C/OpenMP, all host cores) at the benchmark's own
shape, one full iteration per step.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CCSD Omega+Jacobian s/iter & TFLOP/s, mixed vs FP64 on 1 B200 at |dE|<=1e-8 Eh"


def iteration_flops(n_o, n_v, n_J):
    """Algorithmic flops of one ground-state iteration: Omega (eT call sites) + energy + T1 + Fock."""
    o, v, J = float(n_o), float(n_v), float(n_J)
    ov = o * v
    nop, nom, nvp, nvm = o * (o + 1) / 2, o * (o - 1) / 2, v * (v + 1) / 2, v * (v - 1) / 2
    f = 0.0
    f += 2 * J * ov * ov + 2 * v * o * J * v
    f += 2 * ov * o * o * J + 2 * v * o * o * o * v
    f += 2 * ov * ov
    f += 2 * ov * ov * J + 2 * v * v * v * o * o * 2 + 2 * o * o * o * v * v * 2
    f += 2 * ov * ov * J * 2 + 2 * o ** 4 * J + 2 * o ** 4 * v * v * 2
    f += 2 * v * v * o * o * J + 2 * ov * ov * J * 2 + 8 * ov ** 3
    f += v * v * (v * v + 1) * J + 2 * nop * nvp * nvp + 2 * nom * nvm * nvm
    omega = f
    energy = 2 * ov * ov * J                                     # g_ovov for calculate_energy
    t1 = 2 * J * o * o * v * 2 + 2 * J * v * v * o * 2 + 2 * J * o * v * o   # construct_t1_cholesky
    nmo = o + v
    fock = 2 * J * nmo * nmo + 2 * J * o * nmo * nmo + 4 * nmo * nmo * o   # Coulomb, exchange, h~
    return omega + energy + t1 + fock, omega


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            tok = [x.strip() for x in ln.split(",")]
            try:
                sm.append(float(tok[1]))
                mx = float(tok[2])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, tok[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, local, world


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["bf16_tflops"]), float(pk.get("bf16_tflops_sustained", pk["bf16_tflops"])), \
            float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, 1400.0, 6650.0, "fallback"


TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "tc_gemm_bf16x3_c2d2_10240cubed_full.md")


def gemm_traffic(issued_flops_per_launch):
    """DRAM bytes (read + write) of an average tensor-core GEMM launch: the committed single-kernel
    ncu capture's bytes per issued FLOP (10240^3, profiles/) times the launch's issued FLOPs, or None
    when the capture summary is missing."""
    try:
        for line in open(TRAFFIC_PROFILE):
            if line.startswith("dram_bytes_per_issued_pflop:"):
                return float(line.split(":")[1]) * issued_flops_per_launch / 1e15
    except OSError:
        pass
    return None


# arithmetic of the mixed path's FP64 evaluations (refreshes): int8 digits per operand on the tensor
# cores (ozaki_gemm), or -1 for cuBLAS DGEMM; set from --refresh-digits.  Six digits (~2e-13 of an
# operand's row maximum) converge the o=32, v=320 energy to within 2e-12 Eh of the DGEMM solve.
REFRESH_DIGITS = 6


def converged_solve(gpu, stream, refine, thr=1e-9, ethr=1e-11, L=None, refresh_digits=None):
    """From the MP2 start to |Omega| < thr and |dE| < ethr between iterations (certified by an FP64
    evaluation in mixed precision): (seconds by CUDA events, iterations, energy, converged).  With L
    the Cholesky vectors are set again first (untimed), so every integral kept on the device for a
    Cholesky set is formed inside the timed solve, as in a calculation that solves once."""
    import torch
    if L is not None:
        gpu.set_cholesky_mo(L)
    gpu.set_initial_amplitudes_guess()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e, it, _, rc = gpu.solve_ground_state(max_iterations=60, omega_threshold=thr, energy_threshold=ethr,
                                          refine_threshold=refine, raise_on_failure=False,
                                          refresh_digits=REFRESH_DIGITS if refresh_digits is None else refresh_digits)
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / 1e3, it, e, rc == 0


# the accuracy the benchmark solves for: |dE| <= 1e-8 Eh against the converged FP64 energy, reached with
# |Omega| < 1e-6 and |dE| < 1e-8 between iterations; the timed window refines toward that residual
REFINE_TARGET = 1e-6


def timed_solve(gpu, stream, iters, refine, world, clocks_dev=None):
    """Exactly `iters` ground-state iterations from the MP2 start (no early exit), timed with CUDA
    events; mixed precision refines toward a true residual of REFINE_TARGET."""
    import torch
    gpu.set_initial_amplitudes_guess()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(clocks_dev) if clocks_dev is not None else None
    if clk:
        clk.__enter__()
    ev0.record(stream)
    e, it, hist, rc = gpu.solve_ground_state(max_iterations=iters, omega_threshold=1e-30, energy_threshold=-1.0,
                                             refine_threshold=refine, refine_target=REFINE_TARGET,
                                             refresh_digits=REFRESH_DIGITS,
                                             raise_on_failure=False)
    ev1.record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    barrier(world)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), e, it, hist, clk


def run_gpu(args):
    import torch
    from et_b200 import CCSD, FP64, MIXED
    from et_b200.synthetic import make_system

    rank, local, world = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    n_o, n_v, n_J = args.n_o, args.n_v, args.n_J
    sysd = make_system(n_o, n_v, n_J, seed=2026 + rank)
    prec = MIXED if args.precision == "mixed" else FP64
    gpu = CCSD(n_o, n_v, n_J, precision=prec, device=local)
    stream = torch.cuda.current_stream()
    gpu.set_stream(stream.cuda_stream)
    gpu.set_system(sysd.L_mo, sysd.h_mo, sysd.eps, sysd.e_hf)
    flops_iter, flops_omega = iteration_flops(n_o, n_v, n_J)

    # the integrals kept for a Cholesky set (ladder pairs and ovvv planes in split bf16, and the FP64
    # ones of the refinement evaluations) are formed at set-up, outside the timed window; the solves to
    # a threshold below form them inside their timed region
    if prec == MIXED:
        gpu.set_precision(FP64)
        gpu.set_initial_amplitudes_guess()
        gpu.construct_omega()
        gpu.set_precision(MIXED)
    # warm-up iterations, then exactly K timed iterations from the MP2 start
    timed_solve(gpu, stream, args.warmup, args.refine, world)
    launches0, flops0 = gpu.stats()
    gpu.set_profiling(True)
    nvtx_push("gs_window")                 # profilers can restrict a capture to the timed window
    ms, e, it, hist, clk = timed_solve(gpu, stream, args.steps, args.refine, world, clocks_dev=local)
    nvtx_pop()
    n_gemm, gemm_ms, gemm_flops = gpu.gemm_profile()
    gpu.set_profiling(False)
    launches1, flops1 = gpu.stats()
    ms = max_over_ranks(ms, world)
    ms_step = ms / max(it, 1)
    # s/iter is the headline; TFLOP/s two ways: the contraction flops the window performed (2mnk per
    # GEMM issued, every replica), and eT's flop count of the same iterations (which includes the v^4
    # integral build that eT repeats every iteration and this path does once per Cholesky set)
    tflops_performed = world * (flops1 - flops0) / (ms * 1e-3) / 1e12
    tflops_et = world * flops_iter * it / (ms * 1e-3) / 1e12

    # end to end through the public API with host buffers (eT's per-iteration calls):
    # set_amplitudes(host t) -> calculate_energy -> construct_omega(host Omega), the amplitudes and
    # the residual in pinned host arrays that persist across iterations (as eT keeps t and omega)
    t_host = torch.empty(gpu.n_amp, dtype=torch.float64, pin_memory=True).numpy()
    om_host = torch.empty(gpu.n_amp, dtype=torch.float64, pin_memory=True).numpy()
    t_host[:] = gpu.get_amplitudes()
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        gpu.set_amplitudes(t_host)
        gpu.calculate_energy()
        gpu.construct_omega(out=om_host)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, world)

    peak_burst, peak_sust, hbm, peak_kind = load_peaks()
    roof = None
    if n_gemm:
        achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12
        roof = {"kernel": "split_bf16_gemm_kernel (tcgen05 split-BF16 GEMM)", "bound": "tensor",
                "achieved": round(achieved, 2), "peak": peak_sust, "unit": "TFLOP/s",
                "frac": round(achieved / peak_sust, 4), "peak_kind": f"{peak_kind} bf16 sustained (timed inside a long step)",
                "traffic": gemm_traffic(gemm_flops / n_gemm),
                "traffic_source": "DRAM read + write bytes per issued FLOP of the single-launch ncu capture "
                                  "(profiles/tc_gemm_bf16x3_c2d2_10240cubed_full.md) times the window's average "
                                  "issued FLOPs per launch", "launches": n_gemm, "avg_launch_ms": round(gemm_ms / n_gemm, 4),
                "share_of_step": round(gemm_ms / ms, 4),
                "flops_counted": "issued tensor flops: 3 bf16 products x 2mnk per launch"}

    result = {
        "metric": METRIC, "value": round(ms_step / 1e3, 5), "unit": "s/iter", "n_gpus": world, "steps": it,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "s_per_iter": round(ms_step / 1e3, 5),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "tflops": {"performed": round(tflops_performed, 2), "et_equivalent": round(tflops_et, 2),
                   "performed_flops_per_iter": (flops1 - flops0) / max(it, 1), "et_flops_per_iter": flops_iter,
                   "note": "performed: 2mnk of every GEMM the timed window ran (tensor-core and DGEMM); "
                           "et_equivalent: eT's BLAS call-site count of the same iterations, including the "
                           "v^4 N_J ladder-integral build that this path forms once per Cholesky set, "
                           "outside the window"},
        "dtype": "bf16x3+f64" if prec == MIXED else "f64", "data": "synthetic",
        "config": {"workload": f"CCSD ground-state iteration, synthetic Cholesky system o={n_o} v={n_v} N_J={n_J}",
                   "n_o": n_o, "n_v": n_v, "n_J": n_J, "precision": args.precision,
                   "refine_threshold": args.refine, "refine_target": REFINE_TARGET,
                   "refresh_arithmetic": (f"int8 digit GEMM ({REFRESH_DIGITS} digits) for FP64 products of at "
                                          f"least 1e10 flops" if REFRESH_DIGITS > 0 else "cuBLAS DGEMM"),
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": "inputs larger than L2 (t2 419 MB, L 1.19 GB at full size)",
                   "flops_per_iter": flops_iter},
        "clocks": clk.summary() if clk else None,
        "e2e": {"value": round(e2e_s, 5), "unit": "s/iter", "s_per_iter": round(e2e_s, 5),
                "calls": "set_amplitudes (host t) -> calculate_energy -> construct_omega (host Omega): eT's "
                         "per-iteration calls through the C ABI with pinned host buffers kept across iterations",
                "h2d_bytes_per_step": int(8 * gpu.n_amp), "d2h_bytes_per_step": int(8 * gpu.n_amp + 8)},
        "gpu_launches": int(launches1 - launches0),
        "roofline": roof,
        "solve": {"energy": e, "omega_norm": float(hist[-1, 1]) if len(hist) else None,
                  "omega_history": [float(x) for x in hist[:, 1]]},
    }
    if args.compare and world == 1 and prec == MIXED:
        # the plain FP64 GPU path on the same system: per-iteration time and converged energy
        # time to solution from the MP2 start, FP64 path vs mixed path (mixed convergence is certified
        # by an FP64 evaluation).  The reference energy is the tightly converged FP64 one; the target
        # thresholds (|Omega| < 1e-6, |dE| < 1e-8 between iterations) are those that put both paths
        # within 1e-8 Eh of it; the tight ones (1e-9, 1e-11) are reported beside them.
        # Two FP64 paths: eT's algorithm (the T1-transformed ladder integrals formed in every call,
        # omega_ccsd_a2) and the same residual from FP64 integrals of the untransformed vectors kept
        # for the Cholesky set (the algorithm of the mixed path's ladder, in FP64).  Solves to a
        # threshold set the Cholesky vectors again first, so integrals kept for a Cholesky set are
        # formed inside their timed region.
        L = sysd.L_mo
        gpu.set_precision(FP64)
        gpu.set_fp64_integrals(False)
        ms64, _, it64, _, _ = timed_solve(gpu, stream, 3, args.refine, world)
        s64 = ms64 / 1e3 / it64
        t64, n64, e_ref, ok64 = converged_solve(gpu, stream, args.refine, 1e-9, 1e-11)
        t64b, n64b, e64b, ok64b = converged_solve(gpu, stream, args.refine, 1e-6, 1e-8)
        gpu.set_fp64_integrals(True)
        gpu.construct_omega()              # forms the resident integrals before the per-iteration timing
        ms64r, _, it64r, _, _ = timed_solve(gpu, stream, 3, args.refine, world)
        s64r = ms64r / 1e3 / it64r
        t64r, n64r, e64r, ok64r = converged_solve(gpu, stream, args.refine, 1e-9, 1e-11, L=L)
        t64rb, n64rb, e64rb, ok64rb = converged_solve(gpu, stream, args.refine, 1e-6, 1e-8, L=L)
        gpu.set_precision(MIXED)
        tmb, itmb, emb, okmb = converged_solve(gpu, stream, args.refine, 1e-6, 1e-8, L=L)
        tm, itm, em, okm = converged_solve(gpu, stream, args.refine, 1e-9, 1e-11, L=L)
        # attribution: the same mixed solve with its FP64 evaluations on cuBLAS DGEMM
        tmd, itmd, emd, okmd = converged_solve(gpu, stream, args.refine, 1e-6, 1e-8, L=L, refresh_digits=-1)
        result["fp64_path"] = {"algorithm": "T1-transformed ladder integrals formed in every call (eT)",
                               "s_per_iter": round(s64, 5), "energy": e_ref, "converged": ok64,
                               "to_1e-9": {"s": round(t64, 3), "iterations": n64},
                               "to_target": {"s": round(t64b, 3), "iterations": n64b, "converged": ok64b,
                                             "dE": abs(e64b - e_ref)}}
        result["fp64_resident_path"] = {"algorithm": "integrals of the untransformed vectors kept per Cholesky set "
                                                     "+ T1 corrections (the mixed path's algorithm in FP64)",
                                        "s_per_iter": round(s64r, 5), "converged": ok64r,
                                        "dE_vs_fp64": abs(e64r - e_ref),
                                        "to_1e-9": {"s": round(t64r, 3), "iterations": n64r},
                                        "to_target": {"s": round(t64rb, 3), "iterations": n64rb,
                                                      "converged": ok64rb, "dE": abs(e64rb - e_ref)}}
        result["mixed_path"] = {"refresh_arithmetic": (f"int8 digit GEMM, {REFRESH_DIGITS} digits" if REFRESH_DIGITS > 0
                                                       else "cuBLAS DGEMM"),
                                "to_1e-9": {"s": round(tm, 3), "iterations": itm, "converged": okm,
                                            "dE": abs(em - e_ref)},
                                "to_target": {"s": round(tmb, 3), "iterations": itmb, "converged": okmb,
                                              "dE": abs(emb - e_ref)},
                                "to_target_dgemm_refreshes": {"s": round(tmd, 3), "iterations": itmd,
                                                              "converged": okmd, "dE": abs(emd - e_ref)}}
        result["target"] = "|dE| <= 1e-8 Eh vs converged FP64: thresholds |Omega| < 1e-6, |dE| < 1e-8"
        result["speedup_per_iter_vs_fp64"] = round(s64 / (ms_step / 1e3), 3)
        result["speedup_to_target_vs_fp64"] = round(t64b / tmb, 3)
        result["speedup_to_1e-9_vs_fp64"] = round(t64 / tm, 3)
        result["speedup_per_iter_vs_fp64_resident"] = round(s64r / (ms_step / 1e3), 3)
        result["speedup_to_target_vs_fp64_resident"] = round(t64rb / tmb, 3)
        result["speedup_to_1e-9_vs_fp64_resident"] = round(t64r / tm, 3)
        result["dE_vs_fp64"] = abs(emb - e_ref)
        result["dE_window_vs_fp64"] = abs(e - e_ref)
        result["per_call"] = per_call_times(gpu, stream)
        result["fp64_roofline"] = fp64_roofline(result["per_call"], stream)
    gpu.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if args.extras and world == 1 and prec == MIXED:
        # the other benchmark configurations, each on its own contexts after the headline one is closed
        result["workloads"] = {}
        for name, fn in (("eom", eom_summary), ("adjoint", adjoint_summary), ("batch", batch_summary)):
            t0 = time.perf_counter()
            try:
                result["workloads"][name] = fn(args)
            except Exception as ex:                     # reported in the line, never silently dropped
                result["workloads"][name] = {"error": f"{type(ex).__name__}: {ex}"}
            result["workloads"][name]["wall_s"] = round(time.perf_counter() - t0, 1)
    if rank == 0:
        if args.cpu_baseline and world == 1:
            result["cpu_baseline"] = cpu_sample_isolated(args)
        print(json.dumps(result), flush=True)


def dgemm_peak(stream, n=8192, reps=5):
    """cuBLAS DGEMM (torch.mm on FP64 CUDA tensors) at n^3 timed with CUDA events: the FP64
    tensor-pipe denominator of the FP64 rooflines (not in MEASURED_PEAKS.json)."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.empty_like(a)
    torch.mm(a, b, out=c)
    best = min(_event_time(lambda: torch.mm(a, b, out=c), stream) for _ in range(reps))
    del a, b, c
    return 2.0 * n ** 3 / best / 1e12


def fp64_roofline(per_call, stream):
    """The FP64 residual (resident integrals, the mixed path's refresh) against the measured cuBLAS
    DGEMM rate: performed contraction flops of one evaluation over its median time."""
    peak = dgemm_peak(stream)
    fl, t = per_call.get("omega_fp64_resident_flops"), per_call.get("omega_fp64_resident_s")
    out = {"kernel": "FP64 residual evaluation (cuBLAS DGEMM + this library's bandwidth kernels)", "bound": "tensor",
           "peak": round(peak, 2), "peak_kind": "measured cuBLAS DGEMM 8192^3, CUDA events, this run", "unit": "TFLOP/s"}
    if fl and t:
        out.update({"achieved": round(fl / t / 1e12, 2), "frac": round(fl / t / 1e12 / peak, 4)})
    return out


def nvtx_push(name):
    try:
        import torch
        torch.cuda.nvtx.range_push(name)
    except Exception:
        pass


def nvtx_pop():
    try:
        import torch
        torch.cuda.nvtx.range_pop()
    except Exception:
        pass


def per_call_times(gpu, stream):
    """Seconds per residual (construct_omega into a device buffer) and per one-vector Jacobian
    transform at the converged amplitudes: medians of CUDA-event times after one untimed call, mixed
    and both FP64 algorithms."""
    import torch
    from et_b200 import FP64, MIXED
    om = torch.empty(gpu.n_amp, dtype=torch.float64, device="cuda")
    C = 1e-2 * torch.randn(gpu.n_amp, 1, dtype=torch.float64, device="cuda")
    R = torch.empty_like(C)

    def med(fn, n):
        fn()
        ts = sorted(_event_time(fn, stream) for _ in range(n))
        return round(ts[len(ts) // 2], 4)

    omega = lambda: gpu.construct_omega_device(om.data_ptr())
    jac = lambda: gpu.jacobian_device(1, C.data_ptr(), R.data_ptr())
    out = {}
    gpu.set_precision(MIXED)
    out["omega_mixed_s"] = med(omega, 5)
    out["jacobian_mixed_s"] = med(jac, 3)
    gpu.set_precision(FP64)
    gpu.set_fp64_integrals(True)
    out["omega_fp64_resident_s"] = med(omega, 3)
    f0 = gpu.stats()[1]
    omega()
    out["omega_fp64_resident_flops"] = gpu.stats()[1] - f0
    if REFRESH_DIGITS > 0:
        # the same FP64 evaluation with its large products on the int8 digit GEMM (the refreshes)
        gpu.set_fp64_digits(REFRESH_DIGITS)
        out["omega_fp64_resident_digits_s"] = med(omega, 3)
        gpu.set_profiling(True)
        omega()
        n_oz, ms_oz, ops_oz = gpu.digit_gemm_profile()
        gpu.set_profiling(False)
        gpu.set_fp64_digits(0)
        out["digit_gemm_in_one_evaluation"] = {"launches": n_oz, "device_ms": round(ms_oz, 2),
                                               "int8_tops_issued": round(ops_oz / (ms_oz * 1e-3) / 1e12, 1)
                                               if ms_oz else None}
    out["jacobian_fp64_resident_s"] = med(jac, 1)
    gpu.set_fp64_integrals(False)
    out["omega_fp64_s"] = med(omega, 3)
    out["jacobian_fp64_s"] = med(jac, 1)
    gpu.set_fp64_integrals(True)
    gpu.set_precision(MIXED)
    return out


def _event_time(fn, stream):
    import torch
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    fn()
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / 1e3


def run_eom(args):
    print(json.dumps(eom_summary(args)), flush=True)


def eom_summary(args):
    """EOM-CCSD right roots with a batched Davidson block (o=24, v=240, N_J=792, 12 roots, 24 trials)."""
    import torch
    from et_b200 import CCSD, FP64, MIXED
    from et_b200.synthetic import make_system
    n_o, n_v, n_J = 24, 240, 792
    s = make_system(n_o, n_v, n_J, seed=2026)
    stream = torch.cuda.current_stream()
    gpu = CCSD(n_o, n_v, n_J, precision=MIXED)
    gpu.set_stream(stream.cuda_stream)
    gpu.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
    gpu.set_initial_amplitudes_guess()
    e, it, _, rc = gpu.solve_ground_state(max_iterations=60, omega_threshold=1e-9, energy_threshold=1e-10,
                                          raise_on_failure=False)
    out = {"workload": "EOM-CCSD right roots, synthetic o=24 v=240 N_J=792", "gs_energy": e, "gs_iterations": it}
    n = gpu.n_amp
    C = torch.randn(n, 24, dtype=torch.float64, device="cuda")
    R = torch.empty_like(C)
    # untimed: the GEMM routes of the block sizes Davidson uses are measured once per process
    gpu.set_precision(MIXED)
    t0 = time.perf_counter()
    for nvec in range(1, 25):
        gpu.jacobian_device(nvec, C.data_ptr(), R.data_ptr())
    out["untimed_warmup_s"] = round(time.perf_counter() - t0, 2)
    for prec, name in ((MIXED, "mixed"), (FP64, "fp64")):
        gpu.set_precision(prec)
        gpu.jacobian_device(1, C.data_ptr(), R.data_ptr())                     # warm-up
        t1 = min(_event_time(lambda: gpu.jacobian_device(1, C.data_ptr(), R.data_ptr()), stream) for _ in range(2))
        t24 = _event_time(lambda: gpu.jacobian_device(24, C.data_ptr(), R.data_ptr()), stream)
        out[f"s_per_transform_{name}"] = round(t1, 4)
        out[f"s_per_24_block_{name}"] = round(t24, 4)
    nroots = args.roots
    # mixed Davidson to residual 1e-5, then one FP64 Davidson iteration restarted from its vectors: a
    # Rayleigh-Ritz step with FP64 transforms of the mixed eigenvectors.  (Further FP64 Davidson
    # iterations first move these clustered non-symmetric roots away before converging: after two
    # the largest error was 2.3e-7 Eh, after five 1.1e-7, and eleven were needed for 3e-9.)
    gpu.set_precision(MIXED)
    t0 = time.perf_counter()
    w_mix, X, it_mix = gpu.excited_states(nroots, block=24, residual_threshold=1e-5, energy_threshold=1e-7,
                                          vectors=True, max_iterations=60)
    gpu.set_precision(FP64)
    w_ref, _, it_ref = gpu.excited_states(nroots, block=24, residual_threshold=1e-12, energy_threshold=1e-12,
                                          start=X, max_iterations=1, raise_on_failure=False)
    t_mixed_path = time.perf_counter() - t0
    t0 = time.perf_counter()
    w64, _, it64 = gpu.excited_states(nroots, block=24, residual_threshold=1e-6, energy_threshold=1e-8,
                                      max_iterations=60)
    t_fp64_path = time.perf_counter() - t0
    out.update({"roots": nroots, "omega_mixed_refined": list(map(float, w_ref)), "omega_fp64": list(map(float, w64)),
                "max_abs_domega": float(np.max(np.abs(np.sort(w_ref) - np.sort(w64)))),
                "max_abs_domega_mixed_only": float(np.max(np.abs(np.sort(w_mix) - np.sort(w64)))),
                "speedup": round(t_fp64_path / t_mixed_path, 3),
                "davidson_iterations_mixed_then_fp64": [it_mix, it_ref], "davidson_iterations_fp64": it64,
                "s_mixed_plus_refinement": round(t_mixed_path, 2), "s_fp64": round(t_fp64_path, 2),
                "target_met": bool(np.max(np.abs(np.sort(w_ref) - np.sort(w64))) <= 1e-7)})
    gpu.close()
    return out


def run_adjoint(args):
    print(json.dumps(adjoint_summary(args)), flush=True)


def adjoint_summary(args):
    """Adjoint check at o=16, v=128, N_J=432: VJP into (t, L, h) vs central finite differences, and Lambda."""
    from et_b200 import CCSD
    from et_b200.synthetic import make_system
    n_o, n_v, n_J = 16, 128, 432
    s = make_system(n_o, n_v, n_J, seed=2026)
    gpu = CCSD(n_o, n_v, n_J)
    gpu.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
    gpu.set_initial_amplitudes_guess()
    rng = np.random.default_rng(7)
    t = gpu.get_amplitudes()
    t = t * (1.0 + 0.1 * rng.standard_normal(t.size))
    gpu.set_amplitudes(t)
    b = rng.standard_normal(gpu.n_amp)
    b /= np.linalg.norm(b)
    t0 = time.perf_counter()
    dt, dL, dh = gpu.vjp(b, want_L=True, want_h=True)
    t_vjp = time.perf_counter() - t0
    h = 1e-5
    errs = []

    def f(tt, LL, hh):
        gpu.set_cholesky_mo(LL)
        gpu.set_h_mo(hh, s.eps, s.e_hf)
        gpu.set_amplitudes(tt)
        return float(b @ gpu.construct_omega())

    for _ in range(args.directions):
        # unit directions in each block so that h = 1e-5 is a small step
        d_t = rng.standard_normal(t.size)
        d_t /= np.linalg.norm(d_t)
        d_L = rng.standard_normal(s.L_mo.shape)
        d_L = 0.5 * (d_L + d_L.transpose(0, 2, 1))
        d_L /= np.linalg.norm(d_L)
        d_h = rng.standard_normal(s.h_mo.shape)
        d_h /= np.linalg.norm(d_h)
        fd = (f(t + h * d_t, s.L_mo + h * d_L, s.h_mo + h * d_h) -
              f(t - h * d_t, s.L_mo - h * d_L, s.h_mo - h * d_h)) / (2 * h)
        ad = float(dt @ d_t + np.sum(dL * d_L) + np.sum(dh * d_h))
        errs.append(abs(fd - ad) / max(abs(ad), 1e-300))
    # Lambda equations through the adjoint (transpose transformation) at the converged amplitudes
    gpu.set_cholesky_mo(s.L_mo)
    gpu.set_h_mo(s.h_mo, s.eps, s.e_hf)
    gpu.set_initial_amplitudes_guess()
    gpu.solve_ground_state(omega_threshold=1e-9, energy_threshold=1e-11)
    t0 = time.perf_counter()
    tbar, it_l = gpu.solve_multipliers(residual_threshold=1e-8)
    t_lambda = time.perf_counter() - t0
    resid = float(np.linalg.norm(gpu.jacobian_transpose_transformation(tbar) + gpu.construct_eta()))
    gpu.close()
    return {"workload": "adjoint vs central finite differences, synthetic o=16 v=128 N_J=432",
            "directions": args.directions, "h": h, "max_rel_error": max(errs),
            "median_rel_error": float(np.median(errs)), "target_met": bool(max(errs) <= 1e-6),
            "s_vjp_t_L_h": round(t_vjp, 3), "lambda_iterations": it_l, "lambda_residual": resid,
            "s_lambda": round(t_lambda, 2)}


def run_batch(args):
    """64 independent systems o ~ U{6..24}, v = 8o, N_J = 3(o+v), each from its MP2 start to the
    benchmark's target, |dE| <= 1e-8 Eh from the converged FP64 energy (stopping at |Omega| < 5e-7 and
    |dE| < 5e-9 between iterations, the same for every run): systems/s of the concurrent mixed batch
    (ccsd_gpu_solve_gs_batch, --workers contexts in flight) against 64 sequential plain FP64 solves,
    with the two other combinations for attribution, and |dE| against FP64 energies converged to
    |Omega| < 1e-9 (untimed).  The synthetic inputs are generated before the timed region; each
    solve's device set-up (context, H2D of L and h, MP2 guess) is inside it.  One untimed mixed pass
    over the systems comes first, so the GEMM routes of their shapes are measured (once per process)
    before the timed runs; its duration is reported as untimed_warmup_s."""
    rank, local, world = dist_setup(args.gpus)
    out = batch_summary(args, rank, local, world)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batch_summary(args, rank=0, local=0, world=1):
    """The uneven batch (see run_batch) on this process's share of the systems; the summary on rank 0."""
    import torch
    from et_b200 import FP64, MIXED, solve_ground_states
    from et_b200.synthetic import make_system
    torch.cuda.set_device(local)
    rng = np.random.default_rng(2026)
    sizes = [int(o) for o in rng.integers(6, 25, size=args.systems)]
    mine = list(range(rank, args.systems, world))
    systems = []
    for k in mine:
        o = sizes[k]
        s = make_system(o, 8 * o, 3 * (o + 8 * o), seed=2026 + k)
        systems.append((s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf))
    e_ref, _, st_ref, _ = solve_ground_states(systems, precision=FP64, device=local, workers=args.workers,
                                              max_iterations=80, omega_threshold=1e-9, energy_threshold=1e-11)
    # the stopping thresholds of the timed solves (all four runs alike): |Omega| < 1e-6 and |dE| < 1e-8
    # between iterations put energies at ~4e-9 from the converged one, too close to the 1e-8 target when
    # a solve path shifts; half of each keeps every system inside it
    thr, ethr = 5e-7, 5e-9
    # untimed warm-up of the mixed path: the GEMM routes of every shape are timed once per process
    t0 = time.perf_counter()
    solve_ground_states(systems, precision=MIXED, device=local, workers=1, max_iterations=80,
                        omega_threshold=thr, energy_threshold=ethr)
    tune_s = time.perf_counter() - t0
    runs = {}
    for name, prec, workers in (("mixed_batched", MIXED, args.workers), ("fp64_sequential", FP64, 1),
                                ("fp64_batched", FP64, args.workers), ("mixed_sequential", MIXED, 1)):
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        e, it, st, _ = solve_ground_states(systems, precision=prec, device=local, workers=workers,
                                           max_iterations=80, omega_threshold=thr, energy_threshold=ethr)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0, world)
        runs[name] = (dt, e, st)
    de = max_over_ranks(float(np.abs(runs["mixed_batched"][1] - e_ref).max()), world)
    de64 = max_over_ranks(float(np.abs(runs["fp64_sequential"][1] - e_ref).max()), world)
    sps = {name: round(args.systems / r[0], 3) for name, r in runs.items()}
    return {"workload": f"uneven batch of {args.systems} synthetic systems, o~U{{6..24}}, v=8o, N_J=3(o+v)",
            "n_gpus": world, "workers": args.workers, "systems_per_s": sps,
            "untimed_warmup_s": round(tune_s, 3),
            "speedup_vs_sequential_fp64": round(runs["fp64_sequential"][0] / runs["mixed_batched"][0], 3),
            "thresholds": {"omega": thr, "energy": ethr}, "target": "|dE| <= 1e-8 Eh vs FP64 converged to 1e-9",
            "max_abs_dE_mixed": de, "max_abs_dE_fp64": de64, "target_met": bool(de <= 1e-8),
            "all_converged": all(bool((r[2] == 0).all()) for r in runs.values()) and bool((st_ref == 0).all())}


def run_gemm(args):
    """The tensor-core GEMM alone on one shape (default 10240^3, the (ov)^3 C2/D2 product at o=32,
    v=320): per-launch device time from CUDA events around each launch on the launching stream,
    issued tensor TFLOP/s (3 bf16 products x 2mnk) and FP64-equivalent TFLOP/s (2mnk).  The first
    launch (256^3) is a warm-up, so profilers skip one launch."""
    from et_b200 import CCSD
    m, n, k = args.gemm_m, args.gemm_n, args.gemm_k
    digits = args.gemm_digits
    mode = digits if digits else True
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.standard_normal((m, k)))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    with CCSD(2, 3, 4) as ctx:
        ctx.selftest_gemm(A[:256, :256], B[:256, :256], mixed=mode)
        ctx.set_profiling(True)
        for _ in range(args.gemm_reps):
            ctx.selftest_gemm(A, B, mixed=mode)
        nl, ms, fl = ctx.digit_gemm_profile() if digits else ctx.gemm_profile()
    per = ms / max(nl, 1)
    out = {"workload": "tensor-core GEMM", "kernel": "ozaki_gemm_kernel (int8 digits)" if digits else
           "split_bf16_gemm_kernel", "m": m, "n": n, "k": k, "launches": nl, "ms_per_launch": round(per, 4),
           "fp64_equivalent_tflops": round(2.0 * m * n * k / (per * 1e-3) / 1e12, 1)}
    if digits:
        out.update({"digits": digits, "int8_tops_issued": round(fl / nl / (per * 1e-3) / 1e12, 1)})
    else:
        out["issued_tflops"] = round(fl / nl / (per * 1e-3) / 1e12, 1)
    print(json.dumps(out), flush=True)


def host_cpu():
    """(physical cores, model name) of this host."""
    try:
        import psutil
        cores = psutil.cpu_count(logical=False) or os.cpu_count()
    except ImportError:
        cores = os.cpu_count()
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return int(cores), model


def cpu_sample(args, iterations=None):
    """eT's algorithm on the host cores at the benchmark's own shape: the CPU restatement of
    oracle/et_cpu.py (batched A2 ladder formed from the T1-transformed vectors per (a, b) batch pair
    as omega_ccsd_a2 does, every contraction one OpenBLAS call on all cores, eT's OpenMP sorts and
    packing in C).  The synthetic system, its set-up and the MP2 start are untimed; then `iterations`
    quasi-Newton + DIIS iterations are timed on the wall clock (each ~2.9e13 flop at o=32, v=320)."""
    from et_b200.synthetic import make_system
    from oracle import ccsd as oc
    from oracle import et_cpu
    n_o, n_v, n_J = args.n_o, args.n_v, args.n_J
    n_it = int(iterations if iterations is not None else args.cpu_iterations)
    s = make_system(n_o, n_v, n_J, seed=2026)
    sy = et_cpu.ETSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    sy.mp2_start()
    hist = []
    t0 = time.perf_counter()
    oc.solve_gs(sy, max_iterations=n_it, omega_threshold=0.0, energy_threshold=-1.0, history=hist)
    dt = (time.perf_counter() - t0) / n_it
    fl, _ = iteration_flops(n_o, n_v, n_J)
    cores, model = host_cpu()
    return {"value": round(dt, 3), "unit": "s/iter", "cores": cores, "kind": "port", "cpu_model": model,
            "iterations_timed": n_it, "tflops_et_equivalent": round(fl / dt / 1e12, 4),
            "energy_first_iteration": hist[0][0] if hist else None,
            "sample": f"{n_it} ground-state iteration(s) from the MP2 start of the CPU restatement of eT's "
                      f"algorithm (oracle/et_cpu.py: batched A2, numpy/OpenBLAS + C/OpenMP, all {cores} "
                      f"cores) at the benchmark's own shape o={n_o} v={n_v} N_J={n_J}"}


def cpu_sample_isolated(args, iterations=None, timeout_s=900):
    """cpu_sample in a child process of its own: one OpenMP/OpenBLAS pool sized to the CPUs this
    process may run on (no CUDA runtime, torch threads or GPU-side work beside it), threads that
    sleep instead of spinning when idle, and a bound on the wall time.  A sample that runs out of
    time is reported as such instead of holding the benchmark."""
    try:
        ncpu = len(os.sched_getaffinity(0))
    except AttributeError:
        ncpu = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(ncpu), OPENBLAS_NUM_THREADS=str(ncpu), OMP_WAIT_POLICY="PASSIVE")
    spec = {"n_o": args.n_o, "n_v": args.n_v, "n_J": args.n_J, "cpu_iterations": args.cpu_iterations,
            "iterations": iterations}
    code = ("import json, sys, types; sys.path.insert(0, '.'); import bench; "
            "a = json.loads(sys.argv[1]); it = a.pop('iterations'); "
            "print(json.dumps(bench.cpu_sample(types.SimpleNamespace(**a), it)))")
    root = os.path.dirname(os.path.abspath(__file__))
    try:
        r = subprocess.run([sys.executable, "-c", code, json.dumps(spec)], env=env, cwd=root, capture_output=True,
                           text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        cores, model = host_cpu()
        return {"value": None, "unit": "s/iter", "cores": cores, "kind": "port", "cpu_model": model,
                "iterations_timed": 0, "sample": f"timed out after {timeout_s} s (one iteration of the CPU "
                                                   f"restatement at o={args.n_o} v={args.n_v} N_J={args.n_J})"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        raise RuntimeError("CPU baseline failed: " + r.stderr[-2000:])
    return json.loads(lines[-1])


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_sample_isolated(args)
    line = {"metric": METRIC, "value": cb["value"], "unit": "s/iter", "n_gpus": 0,
            "steps": cb["iterations_timed"], "warmup": 0, "requested_steps": args.steps,
            "requested_warmup": args.warmup,
            "ms_per_step": round(cb["value"] * 1e3, 1) if cb["value"] is not None else None,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"CCSD ground-state iteration, synthetic Cholesky system o={args.n_o} "
                                   f"v={args.n_v} N_J={args.n_J}", "n_o": args.n_o, "n_v": args.n_v,
                       "n_J": args.n_J,
                       "timing": "each step is one full iteration (~2.9e13 flop); the MP2 start is untimed and "
                                 "stands in for the warm-up, so steps = the iterations actually timed"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=15)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="gs", choices=["gs", "eom", "adjoint", "batch", "gemm"],
                   help="gs: the headline ground-state iteration; eom / adjoint / batch: the other workloads; "
                        "gemm: the tensor-core GEMM alone on one shape")
    p.add_argument("--gemm-m", dest="gemm_m", type=int, default=10240)
    p.add_argument("--gemm-n", dest="gemm_n", type=int, default=10240)
    p.add_argument("--gemm-k", dest="gemm_k", type=int, default=10240)
    p.add_argument("--gemm-reps", dest="gemm_reps", type=int, default=3)
    p.add_argument("--gemm-digits", dest="gemm_digits", type=int, default=0,
                   help="gemm workload: 4..7 = the FP64-accurate int8 digit GEMM, 0 = the split-BF16 GEMM")
    p.add_argument("--roots", type=int, default=12)
    p.add_argument("--directions", type=int, default=256)
    p.add_argument("--systems", type=int, default=64)
    p.add_argument("--workers", type=int, default=8, help="batch workload: systems in flight")
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--refine", type=float, default=1e-4)
    p.add_argument("--no-compare", dest="compare", action="store_false",
                   help="skip the FP64-path comparison (per-iteration time and converged energy)")
    p.add_argument("--n-o", dest="n_o", type=int, default=32)
    p.add_argument("--n-v", dest="n_v", type=int, default=320)
    p.add_argument("--n-J", dest="n_J", type=int, default=1200)
    p.add_argument("--cpu-iterations", dest="cpu_iterations", type=int, default=1,
                   help="ground-state iterations the CPU baseline times at the benchmark shape")
    p.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    p.add_argument("--refresh-digits", dest="refresh_digits", type=int, default=6,
                   help="mixed path: int8 digits of the FP64 evaluations (4..7), -1 = cuBLAS DGEMM")
    p.add_argument("--no-extras", dest="extras", action="store_false",
                   help="skip the EOM, adjoint and uneven-batch workloads in the default line")
    args = p.parse_args()
    global REFRESH_DIGITS
    REFRESH_DIGITS = args.refresh_digits
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "eom":
        run_eom(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "gemm":
        run_gemm(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
