"""Benchmark of the Wstat response operator: dvg -> drho applications per second.

Workload (one "step"): one apply_operator call on 64 perturbations of the
L = 20 bohr, 25 Ry Gamma system (npw 8,440, 64^3 FFT box, 8 Gaussian
pseudo-atoms with s+p Kleinman-Bylander projectors, 32 occupied bands),
seeded complex-normal perturbations scaled by 4 pi / |G|^2, PCG threshold
tr2 = 1e-10, FP64.  Synthetic inputs; the ground state comes from an exact
diagonalisation of the same Hamiltonian.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on stdout (rank 0).  Under torchrun every rank applies its own
64 perturbations (weak scaling, no collective on the data path); the time is
the max over ranks.
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

WORKLOAD = "c2"
M_PERT = 64
TR2 = 1e-10
METRIC = "dvg->drho applications/s (apply_operator, FP64)"
UNIT = "applications/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--m", type=int, default=M_PERT)
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-sample", type=int, default=1, help="perturbations in the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pdep", action="store_true", help="skip the time-to-PDEP Davidson run")
    ap.add_argument("--no-multi", action="store_true", help="skip the three-system uneven batch")
    ap.add_argument("--large-davidson", action="store_true",
                    help="only the 108^3 PDEP Davidson (n_pdep_eigen 256 x 4), FP64 and mixed: one JSON line")
    ap.add_argument("--no-large-pdep", action="store_true",
                    help="skip the 108^3 PDEP Davidson of the default run (about two minutes)")
    ap.add_argument("--trev", type=float, default=1e-6, help="trev_pdep of --large-davidson")
    ap.add_argument("--tr2-dfpt", type=float, default=TR2, help="tr2_dfpt of --large-davidson")
    ap.add_argument("--n-pdep-eigen", type=int, default=256, help="n_pdep_eigen of --large-davidson")
    return ap.parse_args()


def _config(args, extra=None):
    from west_b200.system import SPECS
    sp = SPECS[args.workload]
    cfg = {"workload": f"apply_operator {args.workload}: L={sp.L:g} bohr, ecutwfc={sp.ecutwfc:g} Ry, "
                       f"{sp.nr}^3 FFT, {sp.natoms} atoms ({sp.proj}), nbnd_occ={sp.nbnd_occ}, "
                       f"m={args.m} perturbations, tr2={TR2:g}",
           "m_per_rank": args.m, "tr2": TR2, "n_dfpt_maxiter": 250, "precision": "fp64",
           "l2": "working set per step >> 126 MB L2 (PCG vectors and stick buffers, GBs)"}
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.skip = 0
        self.end = None
        self._t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            # nvidia-smi's start-up (NVML initialisation) must not overlap the timed
            # region: wait for its first sample, then keep only the later ones
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10.0:
                time.sleep(0.01)
            self.skip = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        lines = self.lines[self.skip:self.end] or self.lines[self.skip:] or self.lines
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def _fp64_gemm_peak(torch):
    """FP64 DGEMM throughput of this GPU (cuBLAS, 8192^3), TFLOP/s, best of 3."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(); torch.matmul(a, b); e1.record(); torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def _cpu_baseline(system, m_sample, seed):
    """The oracle (CPU restatement of WEST's algorithm) on a bounded sample."""
    from oracle import west_oracle as O
    from west_b200.system import perturbations
    dvg = perturbations(system, m_sample, seed=seed)
    t0 = time.perf_counter()
    O.apply_operator(system, dvg, TR2)
    dt = time.perf_counter() - t0
    return {"value": m_sample / dt, "unit": UNIT, "cores": O._WORKERS, "kind": "port",
            "sample": f"{m_sample} perturbation(s) of the same workload through the NumPy/SciPy FP64 oracle "
                      f"(scipy.fft workers={O._WORKERS}, BLAS threads default), {dt:.1f} s"}


def _build_system(name, device):
    from west_b200.system import build_system
    return build_system(name, device=device)


def run_reference(args, rank, world):
    """--impl reference: the CPU restatement of WEST's apply_operator, timed on the host cores."""
    if rank != 0:
        return None
    import torch
    from oracle import west_oracle as O
    from west_b200.system import perturbations
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    s = _build_system(args.workload, dev)           # ground-state synthesis only
    m = max(1, args.cpu_sample)
    times = []
    for it in range(args.warmup + args.steps):
        dvg = perturbations(s, m, seed=1000 + it)
        t0 = time.perf_counter()
        O.apply_operator(s, dvg, TR2)
        if it >= args.warmup:
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = m * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": _config(args, {"reference_sample_m": m}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O._WORKERS, "kind": "port",
                             "sample": f"{m} perturbation(s) per step through the NumPy/SciPy FP64 restatement "
                                       f"of WEST's apply_operator (the Fortran reference cannot be built here)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from west_b200.system import perturbations
    from west_b200.wstat import ResponseOperator

    torch.cuda.set_device(local_rank)
    t0 = time.time()
    s = _build_system(args.workload, "cuda")
    t_sys = time.time() - t0
    m = args.m
    op = ResponseOperator(s, device=local_rank, verbose=False)
    npw = s.npw
    # one global batch of m * world perturbations, cyclically sharded over the
    # ranks as WEST shards them over images (weak scaling: m per rank)
    from west_b200.distribute import PertDistribution
    dist_p = PertDistribution(m * world, world, rank)
    dvg_h = np.asfortranarray(perturbations(s, m * world, seed=1234)[:, dist_p.local_columns()])
    dvg_d = torch.from_numpy(np.ascontiguousarray(dvg_h.T)).cuda()      # [m, npw] = Fortran [npw, m]
    dng_d = torch.zeros_like(dvg_d)
    dvg_p = torch.from_numpy(np.ascontiguousarray(dvg_h.T)).pin_memory()
    dng_p = torch.zeros_like(dvg_p).pin_memory()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the clock sampler starts before the warm-up: its start-up leaves the GPU
    # idle for up to a second, which must not precede the first timed step
    clk = ClockSampler(local_rank).__enter__()
    # warm-up (also settles the device workspace), then further untimed steps
    # until two in a row agree within 3% (at most 12): steps right after the GPU
    # idled, or after an nvidia-smi process started, ran 10-50% slower
    def one_step_ms():
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(); op.apply_operator(m, dvg_d, dng_d, TR2); e1.record(); torch.cuda.synchronize()
        return e0.elapsed_time(e1)
    prev = None
    for _ in range(args.warmup):
        prev = one_step_ms()
    settle = 0
    while settle < 12:
        cur = one_step_ms()
        settle += 1
        if prev is not None and abs(cur - prev) <= 0.03 * prev:
            break
        prev = cur
    settle = max_over_ranks(settle) if world > 1 else settle
    torch.cuda.synchronize()

    # timed region: inputs resident in HBM, the library's default path (each
    # call's PCG loop is one CUDA-graph launch), no stage events
    launches = 0
    iters, act_sum, boxes = [], 0, 0
    barrier(); torch.cuda.synchronize()
    clk.skip = len(clk.lines)  # clock samples of the timed region only
    try:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev[0].record()
        for i in range(args.steps):
            ierr = op.apply_operator(m, dvg_d, dng_d, TR2)
            ev[i + 1].record()
            st = op.stats()
            launches += st["launches"]
            iters.append(st["cg_iterations"]); act_sum += st["cg_active_sum"]; boxes += st["fft_boxes"]
        torch.cuda.synchronize()
        barrier()
        clk.end = len(clk.lines)
    finally:
        clk.__exit__(None, None, None)
    ms = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    step_ms = [round(ev[i].elapsed_time(ev[i + 1]), 2) for i in range(args.steps)]
    # roofline: the same steps with CUDA events on the library stream around the
    # dominant stage (the local-potential FFT); events need the eager loop, and
    # cost 2-5% of a step, so they stay out of the timed region above
    op.set_profiling(["vloc_zinv", "vloc_plane", "vloc_zfwd"])
    stage_tot = {}
    ms_eager = _timed_steps(op, m, dvg_d, dng_d, args, barrier, max_over_ranks, warmup=1, stage_tot=stage_tot)
    # one extra untimed step with every stage timed, for the stage shares
    op.set_profiling("all")
    op.apply_operator(m, dvg_d, dng_d, TR2)
    share_stats = op.stats()["stages"]
    op.set_profiling(None)
    value = world * m * args.steps / (ms * 1e-3)
    dng_val = dng_d.cpu().numpy().T.copy()

    # end-to-end through the host-pointer entry point, pinned host buffers
    dvg_np = dvg_p.numpy().T      # Fortran-ordered view of pinned memory
    dng_np = dng_p.numpy().T
    op.apply_operator(m, dvg_np, dng_np, TR2)   # untimed: sizes the host staging buffers
    barrier(); torch.cuda.synchronize()
    t_e2e0 = time.perf_counter()
    e2e_marks, e2e_lib = [], []
    for _ in range(args.steps):
        op.apply_operator(m, dvg_np, dng_np, TR2)
        e2e_marks.append(time.perf_counter())
        e2e_lib.append(round(op.stats()["ms_total"], 2))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t_e2e0)
    e2e_steps = [round(1e3 * (b - a), 2) for a, b in zip([t_e2e0] + e2e_marks[:-1], e2e_marks)]
    barrier()
    e2e_val = world * m * args.steps / e2e_s
    e2e_ok = bool(np.allclose(dng_np, dng_val, rtol=0, atol=1e-12 * np.abs(dng_val).max()))

    line = None
    if rank == 0:
        peaks = _measured_peaks()
        hbm = peaks.get("hbm_gbs", 6650.0)
        fp64_peak = _fp64_gemm_peak(torch)
        N = s.nr
        # dominant stage: the local-potential FFT (zinv + plane + zfwd = 2 box FFTs per item)
        vz = [stage_tot[k] for k in ("vloc_zinv", "vloc_plane", "vloc_zfwd")]
        items = vz[1]["items"]; nl = max(1, vz[1]["launches"])
        t_ms = sum(v["ms"] for v in vz)
        alg_bytes = 2.0 * items * 2.0 * N ** 3 * 16.0           # B_fft = 2 N^3 s per FFT, 2 FFTs per item
        per_launch_bytes = alg_bytes / nl
        per_launch_s = t_ms * 1e-3 / nl
        achieved = per_launch_bytes / per_launch_s / 1e9
        flops = 2.0 * items * 5.0 * N ** 3 * math.log2(N ** 3)  # nominal radix-2 count, full box
        fp64_ach = flops / (t_ms * 1e-3) / 1e12
        traffic = _profiled_traffic(items / nl)
        steps_ms = ms / args.steps
        stage_share = {k: round(v["ms"] / max(1e-9, sum(x["ms"] for x in share_stats.values())), 4)
                       for k, v in share_stats.items()}
        # in-place rates of the FP64 projector GEMMs (stage timers of the profiled step):
        # 2 M K flops per active system, M = nkb + nbnd_occ, K = 2 npw real rows
        gemm_rates = {}
        for k in ("gemm_tn", "gemm_nn"):
            v = share_stats.get(k)
            if v and v["ms"] > 0:
                tf = 2.0 * (s.nkb + s.nbnd_occ) * 2 * npw * v["items"] / (v["ms"] * 1e-3) / 1e12
                gemm_rates[k] = {"tflops": tf, "frac_of_dgemm": tf / fp64_peak, "systems": int(v["items"]),
                                 "ms": v["ms"]}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": steps_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian pseudo-atoms, exact ground state)",
            "config": _config(args, {"parallelism": f"perturbation shards x{world}", "npw": npw,
                                     "cg_iterations": iters, "system_build_s": round(t_sys, 1),
                                     "step_ms": step_ms, "settle_steps": int(settle)}),
            "clocks": clk.summary(),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(m * npw * 16),
                    "d2h_bytes_per_step": int(m * npw * 16), "matches_device_path": e2e_ok,
                    "step_ms": e2e_steps, "library_ms": e2e_lib},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "vloc FFT stage (k_zinv + k_plane_vloc + k_zfwd), per launch",
                         "timed_over": f"{args.steps} steps of the same workload right after the timed region, "
                                       "CUDA events on the library stream around the stage",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                         "algorithmic_bytes_per_launch": per_launch_bytes,
                         "fp64": {"achieved_tflops_nominal": fp64_ach, "dgemm_peak_tflops": fp64_peak,
                                  "frac": fp64_ach / fp64_peak}},
            "stage_share": stage_share,
            "gemm_fp64": dict(gemm_rates, note="bra-ket (k_gemm_tn, DMMA, split K) and update (k_gemm_nn) "
                                                "in the PCG operator, against the measured cuBLAS DGEMM"),
            "work": {"cg_active_sum": act_sum, "fft_boxes": boxes},
            "eager_profiled": {"value": world * m * args.steps / (ms_eager * 1e-3), "unit": UNIT,
                               "ms_per_step": ms_eager / args.steps,
                               "note": "the roofline steps: eager PCG loop with CUDA events around the vloc "
                                       "stages; the headline value times the graph-launched loop without events"},
        }
        if not args.no_pdep:
            line["time_to_pdep"] = _time_to_pdep(local_rank, "fp64")
    # the mixed form on the same inputs: throughput and its dng error against FP64
    op.set_precision("mixed")
    ms_mixed = _timed_steps(op, m, dvg_d, dng_d, args, barrier, max_over_ranks)
    st_mixed = op.stats()
    dng_mixed = dng_d.cpu().numpy().T
    err_mixed = float(np.linalg.norm(dng_mixed - dng_val) / np.linalg.norm(dng_val))
    op.set_profiling("all")
    op.apply_operator(m, dvg_d, dng_d, TR2)
    mixed_stages = op.stats()["stages"]
    op.set_profiling(None)
    op.set_precision("fp64")
    if rank == 0:
        v_mixed = world * m * args.steps / (ms_mixed * 1e-3)
        line["mixed"] = {"value": v_mixed, "unit": UNIT, "ms_per_step": ms_mixed / args.steps,
                         "speedup_vs_fp64": v_mixed / value, "dng_rel_err_vs_fp64": err_mixed,
                         "refinements": st_mixed["refinements"], "inner_iterations": st_mixed["cg_iterations"],
                         "stage_share": {k: round(v["ms"] / max(1e-9, sum(x["ms"] for x in mixed_stages.values())), 4)
                                         for k, v in mixed_stages.items()},
                         "precision": "FP32 PCG corrections + FP32 FFTs and projector GEMMs, FP64 refinement"}
        if not args.no_pdep:
            line["mixed"]["time_to_pdep"] = _time_to_pdep(local_rank, "mixed")
    del op
    if rank == 0 and world == 1 and not args.no_multi:
        for key, fn in (("batched_uneven", _batched_uneven), ("large_cell", _large_cell)):
            try:
                line[key] = fn(local_rank, args)
            except Exception as e:  # a failed side measurement must not lose the headline line
                line[key] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
    if rank == 0 and world == 1 and not args.no_large_pdep:
        try:
            ld = _large_davidson(args, local_rank)
            line["large_cell_pdep"] = {k: ld[k] for k in ("config", "fp64", "mixed", "mixed_vs_fp64", "clocks")}
        except Exception as e:
            line["large_cell_pdep"] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
    # the CPU baseline last: its BLAS and FFT worker threads keep spinning on the
    # host cores for a while after each call, which slowed the latency-bound
    # Davidson host loop measured right after it (warm c1 runs of 0.06-0.32 s)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_baseline(s, args.cpu_sample, seed=77)
    return line


def _timed_steps(op, m, dvg_d, dng_d, args, barrier, max_over_ranks, warmup=None, stage_tot=None):
    """Warm-up then args.steps calls, CUDA events around them; ms (max over ranks).
    stage_tot, if given, accumulates the library's per-stage times of the timed calls."""
    import torch
    for _ in range(args.warmup if warmup is None else warmup):
        op.apply_operator(m, dvg_d, dng_d, TR2)
    barrier(); torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True); f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        op.apply_operator(m, dvg_d, dng_d, TR2)
        if stage_tot is not None:
            for k, v in op.stats()["stages"].items():
                a = stage_tot.setdefault(k, {"ms": 0.0, "launches": 0, "items": 0})
                a["ms"] += v["ms"]; a["launches"] += v["launches"]; a["items"] += v["items"]
    f1.record(); torch.cuda.synchronize()
    return max_over_ranks(f0.elapsed_time(f1))


def _large_cell(device, args):
    """The L = 30 bohr, 30 Ry, 108^3 cell (npw 37,387, 20 atoms s+p, nbnd_occ 128):
    apply_operator on 16 perturbations (2,048 Sternheimer systems), FP64 and mixed."""
    import torch
    from west_b200.system import build_system, perturbations
    from west_b200.wstat import ResponseOperator
    t0 = time.time()
    s = build_system("c5", device="cuda")
    t_sys = time.time() - t0
    m = 16
    op = ResponseOperator(s, device=device, verbose=False)
    d = torch.from_numpy(np.ascontiguousarray(perturbations(s, m, seed=1234).T)).cuda()
    out = {}
    res = {}
    steps = 2
    for prec in ("fp64", "mixed"):
        op.set_precision(prec)
        o = torch.zeros_like(d)
        ierr = op.apply_operator(m, d, o, TR2)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True); f1 = torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(steps):
            ierr = op.apply_operator(m, d, o, TR2)
        f1.record(); torch.cuda.synchronize()
        st = op.stats()
        res[prec] = o
        out[prec] = {"value": m * steps / (f0.elapsed_time(f1) * 1e-3), "cg_iterations": st["cg_iterations"],
                     "refinements": st["refinements"], "unconverged": int(np.count_nonzero(ierr))}
    err = float(torch.linalg.norm(res["mixed"] - res["fp64"]) / torch.linalg.norm(res["fp64"]))
    return {"workload": "apply_operator c5: L=30 bohr, ecutwfc=30 Ry, 108^3 FFT, 20 atoms (sp), nbnd_occ=128, "
                        "m=16 perturbations, tr2=1e-10",
            "unit": UNIT, "npw": int(s.npw), "steps": steps, "system_build_s": round(t_sys, 1),
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_speedup_vs_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "dng_rel_err_mixed_vs_fp64": err,
            "ground_state": "matrix-free block LOBPCG on the GPU (lowest 132 bands, residual < 1e-9)"}


def _batched_uneven(device, args):
    """Three ground states of uneven size in one wb_apply_operator_multi call, mixed
    form: L = 15/20/25 bohr, 48^3/64^3/80^3, nbnd_occ 8/32/64, 64/128/64
    perturbations (256 applications per step), against the same three calls
    made one after another."""
    import torch
    from west_b200.system import build_system, perturbations
    from west_b200.wstat import ResponseOperator, apply_operator_multi
    names, ms = ("c4a", "c4b", "c4c"), (64, 128, 64)
    t0 = time.time()
    systems = [build_system(n, device="cuda") for n in names]
    t_sys = time.time() - t0
    ops = [ResponseOperator(s, device=device, verbose=False) for s in systems]
    for op in ops:
        op.set_precision("mixed")
    dvgs = [torch.from_numpy(np.ascontiguousarray(perturbations(s, m, seed=1234 + i).T)).cuda()
            for i, (s, m) in enumerate(zip(systems, ms))]
    dngs = [torch.zeros_like(d) for d in dvgs]
    steps = max(1, min(args.steps, 3))

    def multi():
        apply_operator_multi(ops, dvgs, dngs, TR2)

    def sequential():
        for op, d, o, m in zip(ops, dvgs, dngs, ms):
            op.apply_operator(m, d, o, TR2)

    out = {}
    for name, fn in (("multi", multi), ("sequential", sequential)):
        fn()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(steps):
            fn()
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - w0) / steps
    napp = sum(ms)
    # the reference's order: one perturbation per call (dfpt_module.f90:227 loops over
    # perturbations), timed on a sample of 4 per system and scaled to all of them
    nsample = 4
    t_one = 0.0
    for op, d, o, m in zip(ops, dvgs, dngs, ms):
        op.apply_operator(1, d[:1], o[:1], TR2)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for j in range(nsample):
            op.apply_operator(1, d[j:j + 1], o[j:j + 1], TR2)
        torch.cuda.synchronize()
        t_one += (time.perf_counter() - w0) / nsample * m
    return {"workload": "c4 mixed: L=15/20/25 bohr, 48^3/64^3/80^3, nbnd_occ=8/32/64, m=64/128/64 "
                        "(256 perturbations), tr2=1e-10, one wb_apply_operator_multi call per step",
            "value": napp / out["multi"], "unit": UNIT, "ms_per_step": 1e3 * out["multi"],
            "sequential_value": napp / out["sequential"], "speedup_vs_sequential": out["sequential"] / out["multi"],
            "per_perturbation_value": napp / t_one, "speedup_vs_per_perturbation": t_one / out["multi"],
            "per_perturbation_sample": f"{nsample} single-perturbation calls per system, scaled to its m",
            "npw": [int(s.npw) for s in systems], "steps": steps, "system_build_s": round(t_sys, 1),
            "cg_iterations": [op.stats()["cg_iterations"] for op in ops],
            "timing": "host wall clock around the synchronous call (several library streams)"}


def _time_to_pdep(device, precision):
    """Wstat time-to-PDEP on the L = 15 bohr, 20 Ry, 48^3 system: n_pdep_eigen 16,
    n_pdep_times 4, PCG threshold 1e-10, Davidson tolerance 1e-6."""
    from west_b200.system import build_system, randomized_basis
    from west_b200.wstat import ResponseOperator
    s = build_system("c1", device="cuda")
    op = ResponseOperator(s, device=device, verbose=False)
    op.set_precision(precision)
    dvg0 = randomized_basis(s, 16)
    runs = []
    for _ in range(10):  # cold (first use: autotuning, graph capture, kernel loading), then 9 warm
        ev, conv, _, info = op.davidson(dvg0, 16, n_pdep_times=4, n_pdep_maxiter=100, tr2_dfpt=1e-10,
                                        trev_pdep=1e-6, trev_pdep_rel=1e-1)
        runs.append(info)
    info = runs[0]
    warm = [r["seconds"] for r in runs[1:]]
    return {"workload": "Davidson c1: L=15 bohr, 20 Ry, 48^3, 4 atoms (s), nbnd_occ=8, n_pdep_eigen=16, "
                        f"n_pdep_times=4, tr2_dfpt=1e-10, trev_pdep=1e-6, {precision}",
            "seconds": info["seconds"], "seconds_warm": float(np.median(warm)), "seconds_warm_runs": warm,
            "seconds_warm_apply": [round(r["seconds_apply"], 4) for r in runs[1:]],
            "dav_iter": info["dav_iter"],
            "converged": bool(info["converged"]), "perturbations_applied": info["perturbations"],
            "ev": [float(x) for x in ev]}


def _large_davidson(args, device):
    """Wstat time-to-PDEP on the large cell: L = 30 bohr, 30 Ry, 108^3, 20 atoms (s+p),
    nbnd_occ 128, n_pdep_eigen 256 x n_pdep_times 4 (basis 1024), PCG threshold
    tr2_dfpt, Davidson tolerance trev_pdep; FP64 then mixed from the same
    starting basis, with the largest relative eigenvalue difference."""
    import torch
    from west_b200.system import build_system, randomized_basis
    from west_b200.wstat import ResponseOperator
    t0 = time.time()
    s = build_system("c5", device="cuda")
    t_sys = time.time() - t0
    nvec = args.n_pdep_eigen
    dvg0 = randomized_basis(s, nvec)
    out = {"metric": "Wstat time-to-PDEP (s), 108^3 large cell", "unit": "s", "higher_is_better": False,
           "n_gpus": 1, "dtype": "f64 / mixed", "data": "synthetic (seeded Gaussian pseudo-atoms, LOBPCG ground state)",
           "config": {"workload": f"Davidson c5: L=30 bohr, 30 Ry, 108^3, 20 atoms (sp), nbnd_occ=128, npw={s.npw}, "
                                  f"n_pdep_eigen={nvec}, n_pdep_times=4, tr2_dfpt={args.tr2_dfpt:g}, "
                                  f"trev_pdep={args.trev:g}, trev_pdep_rel=0.1",
                      "system_build_s": round(t_sys, 1)}}
    evs = {}
    with ClockSampler(device) as clk:
        for prec in ("fp64", "mixed"):
            op = ResponseOperator(s, device=device, verbose=False)
            op.set_precision(prec)
            torch.cuda.synchronize()
            ev, conv, _, info = op.davidson(dvg0, nvec, n_pdep_times=4, n_pdep_maxiter=100, tr2_dfpt=args.tr2_dfpt,
                                            trev_pdep=args.trev, trev_pdep_rel=1e-1)
            evs[prec] = ev
            out[prec] = {"seconds": info["seconds"], "seconds_apply": info["seconds_apply"],
                         "dav_iter": info["dav_iter"], "converged": bool(info["converged"]),
                         "notcnv": info["notcnv"], "apply_calls": info["apply_calls"],
                         "perturbations_applied": info["perturbations"],
                         "ev_lowest": [float(x) for x in ev[:4]], "ev_highest": [float(x) for x in ev[-4:]]}
            op.close()
        clk.end = len(clk.lines)
    rel = np.abs((evs["mixed"] - evs["fp64"]) / evs["fp64"])
    out["mixed_vs_fp64"] = {"speedup": out["fp64"]["seconds"] / out["mixed"]["seconds"],
                            "ev_max_rel_diff": float(rel.max()), "ev_median_rel_diff": float(np.median(rel)),
                            "ev_max_abs_diff": float(np.abs(evs["mixed"] - evs["fp64"]).max())}
    out["value"] = out["fp64"]["seconds"]
    out["clocks"] = clk.summary()
    return out


def main():
    args = _args()
    if args.large_davidson:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(_large_davidson(args, 0)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_b200(args, rank, world, local_rank)
        if line is not None and rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


def _profiled_traffic(items_per_launch):
    """DRAM bytes per launch of the vloc FFT stage: the per-item traffic of the
    committed 1-pass ncu capture (profiles/vloc_fft_traffic.json) times the
    items per launch of this run; None if the summary is missing."""
    p = os.path.join(ROOT, "profiles", "vloc_fft_traffic.json")
    try:
        return json.load(open(p))["dram_bytes_per_item_fp64"] * items_per_launch
    except Exception:
        return None


if __name__ == "__main__":
    main()
