#!/usr/bin/env python
"""Benchmark of the FMM matvec hot path (PBBFMM3D's H2_3D_Compute) on B200.

Metric: N * nCols / s of one forward matvec (binning included, operator
precompute excluded), stated with its rel-L2 error against the float64 direct
sum on 4096 seeded sampled targets.

Workload (the configuration the metric is quoted on): exponential covariance
K = exp(-r/0.3), N = 1,000,000 points uniform in the unit cube (sources =
targets), nCols = 8 weights N(0,1), tree_level 6, uniform interpolation order
5 with FFT M2L (use_chebyshev = 0).  Synthetic seeded data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Multi-GPU (torchrun): every rank runs its own
matvec over its own block of 8 right-hand sides on the same points (columns
are independent; no data-path collective), weak scaling, value = all ranks'
N*nCols / max-over-ranks time.  ``--impl reference`` times the reference's own
CPU code (oracle/_ref, built from the reference sources) on a bounded sample of
the same workload with every host core.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the configuration the metric is quoted on
    "bench": dict(name="expcov0.3_unif5_N1e6_C8_L6", kernel="ExpCov", ell=0.3, N=1_000_000, C=8,
                  L=6, n=5, cheb=0, eps=1e-5, box=1.0, seed=1234),
    # small case of the same kernels for ncu captures (~4.5 GB on the device)
    "profile": dict(name="expcov0.3_unif5_N262144_C8_L5", kernel="ExpCov", ell=0.3, N=262_144,
                    C=8, L=5, n=5, cheb=0, eps=1e-5, box=1.0, seed=1234),
}
WORKLOAD = WORKLOADS["bench"]
# bounded CPU sample: same kernel, order, columns and points per leaf (N / 8^L)
CPU_SAMPLE = dict(N=15_625, L=4)
N_SAMPLED_TARGETS = 4096


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def gen_inputs(wl, rank=0):
    rng = np.random.default_rng(wl["seed"])
    pts = rng.uniform(0.0, 1.0, (wl["N"], 3))
    wr = np.random.default_rng(wl["seed"] + 1000 + rank)
    w = wr.standard_normal(wl["N"] * wl["C"])  # column-major N x C
    return pts, w


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling (200 ms) of SM clocks and throttle reasons during
    the timed region."""

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ helpers
def direct_sum_sampled(pts, w, C, rows, ell, device):
    """float64 direct sum exp(-r/ell) at the sampled target rows (torch, GPU)."""
    import torch

    P = torch.tensor(pts, device=device)
    W = torch.tensor(w.reshape(C, -1), device=device)  # C x N
    T = P[torch.tensor(rows, device=device)]
    out = torch.zeros(C, len(rows), dtype=torch.float64, device=device)
    for a in range(0, P.shape[0], 1 << 16):
        d = torch.cdist(T, P[a:a + (1 << 16)])
        out += W[:, a:a + (1 << 16)] @ torch.exp(-d / ell).T
    return out.cpu().numpy()


def interaction_pairs(tstart, L):
    """Number of (target cell, source cell) M2L pairs per level, counted from
    the built tree (sources = targets)."""
    cnt = np.diff(tstart)
    pairs = {}
    for lvl in range(2, L + 1):
        occ = cnt.reshape(-1, 8 ** (L - lvl)).sum(1) > 0
        side = 1 << lvl
        idx = np.arange(8 ** lvl)
        x = np.zeros_like(idx)
        y = np.zeros_like(idx)
        z = np.zeros_like(idx)
        for b in range(lvl):
            x |= ((idx >> (3 * b + 2)) & 1) << b
            y |= ((idx >> (3 * b + 1)) & 1) << b
            z |= ((idx >> (3 * b)) & 1) << b
        grid = np.zeros((side, side, side), dtype=bool)
        grid[x, y, z] = occ
        total = 0
        px, py, pz = x // 2, y // 2, z // 2
        for ox in range(-3, 4):
            for oy in range(-3, 4):
                for oz in range(-3, 4):
                    if max(abs(ox), abs(oy), abs(oz)) <= 1:
                        continue
                    bx, by, bz = x + ox, y + oy, z + oz
                    ok = (bx >= 0) & (by >= 0) & (bz >= 0) & (bx < side) & (by < side) & (bz < side)
                    # parents adjacent
                    ok &= (np.abs(bx // 2 - px) <= 1) & (np.abs(by // 2 - py) <= 1) & (np.abs(bz // 2 - pz) <= 1)
                    sel = ok & occ
                    total += int(grid[bx[sel], by[sel], bz[sel]].sum())
        pairs[lvl] = total
    return pairs


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ------------------------------------------------------------ reference arm
def cpu_sample_run(wl, steps, warmup, threads):
    """Time the reference's own CPU matvec (oracle/_ref) on the bounded sample."""
    import oracle

    rng = np.random.default_rng(wl["seed"])
    Ns = CPU_SAMPLE["N"]
    pts = rng.uniform(0.0, 1.0, (Ns, 3))
    w = rng.standard_normal(Ns * wl["C"])
    out, timing, wd = oracle.run_reference(wl["kernel"], wl["ell"], wl["box"], CPU_SAMPLE["L"],
                                           wl["n"], wl["eps"], wl["cheb"], pts, w, wl["C"],
                                           repeat=warmup + steps, threads=threads)
    times = timing["matvec_s"][warmup:]
    return Ns * wl["C"] / (sum(times) / len(times)), times, timing["threads"]


def reference_arm(args, rank):
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    sample = ("reference CPU H2_3D_Compute (oracle/_ref, built from the reference sources) on "
              "N=%d points at tree_level %d (same %.2f points/leaf, kernel, order, nCols as the "
              "workload); per-step time of the ctor" % (CPU_SAMPLE["N"], CPU_SAMPLE["L"],
                                                         wl["N"] / 8 ** wl["L"]))
    try:
        value, times, th = cpu_sample_run(wl, args.steps, args.warmup, threads)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build failed: %s" % e}))
        return 0
    ms = 1e3 * sum(times) / len(times)
    line = {
        "impl": "reference", "metric": "FMM matvec N*nCols/s", "value": value,
        "unit": "N*nCols/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded uniform points, N(0,1) weights)",
        "config": {"workload": wl["name"], "sample_N": CPU_SAMPLE["N"],
                   "sample_tree_level": CPU_SAMPLE["L"], "kernel": "exp(-r/0.3)",
                   "interpolation": "uniform n=5, FFT M2L", "nCols": wl["C"]},
        "cpu_baseline": {"value": value, "unit": "N*nCols/s", "cores": th, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "N*nCols/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ our arm
def our_arm(args, rank, world, local_rank):
    import torch

    import pbbfmm3d_b200 as fmm

    wl = WORKLOADS[args.workload]
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811

    pts, w = gen_inputs(wl, rank)
    N, C = wl["N"], wl["C"]
    t0 = time.time()
    tree = fmm.kernel_ExpCov(wl["box"], wl["L"], wl["n"], wl["eps"], wl["cheb"], ell=wl["ell"],
                             device=local_rank)
    tree.buildFMMTree()
    log("precompute %.2fs" % (time.time() - t0))

    d_pts = torch.tensor(pts, device=dev)
    d_w = torch.tensor(w, device=dev)
    d_out = torch.zeros(N * C, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    stream = torch.cuda.current_stream(dev)

    def step(prec):
        fmm.compute_device(tree, d_pts, d_pts, d_w, C, d_out, precision=prec,
                           stream=stream.cuda_stream)

    precisions = [("fp64", fmm.PREC_FP64), ("mixed", fmm.PREC_MIXED)]
    results = {}
    for pname, prec in precisions:
        for _ in range(args.warmup):
            d_out.zero_()
            step(prec)
        torch.cuda.synchronize()
        tree.set_timing(True)
        tree.reset_kernel_times()
        launches0 = fmm.launch_count()
        sampler = ClockSampler(local_rank)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sampler.start()
        evs = []
        for _ in range(args.steps):
            flush.fill_(1.0)  # evict L2 between timed steps (outside the step events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(prec)
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clocks = sampler.stop()
        launches = fmm.launch_count() - launches0
        step_ms = [a.elapsed_time(b) for a, b in evs]
        ktimes = tree.kernel_times()
        tree.set_timing(False)
        total_ms = sum(step_ms)
        if world > 1:
            tt = torch.tensor([total_ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            total_ms = float(tt.item())
        results[pname] = dict(total_ms=total_ms, step_ms=step_ms, ktimes=ktimes, clocks=clocks,
                              launches=launches)
    # accuracy vs FP64 direct sum on sampled targets (outside the timed region)
    rng = np.random.default_rng(7)
    rows = np.sort(rng.choice(N, N_SAMPLED_TARGETS, replace=False))
    ref = direct_sum_sampled(pts, w, C, rows, wl["ell"], dev)
    errs = {}
    for pname, prec in precisions:
        d_out.zero_()
        step(prec)
        out = d_out.view(C, N)[:, torch.tensor(rows, device=dev)].cpu().numpy()
        errs[pname] = float(np.linalg.norm(out - ref) / np.linalg.norm(ref))

    # end to end through the host-buffer public API (H2_3D_Compute)
    e2e = None
    tree.set_precision(fmm.PREC_MIXED)
    if not args.no_e2e:
        host_out = np.zeros(N * C)
        fmm.H2_3D_Compute(tree, pts, pts, w, C, host_out)  # warm-up
        if world > 1:
            dist.barrier()
        ts = []
        for _ in range(max(1, min(args.steps, 5))):
            host_out[:] = 0
            t1 = time.perf_counter()
            fmm.H2_3D_Compute(tree, pts, pts, w, C, host_out)
            ts.append(time.perf_counter() - t1)
        e2e_s = sum(ts) / len(ts)
        if world > 1:
            tt = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt.item())
        e2e = {"value": world * N * C / e2e_s, "unit": "N*nCols/s",
               "h2d_bytes_per_step": int(8 * (3 * N + N * C + N * C)),
               "d2h_bytes_per_step": int(8 * N * C), "ms_per_step": 1e3 * e2e_s,
               "api": "pbbfmm_compute (host buffers, pageable)"}

    # roofline of the dominant kernel (headline = mixed path)
    r = results["mixed"]
    kt = r["ktimes"]
    dom = max(kt, key=lambda k: kt[k][0])
    tstart = tree.debug_copy(2).astype(np.int64)
    pairs = interaction_pairs(tstart, wl["L"])
    n, m = wl["n"], 2 * wl["n"] - 1
    nk = m * m * n
    mac_flops = sum(pairs.values()) * nk * C * 8.0  # one complex MAC = 8 flops
    nonempty = {l: int((np.diff(tstart).reshape(-1, 8 ** (wl["L"] - l)).sum(1) > 0).sum())
                for l in range(2, wl["L"] + 1)}
    mac_bytes = sum(2 * nonempty[l] * nk * C * 16 for l in nonempty)  # read X^, write Y^
    peaks, peak_kind = load_peaks()
    fp64_peak = fmm.measure_fma_peak(local_rank, fmm.PREC_FP64)
    fp32_peak = fmm.measure_fma_peak(local_rank, fmm.PREC_MIXED)
    mac_ms = kt["m2l_mac"][0] / args.steps
    mac_launches = kt["m2l_mac"][1] / args.steps
    achieved_tf = mac_flops / (mac_ms * 1e-3) / 1e12
    mac64_ms = results["fp64"]["ktimes"]["m2l_mac"][0] / args.steps
    roofline = {
        "kernel": "k_m2l_unif_mac<float> (frequency-domain M2L, mixed path)",
        "bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
        "frac": achieved_tf / fp32_peak, "traffic": None,
        "peak_source": "measured in this run: float32 FMA loop on every SM (pbbfmm_measure_fma_peak); "
                       "MEASURED_PEAKS.json has only HBM copy and bf16 tensor figures",
        "fp64_path": {"achieved": mac_flops / (mac64_ms * 1e-3) / 1e12, "peak": fp64_peak,
                      "frac": mac_flops / (mac64_ms * 1e-3) / 1e12 / fp64_peak,
                      "unit": "TFLOP/s"},
        "algorithmic": "%.4g flops per step = %d M2L pairs x %d freqs x %d cols x 8" % (
            mac_flops, sum(pairs.values()), nk, C),
        "launches_per_step": mac_launches,
        "hbm": {"achieved": mac_bytes / (mac_ms * 1e-3) / 1e9, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": mac_bytes / (mac_ms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                "algorithmic_bytes": mac_bytes, "peak_kind": peak_kind},
    }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, times, th = cpu_sample_run(wl, 6, 1, os.cpu_count() or 1)
            cpu = {"value": v, "unit": "N*nCols/s", "cores": th, "kind": "reference",
                   "sample": "reference CPU H2_3D_Compute (oracle/_ref) on N=%d at tree_level %d "
                             "(same points/leaf, kernel, order, nCols); mean of 6 runs %.2fs" % (
                                 CPU_SAMPLE["N"], CPU_SAMPLE["L"], sum(times) / len(times))}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "N*nCols/s", "cores": 0, "kind": "reference",
                   "sample": "failed: %s" % e}

    if rank != 0:
        return 0
    value = world * N * C * args.steps / (r["total_ms"] * 1e-3)
    r64 = results["fp64"]
    value64 = world * N * C * args.steps / (r64["total_ms"] * 1e-3)
    line = {
        "metric": "FMM matvec N*nCols/s (rel-L2 vs FP64 direct sum on 4096 sampled targets)",
        "value": value, "unit": "N*nCols/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded uniform points in the unit cube, N(0,1) weights",
        "config": {"workload": wl["name"], "N": N, "nCols": C, "tree_level": wl["L"],
                   "interpolation_order": wl["n"], "use_chebyshev": 0, "kernel": "exp(-r/0.3)",
                   "precision": "mixed: float32 far field and interpolation with compensated "
                                "sums, float64 positions, operators and output",
                   "l2": "256 MB buffer written between timed steps",
                   "parallelism": "independent 8-column blocks per rank" if world > 1 else "1 GPU"},
        "rel_l2_err": errs["mixed"],
        "fp64": {"value": value64, "unit": "N*nCols/s", "ms_per_step": r64["total_ms"] / args.steps,
                 "rel_l2_err": errs["fp64"],
                 "phase_ms_per_step": {k: v[0] / args.steps for k, v in r64["ktimes"].items()
                                       if v[1]}},
        "mixed_over_fp64": value / value64,
        "phase_ms_per_step": {k: v[0] / args.steps for k, v in kt.items() if v[1]},
        "dominant_kernel": dom,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(r["launches"] / args.steps) * args.steps,
        "gpu_launches_per_step": r["launches"] / args.steps,
        "clocks": r["clocks"],
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="bench", choices=sorted(WORKLOADS))
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    rc = our_arm(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
