"""Benchmark: GLIMPSE2_phase's inner loop on the batched workload.

One step = one complete GLIMPSE2_phase run over the target batch (1 init +
5 burn-in + 15 main Gibbs iterations: PBWT/init selection, two imputation HMM
passes with sampling, phasing HMM, posterior accumulation, finalisation), with
the panel and targets resident on the GPU. `value` = targets / step time (all
ranks). `e2e` = the same run through the C-ABI from pinned host buffers: the
targets' genotype likelihoods are copied in and the dosages/genotypes copied
out inside every timed step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU implementation of the path
(the reference hot-path sources built unmodified as oracle/_ref) on the host
cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from glimpse_b200 import synth  # noqa: E402

METRIC = "samples/s at matched dosage r2 (plain batched GPU path); HMM cells/s vs HBM peak"
BURNIN, MAIN = 5, 15
N_ITER = 1 + BURNIN + MAIN
WORKLOAD = ("batched: 10,000 reference haplotypes x 150,000 sites over 4 Mb (80% rare, sparse), 256 diploid "
            "targets at 0.5-2x coverage, Kpbwt 400-1200 per target, Kinit 1000, 1 init + 5 burn-in + 15 main")


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic_per_cell():
    """DRAM bytes per imputation cell from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "k_impute_warp_batched.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("dram_bytes_per_cell:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = f"/tmp/gp_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def rank_ops(dist, device):
    """Barrier and max-over-ranks of a float (the step time) for the ranks of one job.
    dist is torch.distributed with an initialised process group, or None for one rank."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def cpu_sample(w, n_sample, threads, timed_iters=1):
    """Reference CPU path on a bounded sample: returns (seconds per burn-in iteration, n)."""
    from oracle import oracle as O
    import types
    T = w.targets
    idx = np.arange(min(n_sample, T.n))
    sub = types.SimpleNamespace(n=len(idx), ploidy=T.ploidy[idx], gl=T.gl[idx], flat=T.flat[idx],
                                truth=T.truth[idx], kpbwt=T.kpbwt[idx])
    orc = O.RefOracle(w.panel)
    orc.set_targets(sub)
    orc.configure(kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()), kpbwt_target=sub.kpbwt, seed=15052011)
    orc.iteration(O.STAGE_INIT, 0, threads)
    times = []
    for i in range(timed_iters):
        t0 = time.perf_counter()
        orc.iteration(O.STAGE_BURN, 1 + i, threads)
        times.append(time.perf_counter() - t0)
    return times, len(idx)


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    try:
        from oracle import oracle as O
        if not O.ref_available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libglimpse_ref.so not built"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle import failed: {e}"}))
        return 0
    w = synth.workload(args.config, seed=1)
    threads = os.cpu_count() or 1
    n_sample = threads
    times, n = cpu_sample(w, n_sample, threads, timed_iters=args.warmup + args.steps)
    timed = times[args.warmup:]
    t_iter = sum(timed) / len(timed)
    value = n / (N_ITER * t_iter)
    sample = (f"{n} of the {w.targets.n} targets, one burn-in iteration per step on {threads} threads "
              f"(per-thread replay RNG); samples/s = targets / ({N_ITER} x iteration time)")
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_iter * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    from glimpse_b200 import native
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
        dist = dist_mod
    w = synth.workload(args.config, seed=1)
    T = w.targets
    kmax = int(T.kpbwt.max())
    ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=kmax, seed=15052011, device=local)
    ctx.set_targets(T, kpbwt=T.kpbwt)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", local))

    barrier, max_over_ranks = rank_ops(dist, torch.device("cuda", local))

    def device_step():
        ctx.targets_reset()
        ctx.run(BURNIN, MAIN)

    for _ in range(args.warmup):
        device_step()
    clocks = ClockSampler(local)
    ctx.profile_reset()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        device_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms)
    prof = ctx.profile()
    value = world * T.n / (ms / 1000.0)

    # end to end through the C-ABI from pinned host buffers
    n, L = T.n, w.panel.n_sites
    gl_h = torch.from_numpy(np.ascontiguousarray(T.gl)).pin_memory()
    fl_h = torch.from_numpy(np.ascontiguousarray(T.flat)).pin_memory()
    pl_h = torch.from_numpy(np.ascontiguousarray(T.ploidy, np.int32)).pin_memory()
    kp_h = torch.from_numpy(np.ascontiguousarray(T.kpbwt, np.int32)).pin_memory()
    ds_h = torch.empty((n, L), dtype=torch.float32).pin_memory()
    g0_h = torch.empty((n, L), dtype=torch.uint8).pin_memory()
    g1_h = torch.empty((n, L), dtype=torch.uint8).pin_memory()
    h2d = gl_h.numel() + fl_h.numel() + 4 * pl_h.numel() + 4 * kp_h.numel()
    d2h = 4 * ds_h.numel() + g0_h.numel() + g1_h.numel()

    def e2e_step():
        ctx.set_targets_raw(n, gl_h.data_ptr(), fl_h.data_ptr(), pl_h.data_ptr(), kp_h.data_ptr())
        ctx.run(BURNIN, MAIN)
        ctx.gp_raw(ds_h.data_ptr(), g0_h.data_ptr(), g1_h.data_ptr())

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    e2e_value = world * n / (ms_e2e / 1000.0)
    r2 = synth.dosage_r2(ds_h.numpy(), T.truth.sum(1))

    peak, peak_kind = load_peaks()
    achieved = prof["impute_bytes"] / (prof["impute_ms"] / 1000.0) / 1e9 if prof["impute_ms"] > 0 else 0.0
    per_launch_cells = prof["impute_cells"] / max(1, prof["impute_launches"])
    tpc = read_traffic_per_cell()
    roofline = {"bound": "hbm", "kernel": "k_impute_warp (imputation forward-backward)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "algorithmic_bytes_per_cell": 8.25, "cells_per_launch": per_launch_cells,
                "launch_ms": prof["impute_ms"] / max(1, prof["impute_launches"]),
                "traffic": (tpc * per_launch_cells) if tpc is not None else None}
    hmm_cells = (prof["impute_cells"] + prof["phase_cells"]) / (args.steps)
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "targets_per_gpu": T.n, "iterations_per_step": N_ITER,
                       "l2": "no flush: per-step working set (alpha store, prefix arrays) is tens of GB >> 126 MB L2",
                       "parallelism": f"targets per GPU, {world} rank(s), no collective on the data path"},
            "hmm_cells_per_s": world * hmm_cells / (ms / 1000.0),
            "dosage_r2": r2,
            "gpu_launches": int(prof["kernel_launches"]),
            "clocks": clk,
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times, ns = cpu_sample(w, threads, threads, timed_iters=1)
        cpu_value = ns / (N_ITER * times[0])
        line["cpu_baseline"] = {"value": cpu_value, "unit": "samples/s", "cores": threads, "kind": "reference",
                                "sample": f"{ns} targets, one burn-in iteration on {threads} threads "
                                          f"({times[0]:.1f} s); samples/s = targets / ({N_ITER} x iteration time)"}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="batched")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
