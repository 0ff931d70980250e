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
cores: each step is one complete run (1 init + 5 burn-in + 15 main iterations
and finalisation) over a fixed subset of the workload's targets (the first
--subset targets, default one per host thread up to 32), so the work per target
is the same as in the GPU arm. The GPU arm's line carries the same subset run
on the GPU beside it (`same_subset`), with the dosage r2 of both.

--case iterations|gl|records runs a small single-stage case for profiler
captures (python bench.py --case iterations --targets 16 --iterations 2).
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


def workload_label(name):
    """The workload's shape in words, from its entry in synth.CONFIGS."""
    from glimpse_b200 import synth
    c = synth.CONFIGS[name]

    def spec(x, unit=""):
        kind = x[0]
        if kind == "fixed":
            return f"{x[1]:g}{unit}"
        if kind in ("uniform", "loguniform"):
            return f"{x[1]:g}-{x[2]:g}{unit}" + (" (log-uniform)" if kind == "loguniform" else "")
        return " / ".join(f"{v:g}{unit} ({p:.0%})" for v, p in x[1:])

    return (f"{name}: {c['n_ref_haps']:,} reference haplotypes x {c['n_sites']:,} sites over {c['region_mb']:g} Mb "
            f"({c['rare_frac']:.0%} rare, sparse), {c['n_targets']} diploid targets at {spec(c['cov'], 'x')} "
            f"coverage, Kpbwt {spec(c['k'])} per target, Kinit {c['kinit']}, 1 init + {BURNIN} burn-in + {MAIN} main")


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(kernel):
    """DRAM bytes per algorithmic unit of a kernel from the committed ncu figures
    (profiles/traffic.json: one entry per kernel, with the capture it came from)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    e = d.get(kernel)
    return None if e is None else float(e["dram_bytes_per_unit"])


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


def subset(T, n):
    """The first n targets of a workload's batch (the fixed sample both arms run)."""
    import types
    idx = np.arange(min(n, T.n))
    return types.SimpleNamespace(n=len(idx), ploidy=T.ploidy[idx], gl=T.gl[idx], flat=T.flat[idx],
                                 truth=T.truth[idx], kpbwt=T.kpbwt[idx], coverage=T.coverage[idx])


def reference_ds(orc, n):
    """Dosages of a finished reference run: DS = gp1 + 2 gp2 rounded to 1e-3
    (genotype_writer.cpp:123-126, gp2 = clamp(1 - gp0 - gp1), genotype.h:62-64)."""
    out = []
    for t in range(n):
        g0, g1, _, _, _ = orc.gp(t)
        g2 = np.clip(np.float32(1.0) - g1 - g0, 0.0, 1.0)
        out.append(np.round((g1 + np.float32(2.0) * g2) * 1000.0) / 1000.0)
    return np.stack(out)


class ReferenceRun:
    """The reference's hot path (oracle/_ref: the reference's sources compiled
    unmodified) on the host cores: one step is one complete run, 1 init +
    burn-in + main iterations and finalisation, over a fixed subset of the
    workload's targets, with the reference driver's dynamic assignment of
    targets to threads and per-thread replay streams; or, with native_rng, the
    reference's own generator (std::mt19937 seeded once) on one thread."""

    def __init__(self, w, n_targets, threads, native_rng=False):
        from oracle import oracle as O
        self.O = O
        self.w = w
        self.sub = subset(w.targets, n_targets)
        self.native_rng = native_rng
        self.threads = 1 if native_rng else threads
        self.orc = O.RefOracle(w.panel, native_rng=native_rng)

    def step(self):
        O, sub = self.O, self.sub
        self.orc.set_targets(sub)
        self.orc.configure(kinit=self.w.params["kinit"], kpbwt=int(sub.kpbwt.max()), kpbwt_target=sub.kpbwt,
                           seed=15052011)
        t0 = time.perf_counter()
        self.orc.run(burnin=BURNIN, main=MAIN, threads=self.threads)
        return time.perf_counter() - t0

    def dosage_r2(self):
        return synth.dosage_r2(reference_ds(self.orc, self.sub.n), self.sub.truth.sum(1))

    def sample_text(self, seconds):
        return (f"{self.sub.n} of the {self.w.targets.n} targets (the first {self.sub.n}), one complete run per "
                f"step (1 init + {BURNIN} burn-in + {MAIN} main iterations and finalisation, {seconds:.1f} s) on "
                f"{self.threads} threads ("
                + ("the reference's own std::mt19937" if self.native_rng else "per-thread replay RNG")
                + "); samples/s = targets / run time")


def default_subset(threads):
    return max(1, min(threads, 32))


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    try:
        from oracle import oracle as O
        native = getattr(args, "ref_rng", "replay") == "native"
        if not O.ref_available(native_rng=native):
            lib = "libglimpse_ref_native.so" if native else "libglimpse_ref.so"
            print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/{lib} not built"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle import failed: {e}"}))
        return 0
    w = synth.workload(args.config, seed=1)
    threads = 1 if native else (os.cpu_count() or 1)
    ref = ReferenceRun(w, args.subset or default_subset(threads), threads, native_rng=native)
    for _ in range(args.warmup):
        ref.step()
    times = [ref.step() for _ in range(args.steps)]
    t_run = sum(times) / len(times)
    value = ref.sub.n / t_run
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_run * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_label(args.config), "parallelism": f"{threads} host threads",
                       "targets_timed": ref.sub.n, "rng": "native" if native else "replay"},
            "dosage_r2": ref.dosage_r2(),
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "reference",
                             "sample": ref.sample_text(t_run)},
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
    ctx.set_precision({"full": native.PRECISION_FULL, "f32": native.PRECISION_CKPT_F32,
                       "bf16": native.PRECISION_CKPT_BF16}[args.precision])
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
    # algorithmic bytes per cell: full store 4 B written + 4 B read + 2 x 1/8 B Hvar;
    # checkpoints 2 x 4/32 (FP32) or 2 x 2/32 (BF16) B + 3 x 1/8 B Hvar (forward, recompute, backward)
    bpc = {"full": 8.25, "f32": 0.625, "bf16": 0.5}[args.precision]
    kname = "k_impute_warp" if args.precision == "full" else "k_impute_ckpt"
    achieved = prof["impute_cells"] * bpc / (prof["impute_ms"] / 1000.0) / 1e9 if prof["impute_ms"] > 0 else 0.0
    per_launch_cells = prof["impute_cells"] / max(1, prof["impute_launches"])
    tpc = read_traffic(kname)
    roofline = {"bound": "hbm", "kernel": kname + " (imputation forward-backward)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "algorithmic_bytes_per_cell": bpc, "cells_per_launch": per_launch_cells,
                "launch_ms": prof["impute_ms"] / max(1, prof["impute_launches"]),
                "traffic": (tpc * per_launch_cells) if tpc is not None else None}
    # Phasing (k_phase) is bound by its per-site dependent chain, not by HBM: its
    # messages live in registers. Reported against the FP32 issue rate at the
    # sampled clock: 148 SMs x 128 lanes x 2 flop per FMA.
    sm_mhz = clk.get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    phase_cells_s = prof["phase_cells"] / (prof["phase_ms"] / 1000.0) if prof["phase_ms"] > 0 else 0.0
    phase = {"kernel": "k_phase (phasing backward + forward with diplotype sampling)", "bound": "latency",
             "cells_per_s": phase_cells_s, "launch_ms": prof["phase_ms"] / max(1, prof["phase_launches"]),
             "share_of_step": prof["phase_ms"] / args.steps / ms, "flops_per_cell": 4,
             "fp32_tflops": phase_cells_s * 4 / 1e12, "fp32_peak_tflops": fp32_peak,
             "fp32_frac": phase_cells_s * 4 / 1e12 / fp32_peak,
             "cell": "(VAR site, state, hypothesis) of one pass; 4 flop: transition fma, emission mul, sum add"}
    select = {"kernels": "k_pbwt_sweep + k_pbwt_union + conditioning-set build", "bound": "latency",
              "share_of_step": prof["select_ms"] / args.steps / ms,
              "ms_per_iteration": prof["select_ms"] / args.steps / N_ITER}
    hmm_cells = (prof["impute_cells"] + prof["phase_cells"]) / (args.steps)
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_label(args.config), "targets_per_gpu": T.n, "iterations_per_step": N_ITER,
                       "l2": "no flush: per-step working set (alpha store, prefix arrays) is tens of GB >> 126 MB L2",
                       "parallelism": f"targets per GPU, {world} rank(s), no collective on the data path"},
            "precision": {"full": "every forward row in FP32 (as the reference)",
                          "f32": "FP32 checkpoints every 32 sites, recompute",
                          "bf16": "BF16 checkpoints every 32 sites, FP32 recompute"}[args.precision],
            "autotuned": dict(zip(("chains_per_cta", "sweep_haps_per_warp", "phase_placement", "ms"),
                                  (lambda tu: (*tu[:3], [round(float(x), 3) for x in tu[3]]))(ctx.tuning()))),
            "hmm_cells_per_s": world * hmm_cells / (ms / 1000.0),
            "dosage_r2": r2,
            "dosage_r2_by_maf": [{"maf": [lo, hi], "sites": n_s, "r2": (None if r != r else round(r, 6))}
                                 for lo, hi, n_s, r in synth.dosage_r2_bins(ds_h.numpy(), T.truth.sum(1),
                                                                           synth.panel_maf(w.panel))],
            "gpu_launches": int(prof["kernel_launches"]),
            "clocks": clk,
            "roofline": roofline,
            "phasing": phase,
            "selection": select,
            "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # The same fixed subset on both sides: a complete run of the first
        # targets, on the GPU (device time) and on the host cores (reference).
        threads = os.cpu_count() or 1
        sub = subset(T, args.subset or default_subset(threads))
        ctx.set_targets(sub, kpbwt=sub.kpbwt)
        for _ in range(max(1, min(args.warmup, 3))):
            device_step()
        reps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(reps):
            device_step()
        s1.record(stream)
        torch.cuda.synchronize()
        ms_sub = s0.elapsed_time(s1) / reps
        _, _, ds_sub, _, _ = ctx.gp()
        ref = ReferenceRun(w, sub.n, threads)
        t_ref = ref.step()
        cpu_value = sub.n / t_ref
        line["cpu_baseline"] = {"value": cpu_value, "unit": "samples/s", "cores": threads, "kind": "reference",
                                "sample": ref.sample_text(t_ref)}
        line["same_subset"] = {"targets": sub.n, "gpu_samples_per_s": sub.n / (ms_sub / 1000.0),
                               "gpu_ms_per_run": ms_sub, "reference_samples_per_s": cpu_value,
                               "reference_cores": threads,
                               "gpu_dosage_r2": synth.dosage_r2(ds_sub, sub.truth.sum(1)),
                               "reference_dosage_r2": ref.dosage_r2()}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_learned(args):
    """Learned proposal against plain PBWT selection on one GPU, device-timed
    complete runs (1 init + 5 burn-in + 15 main, finalisation) of the workload's
    benchmark targets. The network is trained first on a separate set of
    simulated targets of the same panel (their own plain init and burn-in
    iterations give the haplotypes; labels are the HMM's window posteriors over
    their PBWT candidates). Reported: samples/s and dosage r2 of plain selection
    at the workload's K; plain and learned at each fraction of K in
    --learned-fracs; and the learned proposal sizing each target's set itself
    (at most the workload's K). Candidates: PBWT at the workload's largest K.
    `value` is the fastest learned run whose r2 is within 0.002 of plain at the
    workload's K (matched_r2), else the learned run with the best r2; the fastest
    plain run at matched r2 is reported beside it."""
    import torch
    from glimpse_b200 import native
    torch.cuda.set_device(0)
    n_test = synth.CONFIGS[args.config]["n_targets"]
    w = synth.workload(args.config, seed=1, n_targets=n_test + args.train_targets)
    test = subset(w.targets, n_test)
    import types
    idx = np.arange(n_test, w.targets.n)
    T = w.targets
    train = types.SimpleNamespace(n=len(idx), ploidy=T.ploidy[idx], gl=T.gl[idx], flat=T.flat[idx],
                                  truth=T.truth[idx], kpbwt=T.kpbwt[idx], coverage=T.coverage[idx])
    kbig = test.kpbwt.copy()
    kcand = int(min(2048, kbig.max()))
    ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=kcand, seed=15052011)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    t0 = time.perf_counter()
    ctx.set_targets(train, kpbwt=np.full(train.n, kcand, np.int32))
    ctx.iteration(native.STAGE_INIT, 0)
    for it in range(1, 3):
        ctx.iteration(native.STAGE_BURN, it)
    losses = ctx.learned_train(kcand=kcand, kpos=8.0, steps=args.train_steps, batch=16384, lr=1e-3, seed=7)
    t_train = time.perf_counter() - t0

    def timed_runs(kp, learned, min_prob=0.5, kmin=0):
        ctx.learned_enable(False, kcand=kcand)
        ctx.set_targets(test, kpbwt=kp)
        ctx.learned_size(min_prob, kmin)
        if learned:
            ctx.learned_enable(True, kcand=kcand)
        for _ in range(args.warmup):
            ctx.targets_reset()
            ctx.run(BURNIN, MAIN)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.targets_reset()
            ctx.run(BURNIN, MAIN)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        _, _, ds, _, _ = ctx.gp()
        kused = float(np.mean([ctx.states(t).size for t in range(test.n)]))  # last iteration's set sizes
        return {"samples_per_s": test.n / (ms / 1000.0), "ms_per_run": ms,
                "dosage_r2": synth.dosage_r2(ds, test.truth.sum(1)), "k_mean": kused}

    plain_big = timed_runs(kbig, False)
    sweep = []
    for frac in [float(x) for x in args.learned_fracs.split(",")]:
        ks = np.maximum(16, np.round(kbig * frac)).astype(np.int32)
        sweep.append({"k_fraction": frac, "plain": timed_runs(ks, False), "learned": timed_runs(ks, True)})
    # the network also sizes the sets: candidates some window scores at 0.5 or
    # more, at least 32, at most the workload's K
    adaptive = timed_runs(kbig, True, 0.5, 32)
    ctx.learned_size(0.5, 0)
    ctx.close()
    r2_ref = plain_big["dosage_r2"]
    learned_runs = [(f"learned at K x {e['k_fraction']}", e["learned"]) for e in sweep] + [("learned, sized by the "
                                                                                            "network", adaptive)]
    matched = [(name, r) for name, r in learned_runs if abs(r["dosage_r2"] - r2_ref) <= 0.002]
    name, best = max(matched, key=lambda nr: nr[1]["samples_per_s"]) if matched else \
        max(learned_runs, key=lambda nr: nr[1]["dosage_r2"])
    plain_matched = [e["plain"] for e in sweep if abs(e["plain"]["dosage_r2"] - r2_ref) <= 0.002]
    line = {"metric": "samples/s at matched dosage r2 (learned + batched vs plain)", "unit": "samples/s",
            "value": best["samples_per_s"], "higher_is_better": True, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "dtype": "f32 HMM, bf16 network", "data": "synthetic",
            "config": {"workload": args.config, "targets": test.n, "training_targets": train.n,
                       "training_steps": args.train_steps, "candidates_per_target": kcand},
            "value_from": name, "matched_r2": bool(matched),
            "speedup_vs_plain_workload_k": best["samples_per_s"] / plain_big["samples_per_s"],
            "fastest_plain_at_matched_r2": max(plain_matched, key=lambda r: r["samples_per_s"]) if plain_matched
            else None,
            "plain_workload_k": plain_big, "k_sweep": sweep, "learned_sized_by_network": adaptive,
            "training": {"seconds": t_train, "loss_first": float(losses[:10].mean()),
                         "loss_last": float(losses[-10:].mean())}}
    print(json.dumps(line))
    return 0


def run_case(args):
    """Small cases of single stages, for profiler captures and quick timings
    (not bench lines): `iterations` runs Gibbs iterations of a workload with a
    reduced batch; `gl` times the target GL input; `records` the output epilogue."""
    from glimpse_b200 import native
    if args.case == "iterations":
        w = synth.workload(args.config, seed=1, n_targets=args.targets)
        T = w.targets
        ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()))
        ctx.set_precision({"full": native.PRECISION_FULL, "f32": native.PRECISION_CKPT_F32,
                           "bf16": native.PRECISION_CKPT_BF16}[args.precision])
        ctx.set_targets(T, kpbwt=T.kpbwt)
        for it in range(args.iterations):
            t0 = time.perf_counter()
            ctx.iteration(0 if it == 0 else 1, it)
            print(f"iteration {it}: {1000 * (time.perf_counter() - t0):.1f} ms, stages (ms) "
                  f"{ctx.stage_times().round(1)}")
        print(ctx.profile())
        ctx.close()
    elif args.case == "gl":
        n, L = args.targets, 150_000
        rng = np.random.default_rng(1)
        if args.fmt == "PL":
            src = rng.integers(0, 300, size=(L, n, 3), dtype=np.int32)
        else:
            src = (-rng.uniform(0, 30, size=(L, n, 3))).astype(np.float32)
        ploidy = np.full(n, 2, np.int32)
        # any panel serves: the conversion does not read it
        w = synth.make_panel_and_targets(600, 4000, 0.4, 0.5, 1, ("uniform", 0.5, 2.0), ("uniform", 80, 300),
                                         seed=7, sparse_maf=0.01, lq_frac=0.02, alt_major_frac=0.1)
        ctx = native.Context(w.panel)
        times = []
        for _ in range(args.reps + 1):
            t0 = time.perf_counter()
            ctx.gl_from_format(args.fmt, src, ploidy)
            times.append(time.perf_counter() - t0)
        t = float(np.median(times[1:]))
        print(f"{args.fmt}: {n} targets x {L} sites, {1e3 * t:.1f} ms per call (median of {args.reps})")
        ctx.close()
    elif args.case == "groups":
        # the workload's targets split over G contexts (one stream each) driven
        # by G host threads: complete runs, device-timed from the first stream
        import threading
        import torch
        w = synth.workload(args.config, seed=1)
        T = w.targets
        G = args.groups
        parts = np.array_split(np.arange(T.n), G)
        ctxs = []
        for idx in parts:
            sub = subset(T, T.n)
            for k in ("ploidy", "gl", "flat", "truth", "kpbwt", "coverage"):
                setattr(sub, k, getattr(T, k)[idx])
            sub.n = len(idx)
            c = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()))
            c.set_targets(sub, kpbwt=sub.kpbwt)
            ctxs.append(c)
        streams = [torch.cuda.ExternalStream(c.stream_handle()) for c in ctxs]

        def one(c):
            c.targets_reset()
            c.run(BURNIN, MAIN)

        def step():
            th = [threading.Thread(target=one, args=(c,)) for c in ctxs]
            for x in th:
                x.start()
            for x in th:
                x.join()

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        for _ in range(args.steps):
            step()
        for st in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(st)
            streams[0].wait_event(ev)
        e1.record(streams[0])
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        print(f"groups={G}: {T.n} targets, {ms:.1f} ms per complete run, {T.n / (ms / 1000.0):.2f} samples/s")
        for c in ctxs:
            c.close()
    elif args.case == "mlp":
        # the learned proposal's fused forward on the tensor cores: rows of
        # random features, timed with CUDA events on the context stream
        import torch
        w = synth.make_panel_and_targets(600, 4000, 0.4, 0.5, 1, ("uniform", 0.5, 2.0), ("uniform", 80, 300),
                                         seed=7, sparse_maf=0.01, lq_frac=0.02, alt_major_frac=0.1)
        ctx = native.Context(w.panel)
        ctx.mlp_init(1)
        n = args.rows
        x = np.random.default_rng(1).random((n, 48), dtype=np.float32)
        ctx.mlp_forward(x[:1024])
        ctx.profile_reset()
        for _ in range(args.reps):
            ctx.mlp_forward(x)
        p = ctx.profile()
        t = (p["mlp_ms"] - 0.0) / max(1, p["mlp_launches"])
        rows = p["mlp_rows"] / max(1, p["mlp_launches"])
        # device time of the fused forward alone (CUDA events around each launch)
        flop = 2.0 * rows * (64 * 256 + 256 * 256 + 256)
        print(f"mlp forward: {rows:.0f} rows per launch (mean over {p['mlp_launches']} launches), {t:.3f} ms, "
              f"{flop / t / 1e9:.1f} TFLOP/s of the 48(64)->256->256->1 network")
        ctx.close()
    elif args.case == "records":
        w = synth.workload(args.config, seed=1, n_targets=args.targets)
        T = w.targets
        ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()))
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.run(0, 1)
        times = []
        for _ in range(args.reps + 1):
            t0 = time.perf_counter()
            ctx.output_records()
            times.append(time.perf_counter() - t0)
        print(f"output records: {T.n} targets, {1e3 * float(np.median(times[1:])):.1f} ms per call")
        ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-rng", choices=["replay", "native"], default="replay",
                    help="reference arm: replay streams on every host thread (default), or the reference's own "
                         "std::mt19937 on one thread")
    ap.add_argument("--config", default="batched")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--subset", type=int, default=0,
                    help="targets of the fixed subset both arms run completely (default: host threads, at most 32)")
    ap.add_argument("--case", choices=["iterations", "gl", "records", "mlp", "groups"], default=None,
                    help="run a small single-stage case (for profiler captures) instead of the bench")
    ap.add_argument("--targets", type=int, default=16)
    ap.add_argument("--iterations", type=int, default=2)
    ap.add_argument("--fmt", choices=["PL", "GL"], default="PL")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--rows", type=int, default=4 << 20)
    ap.add_argument("--groups", type=int, default=2)
    ap.add_argument("--precision", choices=["full", "f32", "bf16"], default="full",
                    help="imputation store: every row (default) or FP32 / BF16 checkpoints")
    ap.add_argument("--learned", action="store_true",
                    help="learned proposal vs plain PBWT selection (separate line; see run_learned)")
    ap.add_argument("--learned-fracs", default="0.4,0.1,0.05",
                    help="fractions of the workload's K at which plain and learned selection are compared")
    ap.add_argument("--train-targets", type=int, default=64)
    ap.add_argument("--train-steps", type=int, default=400)
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.learned:
        return run_learned(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
