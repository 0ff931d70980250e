"""Run a few Gibbs iterations of a synthetic workload, for profiling one kernel.

  python -m glimpse_b200.profile_case [--config batched] [--targets 8] [--iterations 2]

The panel has the shape of the named workload (glimpse_b200.synth.CONFIGS); the
target count is reduced so that a profiler capture stays small. Iteration 0 is
the init stage, the following ones burn-in.
"""
from __future__ import annotations

import argparse
import time

from glimpse_b200 import native, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="batched")
    ap.add_argument("--targets", type=int, default=8)
    ap.add_argument("--iterations", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    w = synth.workload(args.config, seed=args.seed, n_targets=args.targets)
    T = w.targets
    ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()))
    ctx.set_targets(T, kpbwt=T.kpbwt)
    for it in range(args.iterations):
        t0 = time.perf_counter()
        ctx.iteration(0 if it == 0 else 1, it)
        print(f"iteration {it}: {1000 * (time.perf_counter() - t0):.1f} ms, stages (ms) {ctx.stage_times().round(1)}")
    print(ctx.profile())
    ctx.close()


if __name__ == "__main__":
    main()
