"""Time the output epilogue (gp_output_records) after a short run of a workload.

  python -m glimpse_b200.profile_records [--config batched] [--targets 256] [--reps 5]

The run is 1 init + 1 main iteration (enough for finalised posteriors); each
timed call computes GP, RAF, AF and INFO on the device and copies them to the
host (first call excluded; host clock).
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from glimpse_b200 import native, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="batched")
    ap.add_argument("--targets", type=int, default=256)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    w = synth.workload(args.config, seed=1, n_targets=args.targets)
    T = w.targets
    ctx = native.Context(w.panel, kinit=w.params["kinit"], kpbwt=int(T.kpbwt.max()))
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.run(0, 1)
        times = []
        for _ in range(args.reps + 1):
            t0 = time.perf_counter()
            gp, raf, af, info = ctx.output_records()
            times.append(time.perf_counter() - t0)
        t = float(np.median(times[1:]))
        print(f"output records: {T.n} targets x {w.panel.n_sites} sites, {1e3 * t:.1f} ms per call "
              f"(median of {args.reps}, device work and {gp.nbytes / 1e6:.0f} MB copied to the host); "
              f"mean INFO {float(info.mean()):.3f}")
    finally:
        ctx.close()


if __name__ == "__main__":
    main()
