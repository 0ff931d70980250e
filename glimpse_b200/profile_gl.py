"""Time the target GL input (gp_gl_from_pl / gp_gl_from_float) on the batched
workload's shape: 256 diploid targets x 150,000 sites.

  python -m glimpse_b200.profile_gl [--fmt PL] [--targets 256] [--sites 150000] [--reps 5]

Each call copies the FORMAT values in from host memory, converts them on the
device and copies gl/flat back; the printed figures are per call, from the host
clock (first call excluded).
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from glimpse_b200 import native, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--fmt", default="PL", choices=["PL", "GL"])
    ap.add_argument("--targets", type=int, default=256)
    ap.add_argument("--sites", type=int, default=150_000)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    n, L = args.targets, args.sites
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
    try:
        times = []
        for r in range(args.reps + 1):
            t0 = time.perf_counter()
            ctx.gl_from_format(args.fmt, src, ploidy)
            times.append(time.perf_counter() - t0)
        t = float(np.median(times[1:]))
        moved = src.nbytes + n * L * 4
        print(f"{args.fmt}: {n} targets x {L} sites, {1e3 * t:.1f} ms per call (median of {args.reps}), "
              f"{moved / t / 1e9:.1f} GB/s of host data in + out ({moved / 1e6:.0f} MB)")
    finally:
        ctx.close()


if __name__ == "__main__":
    main()
