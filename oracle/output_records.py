"""ORACLE — test infrastructure only.

Restatement of the record fields genotype_writer::writeGenotypes computes
(phase/src/io/genotype_writer.cpp:110-190): FORMAT/GP as written and the per-site
RAF, AF and INFO, from the finalised genotype posteriors. The reference's writer
needs htslib, which is absent here, so this restatement is pinned by known
answers read off those lines (tests/test_output_records.py) rather than by the
reference binary. Only tests/ use this module.

float / double follow the reference's types. Its -mfma build contracts
`ds = gp1 + 2.0f * gp2` and `ds2_sum += ds * ds` into fused multiply-adds; the
first is exact either way (2 * gp2 is exact), the second is computed here with
an exact fma rounded once to float32.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

f32, f64 = np.float32, np.float64
VECTOR_END_BITS = 0x7F800002  # bcf_float_vector_end


def _round_f32(q: Fraction) -> np.float32:
    """q rounded to the nearest float32 (ties to even); normal and subnormal range."""
    if q == 0:
        return f32(0.0)
    sign = -1 if q < 0 else 1
    q = abs(q)
    e = q.numerator.bit_length() - q.denominator.bit_length() - 24
    while q >= Fraction(2) ** (e + 24):
        e += 1
    while q < Fraction(2) ** (e + 23):
        e -= 1
    e = max(e, -149)
    m = q / Fraction(2) ** e
    k = m.numerator // m.denominator
    r = m - k
    if r > Fraction(1, 2) or (r == Fraction(1, 2) and k % 2 == 1):
        k += 1
    return f32(sign * k * 2.0 ** e)


def fmaf(a, b, c) -> np.float32:
    return _round_f32(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def _floor_milli(x) -> np.float32:
    # floorf(x * 1000.0) / 1000.0: double product, float floor, double quotient
    return f32(f64(np.floor(f32(f64(x) * 1000.0))) / 1000.0)


def _roundf(x: np.float32) -> np.float32:
    # roundf: half away from zero (exact in float64 for float32 inputs)
    v = f64(x)
    return f32(np.sign(v) * np.floor(abs(v) + 0.5))


def gp_fields(g0, g1, ploidy_i: int, max_ploidy: int):
    """GP values of one (site, target) as written (genotype_writer.cpp:151-172),
    and the DS and gp2 that enter the INFO sums."""
    g0, g1 = f32(g0), f32(g1)
    if ploidy_i > 1:
        g2 = f32(min(max(f32(f32(1.0) - g1) - g0, f32(0.0)), f32(1.0)))   # genotype.h:62-64
        ds = fmaf(2.0, g2, g1)
    else:
        g2, ds = f32(0.0), g1
    p = [_floor_milli(g0), _floor_milli(g1), f32(0.0)]
    keys = [(f32(1.0) - (g0 - p[0]), 0), (f32(1.0) - (g1 - p[1]), 1)]
    third = max_ploidy > 1 and ploidy_i > 1
    if third:
        p[2] = _floor_milli(max(f32(1.0) - (p[0] + p[1]), f32(0.0)))
        keys.append((f32(1.0) - (g2 - p[2]), 2))
    # std::map<float, float*>: a key equal to an earlier one is not inserted
    kept = []
    for k, idx in keys:
        if all(k != kk for kk, _ in kept):
            kept.append((k, idx))
    kept.sort(key=lambda t: float(t[0]))
    top = 3 if third else 2
    for _, idx in kept:
        s = f32(0.0)
        for j in range(top):
            s = f32(s + p[j])
        if not s < f32(0.9999):
            break
        p[idx] = f32(p[idx] + f32(0.001))
    out = np.array(p, np.float32)
    if not third:
        out[2:] = np.array([VECTOR_END_BITS], np.uint32).view(np.float32)
    return out, ds, g2


def output_records(gp0, gp1, ploidy, calt, cref):
    """gp0, gp1: (n, L) finalised posteriors (1, 0 where none were stored);
    returns gp (n, L, 3), raf, af, info (L,)."""
    gp0 = np.asarray(gp0, np.float32)
    gp1 = np.asarray(gp1, np.float32)
    ploidy = np.asarray(ploidy, np.int32)
    n, L = gp0.shape
    max_ploidy = int(ploidy.max())
    n_haps = int(ploidy.sum())
    mixed = bool((ploidy == 1).any() and (ploidy == 2).any())
    fploidy = -max_ploidy if mixed else max_ploidy                    # genotype_reader.cpp:553-554
    gp = np.zeros((n, L, 3), np.float32)
    raf = np.zeros(L, np.float32)
    af = np.zeros(L, np.float32)
    info = np.zeros(L, np.float32)
    for l in range(L):
        ds_sum = ds2_sum = ds4_sum = f32(0.0)
        for i in range(n):
            out, ds, g2 = gp_fields(gp0[i, l], gp1[i, l], int(ploidy[i]), max_ploidy)
            gp[i, l] = out
            ds_sum = f32(ds_sum + ds)                                   # :175
            if fploidy == 2:
                ds2_sum = fmaf(ds, ds, ds2_sum)                         # :178
                ds4_sum = f32(f64(ds4_sum) + (f64(gp1[i, l]) + 4.0 * f64(g2)))  # :179
        ca, cr = int(calt[l]), int(cref[l])
        raf[l] = f32(f32(ca) * f32(1.0)) / f32(ca + cr)                 # :184
        f = f32(ds_sum / f32(n_haps))                                   # :185
        af[l] = f
        inf = f32(1.0)
        if fploidy == 2 and 0.0 < f < 1.0:                              # :186
            den = f64(f32(f32(n_haps) * f)) * (1.0 - f64(f))
            inf = f32(1.0 - f64(f32(ds4_sum - ds2_sum)) / den)
        inf = f32(0.0) if inf < 0 else inf                              # :187
        info[l] = f32(f64(_roundf(f32(f64(inf) * 1000.0))) / 1000.0)    # :188
    return gp, raf, af, info
