"""ORACLE — test infrastructure only.

numpy restatement of the target GL input of
genotype_reader::readTargetGenotypes (phase/src/io/genotype_reader.cpp:427-500):
FORMAT/PL (int32) or FORMAT/GL (float) per (site, sample) into phred bytes and
flat flags, with the defaults of genotype::allocate (genotype.cpp:50-51).

The reference reads these arrays through htslib inside its VCF reader, which is
not built here (htslib is absent), so this restatement is checked against
known-answer cases derived from those lines (tests/test_gl_input.py), not
against the reference binary. Only tests/ use this module.

Input layout, as htslib returns a site's FORMAT values: src[l, i, c] for site l,
sample i, value c < P, with P = max(ploidy) + 1. site_nval[l] is htslib's
value count for site l (None: n * P everywhere).
"""
from __future__ import annotations

import numpy as np

PL_MISSING = np.int32(-2147483648)      # bcf_int32_missing
PL_VECTOR_END = np.int32(-2147483647)   # bcf_int32_vector_end
GL_MISSING_BITS = 0x7F800001            # bcf_float_missing
GL_VECTOR_END_BITS = 0x7F800002         # bcf_float_vector_end


class GlInputError(ValueError):
    """A negative PL or a positive GL; site and sample of the first one in
    site-then-sample order (the reference stops with vrb.error there)."""

    def __init__(self, fmt, site, sample):
        super().__init__(f"FORMAT/{fmt}: invalid value at site {site}, sample {sample}")
        self.site, self.sample = site, sample


def _phred_pl(v: np.ndarray) -> np.ndarray:
    return v.astype(np.int64)


def _phred_gl(v: np.ndarray) -> np.ndarray:
    """lroundf(-10 * GL) (genotype_reader.cpp:446-448): a float32 product, then
    rounding half away from zero; NaN, infinities and |y| >= 2^63 give LONG_MIN
    on x86-64 (here -1: rejected either way)."""
    with np.errstate(invalid="ignore", over="ignore"):
        y = (np.float32(-10.0) * v.astype(np.float32)).astype(np.float64)
    ok = np.isfinite(y) & (np.abs(y) < 2.0 ** 63)
    r = np.where(ok, np.sign(y) * np.floor(np.abs(np.where(ok, y, 0.0)) + 0.5), -1.0)
    return r.astype(np.int64)


def _absent(fmt, v):
    if fmt == "PL":
        return (v == PL_MISSING) | (v == PL_VECTOR_END)
    b = v.astype(np.float32).view(np.uint32)
    return (b == GL_MISSING_BITS) | (b == GL_VECTOR_END_BITS)


def gl_input(fmt: str, src: np.ndarray, ploidy: np.ndarray, site_nval=None):
    """Returns gl (n, L, 3) uint8 and flat (n, L) uint8; raises GlInputError.
    Vectorised over all (site, sample) entries; each step cites its line."""
    ploidy = np.asarray(ploidy, np.int32)
    n = ploidy.size
    P = int(ploidy.max()) + 1
    L = src.shape[0]
    assert src.shape == (L, n, P)
    dip = (ploidy > 1)[None, :]
    site_ok = np.ones(L, bool) if site_nval is None else (np.asarray(site_nval, np.int64) // n == P)  # :433-435
    ab = _absent(fmt, src)
    use = site_ok[:, None] & ~ab[:, :, 0] & ~ab[:, :, 1]                      # :441-442, :481-482
    if P == 3:
        use &= ~(dip & ab[:, :, 2])                                           # :443, :483
    ph = (_phred_pl if fmt == "PL" else _phred_gl)(src)                       # :446-448
    ph2 = ph[:, :, 2] if P == 3 else np.zeros_like(ph[:, :, 0])
    bad = use & ((ph[:, :, 0] < 0) | (ph[:, :, 1] < 0) | (dip & (ph2 < 0)))   # :450-454, :485-489
    if bad.any():
        first = int(np.argmax(bad.ravel()))                                   # site-then-sample order
        raise GlInputError(fmt, first // n, first % n)
    g0 = np.clip(ph[:, :, 0], 0, 255)                                         # :456-459, :491-494
    g1 = np.clip(ph[:, :, 1], 0, 255)
    g2 = np.where(dip, np.clip(ph2, 0, 255), 0)
    glast = np.where(dip, g2, g1)                                             # gl[ploidy]
    fl = (g0 == g1) & (g0 == glast)                                           # :458-459, :495-496
    gl = np.zeros((n, L, 3), np.uint8)                                        # genotype.cpp:50
    gl[:, :, 0] = np.where(use, g0, 0).T
    gl[:, :, 1] = np.where(use, g1, 0).T
    gl[:, :, 2] = np.where(use, g2, 0).T
    flat = np.where(use, fl, True).T.astype(np.uint8)                         # genotype.cpp:51
    return np.ascontiguousarray(gl), np.ascontiguousarray(flat)
