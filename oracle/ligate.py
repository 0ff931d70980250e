"""ORACLE — test infrastructure only.

Restatement of GLIMPSE2_ligate's phase-flip counting and allele swap
(ligate/src/ligater/ligater_algorithm.cpp): update_distances (:108-127), the
decision and phase quality of scan_overlap (:183-199), and phase_update
(:90-106), on htslib GT values (2 int32 per sample). The reference needs
htslib to read its chunks, so it is not built here; this restatement is pinned
by known answers read off those lines (tests/test_ligate.py). The phase quality
uses the C library's logf, as the reference does. Only tests/ use this module.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

VECTOR_END = -2147483647  # bcf_int32_vector_end

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.logf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]


def gt(allele, phased=True):
    """htslib GT value of one allele (bcf_gt_phased / bcf_gt_unphased); allele -1 = missing."""
    return ((allele + 1) << 1) | (1 if phased else 0)


def _missing(g):
    return (g >> 1) == 0


def _phased(g):
    return (g & 1) != 0


def _allele(g):
    return (g >> 1) - 1


def overlap(gta, gtb, swap_prev):
    gta = np.asarray(gta, np.int64)
    gtb = np.asarray(gtb, np.int64)
    m, n = gta.shape[0], gta.shape[1]
    nmatch = np.zeros(n, np.int32)
    nmism = np.zeros(n, np.int32)
    for s in range(m):
        for i in range(n):
            a0, a1 = int(gta[s, i, 0]), int(gta[s, i, 1])
            b0, b1 = int(gtb[s, i, 0]), int(gtb[s, i, 1])
            if a1 == VECTOR_END or b1 == VECTOR_END:
                continue
            if _missing(a0) or _missing(a1) or _missing(b0) or _missing(b1):
                continue
            if not _phased(a1) or not _phased(b1):
                continue
            x0, x1, y0, y1 = _allele(a0), _allele(a1), _allele(b0), _allele(b1)
            if x0 == x1 or y0 == y1:
                continue
            if x0 == y0 and x1 == y1:
                if swap_prev[i]:
                    nmism[i] += 1
                else:
                    nmatch[i] += 1
            if x0 == y1 and x1 == y0:
                if swap_prev[i]:
                    nmatch[i] += 1
                else:
                    nmism[i] += 1
    swap_next = (nmatch < nmism).astype(np.uint8)
    phaseq = np.full(n, 99.0, np.float32)
    for i in range(n):
        a, b = int(nmatch[i]), int(nmism[i])
        if a and b:
            f0 = np.float32(np.float32(a) / np.float32(a + b))
            t0 = np.float32(f0 * np.float32(_libm.logf(float(f0))))
            g = np.float32(np.float32(1.0) - f0)
            t1 = np.float32(g * np.float32(_libm.logf(float(g))))
            phaseq[i] = np.float32(99 * (0.7 + float(t0) + float(t1)) / 0.7)
    return swap_next, nmatch, nmism, phaseq


def swap(gt_arr, flags):
    out = np.array(gt_arr, np.int64, copy=True)
    m, n = out.shape[0], out.shape[1]
    for s in range(m):
        for i in range(n):
            if not flags[i]:
                continue
            g0, g1 = int(gt_arr[s, i, 0]), int(gt_arr[s, i, 1])
            if _missing(g0) or g1 == VECTOR_END:
                continue
            if not _phased(g1):
                continue
            out[s, i, 0] = gt(1 if _allele(g1) == 1 else 0)
            out[s, i, 1] = gt(1 if _allele(g0) == 1 else 0)
    return out.astype(np.int32)
