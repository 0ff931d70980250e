"""Output epilogue (genotype_writer::writeGenotypes, genotype_writer.cpp:110-190):
FORMAT/GP as written and the per-site RAF, AF and INFO.

The CPU tests pin the restatement (oracle/output_records.py) with known answers
read off those lines. The GPU tests run whole Gibbs runs and compare
gp_output_records with the restatement applied to the run's own finalised
posteriors, bit for bit (the fields are deterministic functions of them)."""
import dataclasses

import numpy as np
import pytest

from oracle import output_records as R

def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_gp_unchanged_when_floors_sum_to_one():
    for g0, g1, want in [(1.0, 0.0, (1.0, 0.0, 0.0)), (0.5, 0.5, (0.5, 0.5, 0.0)), (0.25, 0.75, (0.25, 0.75, 0.0))]:
        out, _, _ = R.gp_fields(g0, g1, 2, 2)
        assert out.tolist() == list(np.array(want, np.float32))


def test_gp_raises_largest_remainder_first():
    # haploid: floors 0.300 and 0.699 sum to 0.999; the key 1 - (gp - floor) of gp1 is smaller, so gp1 is raised
    out, _, _ = R.gp_fields(np.float32(0.3004), np.float32(0.6996), 1, 2)
    assert out[0] == np.float32(0.3)
    assert out[1] == np.float32(np.float32(0.699) + np.float32(0.001))
    assert _bits(out[2]) == R.VECTOR_END_BITS


def test_gp_equal_keys_are_raised_once():
    # both keys equal: the std::map keeps one entry, so only gp0 is raised and the sum stays below 0.9999
    g = np.float32(0.4995)
    out, _, _ = R.gp_fields(g, g, 1, 1)
    assert out[0] == np.float32(np.float32(0.499) + np.float32(0.001)) and out[1] == np.float32(0.499)


def test_info_known_answers():
    # two diploid targets at two sites; the second target has nothing stored (1, 0)
    gp0 = np.array([[0.0, 0.5], [1.0, 1.0]], np.float32)
    gp1 = np.array([[1.0, 0.5], [0.0, 0.0]], np.float32)
    gp, raf, af, info = R.output_records(gp0, gp1, [2, 2], calt=[3, 1], cref=[7, 9])
    assert raf.tolist() == [np.float32(0.3), np.float32(0.1)]
    assert af.tolist() == [np.float32(0.25), np.float32(0.125)]
    # site 0: 1 - (1 - 1) / (4 * 0.25 * 0.75) = 1; site 1: 1 - (0.5 - 0.25) / (4 * 0.125 * 0.875) = 0.4286 -> 0.429
    assert info.tolist() == [np.float32(1.0), np.float32(0.429)]


def test_info_is_one_for_mixed_ploidy():
    gp0 = np.array([[0.0], [0.5]], np.float32)
    gp1 = np.array([[1.0], [0.5]], np.float32)
    gp, raf, af, info = R.output_records(gp0, gp1, [2, 1], calt=[1], cref=[1])
    assert af[0] == np.float32(np.float32(1.5) / np.float32(3.0)) and info[0] == np.float32(1.0)
    assert _bits(gp[1, 0, 2]) == R.VECTOR_END_BITS


def test_exact_fmaf():
    # a = 1 + 2^-12: a * a - 1 = 2^-11 + 2^-24 exactly (a float32); the unfused product drops the 2^-24
    a = np.float32(1.0 + 2.0 ** -12)
    assert R.fmaf(a, a, -1.0) == np.float32(2.0 ** -11 + 2.0 ** -24)
    assert np.float32(a * a) - np.float32(1.0) == np.float32(2.0 ** -11)


def _check_run(w, kw, burnin=2, main=3):
    from glimpse_b200 import native
    P, T = w.panel, w.targets
    ctx = native.Context(P, **kw)
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.run(burnin, main)
        gp0, gp1, ds, gt0, gt1 = ctx.gp()
        gp, raf, af, info = ctx.output_records()
    finally:
        ctx.close()
    want = R.output_records(gp0, gp1, T.ploidy, P.calt, P.cref)
    for name, got, ref in zip(("gp", "raf", "af", "info"), (gp, raf, af, info), want):
        assert np.array_equal(_bits(got), _bits(ref)), f"{name}: {int((_bits(got) != _bits(ref)).sum())} differ"
    # DS of gp_gp_get is the written DS: AF is its mean over haplotypes before rounding
    assert np.allclose(af, ds.sum(0) / T.ploidy.sum(), atol=2e-3)


@pytest.mark.gpu
def test_output_records_match_restatement(small_workload):
    w = small_workload
    _check_run(w, dict(kinit=200, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05))


@pytest.mark.gpu
def test_output_records_mixed_ploidy(small_workload):
    w = small_workload
    T = dataclasses.replace(w.targets, ploidy=w.targets.ploidy.copy())
    T.ploidy[1] = 1
    w = dataclasses.replace(w, targets=T)
    _check_run(w, dict(kinit=200, kpbwt=int(T.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05))
