"""Ligation (GLIMPSE2_ligate, ligate/src/ligater/ligater_algorithm.cpp:90-205):
phase-flip counting over a chunk overlap and the allele swap that follows.

The CPU tests pin the restatement (oracle/ligate.py) with known answers read off
those lines; the GPU tests compare gp_ligate_overlap / gp_ligate_swap with it on
seeded GT arrays that mix phased and unphased hets, homozygotes, missing alleles,
haploid samples and a third allele."""
import numpy as np
import pytest

from oracle import ligate as G

VE = G.VECTOR_END


def _pair(a0, a1, phased=True):
    return [G.gt(a0, phased), G.gt(a1, phased)]


def test_counts_known_answers():
    # one sample, five overlap sites
    gta = np.array([[_pair(0, 1)], [_pair(0, 1)], [_pair(1, 1)], [_pair(0, 1, False)], [[G.gt(0), VE]]], np.int32)
    gtb = np.array([[_pair(0, 1)], [_pair(1, 0)], [_pair(1, 1)], [_pair(0, 1)], [[G.gt(0), VE]]], np.int32)
    sn, nmatch, nmism, pq = G.overlap(gta, gtb, [0])
    # site 0 matches, site 1 is swapped; homozygote, unphased and haploid sites are skipped
    assert (nmatch[0], nmism[0], sn[0]) == (1, 1, 0)
    sn, nmatch, nmism, pq = G.overlap(gta, gtb, [1])  # a swapped first chunk inverts the counts
    assert (nmatch[0], nmism[0]) == (1, 1)


def test_swap_decision_and_quality():
    gta = np.array([[_pair(0, 1)]] * 4, np.int32)
    gtb = np.array([[_pair(0, 1)], [_pair(1, 0)], [_pair(1, 0)], [_pair(1, 0)]], np.int32)
    sn, nmatch, nmism, pq = G.overlap(gta, gtb, [0])
    assert (nmatch[0], nmism[0], sn[0]) == (1, 3, 1)
    # f0 = 0.25: 99 (0.7 + 0.25 ln 0.25 + 0.75 ln 0.75) / 0.7 = 19.47
    assert abs(float(pq[0]) - 19.47) < 0.01
    sn, nmatch, nmism, pq = G.overlap(gta[:1], gtb[:1], [0])
    assert pq[0] == np.float32(99.0)  # one of the counts is zero


def test_swap_known_answers():
    g = np.array([[_pair(0, 1), _pair(1, 1), _pair(0, 1, False), _pair(0, 2), [G.gt(-1), G.gt(1)], [G.gt(1), VE]]],
                 np.int32)
    out = G.swap(g, [1, 1, 1, 1, 1, 1])
    assert out[0, 0].tolist() == _pair(1, 0)
    assert out[0, 1].tolist() == _pair(1, 1)
    assert out[0, 2].tolist() == g[0, 2].tolist()      # unphased: kept
    assert out[0, 3].tolist() == _pair(0, 0)           # alleles become (allele == 1): the third allele is lost
    assert out[0, 4].tolist() == g[0, 4].tolist()      # missing first allele: kept
    assert out[0, 5].tolist() == g[0, 5].tolist()      # haploid: kept
    assert G.swap(g, [0] * 6).tolist() == g.tolist()


def _random_gts(rng, m, n):
    a = rng.integers(0, 2, size=(m, n, 2))
    a[rng.random((m, n, 2)) < 0.03] = 2                 # a third allele
    ph = rng.random((m, n, 2)) < 0.9
    g = ((a + 1) << 1) | ph
    g[rng.random((m, n, 2)) < 0.03] = 0                 # missing (bcf_gt_missing)
    hap = rng.random(n) < 0.1
    g[:, hap, 1] = VE
    return g.astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n", [(1, 1), (500, 77), (64, 1025)])
def test_ligate_matches_restatement(small_workload, m, n):
    from glimpse_b200 import native
    rng = np.random.default_rng(m * 31 + n)
    gta, gtb = _random_gts(rng, m, n), _random_gts(rng, m, n)
    # make the second chunk mostly a consistent relabelling, so both decisions occur
    flip = rng.random(n) < 0.4
    gtb[:, flip] = gtb[:, flip][:, :, ::-1]
    same = rng.random((m, n)) < 0.6
    gtb[same] = gta[same]
    swap_prev = (rng.random(n) < 0.3).astype(np.uint8)
    ctx = native.Context(small_workload.panel)
    try:
        got = ctx.ligate_overlap(gta, gtb, swap_prev)
        swapped = ctx.ligate_swap(gtb, got[0])
    finally:
        ctx.close()
    want = G.overlap(gta, gtb, swap_prev)
    for name, x, y in zip(("swap_next", "nmatch", "nmism"), got[:3], want[:3]):
        assert np.array_equal(x, y), name
    assert np.array_equal(got[3].view(np.uint32), want[3].view(np.uint32)), "phaseq"
    assert np.array_equal(swapped, G.swap(gtb, want[0]))


@pytest.mark.gpu
def test_ligate_empty_overlap_is_an_error(small_workload):
    from glimpse_b200 import native
    ctx = native.Context(small_workload.panel)
    try:
        with pytest.raises(native.GpError, match="Overlap is empty"):
            ctx.ligate_overlap(np.zeros((0, 3, 2), np.int32), np.zeros((0, 3, 2), np.int32), np.zeros(3, np.uint8))
    finally:
        ctx.close()
