"""The accuracy metrics the bench reports: dosage r^2 overall and per
minor-allele-frequency bin, with GLIMPSE2_concordance's bin rule (a site goes
to bin b when edges[b] < maf <= edges[b + 1], call_set_header.h:216-221)."""
import numpy as np

from glimpse_b200 import synth


def test_dosage_r2_is_squared_pearson():
    rng = np.random.default_rng(1)
    truth = rng.integers(0, 3, size=(5, 200)).astype(np.float64)
    ds = truth + rng.normal(0, 0.3, size=truth.shape)
    r = np.corrcoef(ds.ravel(), truth.ravel())[0, 1]
    assert abs(synth.dosage_r2(ds, truth) - r * r) < 1e-12


def test_dosage_r2_bins_follow_the_concordance_rule():
    rng = np.random.default_rng(2)
    maf = np.array([0.0, 0.0005, 0.001, 0.0015, 0.01, 0.3, 0.5, 0.05])
    truth = rng.integers(0, 3, size=(6, maf.size)).astype(np.float64)
    ds = truth + rng.normal(0, 0.2, size=truth.shape)
    bins = synth.dosage_r2_bins(ds, truth, maf)
    assert [b[:2] for b in bins] == list(zip(synth.MAF_BINS[:-1], synth.MAF_BINS[1:]))
    counts = {(lo, hi): n for lo, hi, n, _ in bins}
    assert counts[(0.0, 0.001)] == 2        # 0.0005 and 0.001 (upper edge included); maf 0 is in no bin
    assert counts[(0.001, 0.002)] == 1
    assert counts[(0.005, 0.01)] == 1
    assert counts[(0.02, 0.05)] == 1
    assert counts[(0.2, 0.5)] == 2
    for lo, hi, n, r2 in bins:
        sel = (maf > lo) & (maf <= hi)
        if n:
            assert abs(r2 - synth.dosage_r2(ds[:, sel], truth[:, sel])) < 1e-12
        else:
            assert np.isnan(r2)


def test_panel_maf_from_allele_counts():
    p = type("P", (), {})()
    p.cref = np.array([990, 5, 500, 0], np.uint32)
    p.calt = np.array([10, 995, 500, 0], np.uint32)
    assert np.allclose(synth.panel_maf(p), [0.01, 0.005, 0.5, 0.0])
