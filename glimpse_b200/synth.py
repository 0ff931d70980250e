"""Seeded synthetic panels, targets and genotype likelihoods.

No public dataset ships with the project, so the GLIMPSE2_phase workloads are
generated: a reference panel of haplotypes copied as a Li-Stephens mosaic of a
few founders (with copying errors) at common sites, sparse rare alleles placed
on haplotypes that share a founder segment, held-out mosaic haplotypes paired
into diploid targets, and Poisson read counts turned into phred-scaled genotype
likelihoods the way the reference's GL reader does
(phase/src/io/genotype_reader.cpp:440-500: llk = lroundf(-10 * log10 GL),
clamped to 255; a site is flat when all likelihoods are equal).

The panel is returned in the reference's in-memory representation
(common/src/containers/ref_haplotype_set.h:60-75): per-site cref/calt, major
allele, common flag (MAF >= sparse_maf, genotype_reader.cpp:280-283), the
common-site bit matrix HvarRef (rows = common sites, MSB-first bytes) and the
rare-allele lists ShapRef (per reference haplotype, sites where it carries the
non-major allele).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Panel:
    n_ref_haps: int
    n_sites: int
    bp: np.ndarray          # int32 [L]
    cm: np.ndarray          # float64 [L], relative to the first site
    cref: np.ndarray        # uint32 [L]
    calt: np.ndarray        # uint32 [L]
    lq: np.ndarray          # uint8 [L]
    flag_common: np.ndarray  # uint8 [L]
    major: np.ndarray       # uint8 [L]
    hvar: np.ndarray        # uint8 [n_com, ceil(N/8)] MSB-first
    shap_off: np.ndarray    # int64 [N+1]
    shap_sites: np.ndarray  # int32 [nnz]

    @property
    def n_com(self) -> int:
        return int(self.flag_common.sum())


@dataclasses.dataclass
class Targets:
    n: int
    ploidy: np.ndarray      # int32 [n]
    gl: np.ndarray          # uint8 [n, L, 3] phred
    flat: np.ndarray        # uint8 [n, L]
    truth: np.ndarray       # uint8 [n, 2, L]
    coverage: np.ndarray    # float32 [n]
    kpbwt: np.ndarray       # int32 [n]


@dataclasses.dataclass
class Workload:
    name: str
    panel: Panel
    targets: Targets
    params: dict


# Workload shapes (sites, haplotypes, region, rare fraction, targets, coverage, K).
CONFIGS = {
    "small": dict(n_ref_haps=1000, n_sites=20000, region_mb=2.0, rare_frac=0.0, n_targets=1,
                  cov=("fixed", 1.0), k=("fixed", 500), kinit=500, n_founders=50),
    "batched": dict(n_ref_haps=10000, n_sites=150000, region_mb=4.0, rare_frac=0.8, n_targets=256,
                    cov=("uniform", 0.5, 2.0), k=("uniform", 400, 1200), kinit=1000, n_founders=50),
    "learned": dict(n_ref_haps=20000, n_sites=200000, region_mb=4.0, rare_frac=0.8, n_targets=512,
                    cov=("loguniform", 0.1, 4.0), k=("fixed", 800), kinit=1000, n_founders=50),
    "large": dict(n_ref_haps=100000, n_sites=400000, region_mb=5.0, rare_frac=0.85, n_targets=1000,
                  cov=("mix", (0.5, 0.6), (1.0, 0.3), (4.0, 0.1)), k=("uniform", 600, 2000), kinit=1000,
                  n_founders=50),
}


def _draw(spec, rng, n):
    kind = spec[0]
    if kind == "fixed":
        return np.full(n, spec[1], dtype=np.float64)
    if kind == "uniform":
        return rng.uniform(spec[1], spec[2], n)
    if kind == "loguniform":
        return np.exp(rng.uniform(math.log(spec[1]), math.log(spec[2]), n))
    if kind == "mix":
        vals = np.array([v for v, _ in spec[1:]])
        probs = np.array([p for _, p in spec[1:]])
        return vals[rng.choice(len(vals), size=n, p=probs / probs.sum())]
    raise ValueError(kind)


def make_panel_and_targets(n_ref_haps, n_sites, region_mb, rare_frac, n_targets, cov, k, kinit=1000,
                           n_founders=50, seed=1, maf_min=0.001, sparse_maf=0.001, mutation=0.01,
                           switches_per_cm=10.0, base_error=0.01, alt_major_frac=0.05, lq_frac=0.0,
                           name="custom"):
    """Generate one workload. Sizes follow the arguments; everything is seeded."""
    rng = np.random.default_rng(seed)
    N = int(n_ref_haps)
    L = int(n_sites)
    n_tar_haps = 2 * int(n_targets)
    n_all = N + n_tar_haps

    # Distinct sorted positions over the region, 1 cM/Mb, cM relative to the
    # first site (variant_map.cpp:151-157).
    span = int(region_mb * 1e6)
    bp = np.sort(rng.choice(np.arange(1, span + 1), size=L, replace=False)).astype(np.int32)
    cm = bp.astype(np.float64) / 1e6
    cm -= cm[0]

    n_rare = int(round(rare_frac * L))
    is_rare = np.zeros(L, dtype=bool)
    if n_rare:
        is_rare[rng.choice(L, size=n_rare, replace=False)] = True
    com_idx = np.flatnonzero(~is_rare)
    n_common = com_idx.size

    # Founder alleles at common sites: founder frequency from a 1/x spectrum on
    # [maf_min, 0.5] (inverse CDF), at least one founder carrying each allele.
    u = rng.random(n_common)
    p = maf_min * (0.5 / maf_min) ** u
    F = (rng.random((n_founders, n_common)) < p[None, :]).astype(np.uint8)
    none = F.sum(0) == 0
    F[rng.integers(0, n_founders, none.sum()), np.flatnonzero(none)] = 1
    flip = rng.random(n_common) < alt_major_frac
    F[:, flip] ^= 1

    # Mosaic paths: Poisson(switches_per_cm * length) switch points per hap.
    length_cm = float(cm[-1]) if L > 1 else 1.0
    com_cm = cm[com_idx]

    def founder_path(n_h):
        """Founder index per (hap, common site), uint8 [n_h, n_common]: Poisson
        switch points per haplotype, a fresh founder after each switch."""
        n_sw = rng.poisson(switches_per_cm * length_cm, n_h)
        tot = int(n_sw.sum())
        hap_of = np.repeat(np.arange(n_h), n_sw)
        sw_site = np.searchsorted(com_cm, rng.uniform(0.0, length_cm, tot), side="right")
        delta = np.zeros((n_h, n_common + 1), dtype=np.int16)
        np.add.at(delta, (hap_of, sw_site), 1)
        seg = np.cumsum(delta[:, :n_common], axis=1, dtype=np.int16)
        fids = rng.integers(0, n_founders, (n_h, int(n_sw.max()) + 1 if n_h else 1)).astype(np.uint8)
        return np.take_along_axis(fids, seg.astype(np.int64), axis=1)

    # Haplotypes processed in chunks of 8 so bits pack straight into HvarRef.
    stride = (N + 7) // 8
    hvar_all = np.zeros((n_common, (n_all + 7) // 8), dtype=np.uint8)
    tar_common = np.zeros((n_tar_haps, n_common), dtype=np.uint8)
    rare_idx = np.flatnonzero(is_rare)
    path_all = np.zeros((n_all, n_common), dtype=np.uint8) if rare_idx.size else None
    chunk = 2048
    for h0 in range(0, n_all, chunk):
        h1 = min(n_all, h0 + chunk)
        path = founder_path(h1 - h0)
        bits = F[path, np.arange(n_common)[None, :]]
        bits ^= (rng.random(bits.shape, dtype=np.float32) < mutation).astype(np.uint8)
        if path_all is not None:
            path_all[h0:h1] = path
        if h1 > N:
            lo = max(h0, N)
            tar_common[lo - N:h1 - N] = bits[lo - h0:h1 - h0]
        packed = np.packbits(bits.T, axis=1)  # [n_common, ceil((h1-h0)/8)]
        hvar_all[:, h0 // 8: h0 // 8 + packed.shape[1]] |= packed
    # panel-only HvarRef: clear padding bits beyond N in the last byte
    hvar = np.ascontiguousarray(hvar_all[:, :stride])
    if N % 8:
        hvar[:, -1] &= np.uint8((0xFF << (8 - N % 8)) & 0xFF)

    # Rare alleles: MAC from 1/x on [1, ceil(sparse_maf*N)-1]; carriers are
    # haplotypes that copy the origin's founder at the nearest common site,
    # found among random probes of the population.
    max_mac = max(1, int(math.ceil(sparse_maf * N)) - 1)
    rare_carriers = []
    tar_rare_carriers = []
    if rare_idx.size:
        nr = rare_idx.size
        anchor = np.searchsorted(com_idx, rare_idx).clip(0, max(n_common - 1, 0))
        macs = np.floor(np.exp(rng.uniform(0.0, math.log(max_mac + 1), nr))).astype(np.int64)
        macs = np.clip(macs, 1, max_mac)
        origin = rng.integers(0, N, nr)
        fo = path_all[origin, anchor]
        P = 64 * n_founders // 10 + 64
        probes = rng.integers(0, n_all, (nr, P))
        match = path_all[probes, anchor[:, None]] == fo[:, None]
        probes_ref = np.where(match & (probes < N), probes, -1)
        probes_tar = np.where(match & (probes >= N), probes - N, -1)
        # the origin always carries; other carriers are distinct matching probes in random order
        cand = np.concatenate([origin[:, None], probes_ref], axis=1)
        cand = np.sort(cand, axis=1)
        dup = np.zeros_like(cand, dtype=bool)
        dup[:, 1:] = cand[:, 1:] == cand[:, :-1]
        valid = (cand >= 0) & ~dup
        key = rng.random(cand.shape, dtype=np.float32)
        key[~valid] = 2.0
        key[(cand == origin[:, None]) & valid] = -1.0
        order = np.argsort(key, axis=1)
        cand = np.take_along_axis(cand, order, axis=1)
        valid = np.take_along_axis(valid, order, axis=1)
        take = valid & (np.arange(cand.shape[1])[None, :] < macs[:, None])
        tcand = np.sort(probes_tar, axis=1)
        tdup = np.zeros_like(tcand, dtype=bool)
        tdup[:, 1:] = tcand[:, 1:] == tcand[:, :-1]
        tkeep = (tcand >= 0) & ~tdup & (rng.random(tcand.shape, dtype=np.float32) <
                                         (macs / max(1.0, N / n_founders))[:, None])
        for j in range(nr):
            rare_carriers.append(np.sort(cand[j, take[j]]))
            tar_rare_carriers.append(tcand[j, tkeep[j]])
        del path_all, probes, match

    # Site counts and classes.
    calt = np.zeros(L, dtype=np.int64)
    if n_common:
        unpacked = np.unpackbits(hvar, axis=1, count=N)
        calt[com_idx] = unpacked.sum(1)
        del unpacked
    for j, s in enumerate(rare_idx):
        calt[s] = rare_carriers[j].size
    cref = N - calt
    # keep every common site polymorphic in the panel (the reference drops
    # monomorphic sites); rare sites always have their origin carrier
    if rare_idx.size and (calt[rare_idx] == 0).any():
        raise RuntimeError("rare site without a carrier")
    mono = np.flatnonzero(((calt == 0) | (cref == 0)) & ~is_rare)
    for s in mono:
        ci = int(np.searchsorted(com_idx, s))
        h = int(rng.integers(0, N))
        hvar[ci, h // 8] ^= np.uint8(1 << (7 - h % 8))
        calt[s] += 1 if calt[s] == 0 else -1
    cref = N - calt
    # common-generated sites whose minor count fell below the threshold get extra
    # minor-allele copies so that they stay in HvarRef
    need = int(math.ceil(sparse_maf * N))
    for s in com_idx[np.minimum(cref[com_idx], calt[com_idx]) < need]:
        ci = int(np.searchsorted(com_idx, s))
        row = np.unpackbits(hvar[ci], count=N)
        minor = 1 if calt[s] <= cref[s] else 0
        cand = np.flatnonzero(row != minor)
        add = rng.choice(cand, size=need - int(min(cref[s], calt[s])), replace=False)
        row[add] = minor
        hvar[ci] = np.packbits(row)[:stride]
        calt[s] = int(row.sum())
        cref[s] = N - calt[s]
    major = (calt > cref).astype(np.uint8)
    maf = np.minimum(cref, calt) / N
    flag_common = (maf >= sparse_maf).astype(np.uint8)
    if (flag_common[com_idx] == 0).any() or (flag_common[rare_idx] == 1).any():
        bad_c = com_idx[flag_common[com_idx] == 0]
        bad_r = rare_idx[flag_common[rare_idx] == 1]
        raise RuntimeError(f"site class drift: {bad_c.size} common->rare, {bad_r.size} rare->common")

    # ShapRef: per reference hap, rare sites where it carries the non-major allele.
    if rare_idx.size:
        pairs_h = np.concatenate(rare_carriers)
        pairs_s = np.concatenate([np.full(c.size, s, dtype=np.int64) for c, s in zip(rare_carriers, rare_idx)])
        # carriers hold the alt allele; when alt is major the non-major carriers are the others
        alt_major_rare = major[rare_idx] == 1
        if alt_major_rare.any():
            raise RuntimeError("rare site with alt as major allele")
        order = np.lexsort((pairs_s, pairs_h))
        pairs_h, pairs_s = pairs_h[order], pairs_s[order]
        shap_off = np.zeros(N + 1, dtype=np.int64)
        np.add.at(shap_off, pairs_h + 1, 1)
        shap_off = np.cumsum(shap_off)
        shap_sites = pairs_s.astype(np.int32)
    else:
        shap_off = np.zeros(N + 1, dtype=np.int64)
        shap_sites = np.zeros(0, dtype=np.int32)

    lq = np.zeros(L, dtype=np.uint8)
    if lq_frac > 0:
        lq[rng.random(L) < lq_frac] = 1

    panel = Panel(N, L, bp, cm, cref.astype(np.uint32), calt.astype(np.uint32), lq, flag_common, major, hvar,
                  shap_off, shap_sites)

    # Target truth haplotypes over all sites.
    truth_h = np.zeros((n_tar_haps, L), dtype=np.uint8)
    truth_h[:, com_idx] = tar_common
    for j, s in enumerate(rare_idx):
        truth_h[tar_rare_carriers[j], s] = 1
    nt = int(n_targets)
    truth = truth_h.reshape(nt, 2, L)

    # Reads -> GLs.
    covs = _draw(cov, rng, nt).astype(np.float32)
    gl = np.zeros((nt, L, 3), dtype=np.uint8)
    flat = np.zeros((nt, L), dtype=np.uint8)
    e = base_error
    g = np.array([0.0, 0.5, 1.0])
    p_alt_read = g * (1 - e) + (1 - g) * e  # P(read shows alt | genotype)
    l10_alt = np.log10(p_alt_read)
    l10_ref = np.log10(1 - p_alt_read)
    depth = rng.poisson(covs[:, None].astype(np.float64), (nt, L))
    from_h1 = rng.binomial(depth, 0.5)
    a0 = truth[:, 0].astype(np.int64)
    a1 = truth[:, 1].astype(np.int64)
    alt_true = (depth - from_h1) * a0 + from_h1 * a1
    ref_true = depth - alt_true
    alt_obs = rng.binomial(alt_true, 1 - e) + rng.binomial(ref_true, e)
    ref_obs = depth - alt_obs
    ll = (alt_obs[..., None] * l10_alt + ref_obs[..., None] * l10_ref).astype(np.float32)
    ll -= ll.max(-1, keepdims=True)
    gl[:] = np.minimum(np.rint(-10.0 * ll.astype(np.float64)), 255).astype(np.uint8)
    flat[:] = (gl[..., 0] == gl[..., 1]) & (gl[..., 0] == gl[..., 2])
    kp = np.rint(_draw(k, rng, nt)).astype(np.int32)
    targets = Targets(nt, np.full(nt, 2, dtype=np.int32), gl, flat, truth, covs, kp)
    params = dict(kinit=kinit, kpbwt=int(kp.max()), seed=seed)
    return Workload(name, panel, targets, params)


def workload(name: str, seed: int = 1, **overrides) -> Workload:
    cfg = dict(CONFIGS[name])
    cfg.update(overrides)
    return make_panel_and_targets(seed=seed, name=name, **cfg)


def dosage_r2(ds: np.ndarray, truth: np.ndarray) -> float:
    """Squared Pearson correlation of dosages vs true alt-allele counts over all
    (site, target) pairs (concordance/src/containers/call_set_writing.cpp:85-89,
    common/src/utils/basic_stats.h:120-125)."""
    x = np.asarray(ds, dtype=np.float64).ravel()
    y = np.asarray(truth, dtype=np.float64).ravel()
    if x.size < 2:
        return 0.0
    sx, sy = x.std(), y.std()
    if sx == 0 or sy == 0:
        return 0.0
    r = ((x - x.mean()) * (y - y.mean())).mean() / (sx * sy)
    return float(r * r)


# Allele-frequency bin edges of the r^2 report (GLIMPSE2_concordance --bins style).
MAF_BINS = (0.0, 0.001, 0.002, 0.005, 0.01, 0.02, 0.05, 0.1, 0.2, 0.5)


def dosage_r2_bins(ds: np.ndarray, truth: np.ndarray, maf: np.ndarray, edges=MAF_BINS):
    """Dosage r^2 per minor-allele-frequency bin, as GLIMPSE2_concordance
    reports it: a site goes to bin b when edges[b] < maf <= edges[b + 1]
    (call_set::getFrequencyBin, concordance/src/containers/call_set_header.h:216-221),
    and the bin's r^2 is the squared Pearson correlation of dosage and true
    alt-allele count over all its (site, target) pairs
    (call_set_reading.cpp:707, call_set_writing.cpp:245-249). ds, truth:
    [targets][sites]; maf: [sites]. Returns (low, high, sites, r^2) per bin."""
    ds = np.asarray(ds, np.float64)
    truth = np.asarray(truth, np.float64)
    maf = np.asarray(maf, np.float64)
    out = []
    for b in range(len(edges) - 1):
        sel = (maf > edges[b]) & (maf <= edges[b + 1])
        n = int(sel.sum())
        r2 = dosage_r2(ds[:, sel], truth[:, sel]) if n else float("nan")
        out.append((float(edges[b]), float(edges[b + 1]), n, r2))
    return out


def panel_maf(panel) -> np.ndarray:
    """Minor-allele frequency of every panel site from its allele counts."""
    cref = np.asarray(panel.cref, np.float64)
    calt = np.asarray(panel.calt, np.float64)
    return np.minimum(cref, calt) / np.maximum(cref + calt, 1.0)

