"""CPU tests of the oracle and of the host side of the library (no GPU needed).

The reference ships no tests, fixtures or known-answer vectors for this path,
so the oracle is pinned by (a) published known-answer vectors of the stream
generator (Philox4x32-10, Random123 kat_vectors), (b) the committed fixtures in
tests/golden/ produced by the reference's own compiled code, and (c) the
reference's compiled hot path itself (oracle/_ref) where it is built."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, init_hl

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _ref():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    return O


def test_philox_known_answers():
    O = _ref()
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in kat:
        assert list(O.philox(ctr, key)) == want


def test_stream_words_golden():
    O = _ref()
    with open(os.path.join(GOLDEN, "streams.json")) as f:
        g = json.load(f)
    for case in g["words"]:
        got = O.stream_words(case["seed"], case["purpose"], case["iteration"], case["target"], case["start"],
                             len(case["words"]))
        assert got.tolist() == case["words"]
    for case in g["floats"]:
        got = O.rng_floats(case["seed"], case["purpose"], case["iteration"], case["target"], len(case["values"]))
        assert np.array_equal(got, np.array(case["values"], np.float32))


def test_unphred_table_matches_reference():
    """The library tabulates unphred as printf('%.6e') of 10^(-i/10) read back as
    float; it must equal the reference's literal table (otools.h:98)."""
    ref = np.fromfile(os.path.join(GOLDEN, "unphred.f32"), dtype=np.float32)
    mine = np.array([float("%.6e" % (10.0 ** (-i / 10.0))) for i in range(256)], np.float32)
    assert np.array_equal(ref, mine)
    O = _ref()
    assert np.array_equal(O.unphred_table(), ref)


def test_restatement_pinned_to_reference(small_workload):
    """FP32/FP64 restatement (oracle/restate.c) vs imputation_hmm::computePosteriors."""
    O = _ref()
    w = small_workload
    orc = O.RefOracle(w.panel, w.targets, kinit=200, kpbwt=150)
    rng = np.random.default_rng(2)
    for t in range(w.targets.n):
        for K in (7, 64, 300):
            s = np.sort(rng.choice(w.panel.n_ref_haps, K, replace=False)).astype(np.uint32)
            hl = init_hl(w.targets.gl[t], w.targets.flat[t])
            ref, _ = orc.impute(s, hl, w.targets.flat[t])
            f32, _ = O.restate_impute(w.panel, s, hl, w.targets.flat[t], 32)
            f64, _ = O.restate_impute(w.panel, s, hl, w.targets.flat[t], 64)
            assert np.abs(f32 - ref).max() <= 1e-5
            assert np.abs(f64 - ref).max() <= 1e-5


def test_golden_posteriors(small_workload):
    """Reference posteriors committed as fixtures reproduce through the restatement."""
    O = _ref()
    with open(os.path.join(GOLDEN, "impute_cases.json")) as f:
        g = json.load(f)
    w = small_workload
    for case in g["cases"]:
        s = np.array(case["states"], np.uint32)
        t = case["target"]
        hl = init_hl(w.targets.gl[t], w.targets.flat[t])
        hp = np.array(case["hp_ref"], np.float32)
        f64, _ = O.restate_impute(w.panel, s, hl, w.targets.flat[t], 64)
        assert np.abs(f64 - hp).max() <= 1e-5


def test_sparse_pbwt_builder_bit_exact(small_workload):
    """The library's host sparse-PBWT builder against ref_haplotype_set::build_sparsePBWT."""
    O = _ref()
    from glimpse_b200 import native
    w = small_workload
    orc = O.RefOracle(w.panel)
    y, aoff, aidx = native.build_sparse_pbwt(w.panel)
    ro, rv = orc.a_small_idx()
    assert np.array_equal(y, orc.ypacked())
    assert np.array_equal(aoff, ro) and np.array_equal(aidx, rv)


def test_sparse_pbwt_golden():
    """Builder output on the committed fixture panel equals the reference's bytes."""
    from glimpse_b200 import native
    d = np.load(os.path.join(GOLDEN, "pbwt_panel.npz"))
    from glimpse_b200.synth import Panel
    p = Panel(int(d["N"]), int(d["L"]), d["bp"], d["cm"], d["cref"], d["calt"], d["lq"], d["flag_common"], d["major"],
              d["hvar"], d["shap_off"], d["shap_sites"])
    y, aoff, aidx = native.build_sparse_pbwt(p)
    assert np.array_equal(y, d["ypacked"])
    assert np.array_equal(aoff, d["asmall_off"]) and np.array_equal(aidx, d["asmall_idx"])


def test_inconsistent_panel_is_rejected(small_workload):
    """A panel whose counts disagree with its bits fails with GP_E_DATA instead of
    reading or writing out of bounds."""
    from glimpse_b200 import native
    import copy
    p = copy.deepcopy(small_workload.panel)
    com = np.flatnonzero(p.flag_common)
    p.calt = p.calt.copy()
    p.cref = p.cref.copy()
    p.calt[com[3]] += 1
    p.cref[com[3]] -= 1
    with pytest.raises(native.GpError):
        native.build_sparse_pbwt(p)


def test_library_exports_header_symbols():
    """Every function declared in include/glimpse_b200.h is exported by the library."""
    import ctypes
    import re
    from glimpse_b200 import native
    with open(os.path.join(ROOT, "include", "glimpse_b200.h")) as f:
        hdr = f.read()
    names = set(re.findall(r"\b(gp_[a-z_0-9]+)\s*\(", hdr))
    lib = native.lib()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(native.EXPORTS) <= names


def test_reference_driver_runs(small_workload):
    """The restated reference driver runs a whole (short) Gibbs run."""
    O = _ref()
    from glimpse_b200 import synth
    w = small_workload
    orc = O.RefOracle(w.panel, w.targets, kinit=200, kpbwt=int(w.targets.kpbwt.max()),
                      kpbwt_target=w.targets.kpbwt, pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc.run(burnin=1, main=2)
    ds = []
    for t in range(w.targets.n):
        g0, g1, hds, st, cnt = orc.gp(t)
        assert cnt == 2
        ds.append(g1 + 2 * np.clip(1 - g0 - g1, 0, 1))
    assert synth.dosage_r2(np.stack(ds), w.targets.truth.sum(1)) > 0.5


def test_reference_with_its_own_generator():
    """The native-RNG oracle build runs the reference with its own std::mt19937
    (random_number.h:35-125, seeded once as caller_initialise.cpp:49). The run is
    reproducible for a seed, draws differently from the replay streams, reaches
    the same dosage r2 within sampling noise, and refuses more than one thread
    (the reference's generator is one global stream)."""
    from oracle import oracle as O
    if not O.ref_available(native_rng=True):
        pytest.skip("oracle/_ref native build missing")
    from glimpse_b200 import synth
    w = synth.make_panel_and_targets(800, 6000, 1.0, 0.5, 4, ("uniform", 0.5, 2.0), ("fixed", 150), seed=7,
                                     sparse_maf=0.005)
    kw = dict(kinit=300, kpbwt=150, pbwt_depth=8, pbwt_modulo_cm=0.05)
    truth = w.targets.truth.sum(1)

    def run(native):
        orc = O.RefOracle(w.panel, w.targets, native_rng=native, **kw)
        orc.run(burnin=5, main=15)
        ds = []
        for t in range(w.targets.n):
            g0, g1, _, _, _ = orc.gp(t)
            ds.append(g1 + 2 * np.clip(1 - g0 - g1, 0, 1))
        return np.stack(ds)

    a, b, replay = run(True), run(True), run(False)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, replay)
    assert abs(synth.dosage_r2(a, truth) - synth.dosage_r2(replay, truth)) <= 0.01
    orc = O.RefOracle(w.panel, w.targets, native_rng=True, **kw)
    with pytest.raises(RuntimeError, match="one thread"):
        orc.iteration(O.STAGE_INIT, 0, threads=2)


def test_reference_state_lists(small_workload):
    """The reference's --state-list path as the oracle runs it
    (conditioning_set.cpp:114-121): every set holds the union of its target's
    rows, sorted without duplicates; with Kinit = Kpbwt = 0 it is that union."""
    O = _ref()
    P, T = small_workload.panel, small_workload.targets
    rng = np.random.default_rng(2)
    lists = [np.sort(rng.choice(P.n_ref_haps, int(rng.integers(1, 30)), replace=False)).astype(np.int32)
             for _ in range(int(T.ploidy.sum()))]
    first = np.concatenate([[0], np.cumsum(T.ploidy)])
    for kinit, kp in ((200, 150), (0, 0)):
        orc = O.RefOracle(P, T, kinit=kinit, kpbwt=kp, kpbwt_target=np.full(T.n, kp, np.int32), pbwt_depth=8,
                          pbwt_modulo_cm=0.05)
        orc.set_state_lists(lists)
        for stage, it in ((O.STAGE_INIT, 0), (O.STAGE_BURN, 1)):
            orc.iteration(stage, it)
            for t in range(T.n):
                s = orc.last_states(t).astype(np.int64)
                rows = np.unique(np.concatenate(lists[first[t]:first[t + 1]]))
                assert np.all(np.diff(s) > 0) and np.isin(rows, s).all()
                if kinit == 0:
                    assert np.array_equal(s, rows)
