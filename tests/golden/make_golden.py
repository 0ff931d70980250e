"""Generates the fixtures in tests/golden/ from the reference's own compiled hot
path (oracle/_ref, built from the reference sources by oracle/Makefile).

Run from the repository root, in an environment where the reference tree is
present:  make -C oracle && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from glimpse_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402
from conftest import init_hl  # noqa: E402


def small_workload():
    return synth.make_panel_and_targets(600, 4000, 0.4, 0.5, 3, ("uniform", 0.5, 2.0), ("uniform", 80, 300),
                                        seed=7, sparse_maf=0.01, lq_frac=0.02, alt_major_frac=0.1)


def main():
    O.unphred_table().tofile(os.path.join(HERE, "unphred.f32"))

    streams = {"words": [], "floats": []}
    for seed, purpose, it, tgt, start in [(15052011, 1, 0, 0, 0), (15052011, 4, 7, 3, 1000), (1, 2, 20, 255, 5)]:
        streams["words"].append(dict(seed=seed, purpose=purpose, iteration=it, target=tgt, start=start,
                                     words=O.stream_words(seed, purpose, it, tgt, start, 16).tolist()))
        streams["floats"].append(dict(seed=seed, purpose=purpose, iteration=it, target=tgt,
                                      values=[float(x) for x in O.rng_floats(seed, purpose, it, tgt, 16)]))
    with open(os.path.join(HERE, "streams.json"), "w") as f:
        json.dump(streams, f, indent=1)

    w = small_workload()
    orc = O.RefOracle(w.panel, w.targets, kinit=200, kpbwt=150)
    rng = np.random.default_rng(99)
    cases = []
    for t, K in [(0, 9), (1, 120), (2, 333)]:
        s = np.sort(rng.choice(w.panel.n_ref_haps, K, replace=False)).astype(np.uint32)
        hl = init_hl(w.targets.gl[t], w.targets.flat[t])
        hp, _ = orc.impute(s, hl, w.targets.flat[t])
        cases.append(dict(target=t, states=s.tolist(), hp_ref=[float(x) for x in hp]))
    with open(os.path.join(HERE, "impute_cases.json"), "w") as f:
        json.dump({"cases": cases}, f)

    p = synth.make_panel_and_targets(400, 2000, 0.2, 0.6, 1, ("fixed", 1.0), ("fixed", 50), seed=5,
                                     sparse_maf=0.01, lq_frac=0.03, alt_major_frac=0.1).panel
    po = O.RefOracle(p)
    aoff, aidx = po.a_small_idx()
    np.savez_compressed(os.path.join(HERE, "pbwt_panel.npz"), N=p.n_ref_haps, L=p.n_sites, bp=p.bp, cm=p.cm,
                        cref=p.cref, calt=p.calt, lq=p.lq, flag_common=p.flag_common, major=p.major, hvar=p.hvar,
                        shap_off=p.shap_off, shap_sites=p.shap_sites, ypacked=po.ypacked(), asmall_off=aoff,
                        asmall_idx=aidx)


if __name__ == "__main__":
    main()
