"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libglimpse_b200.so")
    config.addinivalue_line("markers", "slow: larger workloads")


def ref_oracle_or_skip():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return O


@pytest.fixture(scope="session")
def small_workload():
    from glimpse_b200 import synth
    return synth.make_panel_and_targets(600, 4000, 0.4, 0.5, 3, ("uniform", 0.5, 2.0), ("uniform", 80, 300),
                                        seed=7, sparse_maf=0.01, lq_frac=0.02, alt_major_frac=0.1)


def init_hl(gl, flat, ploidy=2, min_gl=1e-10, unphred=None):
    """genotype::initHaplotypeLikelihoods (genotype.cpp:56-91), in numpy float32/float64
    as the reference computes it (used to feed identical HL to both sides)."""
    if unphred is None:
        unphred = np.array([float("%.6e" % (10.0 ** (-i / 10.0))) for i in range(256)], np.float32)
    g = gl.astype(np.int64)
    t0 = unphred[g[:, 0]]
    t1 = unphred[g[:, 1]]
    t2 = unphred[g[:, 2]] if ploidy > 1 else np.zeros_like(t0)
    s = (t0 + t1).astype(np.float32) + t2
    t0, t1, t2 = t0 / s, t1 / s, t2 / s
    hl0 = (t0.astype(np.float64) + 0.5 * t1.astype(np.float64)).astype(np.float32)
    hl1 = (0.5 * t1.astype(np.float64) + t2.astype(np.float64)).astype(np.float32)
    f = flat.astype(bool)
    hl0[f] = 0.5
    hl1[f] = 0.5
    mg = np.float32(min_gl)
    m0 = hl0 < mg
    hl0[m0], hl1[m0] = mg, np.float32(1.0) - mg
    m1 = hl1 < mg
    hl0[m1], hl1[m1] = np.float32(1.0) - mg, mg
    out = np.empty(2 * gl.shape[0], np.float32)
    out[0::2] = hl0
    out[1::2] = hl1
    return out
