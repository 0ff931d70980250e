"""Target GL input (genotype_reader::readTargetGenotypes, genotype_reader.cpp:427-500):
FORMAT/PL or FORMAT/GL per (site, sample) -> phred bytes and flat flags.

The CPU tests pin the numpy restatement (oracle/gl_input.py) with known answers
read off those lines: clamping at 255, lroundf's rounding half away from zero,
htslib's missing and vector-end markers, the per-site value-count check, the
haploid layout, and the first invalid entry in site-then-sample order. The GPU
tests compare gp_gl_from_pl / gp_gl_from_float with the restatement, bit for
bit, on seeded inputs that mix all of these."""
import numpy as np
import pytest

from oracle import gl_input as G

M, VE = G.PL_MISSING, G.PL_VECTOR_END
F_MISSING = np.array([G.GL_MISSING_BITS], np.uint32).view(np.float32)[0]
F_VECTOR_END = np.array([G.GL_VECTOR_END_BITS], np.uint32).view(np.float32)[0]


def test_pl_known_answers():
    # sites x samples x 3; samples 0 and 2 diploid, sample 1 haploid
    pl = np.array([[[0, 10, 300], [3, 7, VE], [5, 5, 5]],
                   [[M, 3, 4], [4, 4, VE], [1, 2, 3]]], np.int32)
    gl, flat = G.gl_input("PL", pl, [2, 1, 2])
    assert gl.tolist() == [[[0, 10, 255], [0, 0, 0]], [[3, 7, 0], [4, 4, 0]], [[5, 5, 5], [1, 2, 3]]]
    assert flat.tolist() == [[0, 1], [0, 1], [1, 0]]


def test_pl_vector_end_in_a_diploid_third_value_skips_the_entry():
    pl = np.array([[[1, 2, VE]]], np.int32)
    gl, flat = G.gl_input("PL", pl, [2])
    assert gl.tolist() == [[[0, 0, 0]]] and flat.tolist() == [[1]]


def test_site_value_count_mismatch_skips_the_site():
    pl = np.array([[[1, 2, 3], [4, 5, 6]], [[7, 8, 9], [1, 1, 1]]], np.int32)
    gl, flat = G.gl_input("PL", pl, [2, 2], site_nval=[4, 6])  # site 0: 4 / 2 = 2 values per sample != 3
    assert gl[:, 0].tolist() == [[0, 0, 0], [0, 0, 0]] and flat[:, 0].tolist() == [1, 1]
    assert gl[:, 1].tolist() == [[7, 8, 9], [1, 1, 1]] and flat[:, 1].tolist() == [0, 1]


def test_gl_rounding_known_answers():
    vals = [-0.0, -1.0, -3.25, -0.05, -0.04, -30.0, 0.01, -25.44]
    want = [0, 10, 33, 1, 0, 255, 0, 254]  # 32.5 -> 33 and 0.5 -> 1 (half away from zero); 0.01 -> -0.1 -> 0
    src = np.array([[[v, v, v]] for v in vals], np.float32)
    gl, flat = G.gl_input("GL", src, [2])
    assert gl[0, :, 0].tolist() == want
    assert flat[0].tolist() == [1] * len(vals)


def test_gl_missing_markers_keep_defaults():
    src = np.array([[[F_MISSING, -1.0, -2.0]], [[-1.0, -2.0, F_VECTOR_END]]], np.float32)
    gl, flat = G.gl_input("GL", src, [2])
    assert gl.tolist() == [[[0, 0, 0], [0, 0, 0]]] and flat.tolist() == [[1, 1]]


@pytest.mark.parametrize("fmt,bad", [("PL", -1), ("GL", 0.1), ("GL", float("nan")), ("GL", float("-inf"))])
def test_first_invalid_entry_is_reported(fmt, bad):
    dt = np.int32 if fmt == "PL" else np.float32
    good = 5 if fmt == "PL" else -0.5
    src = np.full((3, 4, 3), good, dt)
    src[2, 0, 1] = bad
    src[1, 3, 2] = bad  # the first in site-then-sample order
    with pytest.raises(G.GlInputError) as ei:
        G.gl_input(fmt, src, [2, 2, 2, 2])
    assert (ei.value.site, ei.value.sample) == (1, 3)


def _random_case(rng, fmt, n, L, haploid_frac=0.3, absent_frac=0.05, nval_bad_frac=0.03):
    ploidy = np.where(rng.random(n) < haploid_frac, 1, 2).astype(np.int32)
    ploidy[0] = 2
    if fmt == "PL":
        src = rng.integers(0, 400, size=(L, n, 3)).astype(np.int32)
        equal = rng.random((L, n)) < 0.2
        src[equal] = src[equal][:, :1]
        ab = rng.random((L, n, 3)) < absent_frac
        src[ab] = np.where(rng.random(ab.sum()) < 0.5, M, VE)
    else:
        src = (-rng.uniform(0, 40, size=(L, n, 3))).astype(np.float32)
        half = rng.random((L, n, 3)) < 0.1  # exact x.5 after the product by -10
        src[half] = (-(rng.integers(0, 300, half.sum()) + 0.5) / 10).astype(np.float32)
        tiny = rng.random((L, n, 3)) < 0.02  # 0 <= GL < 0.05: rounds to phred 0, accepted
        src[tiny] = rng.uniform(0, 0.0499, tiny.sum()).astype(np.float32)
        equal = rng.random((L, n)) < 0.2
        src[equal] = src[equal][:, :1]
        ab = rng.random((L, n, 3)) < absent_frac
        src[ab] = np.where(rng.random(ab.sum()) < 0.5, F_MISSING, F_VECTOR_END)
    site_nval = np.full(L, n * 3, np.int32)
    site_nval[rng.random(L) < nval_bad_frac] = n * 2
    return src, ploidy, site_nval


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["PL", "GL"])
@pytest.mark.parametrize("n,L", [(1, 1), (37, 1000), (64, 33), (5, 4097)])
def test_gl_input_matches_oracle(small_workload, fmt, n, L):
    from glimpse_b200 import native
    rng = np.random.default_rng(n * 7919 + L)
    src, ploidy, site_nval = _random_case(rng, fmt, n, L)
    ctx = native.Context(small_workload.panel)
    try:
        for nv in (site_nval, None):
            want_gl, want_flat = G.gl_input(fmt, src, ploidy, nv)
            gl, flat = ctx.gl_from_format(fmt, src, ploidy, nv)
            assert np.array_equal(gl, want_gl) and np.array_equal(flat, want_flat)
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,bad", [("PL", -3), ("GL", 0.2)])
def test_gl_input_reports_first_invalid_entry(small_workload, fmt, bad):
    from glimpse_b200 import native
    rng = np.random.default_rng(3)
    src, ploidy, _ = _random_case(rng, fmt, 40, 300, absent_frac=0.0)
    src[200, 5, 0] = bad
    src[17, 39, 1] = bad
    ctx = native.Context(small_workload.panel)
    try:
        with pytest.raises(native.GpError, match=r"target \[39\] at site \[17\]"):
            ctx.gl_from_format(fmt, src, ploidy)
        # the context stays usable after the refusal
        src[200, 5, 0] = src[17, 39, 1] = 0 if fmt == "PL" else -0.0
        gl, flat = ctx.gl_from_format(fmt, src, ploidy)
        want_gl, want_flat = G.gl_input(fmt, src, ploidy)
        assert np.array_equal(gl, want_gl) and np.array_equal(flat, want_flat)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gl_input_batched_shape(small_workload):
    """256 diploid targets x 150,000 sites of PL (the batched workload's shape)."""
    from glimpse_b200 import native
    rng = np.random.default_rng(5)
    n, L = 256, 150_000
    src = rng.integers(0, 300, size=(L, n, 3), dtype=np.int32)
    src[rng.random((L, n)) < 0.3] = 0
    ploidy = np.full(n, 2, np.int32)
    ctx = native.Context(small_workload.panel)
    try:
        gl, flat = ctx.gl_from_format("PL", src, ploidy)
    finally:
        ctx.close()
    want_gl, want_flat = G.gl_input("PL", src, ploidy)
    assert np.array_equal(gl, want_gl) and np.array_equal(flat, want_flat)
