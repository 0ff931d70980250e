"""ORACLE — test infrastructure only.

ctypes bindings for
  * oracle/_ref/libglimpse_ref.so: the reference's own hot-path sources compiled
    unmodified (oracle/Makefile) behind a C-ABI harness (oracle/ref_harness.cpp),
    drawing from the replay streams the GPU path also uses;
  * oracle/_ref/libglimpse_ref_native.so: the same with the reference's own
    random-number generator (std::mt19937 seeded once, one thread);
  * oracle/_ref/librestate.so: the FP64/FP32 restatement (oracle/restate.c).

Only tests/, __graft_entry__.smoke() and bench.py's reference arm load this
module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.environ.get("GP_ORACLE_LIB", os.path.join(HERE, "_ref", "libglimpse_ref.so"))
REF_LIB_NATIVE = os.path.join(HERE, "_ref", "libglimpse_ref_native.so")
RESTATE_LIB = os.path.join(HERE, "_ref", "librestate.so")

STAGE_INIT, STAGE_BURN, STAGE_MAIN = 0, 1, 2

_ref = {}
_restate = None


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def ref_available(native_rng=False) -> bool:
    return os.path.exists(REF_LIB_NATIVE if native_rng else REF_LIB)


def ref_lib(native_rng=False):
    """The harness library: replay streams (default) or the reference's own generator."""
    if native_rng not in _ref:
        lib = C.CDLL(REF_LIB_NATIVE if native_rng else REF_LIB)
        vp = C.c_void_p
        lib.orc_create.restype = vp
        lib.orc_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint8),
                                   C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        lib.orc_destroy.argtypes = [vp]
        lib.orc_last_error.restype = C.c_char_p
        lib.orc_last_error.argtypes = [vp]
        lib.orc_ypacked.restype = C.c_int64
        lib.orc_ypacked.argtypes = [vp, C.POINTER(C.c_uint8), C.c_int64]
        lib.orc_asmall.restype = C.c_int64
        lib.orc_asmall.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.c_int64]
        lib.orc_asmall_rows.argtypes = [vp]
        lib.orc_targets.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]
        lib.orc_config.argtypes = [vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, C.c_int,
                                   C.c_int, C.POINTER(C.c_int), C.c_uint64]
        lib.orc_iteration.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        lib.orc_finalize.argtypes = [vp]
        lib.orc_get_haps.argtypes = [vp, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]
        lib.orc_set_haps.argtypes = [vp, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]
        lib.orc_get_gp.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                   C.POINTER(C.c_uint8)]
        lib.orc_last_states.argtypes = [vp, C.c_int, C.POINTER(C.c_uint32), C.c_int]
        lib.orc_last_hp.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.orc_pbwt_select.argtypes = [vp, C.c_int, C.c_int]
        lib.orc_pbwt_levels.argtypes = [vp, C.c_int]
        lib.orc_pbwt_states.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int32), C.c_int]
        lib.orc_pbwt_nstored.argtypes = [vp]
        lib.orc_pbwt_modulo.restype = C.c_float
        lib.orc_pbwt_modulo.argtypes = [vp]
        lib.orc_pbwt_groups.argtypes = [vp, C.POINTER(C.c_int32), C.c_int]
        lib.orc_select.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.c_int]
        lib.orc_init_select.argtypes = [vp, C.c_int]
        lib.orc_init_states.argtypes = [vp, C.c_int, C.POINTER(C.c_int32), C.c_int]
        lib.orc_state_lists.argtypes = [vp, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        lib.orc_impute.argtypes = [vp, C.POINTER(C.c_uint32), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                   C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        lib.orc_rephase.argtypes = [vp, C.POINTER(C.c_uint32), C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                    C.POINTER(C.c_uint8), C.c_int, C.c_int, C.POINTER(C.c_int32), C.c_int]
        lib.orc_unphred.argtypes = [C.POINTER(C.c_float)]
        lib.orc_stream_words.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int,
                                         C.POINTER(C.c_uint32)]
        if not native_rng:  # the shimmed class's stream draws exist in the replay build only
            lib.orc_rng_floats.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                           C.POINTER(C.c_float)]
            lib.orc_rng_ints.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                         C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint64)]
            lib.orc_std_sample.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                           C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]
        lib.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        lib.orc_native_rng.restype = C.c_int
        if lib.orc_native_rng() != int(bool(native_rng)):
            raise RuntimeError("oracle library built with the other random-number generator")
        _ref[native_rng] = lib
    return _ref[native_rng]


class RefOracle:
    """The reference's GLIMPSE2_phase hot path on the host (one object per panel).

    native_rng=True runs it with the reference's own generator (std::mt19937
    seeded once, caller_initialise.cpp:49; draws in the reference's call order,
    so on one thread only) in place of the replay streams; call-level parity
    with the GPU then no longer holds, only run-level statistics such as r2."""

    def __init__(self, panel, targets=None, *, ne=100000, err_imp=1e-12, err_phase=1e-4, min_gl=1e-10,
                 pbwt_depth=12, pbwt_modulo_cm=0.1, kinit=1000, kpbwt=2000, kpbwt_target=None, seed=15052011,
                 native_rng=False):
        lib = ref_lib(native_rng)
        self.native_rng = bool(native_rng)
        self.lib = lib
        self.panel = panel
        p = panel
        self._keep = [np.ascontiguousarray(x) for x in (p.bp.astype(np.int32), p.cm.astype(np.float64),
                                                        p.cref.astype(np.uint32), p.calt.astype(np.uint32),
                                                        p.lq.astype(np.uint8), p.flag_common.astype(np.uint8),
                                                        p.major.astype(np.uint8), p.hvar.astype(np.uint8),
                                                        p.shap_off.astype(np.int64), p.shap_sites.astype(np.int32))]
        k = self._keep
        self.h = lib.orc_create(p.n_ref_haps, p.n_sites, _p(k[0], C.c_int), _p(k[1], C.c_double),
                                _p(k[2], C.c_uint32), _p(k[3], C.c_uint32), _p(k[4], C.c_uint8), _p(k[5], C.c_uint8),
                                _p(k[6], C.c_uint8), _p(k[7], C.c_uint8), _p(k[8], C.c_int64), _p(k[9], C.c_int32))
        if not self.h:
            raise RuntimeError("orc_create failed")
        self.L = p.n_sites
        self.seed = seed
        self.n_targets = 0
        if targets is not None:
            self.set_targets(targets)
            self.configure(ne=ne, err_imp=err_imp, err_phase=err_phase, min_gl=min_gl, pbwt_depth=pbwt_depth,
                           pbwt_modulo_cm=pbwt_modulo_cm, kinit=kinit, kpbwt=kpbwt, kpbwt_target=kpbwt_target,
                           seed=seed)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error(self.h).decode())

    def ypacked(self) -> np.ndarray:
        n = self.lib.orc_ypacked(self.h, None, 0)
        out = np.zeros(n, dtype=np.uint8)
        self.lib.orc_ypacked(self.h, _p(out, C.c_uint8), n)
        return out

    def a_small_idx(self):
        rows = self.lib.orc_asmall_rows(self.h)
        off = np.zeros(rows + 1, dtype=np.int64)
        tot = self.lib.orc_asmall(self.h, _p(off, C.c_int64), None, 0)
        vals = np.zeros(max(tot, 1), dtype=np.int32)
        self.lib.orc_asmall(self.h, _p(off, C.c_int64), _p(vals, C.c_int32), tot)
        return off, vals[:tot]

    def set_targets(self, targets):
        self.targets = targets
        self.n_targets = targets.n
        self._tk = [np.ascontiguousarray(targets.ploidy.astype(np.int32)),
                    np.ascontiguousarray(targets.gl.astype(np.uint8)),
                    np.ascontiguousarray(targets.flat.astype(np.uint8))]
        self._check(self.lib.orc_targets(self.h, targets.n, _p(self._tk[0], C.c_int), _p(self._tk[1], C.c_uint8),
                                         _p(self._tk[2], C.c_uint8)))

    def configure(self, *, ne=100000, err_imp=1e-12, err_phase=1e-4, min_gl=1e-10, pbwt_depth=12,
                  pbwt_modulo_cm=0.1, kinit=1000, kpbwt=2000, kpbwt_target=None, seed=15052011):
        self.seed = seed
        kt = None
        if kpbwt_target is not None:
            kt = np.ascontiguousarray(np.asarray(kpbwt_target, dtype=np.int32))
            self._kt = kt
        self._check(self.lib.orc_config(self.h, ne, err_imp, err_phase, min_gl, pbwt_depth, pbwt_modulo_cm, kinit,
                                        kpbwt, _p(kt, C.c_int), seed))

    def iteration(self, stage, iter_index, threads=1):
        self._check(self.lib.orc_iteration(self.h, stage, iter_index, threads))

    def run(self, burnin=5, main=15, threads=1):
        it = 0
        self.iteration(STAGE_INIT, it, threads)
        it += 1
        for _ in range(burnin):
            self.iteration(STAGE_BURN, it, threads)
            it += 1
        for _ in range(main):
            self.iteration(STAGE_MAIN, it, threads)
            it += 1
        self._check(self.lib.orc_finalize(self.h))

    def haps(self, ind):
        h0 = np.zeros(self.L, dtype=np.uint8)
        h1 = np.zeros(self.L, dtype=np.uint8)
        self.lib.orc_get_haps(self.h, ind, _p(h0, C.c_uint8), _p(h1, C.c_uint8))
        return h0, h1

    def set_haps(self, ind, h0, h1):
        h0 = np.ascontiguousarray(h0, dtype=np.uint8)
        h1 = np.ascontiguousarray(h1, dtype=np.uint8)
        self.lib.orc_set_haps(self.h, ind, _p(h0, C.c_uint8), _p(h1, C.c_uint8))

    def gp(self, ind):
        L = self.L
        gp0 = np.zeros(L, np.float32)
        gp1 = np.zeros(L, np.float32)
        hds = np.zeros(L, np.uint8)
        st = np.zeros(L, np.uint8)
        cnt = self.lib.orc_get_gp(self.h, ind, _p(gp0, C.c_float), _p(gp1, C.c_float), _p(hds, C.c_uint8),
                                  _p(st, C.c_uint8))
        return gp0, gp1, hds, st, cnt

    def last_states(self, ind):
        out = np.zeros(self.panel.n_ref_haps, np.uint32)
        n = self.lib.orc_last_states(self.h, ind, _p(out, C.c_uint32), out.size)
        return out[:n].copy()

    def last_hp(self, ind):
        hp0 = np.zeros(2 * self.L, np.float32)
        hp1 = np.zeros(2 * self.L, np.float32)
        npoly = self.lib.orc_last_hp(self.h, ind, _p(hp0, C.c_float), _p(hp1, C.c_float))
        return hp0, hp1, npoly

    def pbwt_select(self, iter_index, main_iteration=False):
        self._check(self.lib.orc_pbwt_select(self.h, iter_index, int(main_iteration)))

    def pbwt_states(self, ind):
        lv = self.lib.orc_pbwt_levels(self.h, ind)
        out = []
        buf = np.zeros(1 << 20, np.int32)
        for i in range(lv):
            n = self.lib.orc_pbwt_states(self.h, ind, i, _p(buf, C.c_int32), buf.size)
            out.append(buf[:n].copy())
        return out

    def pbwt_groups(self):
        buf = np.zeros(1 << 20, np.int32)
        n = self.lib.orc_pbwt_groups(self.h, _p(buf, C.c_int32), buf.size)
        return buf[:n].copy(), float(self.lib.orc_pbwt_modulo(self.h))

    def select(self, ind, stage):
        out = np.zeros(self.panel.n_ref_haps, np.uint32)
        n = self.lib.orc_select(self.h, ind, stage, _p(out, C.c_uint32), out.size)
        if n < 0:
            raise RuntimeError(self.lib.orc_last_error(self.h).decode())
        return out[:n].copy()

    def init_select(self, iter_index=0):
        self._check(self.lib.orc_init_select(self.h, iter_index))

    def set_state_lists(self, lists):
        """Per target haplotype (rows of --state-list), reference haplotype ids;
        None or [] clears."""
        lists = lists or []
        off = np.zeros(len(lists) + 1, np.int64)
        off[1:] = np.cumsum([len(x) for x in lists])
        ids = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in lists]) if lists
                                   else np.zeros(1, np.int32))
        self._check(self.lib.orc_state_lists(self.h, len(lists), _p(off, C.c_int64), _p(ids, C.c_int32)))

    def init_states(self, ind):
        out = np.zeros(self.panel.n_ref_haps, np.int32)
        n = self.lib.orc_init_states(self.h, ind, _p(out, C.c_int32), out.size)
        return out[:n].copy()

    def impute(self, states, HL, flat):
        states = np.ascontiguousarray(states, dtype=np.uint32)
        HL = np.ascontiguousarray(HL, dtype=np.float32)
        flat = np.ascontiguousarray(flat, dtype=np.uint8)
        HP = np.zeros(2 * self.L, np.float32)
        poly = np.zeros(self.L, np.int32)
        n = self.lib.orc_impute(self.h, _p(states, C.c_uint32), states.size, _p(HL, C.c_float), _p(flat, C.c_uint8),
                                _p(HP, C.c_float), _p(poly, C.c_int32))
        if n < 0:
            raise RuntimeError(self.lib.orc_last_error(self.h).decode())
        return HP, poly[:n].copy()

    def rephase(self, states, H0, H1, flat, iter_index, target):
        states = np.ascontiguousarray(states, dtype=np.uint32)
        H0 = np.array(H0, dtype=np.uint8, copy=True)
        H1 = np.array(H1, dtype=np.uint8, copy=True)
        flat = np.ascontiguousarray(flat, dtype=np.uint8)
        dip = np.zeros(1 << 20, np.int32)
        n = self.lib.orc_rephase(self.h, _p(states, C.c_uint32), states.size, _p(H0, C.c_uint8), _p(H1, C.c_uint8),
                                 _p(flat, C.c_uint8), iter_index, target, _p(dip, C.c_int32), dip.size)
        if n < 0:
            raise RuntimeError(self.lib.orc_last_error(self.h).decode())
        return H0, H1, dip[:n].copy()


def unphred_table() -> np.ndarray:
    out = np.zeros(256, np.float32)
    ref_lib().orc_unphred(_p(out, C.c_float))
    return out


def stream_words(seed, purpose, iteration, target, start, n):
    out = np.zeros(n, np.uint32)
    ref_lib().orc_stream_words(seed, purpose, iteration, target, start, n, _p(out, C.c_uint32))
    return out


def rng_floats(seed, purpose, iteration, target, n):
    out = np.zeros(n, np.float32)
    ref_lib().orc_rng_floats(seed, purpose, iteration, target, n, _p(out, C.c_float))
    return out


def rng_ints(seed, purpose, iteration, target, lo, hi):
    lo = np.ascontiguousarray(lo, np.uint32)
    hi = np.ascontiguousarray(hi, np.uint32)
    out = np.zeros(lo.size, np.uint32)
    used = C.c_uint64(0)
    ref_lib().orc_rng_ints(seed, purpose, iteration, target, lo.size, _p(lo, C.c_uint32), _p(hi, C.c_uint32),
                           _p(out, C.c_uint32), C.byref(used))
    return out, used.value


def std_sample(seed, purpose, iteration, target, pop, n):
    out = np.zeros(max(n, 1), np.int32)
    used = C.c_uint64(0)
    k = ref_lib().orc_std_sample(seed, purpose, iteration, target, pop, n, _p(out, C.c_int32), C.byref(used))
    return out[:k].copy(), used.value


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    ref_lib().orc_philox(_p(c, C.c_uint32), _p(k, C.c_uint32), _p(out, C.c_uint32))
    return out


def restate_lib():
    global _restate
    if _restate is None:
        lib = C.CDLL(RESTATE_LIB)
        lib.rs_impute.restype = C.c_double
        lib.rs_impute.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                  C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.c_int,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_uint32), C.c_int,
                                  C.c_double, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                  C.POINTER(C.c_float)]
        lib.rs_state_post.restype = None
        lib.rs_state_post.argtypes = [C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                      C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.c_int,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_uint32), C.c_int,
                                      C.c_double, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                      C.POINTER(C.c_int32), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
        _restate = lib
    return _restate


def restate_impute(panel, states, HL, flat, precision=64, ne=100000, err_imp=1e-12):
    """FP64 (or FP32) restatement of imputation_hmm::computePosteriors; returns (HP, loglik)."""
    lib = restate_lib()
    L = panel.n_sites
    comrow = np.full(L, -1, np.int32)
    com = np.flatnonzero(panel.flag_common)
    comrow[com] = np.arange(com.size, dtype=np.int32)
    keep = [np.ascontiguousarray(x) for x in (panel.flag_common.astype(np.uint8), panel.lq.astype(np.uint8),
                                              panel.major.astype(np.uint8), panel.cm.astype(np.float64), comrow,
                                              panel.hvar.astype(np.uint8), panel.shap_off.astype(np.int64),
                                              panel.shap_sites.astype(np.int32),
                                              np.asarray(states, np.uint32), np.asarray(HL, np.float32),
                                              np.asarray(flat, np.uint8))]
    HP = np.zeros(2 * L, np.float32)
    err = float(np.clip(np.float32(err_imp), np.float32(1e-12), np.float32(1e-3)))
    ed = np.float32(err)
    ee = np.float32(1.0 - float(ed))
    nrho = (-0.04 * ne) / panel.n_ref_haps
    ll = lib.rs_impute(precision, L, _p(keep[0], C.c_uint8), _p(keep[1], C.c_uint8), _p(keep[2], C.c_uint8),
                       _p(keep[3], C.c_double), _p(keep[4], C.c_int32), _p(keep[5], C.c_uint8),
                       (panel.n_ref_haps + 7) // 8, _p(keep[6], C.c_int64), _p(keep[7], C.c_int32),
                       _p(keep[8], C.c_uint32), keep[8].size, nrho, float(ed), float(ee), _p(keep[9], C.c_float),
                       _p(keep[10], C.c_uint8), _p(HP, C.c_float))
    return HP, ll


def panel_windows(panel, win_sites=256):
    """Window of every panel site for the learned proposal: that of the last
    common site at or before it, windows of win_sites common sites."""
    com = np.asarray(panel.flag_common, bool)
    r = np.cumsum(com) - 1
    return (np.maximum(r, 0) // win_sites).astype(np.int32), max(1, (int(com.sum()) + win_sites - 1) // win_sites)


def restate_state_post(panel, states, HL, flat, ne=100000, err_imp=1e-12):
    """FP64 per-window state posteriors (mass (nwin, K), nsites (nwin,))."""
    lib = restate_lib()
    L = panel.n_sites
    comrow = np.full(L, -1, np.int32)
    com = np.flatnonzero(panel.flag_common)
    comrow[com] = np.arange(com.size, dtype=np.int32)
    sw, nwin = panel_windows(panel)
    keep = [np.ascontiguousarray(x) for x in (panel.flag_common.astype(np.uint8), panel.lq.astype(np.uint8),
                                              panel.major.astype(np.uint8), panel.cm.astype(np.float64), comrow,
                                              panel.hvar.astype(np.uint8), panel.shap_off.astype(np.int64),
                                              panel.shap_sites.astype(np.int32),
                                              np.asarray(states, np.uint32), np.asarray(HL, np.float32),
                                              np.asarray(flat, np.uint8), sw)]
    K = keep[8].size
    mass = np.zeros(nwin * K, np.float64)
    ns = np.zeros(nwin, np.int32)
    err = float(np.clip(np.float32(err_imp), np.float32(1e-12), np.float32(1e-3)))
    ed = np.float32(err)
    ee = np.float32(1.0 - float(ed))
    lib.rs_state_post(L, _p(keep[0], C.c_uint8), _p(keep[1], C.c_uint8), _p(keep[2], C.c_uint8),
                      _p(keep[3], C.c_double), _p(keep[4], C.c_int32), _p(keep[5], C.c_uint8),
                      (panel.n_ref_haps + 7) // 8, _p(keep[6], C.c_int64), _p(keep[7], C.c_int32),
                      _p(keep[8], C.c_uint32), K, (-0.04 * ne) / panel.n_ref_haps, float(ed), float(ee),
                      _p(keep[9], C.c_float), _p(keep[10], C.c_uint8), _p(keep[11], C.c_int32), nwin,
                      _p(mass, C.c_double), _p(ns, C.c_int32))
    return mass.reshape(nwin, K), ns
