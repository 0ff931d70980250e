"""ctypes binding of libglimpse_b200.so (the C-ABI declared in include/glimpse_b200.h).

There is no CPU fallback: every call runs on the GPU, and loading fails loudly
when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libglimpse_b200.so")

GP_OK = 0
STAGE_INIT, STAGE_BURN, STAGE_MAIN = 0, 1, 2

# Symbols declared in include/glimpse_b200.h.
EXPORTS = [
    "gp_config_defaults", "gp_ctx_create", "gp_ctx_destroy", "gp_last_error", "gp_targets_set", "gp_iteration",
    "gp_run", "gp_haps_get", "gp_haps_set", "gp_posteriors_get", "gp_states_get", "gp_finalize", "gp_gp_get",
    "gp_impute_batch", "gp_rephase_batch", "gp_select", "gp_pbwt_states_get", "gp_sparse_pbwt_get",
    "gp_stage_times", "gp_build_sparse_pbwt", "gp_profile_get", "gp_profile_reset", "gp_stream",
    "gp_impute_one_static",
    "gp_targets_reset", "gp_gl_from_pl", "gp_gl_from_float", "gp_output_records", "gp_ligate_overlap",
    "gp_ligate_swap", "gp_gp_accum_get",
    "gp_mlp_param_count", "gp_mlp_init", "gp_mlp_set_params", "gp_mlp_get_params", "gp_mlp_forward",
    "gp_mlp_train_step", "gp_learned_enable", "gp_learned_train", "gp_learned_windows", "gp_state_posteriors",
    "gp_set_precision", "gp_loglik_get", "gp_tuning_set", "gp_tuning_get", "gp_learned_size",
    "gp_state_lists_set",
]
PRECISION_FULL, PRECISION_CKPT_F32, PRECISION_CKPT_BF16 = 0, 1, 2


class gp_profile(C.Structure):
    _fields_ = [
        ("impute_ms", C.c_double), ("impute_cells", C.c_double), ("impute_bytes", C.c_double),
        ("phase_ms", C.c_double), ("phase_cells", C.c_double), ("select_ms", C.c_double),
        ("impute_launches", C.c_int64), ("phase_launches", C.c_int64), ("kernel_launches", C.c_int64),
        ("mlp_ms", C.c_double), ("mlp_rows", C.c_double), ("mlp_launches", C.c_int64),
    ]


class gp_panel_desc(C.Structure):
    _fields_ = [
        ("n_ref_haps", C.c_int32), ("n_sites", C.c_int32), ("cm", C.POINTER(C.c_double)),
        ("cref", C.POINTER(C.c_uint32)), ("calt", C.POINTER(C.c_uint32)), ("lq", C.POINTER(C.c_uint8)),
        ("flag_common", C.POINTER(C.c_uint8)), ("major", C.POINTER(C.c_uint8)), ("hvar", C.POINTER(C.c_uint8)),
        ("shap_off", C.POINTER(C.c_int64)), ("shap_sites", C.POINTER(C.c_int32)),
        ("ypacked", C.POINTER(C.c_uint8)), ("ypacked_len", C.c_int64), ("asmall_off", C.POINTER(C.c_int64)),
        ("asmall_idx", C.POINTER(C.c_int32)),
    ]


class gp_config(C.Structure):
    _fields_ = [
        ("ne", C.c_int32), ("err_imp", C.c_float), ("err_phase", C.c_float), ("min_gl", C.c_float),
        ("pbwt_depth", C.c_int32), ("pbwt_modulo_cm", C.c_float), ("kinit", C.c_int32), ("kpbwt", C.c_int32),
        ("seed", C.c_uint64), ("device", C.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m glimpse_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _lib.gp_last_error.restype = C.c_char_p
        _lib.gp_last_error.argtypes = [C.c_void_p]
        _lib.gp_stream.restype = C.c_void_p
        _lib.gp_stream.argtypes = [C.c_void_p]
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class GpError(RuntimeError):
    pass


def _panel_desc(p, keep, ypacked=None, asmall=None):
    keep.update(cm=np.ascontiguousarray(p.cm, np.float64), cref=np.ascontiguousarray(p.cref, np.uint32),
                calt=np.ascontiguousarray(p.calt, np.uint32), lq=np.ascontiguousarray(p.lq, np.uint8),
                common=np.ascontiguousarray(p.flag_common, np.uint8), major=np.ascontiguousarray(p.major, np.uint8),
                hvar=np.ascontiguousarray(p.hvar, np.uint8), soff=np.ascontiguousarray(p.shap_off, np.int64),
                ssites=np.ascontiguousarray(p.shap_sites, np.int32))
    k = keep
    d = gp_panel_desc()
    d.n_ref_haps, d.n_sites = p.n_ref_haps, p.n_sites
    d.cm, d.cref, d.calt = _p(k["cm"], C.c_double), _p(k["cref"], C.c_uint32), _p(k["calt"], C.c_uint32)
    d.lq, d.flag_common, d.major = _p(k["lq"], C.c_uint8), _p(k["common"], C.c_uint8), _p(k["major"], C.c_uint8)
    d.hvar, d.shap_off, d.shap_sites = _p(k["hvar"], C.c_uint8), _p(k["soff"], C.c_int64), _p(k["ssites"], C.c_int32)
    if ypacked is not None:
        k["yp"] = np.ascontiguousarray(ypacked, np.uint8)
        d.ypacked, d.ypacked_len = _p(k["yp"], C.c_uint8), k["yp"].size
    if asmall is not None:
        k["aoff"] = np.ascontiguousarray(asmall[0], np.int64)
        k["aidx"] = np.ascontiguousarray(asmall[1], np.int32)
        d.asmall_off, d.asmall_idx = _p(k["aoff"], C.c_int64), _p(k["aidx"], C.c_int32)
    return d


def build_sparse_pbwt(panel):
    """Host-only sparse PBWT of a panel: (ypacked, asmall_off, asmall_idx)."""
    L = lib()
    keep = {}
    d = _panel_desc(panel, keep)
    ylen = C.c_int64(0)
    alen = C.c_int64(0)
    rc = L.gp_build_sparse_pbwt(C.byref(d), None, C.byref(ylen), None, None, C.byref(alen))
    if rc != GP_OK:
        raise GpError(f"gp_build_sparse_pbwt failed with status {rc}")
    n_com_hq = int(((panel.flag_common != 0) & (panel.lq == 0)).sum())
    yp = np.zeros(max(ylen.value, 1), np.uint8)
    aoff = np.zeros(n_com_hq + 2, np.int64)
    aidx = np.zeros(max(alen.value, 1), np.int32)
    rc = L.gp_build_sparse_pbwt(C.byref(d), _p(yp, C.c_uint8), C.byref(ylen), _p(aoff, C.c_int64),
                                _p(aidx, C.c_int32), C.byref(alen))
    if rc != GP_OK:
        raise GpError(f"gp_build_sparse_pbwt failed with status {rc}")
    return yp[:ylen.value], aoff, aidx[:alen.value]


class Context:
    """One device-resident panel plus its targets (a gp_ctx)."""

    def __init__(self, panel, *, ne=100000, err_imp=1e-12, err_phase=1e-4, min_gl=1e-10, pbwt_depth=12,
                 pbwt_modulo_cm=0.1, kinit=1000, kpbwt=2000, seed=15052011, device=0, ypacked=None,
                 asmall=None):
        L = lib()
        self.lib = L
        self.panel = panel
        cfg = gp_config()
        L.gp_config_defaults(C.byref(cfg))
        cfg.ne, cfg.err_imp, cfg.err_phase, cfg.min_gl = ne, err_imp, err_phase, min_gl
        cfg.pbwt_depth, cfg.pbwt_modulo_cm, cfg.kinit, cfg.kpbwt = pbwt_depth, pbwt_modulo_cm, kinit, kpbwt
        cfg.seed, cfg.device = seed, device
        self.cfg = cfg
        p = panel
        self._keep = {}
        d = _panel_desc(p, self._keep, ypacked, asmall)
        h = C.c_void_p()
        rc = L.gp_ctx_create(C.byref(d), C.byref(cfg), C.byref(h))
        if rc != GP_OK:
            raise GpError(f"gp_ctx_create failed with status {rc}")
        self.h = h
        self.L = p.n_sites
        self.N = p.n_ref_haps
        self.n_targets = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.gp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc != GP_OK:
            raise GpError(f"status {rc}: {self.lib.gp_last_error(self.h).decode()}")

    # ---- call-level entry points ----
    def impute_batch(self, states_list, hl, flat):
        """imputation_hmm::computePosteriors for len(states_list) haplotypes."""
        n = len(states_list)
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in states_list])
        st = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint32) for s in states_list]), np.uint32)
        hl = np.ascontiguousarray(hl, np.float32).reshape(n, 2 * self.L)
        flat = np.ascontiguousarray(flat, np.uint8).reshape(n, self.L)
        hp = np.zeros((n, 2 * self.L), np.float32)
        self._check(self.lib.gp_impute_batch(self.h, n, _p(off, C.c_int64), _p(st, C.c_uint32), _p(hl, C.c_float),
                                             _p(flat, C.c_uint8), _p(hp, C.c_float)))
        return hp

    def impute_one_static(self, states, hl, flat):
        """gp_impute_one_static: one haplotype, scratch in the library's fixed device region."""
        st = np.ascontiguousarray(states, np.uint32)
        hl = np.ascontiguousarray(hl, np.float32).reshape(2 * self.L)
        flat = np.ascontiguousarray(flat, np.uint8).reshape(self.L)
        hp = np.zeros(2 * self.L, np.float32)
        self._check(self.lib.gp_impute_one_static(self.h, st.size, _p(st, C.c_uint32), _p(hl, C.c_float),
                                                  _p(flat, C.c_uint8), _p(hp, C.c_float)))
        return hp

    def ligate_overlap(self, gta, gtb, swap_prev):
        """gp_ligate_overlap: gta, gtb (m, n, 2) int32 htslib GT values; swap_prev (n,).
        Returns swap_next, nmatch, nmism, phaseq."""
        gta = np.ascontiguousarray(gta, np.int32)
        gtb = np.ascontiguousarray(gtb, np.int32)
        m, n = gta.shape[0], gta.shape[1]
        sp = np.ascontiguousarray(swap_prev, np.uint8)
        sn = np.zeros(n, np.uint8)
        nmatch, nmism = np.zeros(n, np.int32), np.zeros(n, np.int32)
        pq = np.zeros(n, np.float32)
        self._check(self.lib.gp_ligate_overlap(self.h, n, m, _p(gta, C.c_int32), _p(gtb, C.c_int32), _p(sp, C.c_uint8),
                                               _p(sn, C.c_uint8), _p(nmatch, C.c_int32), _p(nmism, C.c_int32),
                                               _p(pq, C.c_float)))
        return sn, nmatch, nmism, pq

    def ligate_swap(self, gt, swap):
        """gp_ligate_swap on a copy of gt (m, n, 2) int32; returns the swapped copy."""
        gt = np.array(gt, np.int32, copy=True, order="C")
        m, n = gt.shape[0], gt.shape[1]
        sw = np.ascontiguousarray(swap, np.uint8)
        self._check(self.lib.gp_ligate_swap(self.h, n, m, _p(gt, C.c_int32), _p(sw, C.c_uint8)))
        return gt

    def output_records(self):
        """gp_output_records after finalize: gp (n, L, 3) float32 as written, and per
        site raf, af, info (L,) float32."""
        n, L = self.n_targets, self.L
        gp = np.zeros((n, L, 3), np.float32)
        raf, af, info = (np.zeros(L, np.float32) for _ in range(3))
        self._check(self.lib.gp_output_records(self.h, _p(gp, C.c_float), _p(raf, C.c_float), _p(af, C.c_float),
                                               _p(info, C.c_float)))
        return gp, raf, af, info

    def gl_from_format(self, fmt, src, ploidy, site_nval=None):
        """gp_gl_from_pl (fmt "PL", int32 values) or gp_gl_from_float (fmt "GL",
        float values): src[l, i, c] for site l, target i, value c < max(ploidy) + 1.
        Returns gl (n, L, 3) uint8 and flat (n, L) uint8."""
        ploidy = np.ascontiguousarray(ploidy, np.int32)
        n = ploidy.size
        L = src.shape[0]
        dt, ct, fn = ((np.int32, C.c_int32, self.lib.gp_gl_from_pl) if fmt == "PL"
                      else (np.float32, C.c_float, self.lib.gp_gl_from_float))
        src = np.ascontiguousarray(src, dt)
        nval = None if site_nval is None else np.ascontiguousarray(site_nval, np.int32)
        gl = np.zeros((n, L, 3), np.uint8)
        flat = np.zeros((n, L), np.uint8)
        self._check(fn(self.h, n, L, _p(src, ct), _p(nval, C.c_int32), _p(ploidy, C.c_int32), _p(gl, C.c_uint8),
                       _p(flat, C.c_uint8)))
        return gl, flat

    def rephase_batch(self, states_list, h0, h1, flat, iteration, target_ids=None):
        """phasing_hmm::rephaseHaplotypes for len(states_list) diploid targets."""
        n = len(states_list)
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in states_list])
        st = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint32) for s in states_list]), np.uint32)
        h0 = np.array(h0, np.uint8, copy=True).reshape(n, self.L)
        h1 = np.array(h1, np.uint8, copy=True).reshape(n, self.L)
        flat = np.ascontiguousarray(flat, np.uint8).reshape(n, self.L)
        ids = None if target_ids is None else np.ascontiguousarray(target_ids, np.int32)
        self._check(self.lib.gp_rephase_batch(self.h, n, _p(off, C.c_int64), _p(st, C.c_uint32), _p(h0, C.c_uint8),
                                              _p(h1, C.c_uint8), _p(flat, C.c_uint8), iteration,
                                              _p(ids, C.c_int32)))
        return h0, h1

    # ---- target-level entry points ----
    def set_targets(self, targets, kpbwt=None):
        n = targets.n
        self.n_targets = n
        self._tk = dict(gl=np.ascontiguousarray(targets.gl, np.uint8), flat=np.ascontiguousarray(targets.flat, np.uint8),
                        ploidy=np.ascontiguousarray(targets.ploidy, np.int32))
        kp = None
        if kpbwt is not None:
            kp = np.ascontiguousarray(np.broadcast_to(np.asarray(kpbwt, np.int32), (n,)), np.int32)
            self._tk["kp"] = kp
        self._check(self.lib.gp_targets_set(self.h, n, _p(self._tk["gl"], C.c_uint8), _p(self._tk["flat"], C.c_uint8),
                                            _p(self._tk["ploidy"], C.c_int32), _p(kp, C.c_int32)))

    def set_state_lists(self, lists):
        """gp_state_lists_set: per target haplotype (targets in order, ploidy rows
        each), the reference haplotype ids always in its target's conditioning
        sets (the reference's --state-list rows). None or [] clears them."""
        lists = lists or []
        off = np.zeros(len(lists) + 1, np.int64)
        off[1:] = np.cumsum([len(x) for x in lists])
        ids = (np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in lists])) if lists
               else np.zeros(1, np.int32))
        self._check(self.lib.gp_state_lists_set(self.h, len(lists), _p(off, C.c_int64), _p(ids, C.c_int32)))

    def iteration(self, stage, iteration):
        self._check(self.lib.gp_iteration(self.h, stage, iteration))

    def select(self, stage, iteration):
        self._check(self.lib.gp_select(self.h, stage, iteration))

    def run(self, burnin=5, main=15):
        self._check(self.lib.gp_run(self.h, burnin, main))

    def finalize(self):
        self._check(self.lib.gp_finalize(self.h))

    def haps(self):
        h0 = np.zeros((self.n_targets, self.L), np.uint8)
        h1 = np.zeros((self.n_targets, self.L), np.uint8)
        self._check(self.lib.gp_haps_get(self.h, _p(h0, C.c_uint8), _p(h1, C.c_uint8)))
        return h0, h1

    def set_haps(self, h0, h1):
        h0 = np.ascontiguousarray(h0, np.uint8)
        h1 = np.ascontiguousarray(h1, np.uint8)
        self._check(self.lib.gp_haps_set(self.h, _p(h0, C.c_uint8), _p(h1, C.c_uint8)))

    def posteriors(self, target):
        hp0 = np.zeros(2 * self.L, np.float32)
        hp1 = np.zeros(2 * self.L, np.float32)
        self._check(self.lib.gp_posteriors_get(self.h, target, _p(hp0, C.c_float), _p(hp1, C.c_float)))
        return hp0, hp1

    def states(self, target):
        out = np.zeros(self.N, np.uint32)
        n = C.c_int32(0)
        self._check(self.lib.gp_states_get(self.h, target, _p(out, C.c_uint32), C.byref(n)))
        return out[:n.value].copy()

    def pbwt_states(self, target, depth=None):
        depth = depth or self.cfg.pbwt_depth
        counts = np.zeros(depth, np.int32)
        buf = np.zeros(1 << 22, np.int32)
        self._check(self.lib.gp_pbwt_states_get(self.h, target, _p(counts, C.c_int32), _p(buf, C.c_int32), buf.size))
        out, o = [], 0
        for c in counts:
            out.append(buf[o:o + c].copy())
            o += c
        return out

    def gp(self):
        shape = (self.n_targets, self.L)
        gp0, gp1, ds = (np.zeros(shape, np.float32) for _ in range(3))
        gt0, gt1 = np.zeros(shape, np.uint8), np.zeros(shape, np.uint8)
        self._check(self.lib.gp_gp_get(self.h, _p(gp0, C.c_float), _p(gp1, C.c_float), _p(ds, C.c_float),
                                       _p(gt0, C.c_uint8), _p(gt1, C.c_uint8)))
        return gp0, gp1, ds, gt0, gt1

    def gp_accum(self, target):
        """gp_gp_accum_get: (gp0, gp1, flags) of one target, dense over the sites."""
        gp0, gp1 = np.zeros(self.L, np.float32), np.zeros(self.L, np.float32)
        fl = np.zeros(self.L, np.uint8)
        self._check(self.lib.gp_gp_accum_get(self.h, target, _p(gp0, C.c_float), _p(gp1, C.c_float),
                                             _p(fl, C.c_uint8)))
        return gp0, gp1, fl

    # ---- learned state-selection proposal: the scoring network ----
    def mlp_init(self, seed=1):
        self._check(self.lib.gp_mlp_init(self.h, C.c_uint64(seed)))

    def mlp_params(self):
        p = np.zeros(self.lib.gp_mlp_param_count(), np.float32)
        self._check(self.lib.gp_mlp_get_params(self.h, _p(p, C.c_float)))
        return p

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.gp_mlp_set_params(self.h, _p(p, C.c_float)))

    def mlp_forward(self, x, hidden=False):
        """Scores of feature rows x (n, 48); with hidden=True also the BF16 hidden activations."""
        x = np.ascontiguousarray(x, np.float32)
        n = x.shape[0]
        sc = np.zeros(n, np.float32)
        h1 = np.zeros((n, 256), np.float32) if hidden else None
        h2 = np.zeros((n, 256), np.float32) if hidden else None
        self._check(self.lib.gp_mlp_forward(self.h, n, _p(x, C.c_float), _p(sc, C.c_float), _p(h1, C.c_float),
                                            _p(h2, C.c_float)))
        return (sc, h1, h2) if hidden else sc

    def mlp_train_step(self, x, y, wt=None, lr=0.0, grad=False):
        """One step; returns (loss, grad or None)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        wt = None if wt is None else np.ascontiguousarray(wt, np.float32)
        g = np.zeros(self.lib.gp_mlp_param_count(), np.float32) if grad else None
        loss = C.c_float(0.0)
        self._check(self.lib.gp_mlp_train_step(self.h, x.shape[0], _p(x, C.c_float), _p(y, C.c_float),
                                               _p(wt, C.c_float), C.c_float(lr), C.byref(loss), _p(g, C.c_float)))
        return loss.value, g

    def tuning_set(self, chains_per_cta=0, sweep_haps_per_warp=0, phase_placement=0):
        self._check(self.lib.gp_tuning_set(self.h, chains_per_cta, sweep_haps_per_warp, phase_placement))

    def tuning(self):
        """(chains per CTA, haplotypes per sweep warp, phasing placement, measured ms[9]) of the autotuner."""
        a, b, c = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        ms = np.zeros(9, np.float32)
        self._check(self.lib.gp_tuning_get(self.h, C.byref(a), C.byref(b), C.byref(c), _p(ms, C.c_float)))
        return a.value, b.value, c.value, ms

    def set_precision(self, mode):
        """gp_set_precision: PRECISION_FULL, PRECISION_CKPT_F32 or PRECISION_CKPT_BF16."""
        self._check(self.lib.gp_set_precision(self.h, mode))

    def loglik(self, n):
        """gp_loglik_get: FP64 chunk log-likelihoods of the last checkpointed imputation call."""
        out = np.zeros(n, np.float64)
        self._check(self.lib.gp_loglik_get(self.h, n, _p(out, C.c_double)))
        return out

    def learned_size(self, min_prob=0.5, kmin=0):
        """gp_learned_size: kmin = 0 fixed size (the targets' Kpbwt); else adaptive."""
        self._check(self.lib.gp_learned_size(self.h, C.c_float(min_prob), kmin))

    def learned_windows(self):
        n = self.lib.gp_learned_windows(self.h)
        if n < 0:
            self._check(n)
        return n

    def state_posteriors(self, states_list, hl, flat):
        """gp_state_posteriors: per haplotype an array (nwin, K_i) of window masses, and nsites (n, nwin)."""
        n = len(states_list)
        nwin = self.learned_windows()
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in states_list])
        st = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint32) for s in states_list]), np.uint32)
        hl = np.ascontiguousarray(hl, np.float32).reshape(n, 2 * self.L)
        flat = np.ascontiguousarray(flat, np.uint8).reshape(n, self.L)
        mass = np.zeros(nwin * int(off[-1]), np.float32)
        ns = np.zeros((n, nwin), np.int32)
        self._check(self.lib.gp_state_posteriors(self.h, n, _p(off, C.c_int64), _p(st, C.c_uint32), _p(hl, C.c_float),
                                                 _p(flat, C.c_uint8), _p(mass, C.c_float), _p(ns, C.c_int32)))
        out = [mass[nwin * off[i]:nwin * off[i + 1]].reshape(nwin, len(states_list[i])) for i in range(n)]
        return out, ns

    def learned_enable(self, enable=True, kcand=1024):
        self._check(self.lib.gp_learned_enable(self.h, int(enable), kcand))

    def learned_train(self, kcand=1024, kpos=8.0, steps=300, batch=16384, lr=1e-3, seed=1):
        """gp_learned_train on the current targets; returns the per-step losses."""
        losses = np.zeros(max(steps, 1), np.float32)
        self._check(self.lib.gp_learned_train(self.h, kcand, C.c_float(kpos), steps, batch, C.c_float(lr),
                                              C.c_uint64(seed), _p(losses, C.c_float)))
        return losses[:steps]

    def stage_times(self):
        ms = np.zeros(5, np.float32)
        self._check(self.lib.gp_stage_times(self.h, _p(ms, C.c_float), 5))
        return ms

    def sparse_pbwt(self):
        ylen = C.c_int64(0)
        alen = C.c_int64(0)
        self._check(self.lib.gp_sparse_pbwt_get(self.h, None, C.byref(ylen), None, None, C.byref(alen)))
        n_com_hq = int(((self.panel.flag_common != 0) & (self.panel.lq == 0)).sum())
        yp = np.zeros(max(ylen.value, 1), np.uint8)
        aoff = np.zeros(n_com_hq + 2, np.int64)
        aidx = np.zeros(max(alen.value, 1), np.int32)
        self._check(self.lib.gp_sparse_pbwt_get(self.h, _p(yp, C.c_uint8), C.byref(ylen), _p(aoff, C.c_int64),
                                                _p(aidx, C.c_int32), C.byref(alen)))
        return yp[:ylen.value], aoff, aidx[:alen.value]

    def targets_reset(self):
        self._check(self.lib.gp_targets_reset(self.h))

    def profile(self):
        p = gp_profile()
        self._check(self.lib.gp_profile_get(self.h, C.byref(p)))
        return {f: getattr(p, f) for f, _ in gp_profile._fields_}

    def profile_reset(self):
        self._check(self.lib.gp_profile_reset(self.h))

    def stream_handle(self) -> int:
        return int(self.lib.gp_stream(self.h) or 0)

    def set_targets_raw(self, n, gl_ptr, flat_ptr, ploidy_ptr, kpbwt_ptr):
        """gp_targets_set from raw host pointers (e.g. pinned buffers)."""
        self.n_targets = n
        self._check(self.lib.gp_targets_set(self.h, n, C.c_void_p(gl_ptr), C.c_void_p(flat_ptr),
                                            C.c_void_p(ploidy_ptr), C.c_void_p(kpbwt_ptr)))

    def gp_raw(self, ds_ptr, gt0_ptr, gt1_ptr):
        """gp_gp_get of the dosages and called alleles into raw host pointers."""
        self._check(self.lib.gp_gp_get(self.h, None, None, C.c_void_p(ds_ptr), C.c_void_p(gt0_ptr),
                                       C.c_void_p(gt1_ptr)))
