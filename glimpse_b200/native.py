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
    "gp_stage_times",
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
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class GpError(RuntimeError):
    pass


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
        self._keep = dict(cm=np.ascontiguousarray(p.cm, np.float64), cref=np.ascontiguousarray(p.cref, np.uint32),
                          calt=np.ascontiguousarray(p.calt, np.uint32), lq=np.ascontiguousarray(p.lq, np.uint8),
                          common=np.ascontiguousarray(p.flag_common, np.uint8),
                          major=np.ascontiguousarray(p.major, np.uint8), hvar=np.ascontiguousarray(p.hvar, np.uint8),
                          soff=np.ascontiguousarray(p.shap_off, np.int64),
                          ssites=np.ascontiguousarray(p.shap_sites, np.int32))
        k = self._keep
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
