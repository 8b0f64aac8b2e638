"""Learned surrogate of omega on the tensor cores (uc_mlp_* of include/unichem.h).

A 54 -> 256 x 4 (GELU) -> 52 network: inputs T, ln(p/PREF) and ln max(Y_k,
1e-12), standardised; outputs asinh(QDSP_k / s_k), standardised (QDSP is the
reference's -omega). Trained with Adam on states whose omega the exact FP64
kernel computes; evaluated with a per-cell fallback to that kernel.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import unichem
from .unichem import LSP, UniChemError

NF, NO, NIN, NOUT = 54, 52, 64, 64


def raw_features(T, p_over_pref, y) -> np.ndarray:
    """[54, n]: T (K), ln(p/PREF), ln max(Y_k, 1e-12)."""
    return np.vstack([T[None, :], np.log(p_over_pref)[None, :], np.log(np.maximum(y, 1e-12))]).astype(np.float64)


def _lib():
    L = unichem.load_library()
    if not getattr(L, "_mlp_bound", False):
        vp, F, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        U16 = ctypes.POINTER(ctypes.c_uint16)
        L.uc_mlp_create.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.c_long, ctypes.POINTER(vp)]
        L.uc_mlp_nparams.argtypes = [vp]
        L.uc_mlp_params.argtypes = [vp, F, F]
        L.uc_mlp_set_norm.argtypes = [vp, F, F, F, F, F, F, F]
        L.uc_mlp_add_data.argtypes = [vp, vp]
        L.uc_mlp_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_ulonglong, F]
        L.uc_mlp_grad.argtypes = [vp, ctypes.c_int, U16, F, F, F]
        L.uc_mlp_omega.argtypes = [vp, vp, ctypes.c_double, D]
        L.uc_mlp_stat.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        L.uc_mlp_last_error.argtypes = [vp]
        L.uc_mlp_last_error.restype = ctypes.c_char_p
        L.uc_mlp_destroy.argtypes = [vp]
        L.uc_mlp_destroy.restype = None
        L._mlp_bound = True
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Surrogate:
    def __init__(self, capacity: int, seed: int = 0, device: int = 0):
        self.lib = _lib()
        h = ctypes.c_void_p()
        rc = self.lib.uc_mlp_create(device, seed, capacity, ctypes.byref(h))
        if rc != 0:
            raise UniChemError(rc, "uc_mlp_create failed")
        self._h = h
        self.nparams = self.lib.uc_mlp_nparams(h)
        self.norm = None

    def _ck(self, rc):
        if rc != 0:
            raise UniChemError(rc, self.lib.uc_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.uc_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ set-up
    def set_norm(self, feat_mu, feat_sd, hull_lo, hull_hi, tgt_mu, tgt_sd, tgt_scale):
        arrs = [_f32(a) for a in (feat_mu, feat_sd, hull_lo, hull_hi, tgt_mu, tgt_sd, tgt_scale)]
        self._ck(self.lib.uc_mlp_set_norm(self._h, *[_fp(a) for a in arrs]))
        self.norm = dict(zip(("feat_mu", "feat_sd", "hull_lo", "hull_hi", "tgt_mu", "tgt_sd", "tgt_scale"), arrs))

    @staticmethod
    def norm_from_sample(feats: np.ndarray, qdsp: np.ndarray) -> dict:
        """Scales from a sample: feats [54, n] raw features, qdsp [52, n] exact QDSP."""
        s = np.median(np.abs(qdsp), axis=1)
        s = np.where(s > 0, s, 1e-30)
        t = np.arcsinh(qdsp / s[:, None])
        sd_f = feats.std(axis=1)
        sd_t = t.std(axis=1)
        return dict(feat_mu=feats.mean(axis=1), feat_sd=np.where(sd_f > 0, sd_f, 1.0), hull_lo=feats.min(axis=1),
                    hull_hi=feats.max(axis=1), tgt_mu=t.mean(axis=1), tgt_sd=np.where(sd_t > 0, sd_t, 1.0),
                    tgt_scale=s)

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        self._ck(self.lib.uc_mlp_params(self._h, _fp(out), None))
        return out

    def set_params(self, w):
        w = _f32(w)
        self._ck(self.lib.uc_mlp_params(self._h, None, _fp(w)))

    # ------------------------------------------------------------ training
    def add_data(self, u: "unichem.UniChem"):
        self._ck(self.lib.uc_mlp_add_data(self._h, u._h))

    def train(self, steps: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        loss = np.empty(steps, dtype=np.float32)
        self._ck(self.lib.uc_mlp_train(self._h, steps, batch, lr, seed, _fp(loss)))
        return loss

    def grad(self, x_bits: np.ndarray, t: np.ndarray):
        M = x_bits.shape[0]
        g = np.empty(self.nparams, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        x_bits = np.ascontiguousarray(x_bits, dtype=np.uint16)
        t = _f32(t)
        self._ck(self.lib.uc_mlp_grad(self._h, M, x_bits.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), _fp(t),
                                      _fp(g), _fp(loss)))
        return g, float(loss[0])

    # ------------------------------------------------------------ inference
    def omega(self, u: "unichem.UniChem", tol: float = 1e-3, stats: bool = True):
        """QDSP of u's state into u's device outputs, with per-cell fallback to the exact kernel;
        returns the fallback statistics (which cost a synchronisation and copies), or None."""
        if not stats:
            self._ck(self.lib.uc_mlp_omega(self._h, u._h, tol, None))
            return None
        st = np.zeros(3)
        self._ck(self.lib.uc_mlp_omega(self._h, u._h, tol, st.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        out = {}
        for k in ("cells_exact", "cells_outside_hull", "sample_error_p50", "sample_accepted",
                  "sample_accepted_within_tol", "sample_accepted_error_p50", "sample_accepted_error_p99"):
            v = ctypes.c_double(0.0)
            self._ck(self.lib.uc_mlp_stat(self._h, k.encode(), ctypes.byref(v)))
            out[k] = v.value
        return out
