"""TEST INFRASTRUCTURE ONLY -- ctypes wrapper of the CPU oracle library.

Only the tests, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg use
this module, as the checker. It restates the reference's TxModel / Tsvdx4pModel
(see tx_oracle.hpp for the file:line map).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

SCHED_SEQ = 0        # TxModel::fit_epoch (src/tx.rs:734-1115)
SCHED_P = 1          # Tsvdx4pModel parallel epoch (src/tsvdx4p.rs:390-805)

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_fit_epoch.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_uint64]
        L.orc_fit_epoch_p_workers.argtypes = [C.c_void_p, C.c_uint64, C.c_float, C.c_uint64]
        L.orc_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        L.orc_predict_subscores.argtypes = L.orc_predict.argtypes
        L.orc_calc_rmse.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        L.orc_rebuild_ycache.argtypes = [C.c_void_p]
        L.orc_param_count.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_uint64)]
        L.orc_get_param.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64]
        L.orc_set_param.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64]
        L.orc_set_user_order.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64]
        L.orc_get_users.argtypes = [C.c_uint64, C.c_int, C.c_uint64, C.c_uint64, C.c_void_p]
        L.orc_normal_stream.argtypes = [C.c_uint64, C.c_float, C.c_uint64, C.c_void_p]
        L.orc_u32_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p]
        L.orc_chacha_block.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.orc_user_block_p.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        L.orc_apply_deltas_p.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float]
        L.orc_item_block_p.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.orc_last_error.restype = C.c_char_p
        L.orc_time_epochs.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleModel:
    """TxModel restated on the CPU (f32 exact, or the FP64 twin)."""

    def __init__(self, tr, pr, cfg, fp64: bool = False):
        L = lib()
        self._cfg = cfg.to_c()
        self._tv = tr.view()
        self._pv = pr.view(masked=True) if hasattr(pr, "view") and not hasattr(pr, "_ds") else pr.view()
        self.h = L.orc_create(C.byref(self._cfg), C.byref(self._tv), C.byref(self._pv), int(fp64))
        if not self.h:
            raise RuntimeError("oracle create: " + L.orc_last_error().decode())
        self.cfg = cfg
        self.fp64 = fp64

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def n_epochs(self):
        return self.cfg.n_epochs

    def fit_epoch(self, epoch: int, schedule: int = SCHED_SEQ, nsvd_norm_exp: float = 1.0, n_threads: int = 1):
        _check(lib().orc_fit_epoch(self.h, epoch, schedule, nsvd_norm_exp, n_threads))

    def fit_epoch_parallel(self, epoch: int, nsvd_norm_exp: float = 1.0, workers: int = 4):
        """SCHED_P with one chunk, on `workers` host threads (same arithmetic,
        same order; low_memory configurations only)."""
        _check(lib().orc_fit_epoch_p_workers(self.h, epoch, nsvd_norm_exp, workers))

    def predict_batch(self, u, i, day):
        u = np.ascontiguousarray(u, np.int32)
        i = np.ascontiguousarray(i, np.int32)
        d = np.ascontiguousarray(day, np.int16)
        out = np.zeros(len(u), np.float64)
        _check(lib().orc_predict(self.h, _p(u), _p(i), _p(d), len(u), _p(out)))
        return out

    def predict_subscores_batch(self, u, i, day):
        u = np.ascontiguousarray(u, np.int32)
        i = np.ascontiguousarray(i, np.int32)
        d = np.ascontiguousarray(day, np.int16)
        out = np.zeros((len(u), 3), np.float64)
        _check(lib().orc_predict_subscores(self.h, _p(u), _p(i), _p(d), len(u), _p(out)))
        return out

    def calc_rmse(self, ds) -> float:
        v = ds.view()
        out = C.c_double()
        _check(lib().orc_calc_rmse(self.h, C.byref(v), C.byref(out)))
        return out.value

    def rebuild_ycache(self):
        _check(lib().orc_rebuild_ycache(self.h))

    def get_param(self, name: str) -> np.ndarray:
        n = C.c_uint64()
        _check(lib().orc_param_count(self.h, name.encode(), C.byref(n)))
        out = np.zeros(n.value, np.float64)
        _check(lib().orc_get_param(self.h, name.encode(), _p(out), n.value))
        return out

    def set_param(self, name: str, values) -> None:
        v = np.ascontiguousarray(np.asarray(values, np.float64).ravel())
        _check(lib().orc_set_param(self.h, name.encode(), _p(v), len(v)))

    def set_user_order(self, epoch: int, perm) -> None:
        p = np.ascontiguousarray(perm, np.uint32)
        _check(lib().orc_set_user_order(self.h, epoch, _p(p), len(p)))

    # -- the parallel schedule in the steps of a sharded run ----------------
    def user_block_p(self, epoch: int, u_lo: int, u_hi: int):
        """User phase of users u_lo..u_hi-1; returns their NSVD1 deltas
        {dy [I, F], dyb [I], dyd [I, F] or None, nc [I]} in FP64."""
        I, F = self._tv.n_items, self.cfg.n_feat
        dy, dyb, nc = np.zeros((I, F)), np.zeros(I), np.zeros(I)
        dyd = None if self.cfg.low_memory else np.zeros((I, F))
        _check(lib().orc_user_block_p(self.h, epoch, u_lo, u_hi, _p(dy), _p(dyb),
                                      None if dyd is None else _p(dyd), _p(nc)))
        return {"dy": dy, "dyb": dyb, "dyd": dyd, "nc": nc}

    def apply_deltas_p(self, d, nsvd_norm_exp: float = 1.0):
        arrs = [np.ascontiguousarray(d[k], np.float64) if d[k] is not None else None
                for k in ("dy", "dyb", "dyd", "nc")]
        _check(lib().orc_apply_deltas_p(self.h, *[None if a is None else _p(a) for a in arrs], nsvd_norm_exp))

    def item_block_p(self, i_lo: int, i_hi: int):
        _check(lib().orc_item_block_p(self.h, i_lo, i_hi))

    def time_epochs(self, first_epoch: int, epochs: int, schedule: int = SCHED_SEQ) -> float:
        s = C.c_double()
        _check(lib().orc_time_epochs(self.h, first_epoch, epochs, schedule, C.byref(s)))
        return s.value


def get_users(n: int, shuffle: bool, seed: int, epoch: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    _check(lib().orc_get_users(n, int(shuffle), seed, epoch, _p(out)))
    return out


def normal_stream(seed: int, sigma: float, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    _check(lib().orc_normal_stream(seed, sigma, n, _p(out)))
    return out


def u32_stream(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    _check(lib().orc_u32_stream(seed, n, _p(out)))
    return out


def chacha_block(state, rounds: int) -> np.ndarray:
    s = np.ascontiguousarray(state, np.uint32)
    out = np.zeros(16, np.uint32)
    lib().orc_chacha_block(_p(s), _p(out), rounds)
    return out
