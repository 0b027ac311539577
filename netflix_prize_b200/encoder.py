"""Learned warm start: the amortised user encoder and fold-in (C ABI wrappers).

An encoder maps a user's training history to (p_u, b_u, alpha_u) of a trained
model; applied to new users it replaces the standard init before fold-in
(user-side SGD with the item tables frozen, the user phase of the reference's
parallel schedule, src/tsvdx4p.rs:390-639).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .native import TsvdError, load

P = C.c_void_p

_bound = False


def _bind():
    global _bound
    L = load()
    if _bound:
        return L
    L.tsvd_encoder_create.argtypes = [P, P, P, C.c_uint64, C.c_uint64, C.c_float, C.c_float, C.POINTER(P)]
    L.tsvd_encoder_destroy.argtypes = [P]
    L.tsvd_encoder_destroy.restype = None
    L.tsvd_encoder_train_epoch.argtypes = [P, P, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]
    L.tsvd_encoder_loss_grad.argtypes = [P, P, C.c_uint32, C.POINTER(C.c_double)]
    L.tsvd_encoder_forward.argtypes = [P, P, C.c_uint32, P]
    L.tsvd_encoder_apply.argtypes = [P, P, P, C.c_uint64]
    L.tsvd_encoder_get.argtypes = [P, C.c_char_p, P, C.c_uint64]
    L.tsvd_encoder_set.argtypes = [P, C.c_char_p, P, C.c_uint64]
    L.tsvd_encoder_target_stats.argtypes = [P, P, P]
    L.tsvd_encoder_last_error.argtypes = [P]
    L.tsvd_encoder_last_error.restype = C.c_char_p
    L.tsvd_foldin.argtypes = [P, P, C.c_uint64, C.c_uint32]
    L.tsvd_reset_users.argtypes = [P, P, C.c_uint64, C.c_uint64]
    _bound = True
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


SHAPES = {"e_rate": (5, 128), "w1": (128, 512), "b1": (512,), "w2": (512, 512), "b2": (512,)}


class UserEncoder:
    EMB, HID = 128, 512

    def __init__(self, model, train_raw, target_users, seed: int = 7, lr: float = 1e-3, weight_decay: float = 1e-4):
        L = _bind()
        self._L = L
        self.model = model
        self.F = model.cfg.n_feat
        self.O = self.F + 2
        self.n_items = model.n_items
        self.T = model.cfg.n_time_bins
        raw = np.ascontiguousarray(train_raw, np.int8)
        tu = np.ascontiguousarray(target_users, np.uint32)
        h = P()
        rc = L.tsvd_encoder_create(model.h, _p(raw), _p(tu), len(tu), seed, lr, weight_decay, C.byref(h))
        if rc != 0:
            raise TsvdError(rc, L.tsvd_encoder_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise TsvdError(rc, self._L.tsvd_encoder_last_error(self.h).decode())

    def shape(self, name: str):
        base = name[2:] if name.startswith("g.") else name
        return {"e_item": (self.n_items * 5, 128), "e_rate": (5, 128), "e_date": (self.T, 128), "w1": (128, 512),
                "b1": (512,), "w2": (512, 512), "b2": (512,), "w3": (512, self.O), "b3": (self.O,)}[base]

    def get(self, name: str) -> np.ndarray:
        shp = self.shape(name)
        out = np.empty(int(np.prod(shp)), np.float32)
        self._check(self._L.tsvd_encoder_get(self.h, name.encode(), _p(out), out.size))
        return out.reshape(shp)

    def set(self, name: str, values):
        v = np.ascontiguousarray(np.asarray(values, np.float32).ravel())
        self._check(self._L.tsvd_encoder_set(self.h, name.encode(), _p(v), v.size))

    def train_epoch(self, users, batch: int = 1024) -> float:
        u = np.ascontiguousarray(users, np.uint32)
        out = C.c_double()
        self._check(self._L.tsvd_encoder_train_epoch(self.h, _p(u), len(u), batch, C.byref(out)))
        return out.value

    def loss_grad(self, users) -> float:
        u = np.ascontiguousarray(users, np.uint32)
        out = C.c_double()
        self._check(self._L.tsvd_encoder_loss_grad(self.h, _p(u), len(u), C.byref(out)))
        return out.value

    def forward(self, users) -> np.ndarray:
        u = np.ascontiguousarray(users, np.uint32)
        out = np.empty((len(u), self.O), np.float32)
        self._check(self._L.tsvd_encoder_forward(self.h, _p(u), len(u), _p(out)))
        return out

    def apply(self, model, users):
        u = np.ascontiguousarray(users, np.uint32)
        self._check(self._L.tsvd_encoder_apply(self.h, model.h, _p(u), len(u)))

    def target_stats(self):
        mean = np.empty(self.O, np.float32)
        std = np.empty(self.O, np.float32)
        self._check(self._L.tsvd_encoder_target_stats(self.h, _p(mean), _p(std)))
        return mean, std

    def close(self):
        if getattr(self, "h", None):
            self._L.tsvd_encoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def foldin(model, users, passes: int):
    """User-side SGD passes over `users` with every item table frozen."""
    L = _bind()
    u = np.ascontiguousarray(users, np.uint32)
    rc = L.tsvd_foldin(model.h, _p(u), len(u), passes)
    if rc != 0:
        raise TsvdError(rc, L.tsvd_last_error(model.h).decode())


def reset_users(model, users, seed: int):
    """Standard init of `users` (p_u ~ N(0, sigma_u), the rest as TxModel::new)."""
    L = _bind()
    u = np.ascontiguousarray(users, np.uint32)
    rc = L.tsvd_reset_users(model.h, _p(u), len(u), seed)
    if rc != 0:
        raise TsvdError(rc, L.tsvd_last_error(model.h).decode())
