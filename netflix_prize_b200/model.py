"""TxModel on the B200: the reference's `Regressor` surface (src/lib.rs:616-651)
over the C ABI.

Method names, argument meaning and error behaviour follow the reference's
`impl Regressor for TxModel` (src/tx.rs:457-1116): `new(tr, pr, cfg)`,
`n_epochs()`, `fit_epoch(tr, pr, epoch)` with 1-based epochs,
`predict(u, i, day)`, `n_subscores()`, `subscore_names()`,
`predict_subscores(u, i, day)`, `save_artifacts(name, tr_set, preds_dir)`.
Errors raise (the reference panics). Batched forms (`predict_batch`,
`predict_subscores_batch`) are what the driver functions use, since a
per-row call across the FFI would be the wrong granularity.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import SCHED_HOGWILD, SCHED_STRATIFIED, PREC_FP32, TsvdConfig, TsvdGpuOptions, ptr
from .config import TxConfig
from .data import Dataset, MaskedDataset
from .native import TsvdError, load

PARAM_NAMES = ["gbias", "ubias", "ibias", "ufeat", "ufeat2", "ifeat", "yfeat", "ycache", "tu_mean", "alpha_u",
               "but_bin", "bit_bin", "ybias", "ycache_bias", "ubias_day", "ibias_freq", "ifeat_freq", "cu", "cut"]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class TxModel:
    """A device-resident timeSVD++ model (tsvdx4 / TxModel in tx4 mode)."""

    def __init__(self, tr: Dataset, pr, cfg: TxConfig, schedule: int = SCHED_STRATIFIED,
                 precision: int = PREC_FP32, nsvd_norm_exp: float = 1.0, device: int = 0,
                 heavy_item_ratings: int = 0, seq_epochs=()):
        L = load()
        self._L = L
        self.cfg = cfg
        self.device = device
        self.n_users, self.n_items = tr.n_users, tr.n_items
        opts = TsvdGpuOptions()
        opts.schedule = schedule
        opts.precision = precision
        opts.nsvd_norm_exp = nsvd_norm_exp
        opts.device = device
        opts.heavy_item_ratings = heavy_item_ratings
        if len(seq_epochs) > 5:
            raise ValueError("at most 5 seq_epochs (Tsvdx4pConfig::seq_epochs is [usize; 5])")
        for k, e in enumerate(seq_epochs):
            opts.seq_epochs[k] = int(e)
        c = cfg.to_c()
        tv = tr.view()
        pv = pr.view() if isinstance(pr, MaskedDataset) else pr.view(masked=True)
        h = C.c_void_p()
        rc = L.tsvd_create(C.byref(c), C.byref(opts), C.byref(tv), C.byref(pv), C.byref(h))
        if rc != 0:
            raise TsvdError(rc, L.tsvd_last_global_error().decode())
        self.h = h

    # -- Regressor::new ------------------------------------------------------
    @classmethod
    def new(cls, tr: Dataset, pr, cfg: TxConfig, **kw) -> "TxModel":
        return cls(tr, pr, cfg, **kw)

    @classmethod
    def _borrowed(cls, handle, cfg: TxConfig, n_users: int, n_items: int, owner) -> "TxModel":
        """A view of a model owned by a TxGroup (never destroyed here)."""
        m = cls.__new__(cls)
        m._L = load()
        m.cfg = cfg
        m.n_users, m.n_items = n_users, n_items
        m.h = handle
        m._owner = owner
        return m

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self.h = None
            return
        if getattr(self, "h", None):
            self._L.tsvd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise TsvdError(rc, self._L.tsvd_last_error(self.h).decode())

    # -- Regressor -------------------------------------------------------------
    def n_epochs(self) -> int:
        return int(self.cfg.n_epochs)

    def fit_epoch(self, tr=None, pr=None, epoch: int = 1):
        """Regressor::fit_epoch; tr/pr are accepted for signature parity (the
        data were copied to the device at construction)."""
        self._check(self._L.tsvd_fit_epoch(self.h, int(epoch)))

    def predict(self, u: int, i: int, day: int) -> float:
        return float(self.predict_batch(np.array([u]), np.array([i]), np.array([day]))[0])

    def predict_batch(self, u, i, day) -> np.ndarray:
        u = np.ascontiguousarray(u, np.int32)
        i = np.ascontiguousarray(i, np.int32)
        d = np.ascontiguousarray(day, np.int16)
        out = np.empty(len(u), np.float32)
        self._check(self._L.tsvd_predict_batch(self.h, _p(u), _p(i), _p(d), len(u), _p(out)))
        return out

    def n_subscores(self) -> int:
        return 3

    def subscore_names(self):
        return [self._L.tsvd_subscore_name(self.h, k).decode() for k in range(3)]

    def predict_subscores(self, u: int, i: int, day: int) -> np.ndarray:
        return self.predict_subscores_batch(np.array([u]), np.array([i]), np.array([day]))[0]

    def predict_subscores_batch(self, u, i, day) -> np.ndarray:
        u = np.ascontiguousarray(u, np.int32)
        i = np.ascontiguousarray(i, np.int32)
        d = np.ascontiguousarray(day, np.int16)
        out = np.empty((len(u), 3), np.float32)
        self._check(self._L.tsvd_predict_subscores_batch(self.h, _p(u), _p(i), _p(d), len(u), _p(out)))
        return out

    def save_artifacts(self, model_name: str, tr_set: str, preds_dir: str):
        """`{preds_dir}/{name}.ifeat.{tr_set}.npy` when save_ifeat (src/tx.rs:726-732);
        returns the path written (the driver logs it, as the reference's teeln! does), or None."""
        if self.cfg.save_ifeat:
            path = os.path.join(preds_dir, f"{model_name}.ifeat.{tr_set}.npy")
            np.save(path, self.get_param("ifeat"))
            return path
        return None

    # -- driver-level batched helpers -----------------------------------------
    def gen_preds(self, ds: Dataset) -> np.ndarray:
        """gen_preds_parallel (src/lib.rs:710-722)."""
        out = np.empty(ds.n_ratings, np.float32)
        v = ds.view()
        self._check(self._L.tsvd_gen_preds(self.h, C.byref(v), _p(out)))
        return out

    def calc_rmse(self, ds: Dataset) -> float:
        """calc_rmse (src/lib.rs:659-672)."""
        v = ds.view()
        out = C.c_double()
        self._check(self._L.tsvd_calc_rmse(self.h, C.byref(v), C.byref(out)))
        return out.value

    # -- parameters -------------------------------------------------------------
    def param_shape(self, name: str):
        n = C.c_uint64()
        self._check(self._L.tsvd_param_nbytes(self.h, name.encode(), C.byref(n)))
        return n.value // 4

    def get_param(self, name: str) -> np.ndarray:
        n = self.param_shape(name)
        out = np.empty(n, np.float32)
        self._check(self._L.tsvd_get_param(self.h, name.encode(), _p(out), n * 4))
        F = self.cfg.n_feat
        if name in ("ufeat", "ufeat2", "ifeat", "yfeat", "ycache", "ifeat_freq"):
            if F == 0:  # bias-only models: rows without columns
                rows = {"ifeat": self.n_items, "yfeat": self.n_items,
                        "ifeat_freq": self.n_items * self.cfg.n_freq_bins}.get(name, self.n_users)
                return out.reshape(rows, 0)
            return out.reshape(-1, F)
        if name == "but_bin" or name == "bit_bin":
            return out.reshape(-1, self.cfg.n_time_bins)
        if name == "ibias_freq":
            return out.reshape(-1, self.cfg.n_freq_bins)
        if name == "gbias":
            return out[0]
        return out

    def set_param(self, name: str, values) -> None:
        v = np.ascontiguousarray(np.asarray(values, np.float32).ravel())
        self._check(self._L.tsvd_set_param(self.h, name.encode(), _p(v), v.nbytes))

    def rebuild_ycache(self):
        self._check(self._L.tsvd_rebuild_ycache(self.h))

    def set_user_order(self, epoch: int, perm) -> None:
        p = np.ascontiguousarray(perm, np.uint32)
        self._check(self._L.tsvd_set_user_order(self.h, epoch, _p(p), len(p)))

    def get_user_order(self, epoch: int) -> np.ndarray:
        out = np.empty(self.n_users, np.uint32)
        self._check(self._L.tsvd_get_user_order(self.h, epoch, _p(out), self.n_users))
        return out

    # -- streams and timing -----------------------------------------------------
    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.tsvd_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self):
        self._check(self._L.tsvd_synchronize(self.h))

    def set_profiling(self, on: bool):
        self._check(self._L.tsvd_set_profiling(self.h, int(on)))

    def kernel_stats(self, kernel: str):
        n = C.c_uint64()
        ms = C.c_double()
        self._check(self._L.tsvd_kernel_stats(self.h, kernel.encode(), C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def reset_kernel_stats(self):
        self._check(self._L.tsvd_reset_kernel_stats(self.h))

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._check(self._L.tsvd_launch_count(self.h, C.byref(n)))
        return n.value


class TxGroup:
    """Several TxModel variants over one device copy of the data, trained
    together: stratified variants (the default) run their epochs on parallel
    streams, Hogwild variants in one persistent launch per epoch; either way
    an epoch of all variants is one CUDA graph from the second epoch on.
    `models[k]` is the Regressor view of variant k."""

    def __init__(self, tr: Dataset, pr, cfgs, device: int = 0, schedule: int = SCHED_STRATIFIED):
        L = load()
        self._L = L
        self.cfgs = list(cfgs)
        n = len(self.cfgs)
        arr = (TsvdConfig * n)(*[c.to_c() for c in self.cfgs])
        opts = TsvdGpuOptions()
        opts.schedule = schedule
        opts.nsvd_norm_exp = 1.0
        opts.device = device
        tv = tr.view()
        pv = pr.view() if isinstance(pr, MaskedDataset) else pr.view(masked=True)
        h = C.c_void_p()
        rc = L.tsvd_group_create(arr, n, C.byref(opts), C.byref(tv), C.byref(pv), C.byref(h))
        if rc != 0:
            raise TsvdError(rc, L.tsvd_group_last_error(None).decode())
        self.h = h
        self.models = []
        for k in range(n):
            mh = C.c_void_p()
            self._check(L.tsvd_group_model(self.h, k, C.byref(mh)))
            self.models.append(TxModel._borrowed(mh, self.cfgs[k], tr.n_users, tr.n_items, self))

    def _check(self, rc):
        if rc != 0:
            raise TsvdError(rc, self._L.tsvd_group_last_error(self.h).decode())

    def fit_epoch(self, epoch: int):
        self._check(self._L.tsvd_group_fit_epoch(self.h, int(epoch)))

    def set_graphs(self, on: bool):
        self._check(self._L.tsvd_group_set_graphs(self.h, int(on)))

    def last_epoch_ms(self) -> float:
        out = C.c_double()
        self._check(self._L.tsvd_group_last_epoch_ms(self.h, C.byref(out)))
        return out.value

    def autotune(self, sample_users: int = 2000):
        """Hogwild variants: the prefetch depth chosen per variant; stratified
        variants: the item stratum's whole-CTA threshold per variant."""
        out = np.zeros(len(self.cfgs), np.int32)
        self._check(self._L.tsvd_group_autotune(self.h, sample_users, _p(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            for m in self.models:
                m.h = None
            self._L.tsvd_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
