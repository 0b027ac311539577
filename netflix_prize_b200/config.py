"""TxConfig (src/tx.rs:128-204) and the presets the tsvdx4 jobs use.

`TxConfig` keeps the reference's field names and meanings; `to_c()` packs it
into the C ABI struct. `Tsvdx4Config` is the deprecated subset with its
`into_tx_config` shim (src/tsvdx4.rs:10-146).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Optional

from .abi import TsvdConfig, TsvdOrdinalConfig


@dataclass
class OrdinalHeadConfig:
    """src/lib.rs:502-507"""
    th_init: tuple = (0.5, 1.25, 3.75, 5.5)
    th_gap: float = 0.001
    lr_t: float = 0.0
    reg_t: float = 0.0


@dataclass
class TxConfig:
    n_feat: int = 64
    n_epochs: int = 20
    seed: int = 42
    shuffle_users: bool = True
    n_time_bins: int = 29
    beta: float = 0.3
    n_freq_bins: int = 16
    lr_u: float = 0.003
    lr_ud: float = 0.00125
    lr_u2: float = 7e-6
    lr_ub: float = 0.0031
    lr_ubd: float = 0.003
    lr_i: float = 0.0036
    lr_ib: float = 0.0036
    lr_y: float = 0.0005
    lr_yb: float = 2.5e-5
    lr_yd: float = 0.000267
    lr_tu: float = 0.0
    lr_ti: float = 0.000225
    lr_ta: float = 2.25e-5
    lr_ibf: float = 5e-5
    lr_iqf: float = 5e-6
    lr_cu: float = 0.002
    reg_iqf: float = 0.007
    reg_cu: float = 0.01
    reg_u: float = 0.0504
    reg_u2: float = 0.4
    reg_ud: float = 0.04
    reg_i: float = 0.00735
    reg_y: float = 0.04
    reg_yd: float = 0.02667
    sigma_iqf: float = 0.005
    sigma_u: float = 0.0015
    sigma_i: float = 0.005
    sigma_y: float = 0.00333
    sigma_yd: float = 0.009
    reset_u_epoch: int = 13
    max_neighbors: int = 0
    lr_w: float = 0.0
    lr_c: float = 0.0
    reg_w: float = 0.0
    reg_c: float = 0.0
    lr_w_day: float = 0.0
    lr_c_day: float = 0.0
    reg_w_day: float = 0.0
    reg_c_day: float = 0.0
    w_bias: float = 1.0
    w_factor: float = 1.0
    w_nbr: float = 1.0
    sum_err_bug: bool = False
    lambda1: float = 0.0
    lambda2: float = 0.0
    ordinal_head: Optional[OrdinalHeadConfig] = None
    save_ifeat: bool = False
    low_memory: bool = True
    full_su: bool = True

    def replace(self, **kw) -> "TxConfig":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> TsvdConfig:
        c = TsvdConfig()
        for f in dataclasses.fields(self):
            if f.name == "ordinal_head":
                continue
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        if self.ordinal_head is not None:
            c.has_ordinal_head = 1
            o = TsvdOrdinalConfig()
            for k in range(4):
                o.th_init[k] = self.ordinal_head.th_init[k]
            o.th_gap = self.ordinal_head.th_gap
            o.lr_t = self.ordinal_head.lr_t
            o.reg_t = self.ordinal_head.reg_t
            c.ordinal_head = o
        return c


def run_lm(n_feat: int, n_epochs: int, seed: int = 42, n_time_bins: int = 29, low_memory: bool = True,
           save_ifeat: bool = False) -> TxConfig:
    """The `lm` preset of the tsvdx4 jobs (src/bin/tsvdx4-new.rs:130-154)."""
    return TxConfig(n_feat=n_feat, n_epochs=n_epochs, seed=seed, n_time_bins=n_time_bins,
                    low_memory=low_memory, save_ifeat=save_ifeat)


def regression_test_config(**extra) -> TxConfig:
    """The shared `cfg!` of the reference's tiny-fixture regression tests
    (tests/regressors_test.rs:28-73), tsvdx4 variant (:75-93) by default."""
    c = TxConfig(
        n_feat=10, n_epochs=3, seed=42, shuffle_users=True, n_time_bins=4, beta=0.3, n_freq_bins=4,
        lr_u=0.003, lr_ud=0.001, lr_u2=7e-6, lr_ub=0.003, lr_ubd=0.003, lr_i=0.003, lr_ib=0.003,
        lr_y=0.0005, lr_yb=2.5e-5, lr_yd=0.0002, lr_tu=0.0001, lr_ti=0.0002, lr_ta=2e-5,
        lr_ibf=5e-5, lr_iqf=5e-6, reg_iqf=0.007, sigma_iqf=0.005, lr_cu=0.002, reg_cu=0.01,
        reg_u=0.0504, reg_u2=0.4, reg_ud=0.04, reg_i=0.007, reg_y=0.04, reg_yd=0.02,
        sigma_u=0.001, sigma_i=0.005, sigma_y=0.003, sigma_yd=0.009, save_ifeat=False,
        low_memory=False, full_su=True, reset_u_epoch=1, ordinal_head=None, sum_err_bug=False)
    return c.replace(**extra)
