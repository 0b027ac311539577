"""The tsvdx4 base jobs of the reference's job dispatcher
(src/bin/tsvdx4-new.rs:13-40, presets at :118-556) as TxConfig values, with
the driver options each job passes to `fit2!` (src/lib.rs:867-996).

The hyperparameters are the reference's own: the drop-in must train the same
models the `run` orchestrator's jobs train. Every job runs on the default
(stratified) schedule; `JOBS[name].config` is what a Rust shim would pass to
tsvd_create unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from .config import OrdinalHeadConfig, TxConfig


@dataclass(frozen=True)
class Job:
    config: TxConfig
    save_train: bool = False
    save_subscores: bool = False
    save_probe_each_epoch: bool = False
    transpose: bool = False
    extra: dict = field(default_factory=dict)


_ORD = OrdinalHeadConfig((0.5, 1.25, 3.75, 5.5), 0.001, 0.0, 0.0)

# the lm preset (src/bin/tsvdx4-new.rs:118-154); TxConfig's defaults are its values
_LM = dict(lr_yb=2.5e-5, reset_u_epoch=13)


def _lm(n_feat, n_epochs, seed, n_time_bins, save_ifeat, low_memory, save_train, save_subscores, each_epoch):
    cfg = TxConfig(n_feat=n_feat, n_epochs=n_epochs, seed=seed, n_time_bins=n_time_bins, save_ifeat=save_ifeat,
                   low_memory=low_memory, **_LM)
    return Job(cfg, save_train, save_subscores, each_epoch)


def _small_o(n_feat, save_train):
    """run_small_o (src/bin/tsvdx4-new.rs:165-202)."""
    cfg = TxConfig(n_feat=n_feat, n_epochs=28, seed=64, n_time_bins=20, lr_u=0.003, lr_ud=0.0015, lr_u2=1e-5,
                   lr_ub=0.006, lr_ubd=0.006, lr_i=0.0072, lr_ib=0.0072, lr_y=0.0012, lr_yb=2e-6, lr_yd=0.000267,
                   lr_tu=0.0, lr_ti=0.0001, lr_ta=1.5e-5, lr_ibf=5e-5, lr_iqf=5e-6, lr_cu=0.002, reg_iqf=0.007,
                   reg_cu=0.01, reg_u=0.04, reg_u2=0.4, reg_ud=0.04, reg_i=0.007, reg_y=0.04, reg_yd=0.04,
                   sigma_iqf=0.005, sigma_u=0.0, sigma_i=0.005, sigma_y=0.005, sigma_yd=0.005, reset_u_epoch=1024,
                   ordinal_head=_ORD, low_memory=False)
    if save_train:
        return Job(cfg, save_train=True, save_probe_each_epoch=True)
    return Job(cfg, save_subscores=True)


def _cfg(**kw) -> TxConfig:
    """A preset of the 'other base trainers' group: every field is given."""
    base = dict(shuffle_users=True, beta=0.3, n_freq_bins=16, reg_iqf=0.007, reg_cu=0.01, reg_u2=0.4,
                reset_u_epoch=1024, low_memory=True, full_su=True, save_ifeat=False)
    base.update(kw)
    return TxConfig(**base)


JOBS: dict[str, Job] = {
    # lm cluster (src/bin/tsvdx4-new.rs:18-22)
    "tsvdx4-60": _lm(60, 20, 42, 29, False, False, True, False, True),
    "tsvdx4-400lm": _lm(400, 20, 42, 29, True, True, True, True, True),
    "tsvdx4-1600lm": _lm(1600, 2, 1600, 29, False, True, False, False, True),
    "tsvdx4-2400lm": _lm(2400, 25, 2400, 32, False, True, True, True, False),
    "tsvdx4-4800lm": _lm(4800, 27, 2400, 32, True, True, True, False, True),
    # 60o / 80o / 160o (:25-27)
    "tsvdx4-60o": _small_o(60, True),
    "tsvdx4-80o": _small_o(80, False),
    "tsvdx4-160o": _small_o(160, False),
    # other base trainers (:30-40)
    "tsvdx4-d0tb": Job(_cfg(n_feat=0, n_epochs=5, seed=8003, n_time_bins=29, lr_u=0.0, lr_ud=0.0, lr_u2=0.0,
                            lr_ub=0.012, lr_ubd=0.012, lr_i=0.0, lr_ib=0.012, lr_y=0.0, lr_yb=0.0, lr_yd=0.0,
                            lr_tu=0.003, lr_ti=0.001, lr_ta=0.0001, lr_ibf=0.0003, lr_iqf=0.0, lr_cu=0.006,
                            reg_u=0.0504, reg_ud=0.04, reg_i=0.00735, reg_y=0.04, reg_yd=0.02667, sigma_iqf=0.0,
                            sigma_u=0.0, sigma_i=0.0, sigma_y=0.0, sigma_yd=0.0),
                       save_train=True, save_probe_each_epoch=True),
    "tsvdx4-f1": Job(_cfg(n_feat=1, n_epochs=5, seed=8005, n_time_bins=29, lr_u=0.009, lr_ud=0.0, lr_u2=2.1e-5,
                          lr_ub=0.0093, lr_ubd=0.009, lr_i=0.0108, lr_ib=0.0108, lr_y=0.0015, lr_yb=7.5e-5,
                          lr_yd=0.0, lr_tu=0.0, lr_ti=0.000675, lr_ta=6.75e-5, lr_ibf=0.00015, lr_iqf=1.5e-5,
                          lr_cu=0.006, reg_u=0.0504, reg_ud=0.04, reg_i=0.00735, reg_y=0.04, reg_yd=0.02667,
                          sigma_iqf=0.005, sigma_u=0.0015, sigma_i=0.005, sigma_y=0.00333, sigma_yd=0.0),
                     save_probe_each_epoch=True),
    "tsvdx4-h8nb": Job(_cfg(n_feat=8, n_epochs=5, seed=8007, n_time_bins=29, lr_u=0.012, lr_ud=0.0, lr_u2=3e-5,
                            lr_ub=0.0, lr_ubd=0.0, lr_i=0.015, lr_ib=0.0, lr_y=0.003, lr_yb=0.0, lr_yd=0.0,
                            lr_tu=0.0, lr_ti=0.0, lr_ta=0.0, lr_ibf=0.0, lr_iqf=0.0, lr_cu=0.0, reg_u=0.03,
                            reg_ud=0.04, reg_i=0.005, reg_y=0.03, reg_yd=0.02667, sigma_iqf=0.0, sigma_u=0.003,
                            sigma_i=0.008, sigma_y=0.005, sigma_yd=0.0),
                       save_train=True, save_probe_each_epoch=True),
    "tsvdx4-l32nb": Job(_cfg(n_feat=32, n_epochs=5, seed=8011, n_time_bins=29, lr_u=0.01, lr_ud=0.0, lr_u2=2.5e-5,
                             lr_ub=0.0, lr_ubd=0.0, lr_i=0.02, lr_ib=0.0, lr_y=0.002, lr_yb=0.0, lr_yd=0.0,
                             lr_tu=0.0, lr_ti=0.0, lr_ta=0.0, lr_ibf=0.0, lr_iqf=0.0, lr_cu=0.0, reg_u=0.03,
                             reg_ud=0.04, reg_i=0.004, reg_y=0.03, reg_yd=0.02667, sigma_iqf=0.0, sigma_u=0.003,
                             sigma_i=0.008, sigma_y=0.005, sigma_yd=0.0),
                        save_probe_each_epoch=True),
    "tsvdx4-m1n": Job(_cfg(n_feat=1, n_epochs=5, seed=8012, n_time_bins=29, lr_u=0.0, lr_ud=0.0, lr_u2=0.0,
                           lr_ub=0.015, lr_ubd=0.015, lr_i=0.0108, lr_ib=0.0108, lr_y=0.004, lr_yb=0.0002,
                           lr_yd=0.0, lr_tu=0.0, lr_ti=0.000675, lr_ta=6.75e-5, lr_ibf=0.00015, lr_iqf=1.5e-5,
                           lr_cu=0.006, reg_u=0.0504, reg_ud=0.04, reg_i=0.00735, reg_y=0.03, reg_yd=0.02667,
                           sigma_iqf=0.005, sigma_u=0.0, sigma_i=0.005, sigma_y=0.008, sigma_yd=0.0)),
    "tsvdx4-q16tb": Job(_cfg(n_feat=16, n_epochs=8, seed=9001, n_time_bins=48, lr_u=0.005, lr_ud=0.002, lr_u2=1e-5,
                             lr_ub=0.005, lr_ubd=0.005, lr_i=0.006, lr_ib=0.006, lr_y=0.001, lr_yb=5e-5,
                             lr_yd=0.0004, lr_tu=0.0003, lr_ti=0.0004, lr_ta=4e-5, lr_ibf=0.0001, lr_iqf=1e-5,
                             lr_cu=0.004, reg_u=0.04, reg_ud=0.03, reg_i=0.006, reg_y=0.03, reg_yd=0.02,
                             sigma_iqf=0.005, sigma_u=0.002, sigma_i=0.006, sigma_y=0.004, sigma_yd=0.01),
                        save_train=True, save_probe_each_epoch=True),
    "tsvdx4-s20fo": Job(_cfg(n_feat=20, n_epochs=10, seed=9003, n_time_bins=25, n_freq_bins=24, lr_u=0.004,
                             lr_ud=0.002, lr_u2=1.5e-5, lr_ub=0.007, lr_ubd=0.007, lr_i=0.008, lr_ib=0.008,
                             lr_y=0.0015, lr_yb=5e-6, lr_yd=0.0004, lr_tu=0.0, lr_ti=0.00015, lr_ta=2e-5,
                             lr_ibf=8e-5, lr_iqf=8e-6, lr_cu=0.003, reg_iqf=0.005, reg_cu=0.008, reg_u=0.02,
                             reg_u2=0.3, reg_ud=0.02, reg_i=0.004, reg_y=0.02, reg_yd=0.02, sigma_iqf=0.005,
                             sigma_u=0.0, sigma_i=0.005, sigma_y=0.005, sigma_yd=0.005, ordinal_head=_ORD),
                        save_train=True, save_probe_each_epoch=True),
    "tsvdx4-t8cu": Job(_cfg(n_feat=8, n_epochs=8, seed=9004, n_time_bins=29, lr_u=0.006, lr_ud=0.0, lr_u2=1.5e-5,
                            lr_ub=0.006, lr_ubd=0.006, lr_i=0.008, lr_ib=0.008, lr_y=0.005, lr_yb=0.0005,
                            lr_yd=0.0, lr_tu=0.0, lr_ti=0.0003, lr_ta=3e-5, lr_ibf=0.0001, lr_iqf=1e-5, lr_cu=0.05,
                            reg_cu=0.003, reg_u=0.04, reg_ud=0.04, reg_i=0.006, reg_y=0.02, reg_yd=0.02667,
                            sigma_iqf=0.005, sigma_u=0.003, sigma_i=0.008, sigma_y=0.008, sigma_yd=0.0,
                            reset_u_epoch=3),
                       save_train=True, save_probe_each_epoch=True),
    "tsvdx4-16-t": Job(_cfg(n_feat=16, n_epochs=4, seed=9001, n_time_bins=22, beta=0.35, n_freq_bins=12,
                            lr_u=0.004, lr_ud=0.0015, lr_u2=1e-5, lr_ub=0.004, lr_ubd=0.0035, lr_i=0.0025,
                            lr_ib=0.0028, lr_y=0.0004, lr_yb=2e-5, lr_yd=0.0002, lr_tu=0.0, lr_ti=0.0002,
                            lr_ta=2e-5, lr_ibf=4e-5, lr_iqf=0.0, lr_cu=0.0015, reg_cu=0.008, reg_u=0.008,
                            reg_u2=0.3, reg_ud=0.035, reg_i=0.045, reg_y=0.035, reg_yd=0.025, sigma_iqf=0.0,
                            sigma_u=0.006, sigma_i=0.0012, sigma_y=0.003, sigma_yd=0.008, save_ifeat=True),
                       save_train=True, save_probe_each_epoch=True, transpose=True),
    "tsvdx4-n8nbo": Job(_cfg(n_feat=8, n_epochs=5, seed=8013, n_time_bins=20, lr_u=0.015, lr_ud=0.0, lr_u2=0.0,
                             lr_ub=0.0, lr_ubd=0.0, lr_i=0.018, lr_ib=0.0, lr_y=0.003, lr_yb=0.0, lr_yd=0.0,
                             lr_tu=0.0, lr_ti=0.0, lr_ta=0.0, lr_ibf=0.0, lr_iqf=0.0, lr_cu=0.0, reg_u=0.03,
                             reg_ud=0.04, reg_i=0.005, reg_y=0.03, reg_yd=0.02667, sigma_iqf=0.0, sigma_u=0.003,
                             sigma_i=0.008, sigma_y=0.005, sigma_yd=0.0, ordinal_head=_ORD),
                        save_train=True),
    "tsvdx4-p0tbo": Job(_cfg(n_feat=0, n_epochs=5, seed=8014, n_time_bins=29, lr_u=0.0, lr_ud=0.0, lr_u2=0.0,
                             lr_ub=0.018, lr_ubd=0.018, lr_i=0.0, lr_ib=0.015, lr_y=0.0, lr_yb=0.0, lr_yd=0.0,
                             lr_tu=0.003, lr_ti=0.001, lr_ta=0.0001, lr_ibf=0.0003, lr_iqf=0.0, lr_cu=0.006,
                             reg_u=0.0504, reg_ud=0.04, reg_i=0.00735, reg_y=0.04, reg_yd=0.02667, sigma_iqf=0.0,
                             sigma_u=0.0, sigma_i=0.0, sigma_y=0.0, sigma_yd=0.0, ordinal_head=_ORD),
                        save_train=True),
}
