"""Experiment driver: the reference's evaluation helpers and fit/fit2 flow
(src/lib.rs:659-996) over a batched-prediction model.

Output names match the reference exactly: `{preds}/{name}.{pr}.npy`,
`{name}_epNN.{pr}.npy`, `{name}-{bias,mf,nsvd1}.{pr}.npy`, `{name}.{tr}.npy`,
`{name}.ifeat.{tr}.npy` and the `{name}.out` log (src/lib.rs:925,939,946,953;
src/tx.rs:728).
"""
from __future__ import annotations

import os
import sys
from dataclasses import dataclass

import numpy as np

from .data import Dataset, MaskedDataset


class Tee:
    """tee!/teeln! (src/lib.rs:92-135): stdout plus the {name}.out log."""

    def __init__(self, path: str | None):
        self.f = open(path, "w") if path else None

    def write(self, s: str):
        sys.stdout.write(s)
        sys.stdout.flush()
        if self.f:
            self.f.write(s)
            self.f.flush()

    def close(self):
        if self.f:
            self.f.close()
            self.f = None


def calc_rmse(model, ds: Dataset) -> float:
    return model.calc_rmse(ds)


def gen_preds_parallel(model, ds: Dataset) -> np.ndarray:
    return model.gen_preds(ds)


def rmse_from_preds(preds: np.ndarray, ds: Dataset) -> float:
    """src/lib.rs:725-737: FP64 over is_test == 0 rows, against raw ratings."""
    m = ds.is_test == 0
    err = (preds[m].astype(np.float32) - ds.raw_ratings[m].astype(np.float32)).astype(np.float64)
    return float(np.sqrt((err * err).sum() / m.sum()))


def calc_subscores(model, ds: Dataset) -> np.ndarray:
    return model.predict_subscores_batch(ds.user_idxs, ds.item_idxs, ds.dates)


def fmt5(x: float) -> str:
    """`{:.5}` of an f64 as Rust formats it (NaN is "NaN")."""
    return "NaN" if x != x else f"{x:.5f}"


def report_rmse(model, epoch: int, n_epochs: int, ds: Dataset, tee: Tee):
    """src/lib.rs:676-686"""
    tee.write(f"Epoch {epoch:02d}")
    if ds.contains_test_examples() and epoch < n_epochs:
        tee.write("\n")
        return None
    r = calc_rmse(model, ds)
    tee.write(f" | RMSE {fmt5(r)}\n")
    return r


@dataclass
class Fit2Opts:
    """src/lib.rs:838-848"""
    save_train: bool = False
    save_probe_each_epoch: bool = False
    save_subscores: bool = False
    no_fulltrain: bool = False
    transpose: bool = False


def _save_subscores(model, ds: Dataset, model_name: str, set_name: str, preds_dir: str):
    sub = calc_subscores(model, ds)
    for j, name in enumerate(model.subscore_names()):
        np.save(os.path.join(preds_dir, f"{model_name}-{name}.{set_name}.npy"), np.ascontiguousarray(sub[:, j]))


def _train(model_factory, cfg, tr, pr, model_name, preds_dir, save_probe_each_epoch, pr_set, tee, qual=None,
           qual_set=None):
    """Construction and the epoch loop shared by both phases (src/lib.rs:782-795, 921-936)."""
    model = model_factory(tr, MaskedDataset(pr), cfg)
    n_epochs = model.n_epochs()
    curve = []
    for epoch in range(1, n_epochs + 1):
        model.fit_epoch(tr, MaskedDataset(pr), epoch)
        curve.append(report_rmse(model, epoch, n_epochs, pr, tee))
        if save_probe_each_epoch:
            np.save(os.path.join(preds_dir, f"{model_name}_ep{epoch:02d}.{pr_set}.npy"), gen_preds_parallel(model, pr))
            if qual is not None:
                np.save(os.path.join(preds_dir, f"{model_name}_ep{epoch:02d}.{qual_set}.npy"),
                        gen_preds_parallel(model, qual))
    return model, curve


def _artifacts(model, model_name, tr_set, preds_dir, tee):
    """save_artifacts and its log line (src/tx.rs:726-732)."""
    path = model.save_artifacts(model_name, tr_set, preds_dir)
    if path:
        tee.write(f"Saved item factors to {path}\n")


def _arrow(a: str, b: str, transpose: bool) -> str:
    return f"{a} => {b}{' (transposed)' if transpose else ''}\n"


def fit(model_factory, cfg, tr: Dataset, pr: Dataset, model_name: str, preds_dir: str, opts: Fit2Opts,
        tee: Tee, tr_set: str, pr_set: str):
    """fit (src/lib.rs:764-815): the phase-2 run, fulltrain -> qual."""
    tee.write(_arrow(tr_set, pr_set, opts.transpose))
    if opts.transpose:
        tr, pr = tr.transpose(True), pr.transpose(False)
    model, curve = _train(model_factory, cfg, tr, pr, model_name, preds_dir, opts.save_probe_each_epoch, pr_set, tee)
    np.save(os.path.join(preds_dir, f"{model_name}.{pr_set}.npy"), gen_preds_parallel(model, pr))
    if opts.save_subscores:
        _save_subscores(model, pr, model_name, pr_set, preds_dir)
    if opts.save_train:
        np.save(os.path.join(preds_dir, f"{model_name}.{tr_set}.npy"), gen_preds_parallel(model, tr))
    _artifacts(model, model_name, tr_set, preds_dir, tee)
    return model, curve


def fit2_inner(model_factory, cfg, model_name: str, sets: dict, preds_dir: str, opts: Fit2Opts = Fit2Opts(),
               target: str = "rtg"):
    """fit2_inner (src/lib.rs:881-996): tr -> pr, then fulltrain -> qual (or,
    with no_fulltrain, the phase-1 model predicts qual). `sets` maps "tr",
    "pr", "fulltrain_tr", "fulltrain_pr" to (name, Dataset); the fulltrain
    pair may be absent, which skips phase 2."""
    os.makedirs(preds_dir, exist_ok=True)
    tee = Tee(os.path.join(preds_dir, f"{model_name}.out"))
    try:
        tee.write(f"[{model_name}]\n")
        tee.write(f"target = {target!r}\n".replace("'", '"'))
        tee.write(f"{cfg}\n")
        (trn, tr), (prn, pr) = sets["tr"], sets["pr"]
        tee.write(_arrow(trn, prn, opts.transpose))
        qual = qual_name = None
        if opts.no_fulltrain and "fulltrain_pr" in sets:
            qual_name, qual = sets["fulltrain_pr"]
        if opts.transpose:
            tr, pr = tr.transpose(True), pr.transpose(False)
            qual = qual.transpose(False) if qual is not None else None
        model, curve = _train(model_factory, cfg, tr, pr, model_name, preds_dir, opts.save_probe_each_epoch, prn,
                              tee, qual, qual_name)
        pr_preds = gen_preds_parallel(model, pr)
        tee.write(f"{prn} RMSE {fmt5(rmse_from_preds(pr_preds, pr))}\n")
        np.save(os.path.join(preds_dir, f"{model_name}.{prn}.npy"), pr_preds)
        if opts.save_subscores and model.n_subscores() > 0:
            _save_subscores(model, pr, model_name, prn, preds_dir)
        if opts.save_train:
            np.save(os.path.join(preds_dir, f"{model_name}.{trn}.npy"), gen_preds_parallel(model, tr))
        _artifacts(model, model_name, trn, preds_dir, tee)
        if qual is not None:
            tee.write(f"{trn} => {qual_name} (no_fulltrain)\n")
            np.save(os.path.join(preds_dir, f"{model_name}.{qual_name}.npy"), gen_preds_parallel(model, qual))
            if opts.save_subscores and model.n_subscores() > 0:
                _save_subscores(model, qual, model_name, qual_name, preds_dir)
        if hasattr(model, "close"):
            model.close()
        del model
        if not opts.no_fulltrain and "fulltrain_tr" in sets:
            (ftn, ft), (fpn, fp) = sets["fulltrain_tr"], sets["fulltrain_pr"]
            m2, _ = fit(model_factory, cfg, ft, fp, model_name, preds_dir, opts, tee, ftn, fpn)
            if hasattr(m2, "close"):
                m2.close()
        tee.write("\n")
        return curve
    finally:
        tee.close()
