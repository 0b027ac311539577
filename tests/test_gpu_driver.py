"""The driver's file outputs (fit2_inner / fit, src/lib.rs:764-996, and
save_artifacts, src/tx.rs:726-732), with the GPU model behind the reference's
Regressor surface, against the same driver run over the oracle.

Checked: the exact set of output file names, every .npy within 1e-5 of the
oracle's (the sequential schedule, which is the reference's fit_epoch), and
the .out log line for line (RMSE figures within 1e-4).
"""
import os

import numpy as np
import pytest

from netflix_prize_b200 import driver
from netflix_prize_b200.abi import SCHED_SEQUENTIAL
from netflix_prize_b200.config import regression_test_config
from netflix_prize_b200.data import Dataset
from netflix_prize_b200.model import TxModel
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


class OracleRegressor:
    """The oracle behind the same surface the driver calls (test only)."""

    def __init__(self, tr, pr, cfg):
        self.o = po.OracleModel(tr, pr, cfg)
        self.cfg = cfg

    def n_epochs(self):
        return self.cfg.n_epochs

    def fit_epoch(self, tr, pr, epoch):
        self.o.fit_epoch(epoch)

    def calc_rmse(self, ds):
        return self.o.calc_rmse(ds)

    def gen_preds(self, ds):
        # gen_preds_parallel (src/lib.rs:710-722): predict + (raw - residual), f32
        p = self.o.predict_batch(ds.user_idxs, ds.item_idxs, ds.dates).astype(np.float32)
        return p + (ds.raw_ratings.astype(np.float32) - ds.residuals)

    def n_subscores(self):
        return 3

    def subscore_names(self):
        return ["bias", "mf", "nsvd1"]

    def predict_subscores_batch(self, u, i, d):
        return self.o.predict_subscores_batch(u, i, d).astype(np.float32)

    def save_artifacts(self, name, tr_set, preds_dir):
        if self.cfg.save_ifeat:
            path = os.path.join(preds_dir, f"{name}.ifeat.{tr_set}.npy")
            np.save(path, self.o.get_param("ifeat").astype(np.float32).reshape(-1, self.cfg.n_feat))
            return path
        return None


def _qual(pr):
    """A qual-like set: the probe rows marked as test examples."""
    return Dataset.from_ratings(pr.user_idxs, pr.item_idxs, pr.raw_ratings, pr.dates, pr.n_users, pr.n_items,
                                "qual", is_test=np.ones(pr.n_ratings, np.int8))


def _run(factory, tmp, tiny, opts):
    tr, pr = tiny
    sets = {"tr": ("trainx", tr), "pr": ("probex", pr), "fulltrain_tr": ("fulltrain", tr),
            "fulltrain_pr": ("qual", _qual(pr))}
    cfg = regression_test_config(low_memory=True, save_ifeat=True)
    driver.fit2_inner(factory, cfg, "tsvdx4-t", sets, str(tmp), opts)
    return sorted(os.listdir(tmp))


@pytest.mark.parametrize("no_fulltrain", [False, True])
def test_fit2_inner_outputs_match_the_oracle_run(tmp_path, tiny, no_fulltrain):
    opts = driver.Fit2Opts(save_train=True, save_probe_each_epoch=True, save_subscores=True,
                           no_fulltrain=no_fulltrain)
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gfiles = _run(lambda tr, pr, cfg: TxModel(tr, pr, cfg, schedule=SCHED_SEQUENTIAL), gdir, tiny, opts)
    ofiles = _run(OracleRegressor, odir, tiny, opts)
    assert gfiles == ofiles
    want = {"tsvdx4-t.out", "tsvdx4-t.probex.npy", "tsvdx4-t.trainx.npy", "tsvdx4-t.ifeat.trainx.npy",
            "tsvdx4-t.qual.npy", "tsvdx4-t-bias.probex.npy", "tsvdx4-t-mf.probex.npy", "tsvdx4-t-nsvd1.probex.npy",
            "tsvdx4-t-bias.qual.npy", "tsvdx4-t-mf.qual.npy", "tsvdx4-t-nsvd1.qual.npy"}
    want |= {f"tsvdx4-t_ep{e:02d}.probex.npy" for e in (1, 2, 3)}
    if no_fulltrain:
        want |= {f"tsvdx4-t_ep{e:02d}.qual.npy" for e in (1, 2, 3)}
    else:
        want |= {f"tsvdx4-t_ep{e:02d}.qual.npy" for e in (1, 2, 3)}
        want |= {"tsvdx4-t.fulltrain.npy", "tsvdx4-t.ifeat.fulltrain.npy"}
    assert set(gfiles) == want, sorted(set(gfiles) ^ want)
    for f in gfiles:
        if f.endswith(".npy"):
            a, b = np.load(gdir / f), np.load(odir / f)
            assert a.dtype == np.float32 and a.shape == b.shape, f
            assert np.max(np.abs(a - b)) < 1e-5, f
    gl = (gdir / "tsvdx4-t.out").read_text().splitlines()
    ol = (odir / "tsvdx4-t.out").read_text().splitlines()
    assert len(gl) == len(ol)
    for a, b in zip(gl, ol):
        if "RMSE" in a:
            assert a.split("RMSE")[0] == b.split("RMSE")[0]
            x, y = float(a.split("RMSE")[1]), float(b.split("RMSE")[1])
            # a set of test rows only (qual) has no RMSE: NaN, printed "NaN"
            assert (x != x and y != y and a.endswith("NaN")) or abs(x - y) < 1e-4, (a, b)
        elif a.startswith("Saved item factors to "):
            assert os.path.basename(a) == os.path.basename(b)
        else:
            assert a == b
    assert gl[0] == "[tsvdx4-t]" and gl[1] == 'target = "rtg"' and gl[3] == "trainx => probex"
