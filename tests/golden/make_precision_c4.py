#!/usr/bin/env python
"""Writes the FP64 reference of the precision-form workload as a fixture.

The workload: the full-shape synthetic data (480,189 users x 17,770 items,
100,480,507 ratings), the tsvdx4 `lm` preset (src/bin/tsvdx4-new.rs:130-154)
at f=256 with 30 time bins, 60 epochs of the stratified schedule
(Tsvdx4pModel::fit_epoch, src/tsvdx4p.rs:815-822, one chunk, NSVD1 norm
exponent 1). The oracle runs it in FP64 on host threads (the same arithmetic
and order as its one-thread form). Recorded: the held-out RMSE (calc_rmse,
src/lib.rs:659-672) after every epoch, and the final predictions of a seeded
sample of held-out rows. The GPU's precision forms are stated against these.

The file is rewritten after every epoch (the predictions only at the end).

  python tests/golden/make_precision_c4.py --workers 6
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

F, EPOCHS, SAMPLE, SAMPLE_SEED = 256, 60, 4096, 20240


def sample_rows(pr) -> np.ndarray:
    """Row indices of the held-out sample (held-out rows only, seeded)."""
    held = np.flatnonzero(pr.is_test == 0)
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(held, size=min(SAMPLE, held.size), replace=False))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=6)
    ap.add_argument("--epochs", type=int, default=EPOCHS)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "precision_c4_fp64.json"))
    args = ap.parse_args()
    import make_rmse_curves as mk
    from netflix_prize_b200 import synth
    from netflix_prize_b200.config import run_lm
    from netflix_prize_b200.data import MaskedDataset
    from oracle import pyoracle as po

    spec = synth.spec_c2()
    tr, pr = synth.generate(spec)
    cfg = run_lm(F, args.epochs, n_time_bins=30)
    m = po.OracleModel(tr, MaskedDataset(pr), cfg, fp64=True)
    rows = sample_rows(pr)
    rec = {
        "algorithm": "Tsvdx4pModel::fit_epoch (src/tsvdx4p.rs:815-822), one chunk, NSVD1 norm exponent 1, "
                     "FP64 C++ restatement on host threads",
        "generator": {"spec": spec.__dict__.copy(), "fingerprint": mk.fingerprint(tr, pr)},
        "config": {"preset": "lm (src/bin/tsvdx4-new.rs:130-154)", "n_feat": F, "n_epochs": args.epochs,
                   "n_time_bins": 30, "seed": cfg.seed, "low_memory": cfg.low_memory},
        "workers": args.workers, "sample_seed": SAMPLE_SEED, "epochs": [],
    }

    def write():
        tmp = args.out + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(rec, fh, indent=1)
        os.replace(tmp, args.out)

    for e in range(1, args.epochs + 1):
        t = time.time()
        m.fit_epoch_parallel(e, nsvd_norm_exp=1.0, workers=args.workers)
        r = m.calc_rmse(pr)
        rec["epochs"].append({"epoch": e, "heldout_rmse": r, "fit_s": round(time.time() - t, 1)})
        write()
        print(f"epoch {e}: fp64 rmse {r:.7f} ({time.time() - t:.1f} s)", flush=True)
    pred = m.predict_batch(pr.user_idxs[rows], pr.item_idxs[rows], pr.dates[rows])
    rec["sample"] = {"rows": rows.tolist(), "pred_fp64": [float(x) for x in pred]}
    write()


if __name__ == "__main__":
    main()
