#!/usr/bin/env python
"""Writes the reference algorithm's per-epoch held-out RMSE curves as fixtures.

The curve is the CPU oracle's sequential TxModel (tx4 mode, the reference's
`TxModel::fit_epoch`, src/tx.rs:734-1115, followed by `rebuild_ycache`,
src/tx.rs:391-418) trained on the seeded synthetic data of one workload, with
the held-out RMSE of `calc_rmse` (src/lib.rs:659-672) after every epoch. The
GPU tests regenerate the same data from the same seed (a fingerprint of the
generated arrays is stored beside the curve) and compare their own per-epoch
RMSE with it.

Cases (all with the tsvdx4 `lm` preset, src/bin/tsvdx4-new.rs:130-154, T=30):
  c1_f32    10,000 users x 2,000 items, 1,000,000 ratings, f=32, 20 epochs
  c2_f64    480,189 x 17,770, 100,480,507 ratings, f=64, 40 epochs
  c2_f256   the same data, f=256, 60 epochs

The full-shape cases take hours on one core (the reference's epoch is
single-threaded). The output file is rewritten after every epoch, so a run
that stops early leaves the epochs it finished.

  python tests/golden/make_rmse_curves.py --case c1_f32
  python tests/golden/make_rmse_curves.py --case c2_f64 --schedule p --workers 6

The second form writes the curve of the reference's parallel model
(rmse_curve_<case>_p.json), the algorithm the GPU's stratified schedule
restates, on host threads (bitwise the one-thread result).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CASES = {
    # name: (spec function name, n_feat, epochs)
    "c1_f32": ("spec_c1", 32, 20),
    "c2_f64": ("spec_c2", 64, 40),
    "c2_f256": ("spec_c2", 256, 60),
}


def fingerprint(tr, pr) -> str:
    """SHA-256 over the generated columns, so a consumer can check that it
    regenerated the same data."""
    h = hashlib.sha256()
    for d in (tr, pr):
        for name in ("user_idxs", "item_idxs", "raw_ratings", "dates", "is_test"):
            h.update(getattr(d, name).tobytes())
    return h.hexdigest()


def case_setup(case: str):
    """(train, pr, config) for one case; shared with the GPU tests."""
    from netflix_prize_b200 import synth
    from netflix_prize_b200.config import run_lm
    spec_fn, f, epochs = CASES[case]
    spec = getattr(synth, spec_fn)()
    tr, pr = synth.generate(spec)
    return tr, pr, run_lm(f, epochs, n_time_bins=30), spec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=sorted(CASES), required=True)
    ap.add_argument("--out", default=None)
    ap.add_argument("--schedule", choices=["seq", "p"], default="seq",
                    help="seq: TxModel::fit_epoch; p: Tsvdx4pModel (src/tsvdx4p.rs:815-822), one chunk")
    ap.add_argument("--workers", type=int, default=1, help="host threads of the p schedule (same result)")
    args = ap.parse_args()
    from netflix_prize_b200.data import MaskedDataset
    from oracle import pyoracle as po

    out = args.out or os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                   f"rmse_curve_{args.case}{'' if args.schedule == 'seq' else '_p'}.json")
    t0 = time.time()
    tr, pr, cfg, spec = case_setup(args.case)
    gen_s = time.time() - t0
    m = po.OracleModel(tr, MaskedDataset(pr), cfg)
    rec = {
        "case": args.case,
        "algorithm": ("TxModel::fit_epoch (src/tx.rs:734-1115), sequential, C++ restatement, 1 thread"
                      if args.schedule == "seq" else
                      "Tsvdx4pModel::fit_epoch (src/tsvdx4p.rs:815-822), one chunk, NSVD1 norm exponent 1, "
                      "C++ restatement"),
        "generator": {"spec": spec.__dict__.copy(), "fingerprint": fingerprint(tr, pr),
                      "n_train": int(tr.n_ratings), "n_pr": int(pr.n_ratings),
                      "n_heldout": int((pr.is_test == 0).sum())},
        "config": {"preset": "lm (src/bin/tsvdx4-new.rs:130-154)", "n_feat": cfg.n_feat, "n_epochs": cfg.n_epochs,
                   "n_time_bins": cfg.n_time_bins, "seed": cfg.seed, "low_memory": cfg.low_memory},
        "generate_s": gen_s,
        "epochs": [],
    }
    sched = po.SCHED_SEQ if args.schedule == "seq" else po.SCHED_P
    for e in range(1, cfg.n_epochs + 1):
        t = time.time()
        if sched == po.SCHED_SEQ:
            m.fit_epoch(e, sched)
        else:
            m.fit_epoch_parallel(e, nsvd_norm_exp=1.0, workers=args.workers)
        fit_s = time.time() - t
        r = m.calc_rmse(pr)
        rec["epochs"].append({"epoch": e, "heldout_rmse": r, "fit_s": round(fit_s, 2)})
        tmp = out + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(rec, fh, indent=1)
        os.replace(tmp, out)
        print(f"{args.case} epoch {e}: rmse {r:.6f} ({fit_s:.1f} s)", flush=True)


if __name__ == "__main__":
    main()
