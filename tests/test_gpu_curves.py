"""Held-out RMSE curves of the GPU's deterministic schedule against the
reference algorithm, epoch by epoch, at the workloads' own sizes.

The reference curve of each case is a committed fixture written by
tests/golden/make_rmse_curves.py: the oracle's sequential TxModel
(src/tx.rs:734-1115, the reference's `fit_epoch`) on the seeded synthetic
data, with `calc_rmse` (src/lib.rs:659-672) on the held-out rows after every
epoch. Here the same data are regenerated from the same seed (the fixture's
fingerprint is checked first) and the GPU's stratified schedule, the
reference's own parallel schedule (src/tsvdx4p.rs:390-805), is trained with
the same hyperparameters and epoch count.

Tolerance: every epoch's held-out RMSE within +-0.001 of the reference's.
"""
import json
import os

import numpy as np
import pytest

from netflix_prize_b200.abi import SCHED_STRATIFIED
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TOL = 1e-3

_DATA = {}


def _case(case):
    import sys
    sys.path.insert(0, GOLDEN)
    import make_rmse_curves as mk
    with open(os.path.join(GOLDEN, f"rmse_curve_{case}.json")) as fh:
        ref = json.load(fh)
    spec_fn = mk.CASES[case][0]
    if spec_fn not in _DATA:
        _DATA.clear()  # one full-shape dataset in host memory at a time
        tr, pr, _, _ = mk.case_setup(case)
        _DATA[spec_fn] = (tr, pr, mk.fingerprint(tr, pr))
    tr, pr, fp = _DATA[spec_fn]
    from netflix_prize_b200.config import run_lm
    _, f, epochs = mk.CASES[case]
    return ref, tr, pr, fp, run_lm(f, epochs, n_time_bins=30)


def _run_curve(case, **model_kw):
    ref, tr, pr, fp, cfg = _case(case)
    assert ref["generator"]["fingerprint"] == fp, "regenerated data differ from the fixture's"
    # every epoch the committed curve holds (the full-shape curves take hours
    # of one CPU core to write)
    n = len(ref["epochs"])
    assert 1 <= n <= cfg.n_epochs
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, **model_kw)
    rows = []
    for e in range(1, n + 1):
        g.fit_epoch(tr, pr, e)
        rows.append((e, g.calc_rmse(pr), ref["epochs"][e - 1]["heldout_rmse"]))
    g.close()
    worst = max(abs(a - b) for _, a, b in rows)
    print(f"\n{case}: {n} of {cfg.n_epochs} epochs; epoch, gpu stratified, reference sequential, diff")
    for e, a, b in rows:
        print(f"  {e:3d} {a:.6f} {b:.6f} {a - b:+.6f}")
    print(f"{case}: worst |diff| {worst:.6f}")
    return rows, worst


def test_c1_curve_tracks_reference_every_epoch():
    """C1 as written: 10,000 users x 2,000 items, 1,000,000 ratings, f=32,
    20 epochs, T=30."""
    rows, worst = _run_curve("c1_f32")
    assert worst <= TOL, rows


@pytest.mark.parametrize("case", ["c2_f64", "c2_f256"])
def test_full_shape_curve_tracks_reference_every_epoch(case):
    """C2 (480,189 x 17,770, 100,480,507 ratings, f=64, 40 epochs) and the
    same data at f=256 for 60 epochs (C4's shape and length)."""
    rows, worst = _run_curve(case)
    assert worst <= TOL, rows
