"""Held-out RMSE curves of the GPU's deterministic schedule against the
reference algorithms, epoch by epoch, at the workloads' own sizes.

The reference curves are committed fixtures: the oracle's sequential TxModel
(src/tx.rs:734-1115, the reference's `fit_epoch`) written by
tests/golden/make_rmse_curves.py, the oracle's parallel model
(Tsvdx4pModel, src/tsvdx4p.rs:390-822, the algorithm the stratified schedule
restates) written by the same script with `--schedule p`, and the FP64 run of
the parallel model at f=256 written by tests/golden/make_precision_c4.py.
Each curve is `calc_rmse` (src/lib.rs:659-672) on the held-out rows after
every epoch. Here the same data are regenerated from the same seed (the
fixture's fingerprint is checked first) and the GPU's stratified schedule is
trained with the same hyperparameters and epoch count.

Tolerances:
  - against the parallel model: every epoch within +-0.001;
  - against the sequential model at C1: every epoch within +-0.001;
  - against the sequential model at the full shape: the best held-out RMSE
    within +-0.001 (the two reference models' curves part by more than that
    in the middle of training: the parallel model takes one averaged NSVD1
    step per item and epoch where the sequential one takes one per rating);
  - precision forms against the FP64 parallel model: every epoch's held-out
    RMSE within +-0.001, and the final predictions of the sampled held-out
    rows within 2e-2 (after 60 epochs the FP32 and FP64 trajectories have
    parted by rounding alone: the measured FP32 maximum is 1.0e-2, mean
    6e-4; the figures are printed).
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


def _fixture(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} is not committed")
    with open(path) as fh:
        return json.load(fh)


def _data(case):
    import sys
    sys.path.insert(0, GOLDEN)
    import make_rmse_curves as mk
    spec_fn = mk.CASES[case][0]
    if spec_fn not in _DATA:
        _DATA.clear()  # one full-shape dataset in host memory at a time
        tr, pr, _, _ = mk.case_setup(case)
        _DATA[spec_fn] = (tr, pr, mk.fingerprint(tr, pr))
    return _DATA[spec_fn]


def _gpu_curve(case, n, precision=0):
    """The GPU stratified schedule's held-out RMSE after each of n epochs."""
    import make_rmse_curves as mk
    from netflix_prize_b200.config import run_lm
    tr, pr, _ = _data(case)
    _, f, epochs = mk.CASES[case]
    cfg = run_lm(f, epochs, n_time_bins=30)
    g = TxModel(tr, MaskedDataset(pr), cfg, schedule=SCHED_STRATIFIED, precision=precision)
    out = []
    for e in range(1, n + 1):
        g.fit_epoch(tr, pr, e)
        out.append(g.calc_rmse(pr))
    return out, g


def _check_fingerprint(case, ref):
    _, _, fp = _data(case)
    assert ref["generator"]["fingerprint"] == fp, "regenerated data differ from the fixture's"


def _report(title, got, want):
    print(f"\n{title}: epoch, gpu stratified, reference, diff")
    for e, (a, b) in enumerate(zip(got, want), 1):
        print(f"  {e:3d} {a:.6f} {b:.6f} {a - b:+.6f}")
    worst = max(abs(a - b) for a, b in zip(got, want))
    print(f"{title}: worst |diff| {worst:.6f}")
    return worst


def test_c1_curve_tracks_sequential_reference_every_epoch():
    """C1 as written: 10,000 users x 2,000 items, 1,000,000 ratings, f=32,
    20 epochs, T=30, against the sequential reference."""
    ref = _fixture("rmse_curve_c1_f32.json")
    _check_fingerprint("c1_f32", ref)
    want = [x["heldout_rmse"] for x in ref["epochs"]]
    got, g = _gpu_curve("c1_f32", len(want))
    g.close()
    assert _report("c1_f32 vs sequential", got, want) <= TOL


@pytest.mark.parametrize("case", ["c2_f64", "c2_f256"])
def test_full_shape_curve(case):
    """C2 (480,189 x 17,770, 100,480,507 ratings, f=64, 40 epochs) and the
    same data at f=256 for 60 epochs (C4's shape and length): every epoch
    against the parallel reference model, and the best held-out RMSE against
    the sequential one (every epoch printed)."""
    seq = _fixture(f"rmse_curve_{case}.json")
    _check_fingerprint(case, seq)
    par_name = f"rmse_curve_{case}_p.json" if case != "c2_f256" else "precision_c4_fp64.json"
    par = None
    if os.path.exists(os.path.join(GOLDEN, par_name)):
        par = _fixture(par_name)
        _check_fingerprint(case, par)
    n_seq = len(seq["epochs"])
    n_par = len(par["epochs"]) if par else 0
    got, g = _gpu_curve(case, max(n_seq, n_par))
    g.close()
    if par:
        want = [x["heldout_rmse"] for x in par["epochs"]]
        assert _report(f"{case} vs parallel model", got[:n_par], want) <= TOL
    want = [x["heldout_rmse"] for x in seq["epochs"]]
    _report(f"{case} vs sequential model", got[:n_seq], want)
    import make_rmse_curves as mk
    if n_seq == mk.CASES[case][2]:
        best_gpu, best_ref = min(got[:n_seq]), min(want)
        print(f"{case}: best held-out RMSE gpu {best_gpu:.6f} (epoch {int(np.argmin(got[:n_seq])) + 1}), "
              f"sequential reference {best_ref:.6f} (epoch {int(np.argmin(want)) + 1})")
        assert abs(best_gpu - best_ref) <= TOL


@pytest.mark.parametrize("precision,rmse_tol,pred_tol", [(0, 1e-3, 2e-2), (1, 1e-3, 2e-2), (2, 1e-3, 2e-2)])
def test_precision_forms_against_fp64_at_full_shape(precision, rmse_tol, pred_tol):
    """C4: the full shape at f=256 for 60 epochs, FP32 masters with FP32,
    BF16-item-table and BF16-everything read copies, each against the FP64
    run of the same schedule: held-out RMSE every epoch and the final
    predictions of the fixture's sample of held-out rows."""
    ref = _fixture("precision_c4_fp64.json")
    _check_fingerprint("c2_f256", ref)
    want = [x["heldout_rmse"] for x in ref["epochs"]]
    got, g = _gpu_curve("c2_f256", len(want), precision=precision)
    worst = _report(f"precision {precision} vs fp64", got, want)
    if "sample" in ref:
        tr, pr, _ = _data("c2_f256")
        rows = np.asarray(ref["sample"]["rows"], np.int64)
        p64 = np.asarray(ref["sample"]["pred_fp64"], np.float64)
        pg = g.predict_batch(pr.user_idxs[rows], pr.item_idxs[rows], pr.dates[rows]).astype(np.float64)
        err = np.abs(pg - p64)
        print(f"precision {precision}: predictions of {rows.size} held-out rows after {len(want)} epochs: "
              f"max |gpu - fp64| {err.max():.3e}, mean {err.mean():.3e}")
        assert err.max() < pred_tol
    g.close()
    assert worst <= rmse_tol
