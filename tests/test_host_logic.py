"""Host-side logic: dataset I/O in the reference's layout, driver helpers,
and the synthetic generator's invariants."""
import numpy as np
import pytest

from netflix_prize_b200 import synth
from netflix_prize_b200.data import Dataset, calc_user_offsets
from netflix_prize_b200.driver import rmse_from_preds


def test_dataset_npy_round_trip(tmp_path, tiny):
    tr, _ = tiny
    tr.save(str(tmp_path))
    back = Dataset.load("tiny_train", root=str(tmp_path))
    for f in ("user_idxs", "item_idxs", "raw_ratings", "dates", "is_test", "user_cnts", "item_cnts"):
        assert np.array_equal(getattr(tr, f), getattr(back, f))
    assert np.array_equal(back.residuals, tr.raw_ratings.astype(np.float32))
    # items are i16 on disk (src/bin/newsplit.rs:369-387)
    assert np.load(tmp_path / "tiny_train" / "item_idxs.npy").dtype == np.int16


def test_residual_target_spec(tmp_path, tiny):
    tr, _ = tiny
    tr.save(str(tmp_path))
    preds = np.linspace(1, 2, tr.n_ratings).astype(np.float32)
    pd = tmp_path / "preds"
    pd.mkdir()
    np.save(pd / "m1.tiny_train.npy", preds)
    ds = Dataset.load("tiny_train", root=str(tmp_path), target="0.5*m1", preds_dir=str(pd))
    assert np.allclose(ds.residuals, tr.raw_ratings - 0.5 * preds)


def test_rmse_from_preds_skips_test_rows():
    ds = Dataset.from_ratings([0, 0, 1], [0, 1, 0], [3, 4, 5], [1, 2, 3], 2, 2, is_test=[0, 1, 0])
    preds = np.array([3.5, 100.0, 4.0], np.float32)
    assert rmse_from_preds(preds, ds) == pytest.approx(np.sqrt((0.25 + 1.0) / 2))


@pytest.mark.parametrize("spec", [synth.scaled(synth.spec_c1(5), 500, 200, 20000, "t")])
def test_generator_invariants(spec):
    tr, pr = synth.generate(spec)
    assert tr.n_ratings == spec.n_train
    calc_user_offsets(tr)  # user-sorted
    assert np.all(np.diff(tr.user_idxs.astype(np.int64) * spec.n_items + tr.item_idxs) > 0)  # (user, item) order
    assert np.all(np.diff(pr.item_idxs.astype(np.int64) * spec.n_users + pr.user_idxs) > 0)  # (item, user) order
    k = np.concatenate([tr.user_idxs.astype(np.int64) * spec.n_items + tr.item_idxs,
                        pr.user_idxs.astype(np.int64) * spec.n_items + pr.item_idxs])
    assert len(np.unique(k)) == len(k)
    assert tr.raw_ratings.min() >= 1 and tr.raw_ratings.max() <= 5
    held = pr.is_test == 0
    assert pr.raw_ratings[held].min() >= 1 and np.all(pr.raw_ratings[~held] == 0)
    assert np.array_equal(np.bincount(tr.user_idxs, minlength=spec.n_users), tr.user_cnts)
    assert tr.dates.min() >= 0 and tr.dates.max() <= 2242
    # held-out rows are each user's latest-dated ones
    last_train = np.zeros(spec.n_users, np.int64)
    np.maximum.at(last_train, tr.user_idxs, tr.dates)
    first_held = np.full(spec.n_users, 10**9)
    np.minimum.at(first_held, pr.user_idxs[held], pr.dates[held])
    has = first_held < 10**9
    assert np.all(first_held[has] >= last_train[has])


def test_generator_is_seeded():
    s = synth.scaled(synth.spec_c1(11), 200, 100, 5000, "t")
    a, _ = synth.generate(s)
    b, _ = synth.generate(s)
    assert np.array_equal(a.item_idxs, b.item_idxs) and np.array_equal(a.raw_ratings, b.raw_ratings)
