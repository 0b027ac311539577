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


def test_job_table_covers_the_dispatchers_base_jobs():
    """All 19 tsvdx4 base jobs (src/bin/tsvdx4-new.rs:18-40), spot-checked
    against the presets (:118-556)."""
    from netflix_prize_b200.jobs import JOBS
    assert len(JOBS) == 19
    assert JOBS["tsvdx4-4800lm"].config.n_feat == 4800 and JOBS["tsvdx4-4800lm"].config.n_epochs == 27
    assert JOBS["tsvdx4-60"].config.low_memory is False and JOBS["tsvdx4-60"].save_train
    assert JOBS["tsvdx4-d0tb"].config.n_feat == 0 and JOBS["tsvdx4-p0tbo"].config.ordinal_head is not None
    assert JOBS["tsvdx4-q16tb"].config.n_time_bins == 48 and JOBS["tsvdx4-s20fo"].config.n_freq_bins == 24
    assert JOBS["tsvdx4-16-t"].transpose and JOBS["tsvdx4-16-t"].config.beta == 0.35
    assert JOBS["tsvdx4-80o"].save_subscores and not JOBS["tsvdx4-80o"].save_train
    for name, job in JOBS.items():
        c = job.config
        assert c.lr_w == c.lr_c == c.lr_w_day == c.lr_c_day == 0.0, name   # tx4 mode
        assert c.ordinal_head is None or c.ordinal_head.lr_t == 0.0, name


def test_transpose_swaps_roles_and_orders_by_item_then_date():
    """Dataset::transpose (src/lib.rs:295-405): with reorder, a stable order
    by (old item, date); without, the rows keep their order."""
    import numpy as np
    from netflix_prize_b200.data import Dataset
    rng = np.random.default_rng(3)
    u = np.sort(rng.integers(0, 50, 400))
    i = rng.integers(0, 30, 400)
    d = rng.integers(0, 100, 400)
    r = rng.integers(1, 6, 400)
    ds = Dataset.from_ratings(u, i, r, d, 50, 30, "t")
    t = ds.transpose(True)
    assert (t.n_users, t.n_items) == (30, 50) and t.transposed
    key = i.astype(np.int64) * 1000 + d
    o = np.argsort(key, kind="stable")
    assert np.array_equal(t.user_idxs, i[o]) and np.array_equal(t.item_idxs, u[o])
    assert np.array_equal(t.dates, d[o]) and np.array_equal(t.raw_ratings, r[o])
    assert np.array_equal(t.user_cnts, ds.item_cnts) and np.array_equal(t.item_cnts, ds.user_cnts)
    s = ds.transpose(False)
    assert np.array_equal(s.user_idxs, i) and np.array_equal(s.item_idxs, u)
