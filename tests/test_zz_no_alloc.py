"""The allocation-free RMSE entry point, called through the C ABI.

It is for callers that cannot allocate device memory when they evaluate; it
must give the same RMSE as tsvd_calc_rmse (the allocating path) on the same
rows, call after call, although every call reuses the same fixed scratch.
This file is collected last so a stop-at-first-failure run has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from netflix_prize_b200 import native
from netflix_prize_b200.config import run_lm
from netflix_prize_b200.data import MaskedDataset
from netflix_prize_b200.model import TxModel

pytestmark = pytest.mark.gpu


def _rmse_noalloc(model, tensors, n):
    import torch
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the model's stream does not wait for torch's
    u, i, d, t, z = tensors
    rc = native.load().tsvd_calc_rmse_device_noalloc(
        model.h, C.c_void_p(u.data_ptr()), C.c_void_p(i.data_ptr()), C.c_void_p(d.data_ptr()),
        C.c_void_p(t.data_ptr()), C.c_void_p(z.data_ptr()), n, C.c_void_p(out.data_ptr()))
    assert rc == 0, native.load().tsvd_last_error(model.h).decode()
    model.synchronize()
    return out.cpu().numpy()


def test_noalloc_rmse_matches_allocating_path_twice():
    import torch
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=2000, n_items=500, n_train=120000, seed=11)
    model = TxModel(tr, MaskedDataset(pr), run_lm(48, 2, n_time_bins=30))
    model.fit_epoch(tr, pr, 1)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for ds in (pr, tr):  # held-out set (with is_test rows) and the training set
        tensors = (dev(ds.user_idxs), dev(ds.item_idxs), dev(ds.dates), dev(ds.residuals), dev(ds.is_test))
        want = model.calc_rmse(ds)
        first = _rmse_noalloc(model, tensors, ds.n_ratings)
        second = _rmse_noalloc(model, tensors, ds.n_ratings)
        assert first[0] == pytest.approx(want, rel=1e-12, abs=0.0)
        assert np.array_equal(first, second)
        assert first[2] == float((ds.is_test == 0).sum())


def test_noalloc_rejects_rows_beyond_its_scratch():
    from tests.conftest import tiny_sets
    tr, pr = tiny_sets()
    model = TxModel(tr, MaskedDataset(pr), run_lm(8, 1, n_time_bins=4).replace(n_freq_bins=4))
    L = native.load()
    fake = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.tsvd_calc_rmse_device_noalloc(model.h, fake, fake, fake, fake, None, 134217729, fake)
    assert rc == 1
    assert "exceed the maximum of 134217728" in L.tsvd_last_error(model.h).decode()


def test_noalloc_reports_out_of_range_rows_instead_of_reading_them():
    """Device rows are not checked on the host: a user or item index outside
    the model's tables is skipped on the device and reported as
    {NaN, NaN, -(rows out of range)}."""
    import torch
    from tests.conftest import small_sets
    tr, pr = small_sets(n_users=2000, n_items=500, n_train=120000, seed=11)
    model = TxModel(tr, MaskedDataset(pr), run_lm(48, 1, n_time_bins=30))
    u = pr.user_idxs.copy()
    i = pr.item_idxs.copy()
    held = np.nonzero(pr.is_test == 0)[0]
    u[held[0]] = pr.n_users          # one past the last user
    i[held[1]] = -1                  # negative item
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tensors = (dev(u), dev(i), dev(pr.dates), dev(pr.residuals), dev(pr.is_test))
    out = _rmse_noalloc(model, tensors, pr.n_ratings)
    assert np.isnan(out[0]) and np.isnan(out[1]) and out[2] == -2.0
    # the scratch keeps no trace of it: the next call on valid rows is exact
    ok = (dev(pr.user_idxs), dev(pr.item_idxs), dev(pr.dates), dev(pr.residuals), dev(pr.is_test))
    assert _rmse_noalloc(model, ok, pr.n_ratings)[0] == pytest.approx(model.calc_rmse(pr), rel=1e-12, abs=0.0)
