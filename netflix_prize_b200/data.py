"""Dataset / MaskedDataset host types and the on-disk .npy layout.

Mirrors `Dataset` (src/lib.rs:227-242), `Dataset::load` (src/lib.rs:252-290),
`MaskedDataset` (src/lib.rs:421-455), `calc_gbias` (src/lib.rs:463-467),
`calc_user_offsets` (src/lib.rs:470-483) and the per-set file layout written by
the reference's ingest/newsplit tools (src/bin/newsplit.rs:369-387):
data/<set>/{user_idxs i32, user_cnts i32, item_idxs i16, item_cnts i32,
item_years i32, ratings i8, dates i16, is_test i8}.npy.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from .abi import TsvdDatasetView, ptr
import ctypes as C


@dataclass
class Dataset:
    user_idxs: np.ndarray        # i32 [n_ratings]
    user_cnts: np.ndarray        # i32 [n_users]
    item_idxs: np.ndarray        # i32 [n_ratings]
    item_cnts: np.ndarray        # i32 [n_items]
    item_years: np.ndarray       # i32 [n_items]
    raw_ratings: np.ndarray      # i8  [n_ratings]
    residuals: np.ndarray        # f32 [n_ratings]
    dates: np.ndarray            # i16 [n_ratings]
    is_test: np.ndarray          # i8  [n_ratings]
    name: str
    n_users: int
    n_items: int
    n_ratings: int
    transposed: bool = False
    _keep: list = field(default_factory=list, repr=False)

    @staticmethod
    def from_ratings(user_idxs, item_idxs, raw_ratings, dates, n_users, n_items, name="ds", is_test=None):
        """Build in memory, as tests/helpers.rs:9-33 does (residuals = ratings)."""
        u = np.ascontiguousarray(user_idxs, dtype=np.int32)
        i = np.ascontiguousarray(item_idxs, dtype=np.int32)
        r = np.ascontiguousarray(raw_ratings, dtype=np.int8)
        d = np.ascontiguousarray(dates, dtype=np.int16)
        n = len(u)
        t = np.zeros(n, np.int8) if is_test is None else np.ascontiguousarray(is_test, dtype=np.int8)
        return Dataset(
            user_idxs=u, user_cnts=np.bincount(u, minlength=n_users).astype(np.int32),
            item_idxs=i, item_cnts=np.bincount(i, minlength=n_items).astype(np.int32),
            item_years=(2000 + np.arange(n_items)).astype(np.int32),
            raw_ratings=r, residuals=r.astype(np.float32), dates=d, is_test=t,
            name=name, n_users=int(n_users), n_items=int(n_items), n_ratings=n)

    @staticmethod
    def load(name: str, root: str = "data", n_users: int | None = None, n_items: int | None = None,
             target: str = "rtg", preds_dir: str = "preds"):
        """Dataset::load (src/lib.rs:252-290) for target "rtg" or "w*model + ..."
        residual specs. n_users/n_items default to the arrays' lengths (the
        reference hard-codes 480,189 and 17,770 at src/lib.rs:280-281)."""
        base = os.path.join(root, name)
        rd = lambda f: np.load(os.path.join(base, f))
        user_idxs = rd("user_idxs.npy").astype(np.int32)
        user_cnts = rd("user_cnts.npy").astype(np.int32)
        item_idxs = rd("item_idxs.npy").astype(np.int32)
        item_cnts = rd("item_cnts.npy").astype(np.int32)
        item_years = rd("item_years.npy").astype(np.int32)
        raw = rd("ratings.npy").astype(np.int8)
        dates = rd("dates.npy").astype(np.int16)
        is_test = rd("is_test.npy").astype(np.int8)
        residuals = raw.astype(np.float32)
        if target != "rtg":
            for term in target.split(" + "):
                if "*" in term:
                    w, model = term.split("*", 1)
                    w = float(w)
                else:
                    w, model = 1.0, term
                preds = np.load(os.path.join(preds_dir, f"{model.strip()}.{name}.npy")).astype(np.float32)
                residuals = residuals - preds * np.float32(w)
        return Dataset(user_idxs, user_cnts, item_idxs, item_cnts, item_years, raw,
                       np.ascontiguousarray(residuals, np.float32), dates, is_test, name,
                       int(n_users if n_users is not None else len(user_cnts)),
                       int(n_items if n_items is not None else len(item_cnts)), len(raw))

    def save(self, root: str = "data"):
        """Write the reference's per-set .npy layout (items as i16 on disk)."""
        base = os.path.join(root, self.name)
        os.makedirs(base, exist_ok=True)
        np.save(os.path.join(base, "user_idxs.npy"), self.user_idxs.astype(np.int32))
        np.save(os.path.join(base, "user_cnts.npy"), self.user_cnts.astype(np.int32))
        np.save(os.path.join(base, "item_idxs.npy"), self.item_idxs.astype(np.int16))
        np.save(os.path.join(base, "item_cnts.npy"), self.item_cnts.astype(np.int32))
        np.save(os.path.join(base, "item_years.npy"), self.item_years.astype(np.int32))
        np.save(os.path.join(base, "ratings.npy"), self.raw_ratings.astype(np.int8))
        np.save(os.path.join(base, "dates.npy"), self.dates.astype(np.int16))
        np.save(os.path.join(base, "is_test.npy"), self.is_test.astype(np.int8))

    def contains_test_examples(self) -> bool:
        return bool((self.is_test != 0).any())

    def transpose(self, reorder: bool) -> "Dataset":
        """Dataset::transpose (src/lib.rs:295-405): users and items swap roles.
        With `reorder` the ratings are stably sorted by (old item, date), which
        is what the reference's two-pass 16-bit radix sort of the key
        item * n_days + date produces; without it the order is kept."""
        if reorder:
            n_days = int(self.dates.max()) + 1
            key = self.item_idxs.astype(np.uint64) * np.uint64(n_days) + self.dates.astype(np.uint64)
            o = np.argsort(key.astype(np.uint32), kind="stable")
        else:
            o = np.arange(self.n_ratings)
        return Dataset(
            user_idxs=np.ascontiguousarray(self.item_idxs[o], np.int32),
            user_cnts=self.item_cnts.copy(),
            item_idxs=np.ascontiguousarray(self.user_idxs[o], np.int32),
            item_cnts=self.user_cnts.copy(),
            item_years=np.zeros(self.n_users, np.int32),
            raw_ratings=np.ascontiguousarray(self.raw_ratings[o]),
            residuals=np.ascontiguousarray(self.residuals[o]),
            dates=np.ascontiguousarray(self.dates[o]),
            is_test=np.ascontiguousarray(self.is_test[o]),
            name=self.name, n_users=self.n_items, n_items=self.n_users, n_ratings=self.n_ratings,
            transposed=not self.transposed)

    def view(self, masked: bool = False) -> TsvdDatasetView:
        v = TsvdDatasetView()
        v.user_idxs = ptr(self.user_idxs, C.c_int32)
        v.user_cnts = ptr(self.user_cnts, C.c_int32)
        v.item_idxs = ptr(self.item_idxs, C.c_int32)
        v.item_cnts = ptr(self.item_cnts, C.c_int32)
        v.raw_ratings = ptr(None if masked else self.raw_ratings, C.c_int8)
        v.residuals = ptr(None if masked else self.residuals, C.c_float)
        v.dates = ptr(self.dates, C.c_int16)
        v.is_test = ptr(self.is_test, C.c_int8)
        v.n_users = self.n_users
        v.n_items = self.n_items
        v.n_ratings = self.n_ratings
        return v


class MaskedDataset:
    """Training-time view of a pr set without ratings/residuals (src/lib.rs:421-455)."""

    def __init__(self, ds: Dataset):
        self._ds = ds
        for f in ("user_idxs", "user_cnts", "item_idxs", "item_cnts", "item_years", "dates", "is_test",
                  "name", "n_users", "n_items", "n_ratings", "transposed"):
            setattr(self, f, getattr(ds, f))

    @staticmethod
    def from_(ds: Dataset) -> "MaskedDataset":
        return MaskedDataset(ds)

    def view(self) -> TsvdDatasetView:
        return self._ds.view(masked=True)


def calc_gbias(tr: Dataset) -> np.float32:
    """FP64 mean of residuals cast to f32 (src/lib.rs:463-467)."""
    return np.float32(tr.residuals.astype(np.float64).sum() / tr.n_ratings)


def calc_user_offsets(tr: Dataset) -> np.ndarray:
    """Prefix sum of user_cnts; raises on unsorted input (src/lib.rs:470-483)."""
    d = np.diff(tr.user_idxs.astype(np.int64))
    bad = np.nonzero(d < 0)[0]
    if len(bad):
        t = int(bad[0]) + 1
        raise ValueError(f"dataset '{tr.name}' is not user-sorted at index {t}: user "
                         f"{tr.user_idxs[t]} follows user {tr.user_idxs[t - 1]}")
    off = np.zeros(tr.n_users + 1, np.int64)
    np.cumsum(tr.user_cnts, out=off[1:])
    return off
