"""Seeded synthetic stand-in for the Netflix Prize data (absent here).

Produces a training set and a pr set in the reference's in-memory/on-disk
layout (src/lib.rs:227-242; src/bin/newsplit.rs:298-387): train sorted by
(user, item), pr sorted by (item, user); the pr set holds held-out ratings
(is_test = 0, each user's latest-dated ones) and unrated query pairs
(is_test = 1, rating 0), both of which enter N(u) as probe/qual items do
(src/tx.rs:587-598, 402-408).

Ratings follow a planted model: mu + b_u + b_i + per-user linear drift over
time + rank-16 Gaussian factors + N(0, 0.9) noise, rounded and clipped to
1..5. Item popularity is Zipf(s) over a shuffled item order; user activity is
lognormal with the given median, clipped. Each user rates on a few "session"
days inside a personal activity window, so (user, day) frequency bins are
populated as in the real data.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .data import Dataset

N_DAYS = 2243  # days 0..2242 (src/lib.rs:17-20)


@dataclass
class SynthSpec:
    n_users: int
    n_items: int
    n_train: int            # exact number of training ratings
    zipf_s: float
    median_cnt: float
    max_cnt: int
    n_heldout: int | None   # exact total held-out rows, or None for "<= max_heldout per user"
    max_heldout: int
    n_query: int | None     # exact total query pairs, or None for "uniform 0..max_query per user"
    max_query: int
    seed: int
    rank: int = 16
    noise: float = 0.9
    name: str = "synth"


def spec_c1(seed: int = 1) -> SynthSpec:
    """10,000 users x 2,000 items, 1,000,000 training ratings."""
    return SynthSpec(10_000, 2_000, 1_000_000, 1.0, 90.0, 5_000, None, 9, None, 20, seed, name="c1")


def spec_c2(seed: int = 2) -> SynthSpec:
    """Netflix shape: 480,189 x 17,770, 100,480,507 training ratings."""
    return SynthSpec(480_189, 17_770, 100_480_507, 1.1, 96.0, 17_000, 1_408_395, 9, 2_817_131, 20, seed,
                     name="c2")


def spec_c3(seed: int = 3) -> SynthSpec:
    """25M-rating subset shape: 120,000 users x 17,770 items."""
    return SynthSpec(120_000, 17_770, 25_000_000, 1.1, 96.0, 17_000, None, 9, None, 20, seed, name="c3")


def scaled(spec: SynthSpec, n_users: int, n_items: int, n_train: int, name: str) -> SynthSpec:
    """Same generator at another size (held-out/query as per-user caps)."""
    return SynthSpec(n_users, n_items, n_train, spec.zipf_s, spec.median_cnt, min(spec.max_cnt, n_items // 2),
                     None, spec.max_heldout, None, spec.max_query, spec.seed, spec.rank, spec.noise, name)


def _exact_total(rng, w: np.ndarray, total: int, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """Integer vector proportional to w, clipped to [lo, hi], summing to total."""
    w = np.asarray(w, np.float64)
    x = np.clip(np.floor(w * (total / w.sum())), lo, hi).astype(np.int64)
    for _ in range(64):
        d = total - int(x.sum())
        if d == 0:
            return x
        room = (hi - x) if d > 0 else (x - lo)
        cand = np.nonzero(room > 0)[0]
        if len(cand) == 0:
            raise ValueError("cannot reach the requested total within the bounds")
        k = min(abs(d), len(cand))
        pick = rng.choice(cand, size=k, replace=False, p=None)
        x[pick] += 1 if d > 0 else -1
    raise ValueError("total not reached")


def _sample_items(rng, cnt: np.ndarray, cdf: np.ndarray, n_items: int, exclude=None, chunk_draws=1 << 24):
    """Per user, `cnt[u]` distinct items drawn by weight without replacement
    (draw with replacement, keep first occurrences in draw order, top up any
    shortfall). Keys in sorted `exclude` (user * n_items + item) are never
    chosen. Returns (users, items) grouped by user, items in draw order."""
    n_users = len(cnt)
    ex_key = exclude if exclude is not None else np.zeros(0, np.int64)
    out_u, out_i = [], []
    # user chunks of about chunk_draws draws each
    per = np.ceil(cnt * 1.3).astype(np.int64) + 4
    bounds = [0]
    acc = 0
    for u in range(n_users):
        acc += int(per[u])
        if acc >= chunk_draws:
            bounds.append(u + 1)
            acc = 0
    if bounds[-1] != n_users:
        bounds.append(n_users)
    for u0, u1 in zip(bounds[:-1], bounds[1:]):
        need = cnt[u0:u1].astype(np.int64)
        have_k = np.zeros(0, np.int64)   # user * n_items + item
        have_o = np.zeros(0, np.int64)   # draw order
        order_base = 0
        lo = np.searchsorted(ex_key, u0 * n_items)
        hi = np.searchsorted(ex_key, u1 * n_items)
        exk = ex_key[lo:hi]
        for _ in range(200):
            got = np.bincount(have_k // n_items - u0, minlength=u1 - u0) if len(have_k) else np.zeros(u1 - u0, np.int64)
            deficit = need - got
            if deficit.max(initial=0) <= 0:
                break
            draws = np.where(deficit > 0, np.ceil(deficit * 1.3).astype(np.int64) + 4, 0)
            du = np.repeat(np.arange(u0, u1, dtype=np.int64), draws)
            di = np.searchsorted(cdf, rng.random(len(du)), side="right").astype(np.int64)
            np.minimum(di, n_items - 1, out=di)
            dk = du * n_items + di
            do = order_base + np.arange(len(dk), dtype=np.int64)
            order_base += len(dk)
            if len(exk):
                pos = np.minimum(np.searchsorted(exk, dk), len(exk) - 1)
                keep = exk[pos] != dk
                dk, do = dk[keep], do[keep]
            ak = np.concatenate([have_k, dk])
            ao = np.concatenate([have_o, do])
            s = np.argsort(ak, kind="stable")      # equal keys keep draw order
            ak, ao = ak[s], ao[s]
            first = np.ones(len(ak), bool)
            first[1:] = ak[1:] != ak[:-1]
            ak, ao = ak[first], ao[first]
            au = ak // n_items
            s = np.argsort(au * order_base + ao)   # by user, then draw order
            ak, ao, au = ak[s], ao[s], au[s]
            starts = np.searchsorted(au, np.arange(u0, u1))
            rank = np.arange(len(au)) - starts[au - u0]
            keep = rank < need[au - u0]
            have_k, have_o = ak[keep], ao[keep]
        else:
            raise RuntimeError("item sampling did not converge")
        out_u.append(have_k // n_items)
        out_i.append(have_k % n_items)
    return np.concatenate(out_u), np.concatenate(out_i)


def generate(spec: SynthSpec):
    """Returns (train Dataset, pr Dataset)."""
    rng = np.random.default_rng(spec.seed)
    U, I = spec.n_users, spec.n_items
    # --- per-user counts ---------------------------------------------------
    sigma = np.sqrt(2.0 * np.log(max(spec.n_train / U / spec.median_cnt, 1.0001)))
    raw = np.exp(np.log(spec.median_cnt) + sigma * rng.standard_normal(U))
    cap = min(spec.max_cnt, I - spec.max_heldout - spec.max_query - 1)
    n_tr = _exact_total(rng, np.clip(raw, 1, cap), spec.n_train, np.ones(U, np.int64), np.full(U, cap, np.int64))
    if spec.n_heldout is None:
        n_ho = np.minimum(spec.max_heldout, np.maximum(0, n_tr // 10 + rng.integers(0, 2, U)))
    else:
        w = np.minimum(spec.max_heldout, 1 + n_tr / 60.0)
        n_ho = _exact_total(rng, w, spec.n_heldout, np.zeros(U, np.int64), np.full(U, spec.max_heldout, np.int64))
    if spec.n_query is None:
        n_q = rng.integers(0, spec.max_query + 1, U)
    else:
        w = np.minimum(spec.max_query, 1 + n_tr / 40.0)
        n_q = _exact_total(rng, w, spec.n_query, np.zeros(U, np.int64), np.full(U, spec.max_query, np.int64))
    n_rated = n_tr + n_ho
    # --- item popularity ---------------------------------------------------
    pop_rank = rng.permutation(I)            # item id -> popularity rank
    w_rank = 1.0 / np.arange(1, I + 1, dtype=np.float64) ** spec.zipf_s
    w_item = w_rank[pop_rank]
    cdf = np.cumsum(w_item)
    cdf /= cdf[-1]
    ru, ri = _sample_items(rng, n_rated, cdf, I)
    # --- dates: sessions inside a personal window --------------------------
    start = rng.integers(0, N_DAYS - 1, U)
    span = np.minimum(N_DAYS - 1 - start, (rng.exponential(500.0, U) + 1).astype(np.int64))
    n_sess = np.clip((n_rated ** 0.55 * rng.uniform(0.5, 1.5, U)).astype(np.int64), 1, None)
    n_sess = np.minimum(n_sess, np.maximum(span + 1, 1))
    n_sess = np.minimum(n_sess, np.maximum(n_rated, 1))
    sess_off = np.concatenate([[0], np.cumsum(n_sess)])
    sess_day = start.repeat(n_sess) + (rng.random(int(n_sess.sum())) * (span.repeat(n_sess) + 1)).astype(np.int64)
    pick = (rng.random(len(ru)) * n_sess[ru]).astype(np.int64)
    rd = sess_day[sess_off[ru] + pick]
    # --- planted ratings -----------------------------------------------------
    k = spec.rank
    P = rng.standard_normal((U, k)).astype(np.float32) * np.float32(0.3)
    Q = rng.standard_normal((I, k)).astype(np.float32) * np.float32(0.3)
    bu = rng.normal(0, 0.4, U).astype(np.float32)
    bi = (rng.normal(0, 0.5, I) + 0.3 * np.log(w_item / w_item.mean()) / 5).astype(np.float32)
    drift = rng.normal(0, 0.3, U).astype(np.float32)
    mean_day = (start + span / 2).astype(np.float32)
    score = np.empty(len(ru), np.float32)
    for a in range(0, len(ru), 1 << 22):
        b = min(len(ru), a + (1 << 22))
        uu, ii = ru[a:b], ri[a:b]
        s = 3.6 + bu[uu] + bi[ii] + drift[uu] * (rd[a:b] - mean_day[uu]) / 1000.0
        s += np.einsum("nk,nk->n", P[uu], Q[ii])
        s += rng.normal(0, spec.noise, b - a)
        score[a:b] = s
    rating = np.clip(np.rint(score), 1, 5).astype(np.int8)
    # --- split: each user's latest-dated n_ho ratings are held out -----------
    tie = rng.random(len(ru))
    o = np.lexsort((tie, rd, ru))
    ru, ri, rd, rating = ru[o], ri[o], rd[o], rating[o]
    ustart = np.concatenate([[0], np.cumsum(n_rated)])
    pos = np.arange(len(ru)) - ustart[ru]
    held = pos >= n_tr[ru]
    # --- query pairs: unrated items, dated after the user's last rating ----
    ex = np.sort(ru.astype(np.int64) * I + ri)
    qu, qi = _sample_items(rng, n_q, cdf, I, exclude=ex)
    last = np.zeros(U, np.int64)
    np.maximum.at(last, ru, rd)
    qd = np.minimum(N_DAYS - 1, last[qu] + rng.integers(0, 60, len(qu)))
    # --- assemble ------------------------------------------------------------
    tu, ti, td, tr_r = ru[~held], ri[~held], rd[~held], rating[~held]
    o = np.lexsort((ti, tu))
    tu, ti, td, tr_r = tu[o], ti[o], td[o], tr_r[o]
    pu = np.concatenate([ru[held], qu])
    pi = np.concatenate([ri[held], qi])
    pd_ = np.concatenate([rd[held], qd])
    pr_r = np.concatenate([rating[held], np.zeros(len(qu), np.int8)])
    pt = np.concatenate([np.zeros(int(held.sum()), np.int8), np.ones(len(qu), np.int8)])
    o = np.lexsort((pu, pi))
    pu, pi, pd_, pr_r, pt = pu[o], pi[o], pd_[o], pr_r[o], pt[o]
    train = Dataset.from_ratings(tu, ti, tr_r, td, U, I, name=f"{spec.name}_train")
    pr = Dataset.from_ratings(pu, pi, pr_r, pd_, U, I, name=f"{spec.name}_pr", is_test=pt)
    pr.residuals[pt != 0] = 0.0
    return train, pr
