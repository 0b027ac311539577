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


def _argsort(key: np.ndarray) -> np.ndarray:
    """Stable argsort (identical result on every backend)."""
    if len(key) > (1 << 22):
        try:
            import torch
            if torch.cuda.is_available():
                t = torch.from_numpy(np.ascontiguousarray(key)).cuda()
                return torch.sort(t, stable=True).indices.cpu().numpy()
        except ImportError:
            pass
    return np.argsort(key, kind="stable")


def _saturated_counts(n: np.ndarray, w_rank: np.ndarray) -> np.ndarray:
    """Per user with n picks, the number m of most popular items whose
    inclusion probability min(1, c w_k) saturates, where c solves
    sum_k min(1, c w_k) = n (conditional Poisson sampling)."""
    tail = np.concatenate([np.cumsum(w_rank[::-1])[::-1], [0.0]])  # tail[m] = sum_{k >= m} w_k
    lo = np.zeros(len(n), np.int64)
    hi = n.astype(np.int64).copy()
    # smallest m in [0, n] with (n - m) w[m] < tail[m]
    for _ in range(40):
        mid = (lo + hi) // 2
        wm = w_rank[np.minimum(mid, len(w_rank) - 1)]
        ok = (n - mid) * wm < tail[mid]
        hi = np.where(ok, mid, hi)
        lo = np.where(ok, lo, mid + 1)
        if np.all(lo >= hi):
            break
    return hi


def _sample_items(rng, cnt: np.ndarray, w_rank: np.ndarray, rank_item: np.ndarray, exclude=None,
                  chunk_draws=1 << 24):
    """Per user, `cnt[u]` distinct items drawn without replacement with
    popularity weights: the saturated head (see _saturated_counts) is taken
    outright and the rest is drawn from the remaining tail by weight, each
    round drawing exactly the users' shortfall and dropping repeats. Keys in
    sorted `exclude` (user * n_items + item) are never chosen. Returns
    (users, items), sorted by (user, item)."""
    n_users, n_items = len(cnt), len(w_rank)
    cnt = cnt.astype(np.int64)
    ex_key = exclude if exclude is not None else np.zeros(0, np.int64)
    cdf = np.cumsum(w_rank)
    cdf /= cdf[-1]
    m = np.zeros(n_users, np.int64) if exclude is not None else _saturated_counts(cnt, w_rank)
    out = []
    csum = np.cumsum(cnt + 1)
    bounds = [0] + list(np.searchsorted(csum, np.arange(chunk_draws, csum[-1], chunk_draws)) + 1) + [n_users]
    bounds = sorted(set(min(int(b), n_users) for b in bounds))
    for u0, u1 in zip(bounds[:-1], bounds[1:]):
        if u0 == u1:
            continue
        users = np.arange(u0, u1, dtype=np.int64)
        hm = m[u0:u1]
        need = cnt[u0:u1] - hm
        hu = np.repeat(users, hm)
        hr = np.arange(hu.size, dtype=np.int64) - np.repeat(np.cumsum(hm) - hm, hm)
        head_k = np.sort(hu * n_items + rank_item[hr])
        lo_cdf = np.where(hm > 0, cdf[np.maximum(hm - 1, 0)], 0.0)
        exk = ex_key[np.searchsorted(ex_key, u0 * n_items):np.searchsorted(ex_key, u1 * n_items)]
        have = np.zeros(0, np.int64)  # sorted keys
        deficit = need.copy()
        for _ in range(60):
            if deficit.max(initial=0) <= 0:
                break
            du = np.repeat(users, np.maximum(deficit, 0))
            base = lo_cdf[du - u0]
            r = base + rng.random(du.size) * (1.0 - base)
            rank = np.minimum(np.searchsorted(cdf, r, side="right"), n_items - 1)
            dk = du * n_items + rank_item[rank]
            if exk.size:
                pos = np.minimum(np.searchsorted(exk, dk), exk.size - 1)
                dk = dk[exk[pos] != dk]
            ak = np.concatenate([have, dk])
            ak = ak[_argsort(ak)]
            first = np.ones(ak.size, bool)
            first[1:] = ak[1:] != ak[:-1]
            have = ak[first]
            deficit = need - np.bincount(have // n_items - u0, minlength=u1 - u0)
        if deficit.max(initial=0) > 0:
            # rare: fill the remainder uniformly from the items still free
            extra = []
            hs = np.searchsorted(have, users * n_items)
            he = np.searchsorted(have, (users + 1) * n_items)
            xs = np.searchsorted(exk, users * n_items)
            xe = np.searchsorted(exk, (users + 1) * n_items)
            ks = np.searchsorted(head_k, users * n_items)
            ke = np.searchsorted(head_k, (users + 1) * n_items)
            for j in np.nonzero(deficit > 0)[0]:
                uu = u0 + j
                taken = np.zeros(n_items, bool)
                taken[have[hs[j]:he[j]] % n_items] = True
                taken[exk[xs[j]:xe[j]] % n_items] = True
                taken[head_k[ks[j]:ke[j]] % n_items] = True
                free = np.nonzero(~taken)[0]
                pick = rng.choice(free, size=int(min(deficit[j], free.size)), replace=False)
                extra.append(uu * n_items + pick)
            have = np.concatenate([have] + extra)
        out.append(np.sort(np.concatenate([head_k, have])))
    allk = np.concatenate(out)
    return allk // n_items, allk % n_items


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
    rank_item = np.argsort(pop_rank)         # popularity rank -> item id
    w_rank = 1.0 / np.arange(1, I + 1, dtype=np.float64) ** spec.zipf_s
    w_item = w_rank[pop_rank]
    ru, ri = _sample_items(rng, n_rated, w_rank, rank_item)
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
    tie = rng.integers(0, 1 << 16, len(ru), dtype=np.int64)
    o = _argsort((ru.astype(np.int64) << 32) | (rd.astype(np.int64) << 16) | tie)
    ru, ri, rd, rating = ru[o], ri[o], rd[o], rating[o]
    ustart = np.concatenate([[0], np.cumsum(n_rated)])
    pos = np.arange(len(ru)) - ustart[ru]
    held = pos >= n_tr[ru]
    # --- query pairs: unrated items, dated after the user's last rating ----
    ex = np.sort(ru.astype(np.int64) * I + ri)
    n_q = np.minimum(n_q, (I - n_rated) // 4)
    qu, qi = _sample_items(rng, n_q, w_rank, rank_item, exclude=ex)
    last = np.zeros(U, np.int64)
    np.maximum.at(last, ru, rd)
    qd = np.minimum(N_DAYS - 1, last[qu] + rng.integers(0, 60, len(qu)))
    # --- assemble ------------------------------------------------------------
    tu, ti, td, tr_r = ru[~held], ri[~held], rd[~held], rating[~held]
    o = _argsort(tu.astype(np.int64) * I + ti)
    tu, ti, td, tr_r = tu[o], ti[o], td[o], tr_r[o]
    pu = np.concatenate([ru[held], qu])
    pi = np.concatenate([ri[held], qi])
    pd_ = np.concatenate([rd[held], qd])
    pr_r = np.concatenate([rating[held], np.zeros(len(qu), np.int8)])
    pt = np.concatenate([np.zeros(int(held.sum()), np.int8), np.ones(len(qu), np.int8)])
    o = _argsort(pi.astype(np.int64) * U + pu)
    pu, pi, pd_, pr_r, pt = pu[o], pi[o], pd_[o], pr_r[o], pt[o]
    train = Dataset.from_ratings(tu, ti, tr_r, td, U, I, name=f"{spec.name}_train")
    pr = Dataset.from_ratings(pu, pi, pr_r, pd_, U, I, name=f"{spec.name}_pr", is_test=pt)
    pr.residuals[pt != 0] = 0.0
    return train, pr
