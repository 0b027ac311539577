"""The FP64 encoder oracle's gradients against central finite differences
(CPU only): the checker used for the GPU encoder is itself checked."""
import numpy as np

from oracle import encoder_oracle as eo


def small_problem(seed=0, n_items=12, T=5, O=6, n_users=4):
    rng = np.random.default_rng(seed)
    p = {"e_item": rng.normal(0, 0.3, (n_items * 5, 128)), "e_rate": rng.normal(0, 0.3, (5, 128)),
         "e_date": rng.normal(0, 0.3, (T, 128)), "w1": rng.normal(0, 0.1, (128, 512)),
         "b1": rng.normal(0, 0.1, 512), "w2": rng.normal(0, 0.05, (512, 512)), "b2": rng.normal(0, 0.1, 512),
         "w3": rng.normal(0, 0.05, (512, O)), "b3": rng.normal(0, 0.1, O)}
    hist = []
    for _ in range(n_users):
        k = int(rng.integers(1, 6))
        hist.append((rng.choice(n_items, k, replace=False), rng.integers(1, 6, k), rng.integers(0, T, k)))
    t = rng.normal(0, 1, (n_users, O))
    return p, hist, t


def test_oracle_gradients_match_finite_differences():
    p, hist, t = small_problem()
    _, g = eo.loss_and_grads(p, hist, t, mimic_bf16=False)
    rng = np.random.default_rng(1)
    h = 1e-6
    for name in ("e_item", "e_rate", "e_date", "w1", "b1", "w2", "b2", "w3", "b3"):
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in p[name].shape)
            if name == "e_item" and not any(idx[0] in 5 * it + rt - 1 for it, rt, _ in hist):
                continue
            q = {k: v.copy() for k, v in p.items()}
            q[name][idx] += h
            lp, _ = eo.loss_and_grads(q, hist, t, mimic_bf16=False)
            q[name][idx] -= 2 * h
            lm, _ = eo.loss_and_grads(q, hist, t, mimic_bf16=False)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[name][idx]) <= 1e-5 * max(1.0, abs(fd)), (name, idx, fd, g[name][idx])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5], np.float32)
    assert list(eo.bf16(x)) == [1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6, -2.5]
