"""The CPU reference of the term-priority network, pinned by finite differences (no GPU)."""

import numpy as np

from oracle import mlp_ref as M


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, M.N_PARAMS)
    X = rng.normal(0, 1, (37, M.IN))
    t = rng.normal(0, 1, 37)
    _, g = M.loss_and_grad(p, X, t)
    for i in rng.choice(M.N_PARAMS, 60, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, X, t)[0] - M.loss_and_grad(pm, X, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # 1 + 2^-8 is a tie: rounds to even (1.0)
    assert r[2] == 1.0078125            # above the tie: rounds up
    assert abs(r[3] + 3.140625) < 1e-12
    assert r[4] == 65536.0
