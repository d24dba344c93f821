"""Learned padding on the CPU: the oracle's backward formulas against finite
differences, BF16 rounding, label rules, and the host feature/target maps."""
import math

import numpy as np

import scarl_b200.learned as L
from oracle import mlp as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(5378) * 0.3
    X = rng.standard_normal((40, 16))
    T = rng.standard_normal((40, 2))
    loss, g = M.mlp_forward_backward(p, X, T, rounding=False)
    idx = rng.choice(5378, 60, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = M.mlp_forward_backward(q, X, T, rounding=False)
        q[i] -= 2 * eps
        lm, _ = M.mlp_forward_backward(q, X, T, rounding=False)
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 3.0e-39], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0     # 1 + 2^-8 is the tie between 1 and 1 + 2^-7: even
    assert r[3] == 1.0                      # below the tie
    assert r[2] == 1.0 + 2 ** -7 and r[4] == -2.5
    assert abs(r[5] - 3.0e-39) <= 2.0 ** -134  # subnormal: half of the bf16 spacing 2^-133


def test_oracle_labels_follow_the_rules():
    # a short Gaussian correlation needs almost no padding, a long exponential one more
    P1, W1, s1, err1 = M.labels(1, 0.0, 2.0, 64)
    P2, W2, s2, err2 = M.labels(3, 0.5, 18.0, 64)
    assert P1 < P2 and not s1 and not s2
    assert err1(P1) <= 0.01 < err1(P1 - 1) or P1 == 64
    assert err2(P2) <= 0.01 < err2(P2 - 1)
    assert W1 < W2


def test_host_features_and_targets():
    cm = np.array([1, 3, 2], np.int32)
    nu = np.array([0.0, 0.5, 1.2])
    ell = np.array([6.4, 20.0, 3.0])
    N = np.array([64, 100, 256], np.int32)
    X = L.features(cm, nu, ell, N)
    assert X.shape == (3, 16) and np.all(X[:, 8:] == 0)
    np.testing.assert_allclose(X[0, :4], [0.4, math.log2(0.1) / 4, -1.0, math.log2(6.4) / 4], rtol=1e-6)
    np.testing.assert_array_equal(X[:, 4:7], np.eye(3)[[0, 1, 2]])
    np.testing.assert_allclose(X[2, 7], 0.3, rtol=1e-6)
    T = L.targets(ell, N, np.array([80, 228, 256]), np.array([12, 60, 4]))
    np.testing.assert_allclose(T[:, 0], np.log2(np.array([17, 129, 1]) / ell), rtol=1e-6)
    np.testing.assert_allclose(T[:, 1], np.log2(np.array([12, 60, 4]) / ell), rtol=1e-6)


def test_config_sampling_ranges():
    cm, nu, N, ell = L.sample_configs(4096, 1)
    assert set(np.unique(cm)) == {1, 2, 3}
    r = ell / N
    assert r.min() >= 0.01 and r.max() <= 0.3 and N.min() >= 64 and N.max() <= 256
    vk = cm == 2
    assert nu[vk].min() >= 0.3 and nu[vk].max() <= 1.5 and np.all(nu[cm == 3] == 0.5)
