"""Streamed axis-covariance estimator (scarl_axis_cov) against the oracle's
direct FP64 lag sums, and the 2048 x 2048 x 1024 field (4 x 4 x 1 tiles,
Gaussian l = (64, 64, 32), overlap 128) against its target covariance within
Monte Carlo bounds.  Tolerances: FP64 |cov - oracle| <= 1e-11 var, FP32
<= 2e-6 var (the FP32 field's own values, summed in FP64 by the oracle)."""
import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu


def _field(shape, seed, shift=0.0):
    rng = np.random.default_rng(seed)
    f = rng.standard_normal(shape)
    # a little correlation along every axis so that lags carry signal
    for ax in range(3):
        f = f + 0.6 * np.roll(f, 1, axis=ax)
    return np.asfortranarray(f + shift)


@pytest.mark.parametrize("shape,maxlag,shift", [
    ((37, 20, 45), 10, 0.0),
    ((64, 48, 33), 30, 5.0),
    ((130, 7, 9), 6, -2.0),
    ((9, 200, 12), 8, 0.0),
    ((16, 16, 300), 15, 1.0),
    ((257, 31, 17), 16, 0.0),
    ((600, 40, 35), 30, 0.5),   # x line padded to M = 640 (N = 320 = 5 x 64)
    ((64, 700, 62), 60, 0.0),   # y line padded to M = 768 (N = 384 = 3 x 128)
])
def test_axis_cov_vs_oracle(ctx, oracle, shape, maxlag, shift):
    f = _field(shape, sum(shape), shift)
    m_ref, c_ref = oracle.axis_cov(f, maxlag)
    m, v, c = S.axis_cov(ctx, f, shape, maxlag)
    assert m == pytest.approx(m_ref, rel=1e-13, abs=1e-13)
    assert v == c[0, 0]
    np.testing.assert_allclose(c, c_ref, rtol=0, atol=1e-11 * c_ref[0, 0])
    f32 = f.astype(np.float32)
    m_ref32, c_ref32 = oracle.axis_cov(f32.astype(np.float64), maxlag)
    m32, _, c32 = S.axis_cov(ctx, f32, shape, maxlag)
    assert m32 == pytest.approx(m_ref32, rel=1e-12, abs=1e-12)
    np.testing.assert_allclose(c32, c_ref32, rtol=0, atol=2e-6 * c_ref32[0, 0])


def test_axis_cov_device_input_and_limits(ctx, oracle):
    torch = pytest.importorskip("torch")
    f = _field((40, 30, 20), 3)
    dev = torch.from_numpy(f.reshape(-1, order="F")).cuda()
    _, _, c = S.axis_cov(ctx, dev, f.shape, 19)
    np.testing.assert_allclose(c, oracle.axis_cov(f, 19)[1], rtol=0, atol=1e-11)
    with pytest.raises(S.ScarlError):
        S.axis_cov(ctx, f, f.shape, 20)           # maxlag must be below every extent
    with pytest.raises(S.ScarlError):
        S.axis_cov(ctx, np.zeros((4096, 3, 2), order="F"), (4096, 3, 2), 1)  # L + maxlag > 4096


@pytest.mark.parametrize("shape,maxlag", [((64, 48, 33), 30), ((128, 64, 40), 20), ((600, 40, 36), 30)])
def test_axis_cov_staged_equals_direct(ctx, oracle, shape, maxlag):
    """FP32 fields whose lines start on 16-byte boundaries take the staged
    power pass (cp.async copies into shared memory); the same values one
    float off the boundary take the direct one.  Same grid, same order: the
    covariances are identical, and within the FP32 tolerance of the oracle."""
    torch = pytest.importorskip("torch")
    f = _field(shape, 7).astype(np.float32)
    flat = torch.from_numpy(f.reshape(-1, order="F")).cuda()
    buf = torch.empty(flat.numel() + 4, dtype=torch.float32, device="cuda")
    buf[1:1 + flat.numel()] = flat
    off = buf[1:1 + flat.numel()]  # 4 bytes past a 16-byte boundary
    assert flat.data_ptr() % 16 == 0 and off.data_ptr() % 16 == 4
    m1, v1, c1 = S.axis_cov(ctx, flat, shape, maxlag)
    m2, v2, c2 = S.axis_cov(ctx, off, shape, maxlag)
    assert m1 == m2 and v1 == v2
    np.testing.assert_array_equal(c1, c2)
    _, c_ref = oracle.axis_cov(f.astype(np.float64), maxlag)
    np.testing.assert_allclose(c1, c_ref, rtol=0, atol=2e-6 * c_ref[0, 0])


def _blend_kappa(Np, No, T, L, maxlag):
    """Pair-averaged sum over tiles of sqrt(w(x) w(x + h)) of the 1-D
    partition-of-unity weights along one axis (the factor by which blending
    scales the covariance at lag h along that axis)."""
    w = np.zeros((T, L))
    for p in range(T):
        wt = S.unity_partition_weights((Np, 1, 1), (No, 0, 0), (p, 0, 0), (T, 1, 1)).ravel()
        o = (Np - No) * p
        w[p, o:o + Np] = wt
    k = np.empty(maxlag + 1)
    for h in range(maxlag + 1):
        k[h] = np.mean(np.sum(np.sqrt(w[:, :L - h] * w[:, h:]), axis=0))
    return k


def test_large_field_covariance_within_monte_carlo_bounds(ctx):
    """2048 x 2048 x 1024 FP32, Gaussian l = (64, 64, 32), Gaussian marginal
    (mean 0, variance 1), 4 x 4 x 1 tiles with a 128-point overlap.  Bounds:
    one field holds about N / (l_x l_y l_z) = 32768 correlation volumes, so
    the standard error of the variance is sqrt(2 * 0.354 * l^3 / N) ~ 0.005
    and of the mean ~ 0.006; the checks allow 0.03."""
    torch = pytest.importorskip("torch")
    s = S.make_sample((0, 0, 0), (2047, 2047, 1023), (64, 64, 32), (127 / 64, 127 / 64, 0),
                      (65, 65, 33), corrMod=1, margiFirst=1, avg=0.0, std_dev=1.0, seedBase=4)
    lay = S.sample_layout(s, 1, 16, (4, 4, 1))
    L = [int(v) for v in lay["L"]]
    assert L == [2048, 2048, 1024]
    field = torch.empty(L[0] * L[1] * L[2], dtype=torch.float32, device="cuda")
    S.generate_sample(ctx, s, dtype=S.F32, nb_procs=16, topo=(4, 4, 1), pad_policy=S.PAD_AUTO,
                      out=field)
    H = 256
    mean, var, cov = S.axis_cov(ctx, field, L, H)
    del field
    assert abs(mean) < 0.03 and abs(var - 1.0) < 0.03
    h = np.arange(H + 1)
    for d, l in enumerate((64.0, 64.0, 32.0)):
        kap = _blend_kappa(int(lay["Np"][d]), int(lay["Np_ovlp"][d]), int(lay["topo"][d]), L[d], H)
        target = kap * np.exp(-np.pi * h * h / (l * l))
        assert np.max(np.abs(cov[d] - target)) < 0.03, d


def test_axis_cov_known_mean(ctx):
    f = _field((30, 20, 16), 9, 1.0)
    _, _, c = S.axis_cov(ctx, f, f.shape, 6, known_mean=0.25)
    g = f - 0.25
    for d, n in enumerate(f.shape):
        for h in range(7):
            a = np.take(g, range(0, n - h), axis=d)
            b = np.take(g, range(h, n), axis=d)
            assert c[d, h] == pytest.approx(np.mean(a * b), rel=1e-11, abs=1e-12)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_pageable_host_input(ctx, dtype):
    """A pageable host field of 8 MB and more is uploaded through the
    context's pinned ring (32 MB chunks, the last one ragged): the statistics
    equal those of the same field passed as a device tensor, bit for bit, and
    every byte is uploaded once."""
    import torch
    shape = (250, 260, 270)
    f = np.asfortranarray(np.random.default_rng(5).standard_normal(shape).astype(dtype))
    assert f.nbytes > 2 * 32 * 2**20 and f.nbytes % (32 * 2**20) != 0
    c0 = ctx.counters()
    m, v, c = S.axis_cov(ctx, f, shape, 40)
    assert ctx.counters()["h2d_bytes"] - c0["h2d_bytes"] == f.nbytes
    d = torch.from_numpy(f.reshape(-1, order="F").copy()).cuda()
    md, vd, cd = S.axis_cov(ctx, d, shape, 40)
    assert m == md and v == vd
    np.testing.assert_array_equal(c, cd)
    assert abs(m) < 1e-3 and abs(v - 1) < 1e-2
