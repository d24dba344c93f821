"""Monte Carlo statistics of the headline field against its target model.

Field: the 512^3 deck re-fitted to 513^3, exponential correlation
C(r) = exp(-2 |r|_l) with |r|_l = sqrt(sum (r_d / l_d)^2), l = (40, 20, 10) at
spacing 1, lognormal marginal with mean 1 and CV 0.3, 2 x 2 x 2 tiles with
overlap 2 l, split-BF16 path, on the SMOOTH (448 x 384 x 320) and AUTO (512^3)
padded grids; K = 32 realisations (deck seeds 1000 i, i < 32: tile r of a
sample draws with key seedBase + 1 + r, so no two realisations share a tile).

Checked (estimators of SRC_F/Stat_ScaRL/statistics_RF.f90:18-174 (moments)
and the axis covariance of :258-486 as direct FP64 lag sums):
- the marginal: mean of Y = 1 and std of Y = 0.3;
- the Gaussian field under the marginal, X = (ln Y - mu_g) / sigma_g with
  sigma_g^2 = ln(1 + CV^2), mu_g = ln(mean) - sigma_g^2 / 2: mean 0, and its
  axis covariance at lags h <= 2 l_d against the method's exact expectation
  kappa_d(h) rho_d(h), where
    rho_d(h) = sum_k S(k) cos(2 pi k_d h / P_d) / sum_k S(k)
  over the full periodic grid (the covariance of the padded periodic method
  with its FP64 variance normalisation), and
    kappa_d(h) = mean over pairs of sum_tiles sqrt(w(x) w(x + h))
  the factor by which blending tiles of independent fields scales it;
- rho_d(h) against the continuous target exp(-2 h / l_d): the spectrum is
  cut at the grid's Nyquist frequency and renormalised to unit variance,
  which raises the covariance at short lags by up to 0.045 at l_d / dx = 10;
  bounded by 0.05.

Bounds (5 standard errors, from the number of correlation volumes): for a
Gaussian field of N points, Var(mean) <= (1/N) sum_s C(s) = pi l_x l_y l_z / N
and Var(lag-h covariance) <= (2/N) sum_s C(s)^2 = (pi / 4) l_x l_y l_z / N
(sum over lattice lags; C(s+h) C(s-h) <= (C(s+h)^2 + C(s-h)^2) / 2), times 1.1
for the method's slightly higher covariance; each divided by K.  For Y:
Var(mean Y) <= sigma_Y^2 pi l^3 / N, and the CV is held to 1 % (the standard
error of the sample variance of Y over K fields is near 0.1 %).
"""
import math

import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu

K = 32
CL = (40.0, 20.0, 10.0)
MEAN, CV = 1.0, 0.3
SPLIT = S.F32 | S.SPLIT_BF16


def _freqs(P, dx):
    k = np.arange(P)
    return np.where(2 * k <= P, k, k - P) / (P * dx)


def exponential_marginals(corrL, P, dx):
    """Per axis d, sum over the other two axes of the exponential model's
    spectral density S(f) = c (1 + sum 4 pi^2 a_d^2 f_d^2)^-2, a = l / 2 (c
    drops out of rho)."""
    t = [4.0 * math.pi ** 2 * (c / 2.0) ** 2 for c in corrL]
    f2 = [t[d] * _freqs(P[d], dx[d]) ** 2 for d in range(3)]
    M = [np.zeros(P[0]), np.zeros(P[1]), np.zeros(P[2])]
    for z0 in range(0, P[2], 16):
        q = 1.0 + f2[0][:, None, None] + f2[1][None, :, None] + f2[2][None, None, z0:z0 + 16]
        s = q ** -2.0
        M[0] += s.sum(axis=(1, 2))
        M[1] += s.sum(axis=(0, 2))
        M[2][z0:z0 + 16] += s.sum(axis=(0, 1))
    return M


def method_rho(M, P, d, hmax):
    h = np.arange(hmax + 1)
    k = np.arange(P[d])
    return (M[d][None, :] * np.cos(2.0 * np.pi * np.outer(h, k) / P[d])).sum(axis=1) / M[d].sum()


def blend_kappa(Np, No, T, L, hmax):
    """Pair average over the axis of sum over tiles of sqrt(w(x) w(x + h)),
    1-D partition-of-unity weights (the other axes' weights sum to 1)."""
    w = np.zeros((T, L))
    for p in range(T):
        wt = S.unity_partition_weights((Np, 1, 1), (No, 0, 0), (p, 0, 0), (T, 1, 1)).ravel()
        o = (Np - No) * p
        w[p, o:o + Np] = wt
    return np.array([np.mean(np.sum(np.sqrt(w[:, :L - h] * w[:, h:]), axis=0))
                     for h in range(hmax + 1)])


def test_model_spectrum_matches_oracle(oracle):
    for f in ((0.01, 0.02, 0.03), (0.2, 0.1, 0.4), (0.5, 0.0, 0.25)):
        q = 1.0 + sum(4.0 * math.pi ** 2 * (c / 2.0) ** 2 * x * x for c, x in zip(CL, f))
        ratio = oracle.spectrum(3, 0.5, CL, f) / q ** -2.0
        assert ratio == pytest.approx(oracle.spectrum(3, 0.5, CL, (0, 0, 0)), rel=1e-13)


@pytest.mark.parametrize("policy,P", [(S.PAD_SMOOTH, (448, 384, 320)), (S.PAD_AUTO, (512, 512, 512))])
def test_headline_field_statistics(ctx, policy, P):
    import torch
    base = S.make_sample((0, 0, 0), (512, 512, 512), CL, (2, 2, 2), (41, 21, 11), corrMod=3,
                         margiFirst=2, avg=MEAN, std_dev=CV * MEAN)
    lay = S.sample_layout(base, 1, 8, (2, 2, 2))
    L = [int(v) for v in lay["L"]]
    N = L[0] * L[1] * L[2]
    assert [int(v) for v in S.pad_size(policy, 3, CL, lay["xStep"], lay["Np"], 0.5, 1e-3)] == list(P)
    H = [int(2 * c) for c in CL]
    sg2 = math.log(1.0 + CV * CV)
    mug, sg = math.log(MEAN) - sg2 / 2.0, math.sqrt(sg2)

    y = torch.empty(N, dtype=torch.float32, device="cuda")
    ymean, yvar, xmean = [], [], []
    cov = [np.zeros(h + 1) for h in H]
    for i in range(K):
        s = S.make_sample((0, 0, 0), (512, 512, 512), CL, (2, 2, 2), (41, 21, 11), corrMod=3,
                          margiFirst=2, avg=MEAN, std_dev=CV * MEAN, seedBase=1000 * i)
        S.generate_sample(ctx, s, dtype=SPLIT, nb_procs=8, topo=(2, 2, 2), pad_policy=policy, out=y)
        ctx.sync()
        yd = y.double()
        ymean.append(float(yd.mean()))
        yvar.append(float(yd.var(unbiased=False)))
        x = (torch.log(yd) - mug) / sg
        del yd
        # x is written on torch's stream, read on the library's own stream
        torch.cuda.synchronize()
        m, _, c = S.axis_cov(ctx, x, L, max(H), known_mean=0.0)
        xmean.append(m)
        for d in range(3):
            cov[d] += c[d, :H[d] + 1] / K
        del x

    vol = CL[0] * CL[1] * CL[2]
    se_mean = math.sqrt(math.pi * vol / N / K)
    se_cov = math.sqrt(1.1 * (math.pi / 4.0) * vol / N / K)
    se_ymean = math.sqrt(MEAN ** 2 * CV ** 2 * math.pi * vol / N / K)
    print(f"policy {policy}: mean Y {np.mean(ymean):.5f} (se {se_ymean:.1e}), std Y "
          f"{math.sqrt(np.mean(yvar)):.5f}, mean X {np.mean(xmean):+.5f} (se {se_mean:.1e}), "
          f"cov se {se_cov:.1e}")
    assert abs(np.mean(ymean) - MEAN) <= 5 * se_ymean
    assert abs(math.sqrt(np.mean(yvar)) / np.mean(ymean) - CV) <= 0.01 * CV
    assert abs(np.mean(xmean)) <= 5 * se_mean

    M = exponential_marginals(CL, P, lay["xStep"])
    for d in range(3):
        rho = method_rho(M, P, d, H[d])
        kap = blend_kappa(int(lay["Np"][d]), int(lay["Np_ovlp"][d]), int(lay["topo"][d]), L[d], H[d])
        h = np.arange(H[d] + 1)
        target = np.exp(-2.0 * h / CL[d])
        expect = kap * rho
        dev = cov[d] - expect
        print(f"axis {d}: max |cov - kappa rho| {np.max(np.abs(dev)):.4f} (bound {5 * se_cov:.4f}); "
              f"cov at h = l: {cov[d][int(CL[d])]:.4f}, kappa rho {expect[int(CL[d])]:.4f}, "
              f"exp(-2) kappa {target[int(CL[d])] * kap[int(CL[d])]:.4f}; "
              f"max |rho - exp(-2h/l)| {np.max(np.abs(rho - target)):.4f}")
        assert np.max(np.abs(dev)) <= 5 * se_cov, d
        assert np.max(np.abs(rho - target)) <= 0.05, d
        assert abs(rho[0] - 1.0) < 1e-12
