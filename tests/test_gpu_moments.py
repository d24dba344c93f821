"""Moments streamed from the C2R pass (scarl_gen_opts.moments): sum f and
sum f^2 of the output field accumulated in FP64 inside pass 3 as each point
becomes final, compared with FP64 sums over the returned field (the same
values, another summation order: relative difference <= 1e-12), for the
register-transform and engine pass-3 variants, FP32, split BF16 and FP64,
device and host outputs, and the literal Shino generator.  The mean and
variance that follow are the estimators of
SRC_F/Stat_ScaRL/statistics_RF.f90:18-174 over one sample."""
import numpy as np
import pytest

import scarl_b200 as S
from scarl_b200 import _lib

pytestmark = pytest.mark.gpu

HEAD = dict(xMinGlob=(0, 0, 0), xMaxGlob=(512, 512, 512), corrL=(40, 20, 10), overlap=(2, 2, 2),
            pointsPerCorrL=(41, 21, 11), margiFirst=2, avg=1.0, std_dev=0.3, seedBase=0)
SMALL = dict(xMinGlob=(0, 0, 0), xMaxGlob=(60, 50, 40), corrL=(6, 5, 4), overlap=(2, 2, 2),
             pointsPerCorrL=(5, 5, 5), margiFirst=1, avg=0.5, std_dev=2.0, seedBase=3)


def _sums(f):
    f = np.asarray(f, dtype=np.float64).ravel()
    return np.array([f.sum(), (f * f).sum()])


def _check(m, f):
    ref = _sums(f)
    assert np.all(np.abs(m - ref) <= 1e-12 * np.abs(ref)), (m, ref)


@pytest.mark.parametrize("variant", [None, 0])
@pytest.mark.parametrize("dtype", [S.F32, S.F32 | S.SPLIT_BF16, S.F64])
def test_streamed_moments_headline(ctx, dtype, variant):
    """The 513^3 headline deck (8 tiles, lognormal): the streamed sums equal
    FP64 sums of the returned field; variant None is the default pass 3 (the
    register transform in FP32), 0 the shared-memory engine."""
    if variant is not None and dtype == S.F64:
        pytest.skip("FP64 has only the engine")
    torch = pytest.importorskip("torch")
    s = S.make_sample(corrMod=3, nu=0.5, **HEAD)
    tdt = torch.float64 if dtype == S.F64 else torch.float32
    out = torch.empty(513 ** 3, dtype=tdt, device="cuda")
    m = np.zeros(2)
    try:
        if variant is not None:
            ctx.tune_set(S.F32, 3, 224, variant)
        S.generate_sample(ctx, s, dtype=dtype, nb_procs=8, topo=(2, 2, 2), pad=(448, 384, 320),
                          out=out, moments=m)
    finally:
        if variant is not None:
            ctx.tune_set(S.F32, 3, 224, -1)
    _check(m, out.cpu().numpy())
    n = 513 ** 3
    mean, var = m[0] / n, m[1] / n - (m[0] / n) ** 2
    assert abs(mean - 1.0) < 0.05 and abs(np.sqrt(var) / mean - 0.3) < 0.05


@pytest.mark.parametrize("pinned", [False, True])
def test_streamed_moments_host_output(ctx, pinned):
    """Host outputs (the box-by-box copy paths) return the same sums."""
    torch = pytest.importorskip("torch")
    s = S.make_sample(corrMod=3, nu=0.5, **HEAD)
    if pinned:
        out = torch.empty(513 ** 3, dtype=torch.float32, pin_memory=True).numpy()
    else:
        out = np.empty(513 ** 3, dtype=np.float32)
    m = np.zeros(2)
    S.generate_sample(ctx, s, dtype=S.F32, nb_procs=8, topo=(2, 2, 2), pad=(448, 384, 320), out=out,
                      moments=m)
    _check(m, out)


def test_streamed_moments_small_decks(ctx):
    """A small 2 x 2 x 2 Gaussian-marginal deck (padded, FP32 and FP64), the
    literal Shino generator (FP64), a constant field and the refusals."""
    s = S.make_sample(corrMod=1, **SMALL)
    for dtype in (S.F32, S.F64):
        m = np.zeros(2)
        out, _ = S.generate_sample(ctx, s, dtype=dtype, nb_procs=8, pad_policy=S.PAD_AUTO, moments=m)
        _check(m, out)
    m = np.zeros(2)
    out, _ = S.generate_sample(ctx, s, generator=S.GEN_SHINO, dtype=S.F64, nb_procs=8, moments=m)
    _check(m, out)
    c = S.make_sample(corrMod=1, **dict(SMALL, std_dev=0.0))
    m = np.zeros(2)
    out, _ = S.generate_sample(ctx, c, dtype=S.F64, nb_procs=8, moments=m)
    _check(m, out)
    with pytest.raises(S.ScarlError) as e:
        S.generate_sample(ctx, s, dtype=S.F64, nb_procs=8, normalize_field=True, moments=np.zeros(2))
    assert e.value.code == _lib.EUNSUPPORTED
