"""Pass 3 with the line transform in registers and warp shuffles
(scarl_b200/csrc/c2r_shfl.cuh, the FP32 pass-3 variants after the engine's):
every lane count (8, 16, 32 lanes a line) on every half length it serves,
against the FP64 oracle, in crop mode (scarl_gen_padded) and in the blend
epilogue of a whole sample (scarl_generate_sample: PoU weights, overlap sums,
lognormal marginal), and batched over an ensemble."""
import numpy as np
import pytest

import scarl_b200 as S
from scarl_b200 import _lib

pytestmark = pytest.mark.gpu

ENGINE_VARIANTS = 5          # RowVars<float>::n
SHFL = {8: ENGINE_VARIANTS, 16: ENGINE_VARIANTS + 1, 32: ENGINE_VARIANTS + 2}
HALF_LENGTHS = [24, 40, 56, 64, 80, 96, 112, 128, 160, 192, 224, 256, 320, 384, 512, 640, 768, 1024]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _serves(N, L):
    n2 = N // L
    if N % L or n2 < 2 or n2 > 32:
        return False
    m = n2
    while m % 2 == 0:
        m //= 2
    return m in (1, 3, 5, 7)


@pytest.mark.parametrize("N", HALF_LENGTHS)
def test_shfl_variants_crop_vs_oracle(ctx, oracle, N):
    """A tile whose x axis is padded to 2N: each lane count that serves N
    matches the oracle within the FP32 tolerance and the engine variant
    within 1e-6; a lane count that does not serve N is refused as an
    invalid configuration."""
    Np, P = (min(2 * N - 3, N + 37), 6, 5), (2 * N, 8, 8)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), (6, 3, 2), 3, 0.5, 1, seed=5, stream=3)
    try:
        ctx.tune_set(S.F32, 3, N, 0)  # the shared-memory engine
        eng = S.gen_padded(ctx, Np, (1, 1, 1), (6, 3, 2), 3, pad=P, seed=5, stream=3, dtype=S.F32)
        ran = 0
        for L, v in SHFL.items():
            ctx.tune_set(S.F32, 3, N, v)
            if not _serves(N, L):
                with pytest.raises(S.ScarlError) as e:
                    S.gen_padded(ctx, Np, (1, 1, 1), (6, 3, 2), 3, pad=P, seed=5, stream=3, dtype=S.F32)
                assert e.value.code == _lib.EDEVICE and "invalid configuration" in str(e.value)
                continue
            out = S.gen_padded(ctx, Np, (1, 1, 1), (6, 3, 2), 3, pad=P, seed=5, stream=3, dtype=S.F32)
            assert rel(out, ref) < 1e-5, (L, rel(out, ref))
            assert rel(out, eng) < 1e-6, (L, rel(out, eng))
            ran += 1
        assert ran >= 1
    finally:
        ctx.tune_set(S.F32, 3, N, -1)


HEAD = dict(xMinGlob=(0, 0, 0), xMaxGlob=(512, 512, 512), corrL=(40, 20, 10), overlap=(2, 2, 2),
            pointsPerCorrL=(41, 21, 11), margiFirst=2, avg=1.0, std_dev=0.3, seedBase=0)


@pytest.fixture(scope="module")
def headline_ref(oracle):
    g, lay = oracle.generate_sample(S.GEN_PADDED, HEAD["xMinGlob"], HEAD["xMaxGlob"], HEAD["corrL"],
                                    HEAD["overlap"], HEAD["pointsPerCorrL"], 3, 0.5, 2, 1.0, 0.3, 0,
                                    8, (2, 2, 2), (448, 384, 320))
    return g


@pytest.mark.parametrize("L", [8, 16, 32])
def test_shfl_blend_headline_deck_vs_oracle(ctx, headline_ref, L):
    """The 513^3 headline deck (2 x 2 x 2 tiles, SMOOTH 448 x 384 x 320,
    half length 224) with pass 3 on the register transform, FP32 and split
    BF16: field rel-L2 <= 1e-5 and max error <= 2e-5 of the max against the
    oracle; the Gaussian field under the lognormal marginal likewise."""
    s = S.make_sample(corrMod=3, nu=0.5, **HEAD)
    try:
        ctx.tune_set(S.F32, 3, 224, SHFL[L])
        for dtype in (S.F32, S.F32 | S.SPLIT_BF16):
            ctx.profile(True)
            ctx.profile_reset()
            out, _ = S.generate_sample(ctx, s, generator=S.GEN_PADDED, dtype=dtype, nb_procs=8,
                                       topo=(2, 2, 2), pad=(448, 384, 320))
            st = ctx.profile_stats()
            ctx.profile(False)
            assert st["k_c2r_x"][1] == 8
            out = np.asarray(out, np.float64)
            e = rel(out, headline_ref)
            m = float(np.max(np.abs(out - headline_ref)) / np.max(np.abs(headline_ref)))
            gl, gr = np.log(out), np.log(headline_ref)
            eg = float(np.linalg.norm(gl - gr) / np.linalg.norm(gr - gr.mean()))
            assert e <= 1e-5 and m <= 2e-5 and eg <= 1e-5, (L, dtype, e, m, eg)
    finally:
        ctx.tune_set(S.F32, 3, 224, -1)


def test_shfl_batched_ensemble_equals_single_tiles(ctx, oracle):
    """Batched pass 3 with the register transform: every realisation of an
    uneven ensemble equals scarl_gen_padded with the same variants bit for
    bit and stays within 1e-5 of the oracle."""
    Np, cl = S.ensemble_draw(5, 0, 10, (40, 60, 90, 120), 2.0, 8.0)
    pads = [S.pad_size(S.PAD_SMOOTH, 3, c, (1, 1, 1), n) for n, c in zip(Np, cl)]
    halves = sorted({int(p[0]) // 2 for p in pads})
    try:
        for h in halves:
            for L in (8, 16, 32):
                if _serves(h, L):
                    ctx.tune_set(S.F32, 3, h, SHFL[L])
                    break
        out = S.gen_ensemble(ctx, Np, cl, corrMod=3, pad_policy=S.PAD_SMOOTH, dtype=S.F32, graph=False)
        fields = S.ensemble_fields(out, Np)
        for i, (n, c, p) in enumerate(zip(Np, cl, pads)):
            one = S.gen_padded(ctx, n, (1, 1, 1), c, 3, 0.5, pad=p, seed=i, dtype=S.F32)
            np.testing.assert_array_equal(fields[i], one)
            if i % 3 == 0:
                ref = oracle.gen_padded(n, p, (1, 1, 1), c, 3, 0.5, 1, seed=i)
                assert rel(fields[i], ref) < 1e-5, i
    finally:
        for h in halves:
            ctx.tune_set(S.F32, 3, h, -1)
