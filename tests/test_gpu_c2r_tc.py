"""Tensor-core pass 3 (scarl_b200/csrc/c2r_tc.cu): with SCARL_F32 |
SCARL_SPLIT_BF16_X the Hermitian C2R along x runs as two split-BF16
tensor-core DFT stages (N = N1 x N2, N2 = 32 or 16, N1 <= 8) in front of the
same crop / blend epilogue as the CUDA-core pass 3.  Checked against the
FP64 oracle on every half length it serves, in crop mode and in the blend
epilogue of whole samples, with the FP64 moments it streams.
Tolerance: field rel-L2 <= 1e-5 against FP64 (the stated bound of the split
form), max error <= 3e-5 of the field's maximum."""
import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu

SPLIT = S.F32 | S.SPLIT_BF16_X
TC_HALVES = [32, 48, 64, 80, 96, 112, 128, 160, 192, 224, 256]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _stats(ctx, fn):
    ctx.profile(True)
    ctx.profile_reset()
    out = fn()
    st = ctx.profile_stats()
    ctx.profile(False)
    return out, st


@pytest.mark.parametrize("N", TC_HALVES)
def test_tc_pass3_crop_vs_oracle(ctx, oracle, N):
    """One tile, x padded to 2N: the tensor-core pass 3 runs (one launch) and
    the field matches the oracle; Nx = 2N - 3 keeps nearly the whole line,
    Ny Nz = 7 x 5 leaves a ragged last item of 16 lines."""
    Np, P = (2 * N - 3, 7, 5), (2 * N, 16, 16)
    cl = (max(2.0, N / 8), 3.0, 3.0)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), cl, 3, 0.5, 1, seed=21, stream=2)
    out, st = _stats(ctx, lambda: S.gen_padded(ctx, Np, (1, 1, 1), cl, 3, pad=P, seed=21, stream=2,
                                               dtype=SPLIT))
    assert st.get("k_c2r_x_tc", (0, 0))[1] == 1 and "k_c2r_x" not in st
    e = rel(out, ref)
    m = float(np.max(np.abs(out - ref)) / np.max(np.abs(ref)))
    assert e <= 1e-5 and m <= 3e-5, (N, e, m)


@pytest.mark.parametrize("Np,P,cm,nu", [
    ((150, 40, 33), (448, 64, 64), 3, 0.5),    # N = 7 x 32, crop of 150 of 448
    ((100, 77, 20), (256, 128, 32), 1, 0.5),   # N = 4 x 32, Gaussian
    ((60, 50, 45), (224, 64, 64), 2, 1.5),     # N = 7 x 16, von Karman
    ((33, 31, 29), (64, 32, 32), 3, 0.5),      # N = 2 x 16
])
def test_tc_pass3_tiles_vs_oracle(ctx, oracle, Np, P, cm, nu):
    cl = (6.0, 5.0, 4.0)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), cl, cm, nu, 1, seed=5, stream=1)
    out, st = _stats(ctx, lambda: S.gen_padded(ctx, Np, (1, 1, 1), cl, cm, nu, pad=P, seed=5, stream=1,
                                               dtype=SPLIT))
    assert "k_c2r_x_tc" in st
    e = rel(out, ref)
    assert e <= 1e-5, (Np, P, e)
    # the CUDA-core FP32 pass 3 (SCARL_SPLIT_BF16 alone) is the finer one
    out1, st1 = _stats(ctx, lambda: S.gen_padded(ctx, Np, (1, 1, 1), cl, cm, nu, pad=P, seed=5, stream=1,
                                                 dtype=S.F32 | S.SPLIT_BF16))
    assert "k_c2r_x" in st1 and "k_c2r_x_tc" not in st1
    assert rel(out1, ref) < e


@pytest.mark.parametrize("pad", [(448, 384, 320), (512, 512, 512)])
def test_tc_pass3_headline_deck_vs_oracle(ctx, oracle, pad):
    """The 513^3 headline deck (2 x 2 x 2 tiles, exponential, lognormal mean 1
    CV 0.3) on the SMOOTH grid (half length 224 = 7 x 32) and the
    power-of-two grid (256 = 8 x 32): 8 tensor-core pass-3 launches, field
    within 1e-5 of the oracle's, the streamed FP64 moments equal to the
    moments of the field itself."""
    import torch
    head = dict(xMinGlob=(0, 0, 0), xMaxGlob=(512, 512, 512), corrL=(40, 20, 10), overlap=(2, 2, 2),
                pointsPerCorrL=(41, 21, 11))
    s = S.make_sample(corrMod=3, margiFirst=2, avg=1.0, std_dev=0.3, **head)
    ref, _ = oracle.generate_sample(S.GEN_PADDED, head["xMinGlob"], head["xMaxGlob"], head["corrL"],
                                    head["overlap"], head["pointsPerCorrL"], 3, 0.5, 2, 1.0, 0.3, 0, 8,
                                    (2, 2, 2), pad)
    n = 513 ** 3
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    mom = np.zeros(2)
    _, st = _stats(ctx, lambda: S.generate_sample(ctx, s, dtype=SPLIT, nb_procs=8, topo=(2, 2, 2), pad=pad,
                                                  out=y, moments=mom))
    ctx.sync()
    assert st["k_c2r_x_tc"][1] == 8
    got = y.cpu().numpy().astype(np.float64)
    r = np.asarray(ref, np.float64).reshape(-1, order="F")
    e = rel(got, r)
    m = float(np.max(np.abs(got - r)) / np.max(np.abs(r)))
    assert e <= 1e-5 and m <= 3e-5, (pad, e, m)
    s1, s2 = float(np.sum(got)), float(np.sum(got * got))
    assert abs(mom[0] - s1) <= 1e-9 * abs(s1) and abs(mom[1] - s2) <= 1e-9 * s2, (mom, s1, s2)
    del y
    torch.cuda.empty_cache()


def test_tc_pass3_flag_needs_fp32(ctx):
    """SCARL_SPLIT_BF16_X applies to SCARL_F32 only."""
    from scarl_b200 import _lib
    with pytest.raises(S.ScarlError) as e:
        S.gen_padded(ctx, (8, 8, 8), (1, 1, 1), (2, 2, 2), 1, dtype=S.F64 | S.SPLIT_BF16_X)
    assert e.value.code == _lib.EINVAL
