"""Mixed-radix padded lengths (3, 5, 7 times a power of two): every
instantiated line length in each of the three passes against the FP64
oracle (whose FFT handles any length).  Tolerances: FP64 rel-L2 <= 1e-12,
FP32 <= 1e-5, split-BF16 pass 1 <= 1e-5."""
import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)


# (Np, P): every mixed length appears as a z length (pass 1), a y length
# (pass 2) and a half x length (pass 3, N = P0 / 2) somewhere below
CASES = [
    ((20, 30, 40), (48, 80, 112)),        # z 112, y 80, x/2 24
    ((50, 60, 70), (160, 96, 224)),       # z 224, y 96, x/2 80
    ((70, 40, 150), (224, 48, 160)),      # z 160, y 48, x/2 112
    ((30, 100, 90), (80, 112, 192)),      # z 192, y 112, x/2 40
    ((40, 150, 60), (112, 192, 96)),      # z 96, y 192, x/2 56
    ((90, 120, 20), (192, 224, 48)),      # z 48, y 224, x/2 96
    ((100, 9, 300), (320, 16, 320)),      # z 320, x/2 160
    ((7, 300, 8), (16, 384, 16)),         # y 384
    ((9, 7, 400), (448, 16, 448)),        # z 448, x/2 224
    ((6, 500, 5), (640, 640, 8)),         # y 640, x/2 320
    ((5, 6, 600), (768, 16, 768)),        # z 768, x/2 384
    ((5, 800, 6), (896, 896, 16)),        # y 896, x/2 448
    ((6, 5, 1000), (16, 8, 1280)),        # z 1280
    ((5, 1200, 5), (1280, 1536, 8)),      # y 1536, x/2 640
    ((6, 5, 1500), (1536, 8, 1792)),      # z 1792, x/2 768
    ((5, 1600, 5), (1792, 1792, 8)),      # y 1792, x/2 896
]


@pytest.mark.parametrize("Np,P", CASES)
def test_mixed_lengths_vs_oracle(ctx, oracle, Np, P):
    cl, cm = (4.0, 6.0, 9.0), 3
    ref = oracle.gen_padded(Np, P, (1, 1, 1), cl, cm, 0.5, 1, seed=5, stream=1)
    out64 = S.gen_padded(ctx, Np, (1, 1, 1), cl, cm, pad=P, seed=5, stream=1, dtype=S.F64)
    assert rel(out64, ref) < 1e-12
    out32 = S.gen_padded(ctx, Np, (1, 1, 1), cl, cm, pad=P, seed=5, stream=1, dtype=S.F32)
    assert rel(out32, ref) < 1e-5


def test_unsupported_length_rejected(ctx):
    for P in ((88, 64, 64), (64, 64, 2 * 1024 + 512), (64, 56 * 2, 9 * 16)):
        with pytest.raises(S.ScarlError):
            S.gen_padded(ctx, (8, 8, 8), (1, 1, 1), (2, 2, 2), 1, pad=P)


def test_smooth_policy_blended_sample_vs_fp64(ctx, oracle):
    """A blended 2x2x1 sample on the SMOOTH grid: FP32 and FP64 paths against
    the oracle's blended sample on the same padded grid."""
    args = ((0, 0, 0), (60, 50, 40), (6, 5, 4), (1, 1, 1), (7, 6, 5))
    s = S.make_sample(*args, corrMod=3, margiFirst=2, avg=1.0, std_dev=0.3, seedBase=4)
    lay = S.sample_layout(s, 1, 4, (2, 2, 1))
    P = S.pad_size(S.PAD_SMOOTH, 3, args[2], lay["xStep"], lay["Np"], 0.5, 1e-3)
    assert any(p & (p - 1) for p in P)  # at least one length is not a power of two
    ref, _ = oracle.generate_sample(3, *args, 3, 0.5, 2, 1.0, 0.3, 4, nb_procs=4, topo=(2, 2, 1),
                                    pad=[int(v) for v in P])
    for dtype, tol in ((S.F64, 1e-12), (S.F32, 1e-5)):
        out, _ = S.generate_sample(ctx, s, dtype=dtype, nb_procs=4, topo=(2, 2, 1),
                                   pad_policy=S.PAD_SMOOTH)
        assert rel(out, ref) < tol
