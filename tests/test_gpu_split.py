"""Split-precision pass 1 (SCARL_F32 | SCARL_SPLIT_BF16): the z-axis DFT as
BF16 head/tail tensor-core products with FP32 accumulation.  Checked against
the FP64 oracle and the FP64 CUDA path on the same Philox normals.
Tolerance: field rel-L2 <= 1e-5 against FP64 (the stated bound of the split
form); the tensor-core kernel must be the one that ran."""
import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu

TOL = 1e-5
SPLIT = S.F32 | S.SPLIT_BF16


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b))
    return np.linalg.norm((a - b) / s) / np.linalg.norm(b / s)


def _ran_tc(ctx, fn):
    ctx.profile(True)
    ctx.profile_reset()
    out = fn()
    st = ctx.profile_stats()
    ctx.profile(False)
    return out, st


@pytest.mark.parametrize("Np,P,dx,cl,cm,nu", [
    ((12, 10, 300), (16, 16, 512), (1, 1, 1), (3, 3, 40), 3, 0.5),   # exponential
    ((9, 7, 500), (16, 8, 512), (1, 1, 1), (2, 2, 30), 1, 0.5),       # Gaussian, ragged last item
    ((20, 6, 267), (32, 16, 512), (0.5, 1, 1), (4, 3, 12), 2, 1.5),   # von Karman
    ((5, 5, 512), (8, 8, 512), (1, 1, 1), (2, 2, 64), 3, 0.5),        # every z kept
    ((6, 4, 1), (8, 8, 512), (1, 1, 1), (2, 2, 10), 3, 0.5),          # one z plane
    ((11, 9, 200), (32, 16, 256), (1, 1, 1), (3, 3, 20), 3, 0.5),     # N = 16 x 16
    ((7, 5, 256), (16, 8, 256), (1, 1, 1), (2, 2, 30), 1, 0.5),       # N = 16 x 16, all z
    ((9, 6, 600), (16, 16, 1024), (1, 1, 1), (3, 3, 60), 3, 0.5),     # N = 32 x 32, two chunks
    ((5, 7, 1024), (8, 16, 1024), (1, 1, 1), (2, 2, 90), 2, 0.8),     # N = 32 x 32, all z
    ((6, 5, 400), (16, 8, 1024), (1, 1, 1), (2, 2, 40), 1, 0.5),      # first chunk only
    ((10, 7, 267), (32, 16, 320), (1, 1, 1), (3, 3, 10), 3, 0.5),     # N = 8 x 40
    ((9, 5, 320), (16, 8, 320), (1, 1, 1), (2, 2, 30), 1, 0.5),       # N = 8 x 40, all z
    ((5, 6, 100), (8, 16, 320), (1, 1, 1), (2, 2, 15), 2, 0.8),       # first chunk only
    ((12, 8, 300), (48, 16, 384), (1, 1, 1), (3, 3, 25), 3, 0.5),     # N = 16 x 24
    ((6, 5, 384), (16, 8, 384), (1, 1, 1), (2, 2, 40), 1, 0.5),       # N = 16 x 24, all z
])
def test_split_vs_oracle(ctx, oracle, Np, P, dx, cl, cm, nu):
    ref = oracle.gen_padded(Np, P, dx, cl, cm, nu, 1, seed=77, stream=3)
    out, st = _ran_tc(ctx, lambda: S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=P, seed=77,
                                                stream=3, dtype=SPLIT))
    assert "k_gen_z_tc" in st and "k_gen_z" not in st
    err = rel(out, ref)
    print(f"split rel-L2 {err:.2e}, max {np.max(np.abs(out - ref)) / np.max(np.abs(ref)):.2e}")
    assert err < TOL
    out32 = S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=P, seed=77, stream=3, dtype=S.F32)
    assert rel(out32, ref) < err  # the split form is the coarser one


def test_split_deterministic_and_seeded(ctx):
    args = ((30, 20, 200), (1, 1, 1), (5, 5, 20), 3, 0.5)
    a = S.gen_padded(ctx, *args, pad=(64, 32, 512), seed=4, dtype=SPLIT)
    b = S.gen_padded(ctx, *args, pad=(64, 32, 512), seed=4, dtype=SPLIT)
    c = S.gen_padded(ctx, *args, pad=(64, 32, 512), seed=5, dtype=SPLIT)
    assert np.array_equal(a, b)
    assert rel(a, c) > 0.5


def test_split_other_lengths_use_fp32_pass(ctx, oracle):
    # z lengths without a tensor-core kernel (here 128) run the FP32 pass
    Np, P = (10, 10, 100), (16, 16, 128)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), (3, 3, 10), 3, 0.5, 1, seed=2)
    out, st = _ran_tc(ctx, lambda: S.gen_padded(ctx, Np, (1, 1, 1), (3, 3, 10), 3, pad=P, seed=2,
                                                dtype=SPLIT))
    assert "k_gen_z" in st and "k_gen_z_tc" not in st
    assert rel(out, ref) < TOL


def test_split_rejected_for_fp64(ctx):
    with pytest.raises(S.ScarlError):
        S.gen_padded(ctx, (8, 8, 8), (1, 1, 1), (2, 2, 2), 1, dtype=S.F64 | S.SPLIT_BF16)


def test_split_blended_sample_vs_fp64(ctx):
    """The headline deck (512^3 -> 513^3, exponential, l = (40, 20, 10),
    lognormal mean 1 CV 0.3, 2x2x2 tiles, overlap 2 l) on the AUTO padded
    grid 512^3 and the SMOOTH grid 448 x 384 x 320: split FP32 against FP64
    on the same normals."""
    s = S.make_sample((0, 0, 0), (512, 512, 512), (40, 20, 10), (2, 2, 2), (41, 21, 11),
                      corrMod=3, margiFirst=2, avg=1.0, std_dev=0.3)
    for policy in (S.PAD_AUTO, S.PAD_SMOOTH):
        kw = dict(nb_procs=8, topo=(2, 2, 2), pad_policy=policy)
        f64, lay = S.generate_sample(ctx, s, dtype=S.F64, **kw)
        (f32s, _), st = _ran_tc(ctx, lambda: S.generate_sample(ctx, s, dtype=SPLIT, **kw))
        assert st["k_gen_z_tc"][1] == 4  # host output: one batched launch per row of 2 tiles
        err = rel(f32s, f64)
        print(f"513^3 split rel-L2 {err:.2e} (policy {policy})")
        assert err < TOL


def test_batched_tiles_equal_per_tile_launches(ctx):
    """With the tensor-core pass 1 and the field in device memory, passes 1
    and 2 of a sample's 8 tiles run as one batched launch each; a context
    whose memory budget holds one tile's work buffer only runs them per tile;
    a host output takes one row of tiles per launch.  All three fields are
    bit-identical (513^3 headline deck)."""
    import torch
    s = S.make_sample((0, 0, 0), (512, 512, 512), (40, 20, 10), (2, 2, 2), (41, 21, 11),
                      corrMod=3, margiFirst=2, avg=1.0, std_dev=0.3)
    kw = dict(dtype=SPLIT, nb_procs=8, topo=(2, 2, 2), pad_policy=S.PAD_SMOOTH)
    n = 513 ** 3
    a = torch.empty(n, dtype=torch.float32, device="cuda")
    _, st = _ran_tc(ctx, lambda: S.generate_sample(ctx, s, out=a, **kw))
    ctx.sync()
    assert st["k_gen_z_tc"][1] == 1 and st["k_mid_y"][1] == 1 and st["k_c2r_x"][1] == 8
    b = torch.empty(n, dtype=torch.float32, device="cuda")
    small = S.Context(0, budget_bytes=1 << 30)  # one 185 MB work buffer fits, eight do not
    try:
        _, st1 = _ran_tc(small, lambda: S.generate_sample(small, s, out=b, **kw))
        small.sync()
    finally:
        small.close()
    assert st1["k_gen_z_tc"][1] == 8 and st1["k_mid_y"][1] == 8
    assert torch.equal(a, b)
    (h, _), st2 = _ran_tc(ctx, lambda: S.generate_sample(ctx, s, **kw))
    assert st2["k_gen_z_tc"][1] == 4
    np.testing.assert_array_equal(h.reshape(-1, order="F"), a.cpu().numpy())


def test_split_bounded_wait_reports_timeout(ctx, oracle):
    """With the test hook no matrix product is issued: every CTA's bounded wait
    on the tensor core runs out, the call returns SCARL_ETIMEOUT, and the
    context generates correctly afterwards."""
    from scarl_b200 import _lib
    Np, P, cl = (12, 10, 300), (16, 16, 512), (3, 3, 40)
    ctx.tc_wait_test(True)
    try:
        with pytest.raises(S.ScarlError) as e:
            S.gen_padded(ctx, Np, (1, 1, 1), cl, 3, pad=P, seed=77, stream=3, dtype=SPLIT)
        assert e.value.code == _lib.ETIMEOUT
    finally:
        ctx.tc_wait_test(False)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), cl, 3, 0.5, 1, seed=77, stream=3)
    out = S.gen_padded(ctx, Np, (1, 1, 1), cl, 3, pad=P, seed=77, stream=3, dtype=SPLIT)
    assert rel(out, ref) < TOL
    ctx.sync()


def test_batched_tiles_ragged_groups(ctx):
    """Tiles of 555 MB work buffers (991^3 field, 2x2x2 tiles on the 512^3 grid):
    the 4 GB batching cap takes them in groups of 7 and 1; the field equals
    per-tile launches bit for bit."""
    import torch
    s = S.make_sample((0, 0, 0), (990, 990, 990), (4, 4, 4), (1, 1, 1), (5, 5, 5), corrMod=3)
    kw = dict(dtype=SPLIT, nb_procs=8, topo=(2, 2, 2), pad_policy=S.PAD_SMOOTH)
    n = 991 ** 3
    a = torch.empty(n, dtype=torch.float32, device="cuda")
    _, st = _ran_tc(ctx, lambda: S.generate_sample(ctx, s, out=a, **kw))
    ctx.sync()
    assert st["k_gen_z_tc"][1] == 2 and st["k_mid_y"][1] == 2 and st["k_c2r_x"][1] == 8
    b = torch.empty(n, dtype=torch.float32, device="cuda")
    small = S.Context(0, budget_bytes=1 << 30)
    try:
        _, st1 = _ran_tc(small, lambda: S.generate_sample(small, s, out=b, **kw))
        small.sync()
    finally:
        small.close()
    assert st1["k_gen_z_tc"][1] == 8
    assert torch.equal(a, b)
    del a, b
    torch.cuda.empty_cache()


def test_fp32_tiles_run_per_tile(ctx):
    """The CUDA-core FP32 passes run per tile (batching measured slower)."""
    s = S.make_sample((0, 0, 0), (120, 100, 90), (8, 6, 5), (1, 1, 1), (5, 5, 5), corrMod=3)
    (_, _), st = _ran_tc(ctx, lambda: S.generate_sample(ctx, s, dtype=S.F32, nb_procs=8, topo=(2, 2, 2)))
    assert st["k_gen_z"][1] == 8 and st["k_mid_y"][1] == 8 and st["k_c2r_x"][1] == 8

