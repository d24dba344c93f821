"""CUDA path (through the C ABI) against the CPU oracle and the golden
fixtures.  Tolerances: FP64 fields rel-L2 <= 1e-12; FP32 fields rel-L2 <=
1e-5 against FP64; weights, overlap sums and index maps bit-exact."""
import os

import numpy as np
import pytest

import scarl_b200 as S

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))

TOL64 = 1e-12
TOL32 = 1e-5


def rel(a, b):
    """rel-L2 error, scaled first so that huge fields cannot overflow the norm."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b))
    return np.linalg.norm((a - b) / s) / np.linalg.norm(b / s)


# ---------------------------------------------------------------------------
# padded periodic generator
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("tag", ["g", "e", "v"])
@pytest.mark.parametrize("dtype,tol", [(S.F64, TOL64), (S.F32, TOL32)])
def test_gen_padded_injected_golden(ctx, tag, dtype, tol):
    xi = GOLD[f"pad_{tag}_xi"]
    if dtype == S.F32:
        xi = xi.astype(np.float32)
    out = S.gen_padded(ctx, GOLD[f"pad_{tag}_Np"], GOLD[f"pad_{tag}_dx"], GOLD[f"pad_{tag}_corrL"],
                       int(GOLD[f"pad_{tag}_cm"]), float(GOLD[f"pad_{tag}_nu"]),
                       pad=GOLD[f"pad_{tag}_P"], xi=xi, dtype=dtype)
    assert rel(out, GOLD[f"pad_{tag}_out"]) < tol


@pytest.mark.parametrize("Np,P,dx,cl,cm,nu", [
    ((20, 20, 20), (64, 64, 64), (1, 1, 1), (5, 5, 5), 1, 0.5),
    ((30, 17, 11), (64, 32, 32), (0.5, 1, 2), (3, 6, 9), 3, 0.5),
    ((33, 40, 25), (128, 64, 64), (1, 1, 1), (8, 4, 6), 2, 1.5),
    ((16, 16, 16), (32, 32, 32), (1, 1, 1), (4, 4, 4), 2, 0.3),
    ((100, 7, 9), (256, 16, 32), (1, 1, 1), (10, 2, 3), 3, 0.5),
    ((5, 60, 3), (32, 128, 32), (1, 1, 1), (2, 10, 2), 1, 0.5),
    ((300, 6, 5), (512, 16, 16), (1, 1, 1), (40, 3, 3), 3, 0.5),
    ((600, 5, 4), (2048, 8, 8), (1, 1, 1), (60, 2, 2), 3, 0.5),
    ((6, 400, 5), (16, 1024, 16), (1, 1, 1), (3, 30, 3), 2, 0.8),
    ((5, 6, 700), (16, 16, 2048), (1, 1, 1), (3, 3, 50), 1, 0.5),
    ((7, 5, 297), (16, 8, 1024), (1, 1, 1), (3, 3, 10), 3, 0.5),
])
def test_gen_padded_philox_vs_oracle(ctx, oracle, Np, P, dx, cl, cm, nu):
    ref = oracle.gen_padded(Np, P, dx, cl, cm, nu, 1, seed=77, stream=3)
    out64 = S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=P, seed=77, stream=3, dtype=S.F64)
    assert rel(out64, ref) < TOL64
    out32 = S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=P, seed=77, stream=3, dtype=S.F32)
    assert rel(out32, ref) < TOL32


def test_gen_padded_unnormalised_vs_oracle(ctx, oracle):
    Np, P = (24, 24, 24), (64, 64, 64)
    ref = oracle.gen_padded(Np, P, (1, 1, 1), (6, 6, 6), 3, 0.5, 0, seed=5)
    out = S.gen_padded(ctx, Np, (1, 1, 1), (6, 6, 6), 3, pad=P, normalise=False, seed=5,
                       dtype=S.F64)
    assert rel(out, ref) < TOL64


def test_gen_padded_default_pad_and_determinism(ctx):
    a = S.gen_padded(ctx, (40, 30, 20), (1, 1, 1), (5, 5, 5), 1, seed=9)
    b = S.gen_padded(ctx, (40, 30, 20), (1, 1, 1), (5, 5, 5), 1, seed=9)
    c = S.gen_padded(ctx, (40, 30, 20), (1, 1, 1), (5, 5, 5), 1, seed=10)
    assert np.array_equal(a, b)
    assert not np.allclose(a, c)


def test_gen_padded_device_pointer(ctx):
    torch = pytest.importorskip("torch")
    host = S.gen_padded(ctx, (32, 16, 8), (1, 1, 1), (4, 4, 4), 1, seed=1, dtype=S.F32)
    dev = torch.empty(8 * 16 * 32, dtype=torch.float32, device="cuda")
    S.gen_padded(ctx, (32, 16, 8), (1, 1, 1), (4, 4, 4), 1, seed=1, dtype=S.F32, out=dev)
    ctx.sync()
    np.testing.assert_array_equal(dev.cpu().numpy(), host.reshape(-1, order="F"))


# ---------------------------------------------------------------------------
# reference generators
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("tag", ["a", "b"])
def test_dct_generator_golden(ctx, tag):
    out = S.gen_std_gauss_FFT(ctx, GOLD[f"dct_{tag}_Np"], GOLD[f"dct_{tag}_xRange"],
                              GOLD[f"dct_{tag}_corrL"], 1, 0, 0, phiK=GOLD[f"dct_{tag}_phi"])
    assert rel(out, GOLD[f"dct_{tag}_out"]) < TOL64


@pytest.mark.parametrize("Np", [(64, 64, 64), (37, 50, 29), (128, 20, 3)])
def test_dct_generator_vs_oracle(ctx, oracle, Np):
    rng = np.random.default_rng(sum(Np))
    phi = np.asfortranarray(rng.random([n // 2 for n in Np]))
    gam = np.asfortranarray(rng.random([n // 2 for n in Np]))
    xr = [(n - 1) * 0.5 for n in Np]
    cl = (3.0, 4.0, 5.0)
    ref = oracle.gen_std_gauss_fft(Np, xr, cl, phi, gam)
    out = S.gen_std_gauss_FFT(ctx, Np, xr, cl, 1, 0, 0, phiK=phi, gammaK=gam)
    assert rel(out, ref) < TOL64


def test_dct_generator_default_phases(ctx, oracle):
    Np = (20, 22, 18)
    xr = [19.0, 21.0, 17.0]
    seed, rank = 41, 3
    phi = oracle.uniforms(seed + rank, 0, 0, 10 * 11 * 9).reshape((10, 11, 9), order="F")
    ref = oracle.gen_std_gauss_fft(Np, xr, (2, 2, 2), phi)
    out = S.gen_std_gauss_FFT(ctx, Np, xr, (2, 2, 2), 1, seed, rank)
    assert rel(out, ref) < TOL64


@pytest.mark.parametrize("tag", ["a", "b"])
def test_shino_generator_golden(ctx, tag):
    out = S.gen_std_gauss_Shino_FFT(ctx, GOLD[f"shino_{tag}_Np"], GOLD[f"shino_{tag}_xRange"],
                                    GOLD[f"shino_{tag}_corrL"], seed=int(GOLD[f"shino_{tag}_seed"]))
    assert rel(out, GOLD[f"shino_{tag}_out"]) < TOL64


@pytest.mark.parametrize("Np,xr,cl,seed", [
    ((40, 40, 40), (39.0, 39.0, 39.0), (4.0, 4.0, 4.0), 1),
    ((25, 70, 33), (24.0, 34.5, 64.0), (3.0, 2.0, 5.0), -17),
    ((100, 12, 9), (99.0, 11.0, 8.0), (9.0, 1.0, 1.0), 2147483000),
])
def test_shino_generator_vs_oracle(ctx, oracle, Np, xr, cl, seed):
    ref = oracle.gen_std_gauss_shino_fft(Np, xr, cl, seed, 0)
    out = S.gen_std_gauss_Shino_FFT(ctx, Np, xr, cl, seed=seed)
    assert rel(out, ref) < TOL64


# ---------------------------------------------------------------------------
# full sample: tiles, PoU, overlap, marginal
# ---------------------------------------------------------------------------
SAMPLES = [
    # xmin, xmax, corrL, overlap, ppcl, corrMod, nu, margi, avg, std, seed, nb, topo
    ((0, 0, 0), (30, 24, 20), (4, 3, 5), (1, 1, 1), (5, 4, 6), 1, 0.5, 1, 0.0, 1.0, 0, 8, None),
    ((0, 0, 0), (40, 20, 12), (5, 5, 3), (2, 1, 0.5), (6, 6, 5), 3, 0.5, 2, 1.0, 0.3, 3, 6, (3, 2, 1)),
    ((-5, 2, 1), (20, 30, 14), (3, 6, 2), (0, 1, 1), (4, 5, 5), 2, 1.5, 2, 2.0, 0.5, 11, 4, (2, 1, 2)),
    ((0, 0, 0), (16, 16, 16), (2, 2, 2), (0, 0, 0), (5, 5, 5), 1, 0.5, 1, 1.0, 2.0, 7, 8, (2, 2, 2)),
    ((0, 0, 0), (24, 18, 10), (2, 3, 2), (0.25, 0.34, 0.1), (5, 4, 4), 3, 0.5, 1, 0.0, 1.0, 2, 8, None),
]


@pytest.mark.parametrize("case", range(len(SAMPLES)))
@pytest.mark.parametrize("generator", [S.GEN_PADDED, S.GEN_DCT, S.GEN_SHINO])
def test_generate_sample_vs_oracle(ctx, oracle, case, generator):
    (xmin, xmax, cl, ov, ppcl, cm, nu, mf, avg, sd, seed, nb, topo) = SAMPLES[case]
    if generator != S.GEN_PADDED:
        cm = 1
    s = S.make_sample(xmin, xmax, cl, ov, ppcl, cm, mf, avg, sd, seed, nu)
    ref, lay = oracle.generate_sample(generator, xmin, xmax, cl, ov, ppcl, cm, nu, mf, avg, sd,
                                      seed, nb, topo)
    out, glay = S.generate_sample(ctx, s, generator=generator, dtype=S.F64, nb_procs=nb, topo=topo)
    np.testing.assert_array_equal(glay["L"], lay["L"])
    assert rel(out, ref) < TOL64
    if generator == S.GEN_PADDED:
        out32, _ = S.generate_sample(ctx, s, generator=generator, dtype=S.F32, nb_procs=nb, topo=topo)
        assert rel(out32, ref) < TOL32


@pytest.mark.parametrize("topo,generator,dtype,ov", [
    ((2, 2, 2), S.GEN_PADDED, S.F32, (1, 1, 1.5)),
    ((2, 1, 3), S.GEN_PADDED, S.F64, (1, 1, 1.5)),
    ((1, 2, 4), S.GEN_PADDED, S.F32 | S.SPLIT_BF16, (1, 1, 1.5)),
    ((2, 1, 2), S.GEN_DCT, S.F64, (1, 1, 1.5)),
    ((2, 3, 1), S.GEN_PADDED, S.F32, (1, 1, 1.5)),
    ((1, 1, 1), S.GEN_PADDED, S.F32, (1, 1, 1.5)),
    ((1, 3, 2), S.GEN_PADDED, S.F32, (0, 0, 0)),      # overlap 0: neighbours share one plane
])
def test_generate_sample_pinned_host_output(ctx, topo, generator, dtype, ov):
    """Into pinned host memory the field comes back box by box (the y rows
    and z planes a row of tiles finishes) while later tile rows are
    generated: bit-identical to the device output and to a pageable host
    output, every byte copied once."""
    import torch
    cm = 3 if generator == S.GEN_PADDED else 1
    s = S.make_sample((0, 0, 0), (60, 50, 90), (4, 5, 6), ov, (5, 5, 5), cm, 2, 1.0, 0.3, 9)
    nb = topo[0] * topo[1] * topo[2]
    kw = dict(generator=generator, dtype=dtype, nb_procs=nb, topo=topo)
    ref, lay = S.generate_sample(ctx, s, **kw)  # pageable host memory
    L = tuple(int(v) for v in lay["L"])
    tdt = torch.float64 if ref.dtype == np.float64 else torch.float32
    dev = torch.empty(int(np.prod(L)), dtype=tdt, device="cuda")
    S.generate_sample(ctx, s, out=dev, **kw)
    ctx.sync()
    pin = torch.empty(int(np.prod(L)), dtype=tdt, pin_memory=True)
    hp = pin.numpy().reshape(L, order="F")
    for _ in range(2):
        hp[...] = np.nan
        c0 = ctx.counters()
        S.generate_sample(ctx, s, out=hp, **kw)
        c1 = ctx.counters()
        assert c1["d2h_bytes"] - c0["d2h_bytes"] == ref.nbytes
        np.testing.assert_array_equal(hp, ref)
    np.testing.assert_array_equal(dev.cpu().numpy().reshape(L, order="F"), ref)


@pytest.mark.parametrize("dtype,topo", [(S.F32, (2, 2, 1)), (S.F64, (2, 2, 1)), (S.F32, (1, 2, 3))])
def test_large_pageable_host_output(ctx, dtype, topo):
    """Outputs of 8 MB and more into pageable host memory pass through the
    context's pinned ring in pieces of at most 32 MB (the boxes that each row
    of tiles finishes, copied while later rows generate; for a single tile,
    32 MB chunks with a ragged last one), moved out by host threads:
    bit-identical to the device output, into fresh and into reused arrays."""
    import torch
    s = S.make_sample((0, 0, 0), (300, 300, 200), (6, 8, 5), (1, 1, 1), (9, 9, 9), 3, 2, 1.0, 0.3, 4)
    kw = dict(dtype=dtype, nb_procs=topo[0] * topo[1] * topo[2], topo=topo)
    a, lay = S.generate_sample(ctx, s, **kw)  # fresh pageable array
    L = tuple(int(v) for v in lay["L"])
    assert a.nbytes > 2 * 32 * 2**20 and a.nbytes % (32 * 2**20) != 0
    tdt = torch.float64 if a.dtype == np.float64 else torch.float32
    dev = torch.empty(int(np.prod(L)), dtype=tdt, device="cuda")
    S.generate_sample(ctx, s, out=dev, **kw)
    ctx.sync()  # device outputs return once the work is queued
    ref = dev.cpu().numpy().reshape(L, order="F")
    np.testing.assert_array_equal(a, ref)
    b = np.full(L, np.nan, dtype=a.dtype, order="F")
    for _ in range(2):
        c0 = ctx.counters()
        S.generate_sample(ctx, s, out=b, **kw)
        assert ctx.counters()["d2h_bytes"] - c0["d2h_bytes"] == b.nbytes
        np.testing.assert_array_equal(b, ref)
    # the single-tile generator through the same path
    g = S.gen_padded(ctx, (260, 250, 130), (1, 1, 1), (5, 5, 5), 3, pad=(512, 512, 256), seed=3,
                     dtype=dtype)
    gd = torch.empty(260 * 250 * 130, dtype=tdt, device="cuda")
    S.gen_padded(ctx, (260, 250, 130), (1, 1, 1), (5, 5, 5), 3, pad=(512, 512, 256), seed=3,
                 dtype=dtype, out=gd)
    ctx.sync()
    np.testing.assert_array_equal(g, gd.cpu().numpy().reshape(g.shape, order="F"))


def test_generate_sample_normalize_field(ctx, oracle):
    args = ((0, 0, 0), (30, 24, 20), (4, 3, 5), (1, 1, 1), (5, 4, 6))
    s = S.make_sample(*args, 1, 2, 1.0, 0.4, 5)
    ref, _ = oracle.generate_sample(3, *args, 1, 0.5, 2, 1.0, 0.4, 5, 8, None, normalize_field=1)
    out, _ = S.generate_sample(ctx, s, dtype=S.F64, nb_procs=8, normalize_field=True)
    assert rel(out, ref) < TOL64


def test_generate_sample_constant_field(ctx):
    s = S.make_sample((0, 0, 0), (10, 10, 10), (1, 1, 1), (1, 1, 1), (3, 3, 3), 1, 1, 2.5, 0.0, 0)
    out, _ = S.generate_sample(ctx, s, nb_procs=2)
    assert np.all(out == np.float32(2.5))


def test_generate_sample_dct_injected_phases(ctx, oracle):
    args = ((0, 0, 0), (12, 10, 8), (2, 2, 2), (1, 1, 1), (4, 4, 4))
    lay = oracle.sample_layout(*args, 1, 4)
    K = int(np.prod(lay["Np"] // 2))
    phi = np.random.default_rng(0).random(4 * K)
    s = S.make_sample(*args, 1, 1, 0.0, 1.0, 0)
    ref, _ = oracle.generate_sample(1, *args, 1, 0.5, 1, 0.0, 1.0, 0, 4, None, phiK_all=phi)
    out, _ = S.generate_sample(ctx, s, generator=S.GEN_DCT, dtype=S.F64, nb_procs=4, phiK=phi)
    assert rel(out, ref) < TOL64


# ---------------------------------------------------------------------------
# post steps
# ---------------------------------------------------------------------------
def test_apply_unity_partition_bit_exact(ctx, oracle):
    rng = np.random.default_rng(1)
    for Np, No, pos, shape in [((9, 8, 7), (4, 3, 2), (1, 0, 1), (3, 2, 2)),
                               ((16, 12, 10), (5, 1, 3), (0, 1, 0), (2, 2, 2)),
                               ((7, 7, 7), (3, 3, 3), (1, 1, 1), (3, 3, 3))]:
        f = np.asfortranarray(rng.standard_normal(Np))
        ref = oracle.apply_unity_partition(f, Np, No, pos, shape)
        g = f.copy(order="F")
        S.apply_UnityPartition_mtx(ctx, g, Np, No, 1, pos, shape)
        np.testing.assert_array_equal(g, ref)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_add_overlap_bit_exact(ctx, tag):
    tiles = np.ascontiguousarray(GOLD[f"ovl_{tag}_in"])
    shape = GOLD[f"ovl_{tag}_shape"]
    Np = GOLD[f"ovl_{tag}_Np"]
    # tiles are stored rank-major, each tile in Fortran order
    flat = np.concatenate([t.reshape(-1, order="F") for t in tiles])
    S.add_overlap(ctx, flat, Np, GOLD[f"ovl_{tag}_No"], shape)
    ref = np.concatenate([t.reshape(-1, order="F") for t in GOLD[f"ovl_{tag}_out"]])
    np.testing.assert_array_equal(flat, ref)


@pytest.mark.parametrize("mf,avg,sd", [(1, 0.5, 2.0), (2, 1.0, 0.3), (2, 3.0, 1.5)])
def test_multivariate_transformation(ctx, oracle, mf, avg, sd):
    f = np.random.default_rng(2).standard_normal(1000)
    ref = oracle.multivariate_transformation(avg, sd, mf, f)
    g = f.copy()
    S.multiVariateTransformation(ctx, avg, sd, mf, g)
    np.testing.assert_allclose(g, ref, rtol=1e-15, atol=1e-15)
    g32 = f.astype(np.float32)
    S.multiVariateTransformation(ctx, avg, sd, mf, g32)
    assert rel(g32, ref) < TOL32


def test_normalize_field(ctx, oracle):
    f = np.asfortranarray(np.random.default_rng(3).standard_normal((20, 15, 10)) * 3 + 1)
    (ref,), a, s = oracle.normalize_field([f], [20, 15, 10], [0, 0, 0], [1, 1, 1])
    g = f.copy(order="F")
    a2, s2 = S.normalize_field(ctx, g)
    assert a2 == pytest.approx(a, rel=1e-13) and s2 == pytest.approx(s, rel=1e-13)
    assert rel(g, ref) < TOL64


def test_marginal_rejects_nonpositive_lognormal_mean(ctx):
    with pytest.raises(S.ScarlError) as e:
        S.multiVariateTransformation(ctx, 0.0, 1.0, 2, np.zeros(4))
    assert e.value.code == 1


# ---------------------------------------------------------------------------
# estimators
# ---------------------------------------------------------------------------
def test_moments_vs_oracle(ctx, oracle):
    f = np.random.default_rng(4).standard_normal((7000, 5)) * 2 + 0.5
    ref = oracle.moments(f)
    got = S.calculate_average_and_stdVar(ctx, np.asfortranarray(f), Nmc=5)
    np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(got[1], ref[1], rtol=1e-12)
    assert got[2] == pytest.approx(ref[2], rel=1e-12) and got[3] == pytest.approx(ref[3], rel=1e-12)
    got32 = S.calculate_average_and_stdVar(ctx, np.asfortranarray(f.astype(np.float32)), Nmc=5)
    assert got32[3] == pytest.approx(ref[3], rel=1e-6)


def test_rebuild_sk_golden(ctx):
    f = GOLD["sk_field"]
    sk = S.rebuild_Sk(ctx, f, f.shape, float(GOLD["sk_avg"]), float(GOLD["sk_sd"]))
    off = 0
    for d in range(3):
        n = f.shape[d] // 2
        np.testing.assert_allclose(sk[off:off + n], GOLD[f"sk_dir{d}"][:n], rtol=1e-12, atol=1e-14)
        off += n


@pytest.mark.parametrize("shape", [(33, 20, 17), (64, 8, 40), (5, 6, 7)])
@pytest.mark.parametrize("literal", [True, False])
def test_rebuild_sk_vs_oracle(ctx, oracle, shape, literal):
    f = np.asfortranarray(np.random.default_rng(sum(shape)).standard_normal(shape))
    avg, sd = float(f.mean()), float(f.std())
    sk = S.rebuild_Sk(ctx, f, shape, avg, sd, tukey_literal=literal)
    off = 0
    for d in range(3):
        n = shape[d] // 2
        ref = oracle.rebuild_sk_fft(f, d, avg, sd, int(literal))
        np.testing.assert_allclose(sk[off:off + n], ref[:n], rtol=1e-11, atol=1e-13)
        off += n
    cl = S.rebuild_corrL(sk, shape, (1.0, 0.5, 2.0))
    np.testing.assert_array_equal(cl, oracle.rebuild_corrL(sk, [v // 2 for v in shape], (1.0, 0.5, 2.0)))


# ---------------------------------------------------------------------------
# error paths
# ---------------------------------------------------------------------------
def test_error_paths(ctx):
    with pytest.raises(S.ScarlError) as e:
        S.gen_padded(ctx, (10, 10, 10), (1, 1, 1), (2, 2, 2), 1, pad=(24, 32, 32))
    assert e.value.code == 5
    with pytest.raises(S.ScarlError) as e:
        S.gen_padded(ctx, (40, 10, 10), (1, 1, 1), (2, 2, 2), 1, pad=(32, 32, 32))
    assert e.value.code == 1
    with pytest.raises(S.ScarlError) as e:
        S.gen_std_gauss_FFT(ctx, (8, 8, 8), (7, 7, 7), (1, 1, 1), corrMod=2)
    assert e.value.code == 1
    small = S.Context(0, budget_bytes=1 << 20)
    try:
        with pytest.raises(S.ScarlError) as e:
            S.gen_padded(small, (200, 200, 200), (1, 1, 1), (8, 8, 8), 1)
        assert e.value.code == 2
    finally:
        small.close()


@pytest.mark.parametrize("cm,nu", [(3, 0.5), (1, 0.5), (2, 1.2)])
def test_generate_sample_auto_padding_vs_oracle(ctx, oracle, cm, nu):
    args = ((0, 0, 0), (40, 30, 20), (6, 4, 3), (1, 1, 1), (7, 5, 4))
    s = S.make_sample(*args, cm, 2, 1.0, 0.3, 9, nu)
    lay = S.sample_layout(s, 1, 8)
    P = S.pad_size(S.PAD_AUTO, cm, args[2], lay["xStep"], lay["Np"], nu, 1e-3)
    assert np.prod(P) < np.prod(S.pad_size(S.PAD_FULL, cm, args[2], lay["xStep"], lay["Np"]))
    ref, _ = oracle.generate_sample(3, *args, cm, nu, 2, 1.0, 0.3, 9, 8, None, pad=P)
    out, _ = S.generate_sample(ctx, s, dtype=S.F64, nb_procs=8, pad_policy=S.PAD_AUTO)
    assert rel(out, ref) < TOL64


# ---------------------------------------------------------------------------
# global (FFT_MPI) path: one transform over the whole re-fitted grid
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("L", [(16, 12, 10), (33, 20, 17), (64, 48, 40)])
def test_gen_std_gauss_fft_mpi_vs_oracle(ctx, oracle, L):
    rng = np.random.default_rng(sum(L))
    phi = rng.random((L[0] // 2, L[1] // 2, L[2]))
    gam = rng.random((L[0] // 2, L[1] // 2, L[2]))
    xr = tuple((n - 1) * 0.5 for n in L)
    ref = oracle.gen_std_gauss_fft_mpi(L, xr, (3, 2, 4), phi, gam)
    out = S.gen_std_gauss_FFT_MPI(ctx, xr, (3, 2, 4), 1, 5, 0, L=L, phiK=phi, gammaK=gam)
    assert rel(out, ref) < TOL64
    with pytest.raises(S.ScarlError) as e:
        S.gen_std_gauss_FFT_MPI(ctx, xr, (3, 2, 4), 1, 5, 0, L=L, Np=(L[0], L[1], L[2] // 2))
    assert e.value.code == 5


def test_generate_sample_fft_mpi_global(ctx, oracle):
    """gen_meth = FFT_MPI: the slabs of 3 ranks re-fit the grid (L2 a multiple
    of 3); the GPU generates it as one global DCT field with the marginal."""
    s = S.make_sample((0, 0, 0), (30, 20, 25), (4, 3, 5), (1, 1, 1), (5, 4, 6), corrMod=1,
                      margiFirst=1, avg=2.0, std_dev=0.5)
    lay = S.sample_layout(s, 2, 3)
    L = [int(v) for v in lay["L"]]
    assert L[2] % 3 == 0 and list(lay["Np_ovlp"]) == [0, 0, 0]
    rng = np.random.default_rng(2)
    phi = rng.random((L[0] // 2, L[1] // 2, L[2]))
    out, glay = S.generate_sample(ctx, s, generator=S.GEN_DCT, dtype=S.F64, nb_procs=3,
                                  gen_meth=2, phiK=phi.reshape(-1, order="F"))
    assert list(glay["L"]) == L
    xr = [(n - 1) * float(dx) for n, dx in zip(L, lay["xStep"])]
    base = oracle.gen_std_gauss_fft_mpi(L, xr, (4, 3, 5), phi)
    # the reference's DCT field is unnormalised, so the Gaussian marginal
    # (x * std + avg) is the one that stays finite
    assert rel(out, base * 0.5 + 2.0) < TOL64
    # the padded method over the global grid: one tile, no blend
    s.margiFirst = 2
    pad, _ = S.generate_sample(ctx, s, dtype=S.F64, nb_procs=3, gen_meth=2, pad_policy=S.PAD_AUTO)
    s.margiFirst = 1
    s.avg, s.std_dev = 0.0, 1.0
    std, _ = S.generate_sample(ctx, s, dtype=S.F64, nb_procs=3, gen_meth=2, pad_policy=S.PAD_AUTO)
    P = S.pad_size(S.PAD_AUTO, 1, (4, 3, 5), lay["xStep"], L)
    ref2 = oracle.gen_padded(L, P, lay["xStep"], (4, 3, 5), 1, 0.5, 1, seed=1)
    assert rel(std, ref2) < TOL64
    assert np.all(pad > 0)
