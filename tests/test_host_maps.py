"""Host-side C++ of libscarl_b200 (index maps, topology, tile geometry,
partition-of-unity weights, Shino sizes, validation) against the oracle's
restatement: bit-exact, on the CPU, no GPU needed."""
import os

import numpy as np
import pytest

import scarl_b200 as S

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def _random_decks(n, seed=0):
    rng = np.random.default_rng(seed)
    for _ in range(n):
        xmin = rng.uniform(-50, 50, 3)
        xmax = xmin + rng.uniform(0.5, 300, 3)
        corrL = rng.uniform(0.3, 40, 3)
        ov = rng.choice([0.0, 0.5, 1.0, 2.0, 127 / 64, rng.uniform(0, 3)], 3)
        ppcl = rng.integers(2, 70, 3)
        yield xmin, xmax, corrL, ov, ppcl


@pytest.mark.parametrize("nb_procs", [1, 2, 3, 4, 6, 7, 8, 12, 16, 27, 64])
def test_sample_layout_matches_oracle(oracle, nb_procs):
    for xmin, xmax, corrL, ov, ppcl in _random_decks(40, nb_procs):
        s = S.make_sample(xmin, xmax, corrL, ov, ppcl)
        got = S.sample_layout(s, 1, nb_procs)
        ref = oracle.sample_layout(xmin, xmax, corrL, ov, ppcl, 1, nb_procs)
        for k in ("L", "Np", "Np_ovlp", "topo"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
        np.testing.assert_array_equal(got["xStep"], ref["xStep"])


def test_sample_layout_fft_mpi_and_explicit_topology(oracle):
    for xmin, xmax, corrL, ov, ppcl in _random_decks(20, 99):
        s = S.make_sample(xmin, xmax, corrL, ov, ppcl)
        for gm, nb, topo in ((2, 5, None), (1, 8, (2, 2, 2)), (1, 6, (3, 1, 2))):
            got = S.sample_layout(s, gm, nb, topo)
            ref = oracle.sample_layout(xmin, xmax, corrL, ov, ppcl, gm, nb, topo)
            for k in ("L", "Np", "Np_ovlp", "topo"):
                np.testing.assert_array_equal(got[k], ref[k])
    with pytest.raises(S.ScarlError):
        S.sample_layout(S.make_sample(), 1, 8, (2, 2, 3))


def test_worked_configurations():
    # 512^3 deck with l = (40, 20, 10), spacing 1, overlap 2 l, 2x2x2 tiles
    s = S.make_sample((0, 0, 0), (512, 512, 512), (40, 20, 10), (2, 2, 2), (41, 21, 11))
    lay = S.sample_layout(s, 1, 8)
    assert list(lay["L"]) == [513, 513, 513]
    assert list(lay["Np"]) == [297, 277, 267] and list(lay["Np_ovlp"]) == [81, 41, 21]
    assert list(lay["topo"]) == [2, 2, 2]
    # 128^3, l = 10, spacing 1, one tile
    s = S.make_sample((0, 0, 0), (127, 127, 127), (10, 10, 10), (0, 0, 0), (11, 11, 11))
    lay = S.sample_layout(s, 1, 1)
    assert list(lay["L"]) == [128] * 3 and list(lay["Np"]) == [128] * 3
    # 2048 x 2048 x 1024 with 4x4x1 tiles and a 128-point overlap
    s = S.make_sample((0, 0, 0), (2047, 2047, 1023), (64, 64, 32), (127 / 64, 127 / 64, 0),
                      (65, 65, 33))
    lay = S.sample_layout(s, 1, 16, (4, 4, 1))
    assert list(lay["L"]) == [2048, 2048, 1024] and list(lay["Np"]) == [608, 608, 1024]
    assert list(lay["Np_ovlp"])[:2] == [128, 128]


def test_decide_topo_shape_matches_oracle(oracle):
    rng = np.random.default_rng(5)
    for _ in range(300):
        L = rng.integers(1, 3000, 3)
        ov = rng.integers(0, 200, 3)
        nb = int(rng.integers(1, 200))
        np.testing.assert_array_equal(S.decide_topo_shape(nb, L, ov),
                                      oracle.decide_topo_shape(nb, L, ov))


def test_topo_pos_rank_roundtrip(oracle):
    for shape in [(1, 1, 1), (2, 2, 2), (3, 1, 2), (4, 4, 1), (5, 3, 7)]:
        for r in range(int(np.prod(shape))):
            p = S.get_topo_pos(r, shape)
            np.testing.assert_array_equal(p, oracle.get_topo_pos(r, shape))
            assert S.get_topo_rank(shape, p) == r
            assert p[0] + shape[0] * (p[1] + shape[1] * p[2]) == r


def test_tile_geometry_matches_oracle(oracle):
    for xmin, xmax, corrL, ov, ppcl in _random_decks(30, 7):
        s = S.make_sample(xmin, xmax, corrL, ov, ppcl)
        lay = S.sample_layout(s, 1, 8)
        for r in range(lay["nb_tiles"]):
            g = S.tile_geometry(lay, xmin, r)
            ref = oracle.tile_geometry(lay["Np"], lay["Np_ovlp"], g["topo_pos"], lay["xStep"], xmin)
            for k in ("pos_0", "pos_N", "coord_0", "coord_N", "xRange"):
                np.testing.assert_array_equal(g[k], ref[k], err_msg=k)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_pou_weights_golden_bit_exact(tag):
    w = S.unity_partition_weights(GOLD[f"pou_{tag}_Np"], GOLD[f"pou_{tag}_No"],
                                  GOLD[f"pou_{tag}_pos"], GOLD[f"pou_{tag}_shape"])
    np.testing.assert_array_equal(w, GOLD[f"pou_{tag}_w"])


def test_pou_weights_match_oracle_bit_exact(oracle):
    rng = np.random.default_rng(11)
    for _ in range(40):
        shape = rng.integers(1, 4, 3)
        pos = np.array([rng.integers(0, s) for s in shape])
        No = rng.integers(0, 6, 3)
        Np = np.maximum(2 * No, rng.integers(2, 12, 3))
        w = S.unity_partition_weights(Np, No, pos, shape)
        np.testing.assert_array_equal(w, oracle.unity_partition_weights(Np, No, pos, shape))


def test_pou_is_partition_of_unity():
    # weights of overlapping tiles sum to one on every shared point
    Np, No, shape = [10, 8, 6], [4, 3, 2], [2, 2, 2]
    L = [Np[d] * shape[d] - (shape[d] - 1) * No[d] for d in range(3)]
    tot = np.zeros(L, order="F")
    for r in range(8):
        p = S.get_topo_pos(r, shape)
        o = [(Np[d] - No[d]) * p[d] for d in range(3)]
        tot[o[0]:o[0] + Np[0], o[1]:o[1] + Np[1], o[2]:o[2] + Np[2]] += \
            S.unity_partition_weights(Np, No, p, shape)
    np.testing.assert_allclose(tot, 1.0, atol=1e-15)


def test_shino_sizes_match_oracle(oracle):
    rng = np.random.default_rng(2)
    for _ in range(50):
        Np = rng.integers(2, 700, 3)
        cl = rng.uniform(0.5, 50, 3)
        xr = (Np - 1) * rng.uniform(0.05, 2, 3)
        got = S.shino_sizes(Np, xr, cl)
        ref = oracle.shino_sizes(Np, xr, cl)
        for k in ("sz_c", "sz_Sk", "delta_k"):
            np.testing.assert_array_equal(got[k], ref[k])


@pytest.mark.parametrize("field,value,msg", [
    ("xMaxGlob", (0, 1, 1), "xMinGlob >= xMaxGlob"),
    ("corrL", (1, -1, 1), "corrL < 0d0"),
    ("corrMod", 7, "Correlation model not implemented"),
    ("margiFirst", 3, "First-order marginal not implemented"),
    ("std_dev", -1.0, "Standard deviation"),
    ("pointsPerCorrL", (5, 1, 5), "PointsPerCorrL < 2"),
])
def test_verify_inputs_rules(oracle, field, value, msg):
    kw = dict(xMinGlob=(0, 0, 0), xMaxGlob=(1, 1, 1), corrL=(1, 1, 1), overlap=(0, 0, 0),
              pointsPerCorrL=(5, 5, 5), corrMod=1, margiFirst=1, avg=1.0, std_dev=1.0)
    kw[field] = value
    s = S.make_sample(**kw)
    with pytest.raises(S.ScarlError) as e:
        S.verify_inputs(s)
    assert msg in str(e.value)
    rule = oracle.verify_inputs(kw["xMinGlob"], kw["xMaxGlob"], kw["corrL"], kw["overlap"],
                                kw["avg"], kw["std_dev"], kw["corrMod"], kw["margiFirst"],
                                kw["pointsPerCorrL"])
    assert rule != 0


def test_verify_inputs_lognormal_and_method():
    s = S.make_sample(margiFirst=2, avg=0.0)
    with pytest.raises(S.ScarlError, match="lognormal"):
        S.verify_inputs(s)
    with pytest.raises(S.ScarlError, match="Generation Method"):
        S.verify_inputs(S.make_sample(), gen_meth=3)
    S.verify_inputs(S.make_sample(corrMod=3))
    S.verify_inputs(S.make_sample(corrMod=2, nu=1.5))


def test_rebuild_corrL_matches_oracle(oracle):
    rng = np.random.default_rng(4)
    L = [12, 9, 16]
    sk = rng.random(sum(v // 2 for v in L))
    xs = [0.5, 1.0, 2.0]
    np.testing.assert_array_equal(S.rebuild_corrL(sk, L, xs),
                                  oracle.rebuild_corrL(sk, [v // 2 for v in L], xs))


@pytest.mark.parametrize("cm,nu", [(1, 0.5), (3, 0.5), (2, 0.3), (2, 1.5)])
def test_pad_size_auto_is_minimal(cm, nu):
    """AUTO picks the smallest power of two whose nearest periodic image of the
    farthest tile pair has correlation <= tol (checked against scipy)."""
    from scipy.special import gamma, kv

    def corr(l, r):
        if cm == 1:
            return np.exp(-np.pi * r * r / (l * l))
        v = 0.5 if cm == 3 else nu
        a = l * gamma(v) / (2 * np.sqrt(np.pi) * gamma(v + 0.5))
        x = r / a
        return 2 ** (1 - v) / gamma(v) * x ** v * kv(v, x)
    for Np, cl, dx in [((297, 277, 267), (40, 20, 10), (1, 1, 1)), ((50, 9, 120), (3, 7, 12), (0.5, 1, 2))]:
        for tol in (1e-2, 1e-3, 1e-6):
            P = S.pad_size(S.PAD_AUTO, cm, cl, dx, Np, nu, tol)
            for d in range(3):
                assert P[d] >= 8 and P[d] & (P[d] - 1) == 0 and P[d] >= Np[d]
                assert corr(cl[d], (P[d] - Np[d] + 1) * dx[d]) <= tol * (1 + 1e-9)
                if P[d] > 8 and P[d] // 2 >= Np[d]:
                    assert corr(cl[d], (P[d] // 2 - Np[d] + 1) * dx[d]) > tol
    full = S.pad_size(S.PAD_FULL, cm, (40, 20, 10), (1, 1, 1), (297, 277, 267))
    assert list(full) == [1024, 1024, 1024]


SMOOTH_LENGTHS = sorted({2 ** a for a in range(3, 12)} |
                        {m * 2 ** a for m in (3, 5, 7) for a in range(4, 10) if m * 2 ** a <= 2048})


@pytest.mark.parametrize("cm,nu", [(1, 0.5), (3, 0.5), (2, 0.8)])
def test_pad_size_smooth_is_minimal(cm, nu):
    """SMOOTH applies AUTO's rule over every supported length (powers of two
    and 3, 5, 7 times 2^a >= 16, up to 2048): the chosen length passes, every
    smaller supported length >= Np fails, and it is never above AUTO's."""
    for Np, cl, dx in [((297, 277, 267), (40, 20, 10), (1, 1, 1)), ((50, 9, 120), (3, 7, 12), (0.5, 1, 2)),
                       ((608, 608, 1024), (64, 64, 32), (1, 1, 1))]:
        for tol in (1e-2, 1e-3):
            P = S.pad_size(S.PAD_SMOOTH, cm, cl, dx, Np, nu, tol)
            A = S.pad_size(S.PAD_AUTO, cm, cl, dx, Np, nu, tol)
            for d in range(3):
                assert P[d] in SMOOTH_LENGTHS and P[d] >= Np[d] and P[d] <= A[d]
                ok = lambda p: S.axis_correlation(cm, cl[d], (p - Np[d] + 1) * dx[d], nu) <= tol
                assert ok(P[d])
                assert not any(ok(p) for p in SMOOTH_LENGTHS if Np[d] <= p < P[d])
    # the headline deck: 513^3 field, exponential l = (40, 20, 10), 2x2x2 tiles
    P = S.pad_size(S.PAD_SMOOTH, 3, (40, 20, 10), (1, 1, 1), (297, 277, 267), 0.5, 1e-3)
    assert list(P) == [448, 384, 320]


def test_ensemble_draw_matches_oracle(oracle):
    """Shapes and correlation lengths of ensemble realisations: library and
    oracle draw the same Philox words, bit-exact."""
    for seed, first, n in ((0, 0, 256), (12345, 1000, 64), (2 ** 40 + 3, 2 ** 33, 16)):
        Np, cl = S.ensemble_draw(seed, first, n)
        rNp, rcl = oracle.ensemble_draw(seed, first, n, S.ENSEMBLE_AXES, 4.0, 32.0)
        np.testing.assert_array_equal(Np, rNp)
        np.testing.assert_array_equal(cl, rcl)
    Np, cl = S.ensemble_draw(0, 0, 256)
    assert set(np.unique(Np)) <= set(S.ENSEMBLE_AXES) and len(np.unique(Np)) == 6
    assert np.all((cl >= 4) & (cl <= 32)) and np.all(cl[:, 0] == cl[:, 2])
    # the first realisations do not depend on how many are drawn
    np.testing.assert_array_equal(S.ensemble_draw(0, 0, 10)[0], Np[:10])
    np.testing.assert_array_equal(S.ensemble_draw(0, 5, 3)[0], Np[5:8])
