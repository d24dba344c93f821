"""Generate tests/golden/golden.npz: an independent numpy/scipy restatement of
the ScaRL routines on the generation path, at small sizes and fixed seeds.

It shares no code with the C oracle.  The transforms are scipy.fft.dctn(type=3)
(= FFTW REDFT01, unnormalised) and numpy.fft.ifftn * N (= FFTW BACKWARD,
unnormalised); Park-Miller is plain Python integers.  Paths cite the ScaRL
source tree.

    python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy.fft as sfft
from scipy.special import gamma as G

HERE = os.path.dirname(os.path.abspath(__file__))
PI_REF = 3.1415926535898  # SRC_F/constants_ScaRL.f90:5


# --- SRC_F/normal_ScaRL.f90:827-838 -----------------------------------------
def pm_uniforms(seed, n):
    s = int(seed)
    out = np.empty(n)
    for i in range(n):
        k = int(s / 127773)  # Fortran integer division truncates toward zero
        s = 16807 * (s - k * 127773) - k * 2836
        if s < 0:
            s += 2147483647
        out[i] = float(s) * 4.656612875e-10
    return out


# --- SRC_F/fftw_ScaRL.f90:261-418 (gen_std_gauss_FFT, Gaussian) --------------
def gen_std_gauss_fft(Np, xRange, corrL, phiK):
    K = [n // 2 for n in Np]
    Sk = np.zeros(Np, order="F")
    S = np.ones(K)
    for d in range(3):
        dx = xRange[d] / (Np[d] - 1)
        dk = (1.0 / dx) / (Np[d] - 1)
        kp = np.arange(K[d]) * dk / corrL[d]
        f = corrL[d] * np.exp(-PI_REF * kp * kp)
        shape = [1, 1, 1]
        shape[d] = K[d]
        S = S * f.reshape(shape)
    Sk[:K[0], :K[1], :K[2]] = np.sqrt(S) * np.cos(2.0 * PI_REF * phiK)
    return sfft.dctn(Sk, type=3)


# --- SRC_F/spectra_ScaRL.f90:10-142 + SRC_F/fftw_ScaRL.f90:157-255 ----------
def shino(Np, xRange, corrL, seed):
    sz_c, sz, dk = [], [], []
    for d in range(3):
        xr = xRange[d] / corrL[d]
        c = 2 ** int(np.ceil(np.log(2.0 * Np[d]) / np.log(2.0)))
        dx = xr / (Np[d] - 1)
        kmax = 1.0 / dx
        delta = kmax / (c // 2)
        kcut = min(7.355, kmax)
        sz_c.append(c)
        dk.append(delta)
        sz.append(min(int(np.ceil(kcut / delta)), c // 2))
    n1, n2, n3 = sz[0], 2 * sz[1], 2 * sz[2]
    u = pm_uniforms(np.int32(np.uint32(seed) + np.uint32(1000000)).item(), n1 * n2 * n3)
    ph = 2.0 * PI_REF * u.reshape((n1, n2, n3), order="F")
    Sk = (np.cos(ph).astype(np.float32).astype(np.float64)
          + 1j * np.sin(ph).astype(np.float32).astype(np.float64))
    Sk[0, :, :] = 0
    Sk[:, 0, :] = 0
    Sk[:, :, 0] = 0
    Sk[:, n2 - 1, :] = 0
    Sk[:, :, n3 - 1] = 0
    de = [(PI_REF ** 2 / 2.0) * (d * d) for d in dk]
    ii = np.arange(n1)[:, None, None].astype(float)
    jj = np.arange(n2)
    jm = np.where(jj < sz[1], jj, n2 - 1 - jj)[None, :, None].astype(float)
    kk = np.arange(n3)
    km = np.where(kk < sz[2], kk, n3 - 1 - kk)[None, None, :].astype(float)
    sv = np.sqrt(np.exp(-((ii * ii * de[0] + jm * jm * de[1]) + km * km * de[2])))
    Sk = Sk * sv
    Sk = np.sqrt(8.0) * Sk
    Sk = 2.0 * np.sqrt(dk[0] * dk[1] * dk[2]) * Sk
    c = np.zeros(sz_c, complex)
    cj = np.where(jj < sz[1], jj, sz_c[1] - n2 + jj)
    ck = np.where(kk < sz[2], kk, sz_c[2] - n3 + kk)
    c[np.ix_(np.arange(n1), cj, ck)] = Sk
    out = np.fft.ifftn(c) * np.prod(sz_c)
    return np.asfortranarray(out.real[:Np[0], :Np[1], :Np[2]])


# --- padded periodic method, normalised spectra (no reference counterpart) ---
def spectrum(corrMod, nu, corrL, f):
    if corrMod == 1:
        S = 1.0
        for d in range(3):
            S = S * corrL[d] * np.exp(-np.pi * corrL[d] ** 2 * f[d] ** 2)
        return S
    if corrMod == 3:
        nu = 0.5
    sc = G(nu) / (2 * np.sqrt(np.pi) * G(nu + 0.5))
    a = [c * sc for c in corrL]
    q = sum(4 * np.pi ** 2 * a[d] ** 2 * f[d] ** 2 for d in range(3))
    C = 8 * np.pi ** 1.5 * G(nu + 1.5) / G(nu) * a[0] * a[1] * a[2]
    return C * (1 + q) ** (-(nu + 1.5))


def padded(Np, P, dx, corrL, corrMod, nu, xi):
    Hx = P[0] // 2 + 1
    fr = []
    for d, n in enumerate([Hx, P[1], P[2]]):
        k = np.arange(n)
        s = np.where(2 * k <= P[d], k, k - P[d])
        fr.append(s / (P[d] * dx[d]))
    FX, FY, FZ = np.meshgrid(fr[0], fr[1], fr[2], indexing="ij")
    dk3 = np.prod([1.0 / (P[d] * dx[d]) for d in range(3)])
    S = spectrum(corrMod, nu, corrL, (FX, FY, FZ)) * dk3
    kx = np.arange(Hx)[:, None, None]
    c = np.where((kx == 0) | (2 * kx == P[0]), 1.0, 2.0)
    norm = np.sum(c * S)
    g = np.where((kx == 0) | (2 * kx == P[0]), 1.0, np.sqrt(0.5))
    A = np.sqrt(S / norm) * g
    H = A * (xi[..., 0] + 1j * xi[..., 1])
    # C2R: z, y complex inverse, then Hermitian inverse along x (irfft)
    field = np.fft.irfftn(H.transpose(2, 1, 0), s=(P[2], P[1], P[0]), axes=(0, 1, 2))
    field = field.transpose(2, 1, 0) * np.prod(P)
    return np.asfortranarray(field[:Np[0], :Np[1], :Np[2]]), norm


# --- SRC_F/main_ScaRL.f90:1236-1294 -------------------------------------------
def pou_weights(Np, No, pos, shape):
    w = np.ones(Np, order="F")
    for side in (0, 1):
        for ax in range(3):
            shift = -1 if side == 0 else 1
            if No[ax] < 2 or not (0 <= pos[ax] + shift <= shape[ax] - 1):
                continue
            p = np.arange(No[ax]) / (No[ax] - 1)
            if side == 0:
                p = p[::-1]
            p = (1.0 + np.cos(PI_REF * p)) / 2.0
            D = 0 if side == 0 else Np[ax] - No[ax]
            sl = [slice(None)] * 3
            for t in range(No[ax]):
                sl[ax] = D + t
                w[tuple(sl)] *= p[t]
    return w


def topo_pos(r, shape):
    z = r // (shape[0] * shape[1])
    r -= z * shape[0] * shape[1]
    y = r // shape[0]
    return [r - y * shape[0], y, z]


# --- SRC_F/main_ScaRL.f90:984-1210 over simulated ranks ----------------------
def add_overlap(RF, Np, No, shape):
    nb = len(RF)
    acc = [np.zeros(Np, order="F") for _ in range(nb)]
    for r in range(nb):
        pos = topo_pos(r, shape)
        for kk in (-1, 0, 1):
            for jj in (-1, 0, 1):
                for ii in (-1, 0, 1):
                    s = (ii, jj, kk)
                    if s == (0, 0, 0):
                        continue
                    src = [pos[d] - s[d] for d in range(3)]
                    if any(src[d] < 0 or src[d] > shape[d] - 1 for d in range(3)):
                        continue
                    rs, ss = [], []
                    ok = True
                    for d in range(3):
                        if s[d] == 1:
                            rs.append(slice(0, No[d])); ss.append(slice(Np[d] - No[d], Np[d]))
                            ok &= No[d] > 1
                        elif s[d] == -1:
                            rs.append(slice(Np[d] - No[d], Np[d])); ss.append(slice(0, No[d]))
                            ok &= No[d] > 1
                        else:
                            rs.append(slice(0, Np[d])); ss.append(slice(0, Np[d]))
                            ok &= Np[d] > 1
                    if not ok:
                        continue
                    R = src[0] + shape[0] * (src[1] + shape[1] * src[2])
                    acc[r][tuple(rs)] = acc[r][tuple(rs)] + RF[R][tuple(ss)]
    return [RF[r] + acc[r] for r in range(nb)]


# --- SRC_F/Stat_ScaRL/statistics_RF.f90:258-462 -------------------------------
def tukey_literal(n):
    r = float(np.float32(0.1))
    w = np.ones(n)
    for i in range(n):
        ratio = i / (n - 1)
        if ratio < r:
            w[i] = 0.5 * (1 + np.cos(2 * PI_REF / r * (ratio - r / 2)))
        elif ratio > r:
            w[i] = 0.5 * (1 + np.cos(2 * PI_REF / r * (ratio - 1 + r / 2)))
    return w


def rebuild_sk(f, d, avg, sd):
    n = f.shape[d]
    w = tukey_literal(n)
    shape = [1, 1, 1]
    shape[d] = n
    t = (f - avg) / sd * w.reshape(shape)
    X = np.fft.fft(t, axis=d) / n
    P = (X * np.conj(X)).real
    other = tuple(a for a in range(3) if a != d)
    m = P.mean(axis=other)
    return (np.fft.ifft(m) * n).real


def main():
    rng = np.random.default_rng(20240601)
    g = {}
    g["pm_12345"] = pm_uniforms(12345, 3)
    # DCT path
    for tag, Np, xs, cl in [("a", (16, 12, 10), (1.0, 1.0, 1.0), (4.0, 3.0, 2.0)),
                            ("b", (13, 9, 11), (0.5, 1.0, 2.0), (2.0, 5.0, 7.0))]:
        xr = [(n - 1) * s for n, s in zip(Np, xs)]
        phi = rng.random([n // 2 for n in Np])
        phi = np.asfortranarray(phi)
        g[f"dct_{tag}_Np"] = np.array(Np)
        g[f"dct_{tag}_xRange"] = np.array(xr)
        g[f"dct_{tag}_corrL"] = np.array(cl)
        g[f"dct_{tag}_phi"] = phi
        g[f"dct_{tag}_out"] = gen_std_gauss_fft(Np, xr, cl, phi)
    # Shino padded c2c path
    for tag, Np, xr, cl, seed in [("a", (20, 18, 16), (3.8, 3.4, 3.0), (1.0, 1.0, 1.0), 7),
                                  ("b", (12, 14, 10), (11.0, 13.0, 9.0), (1.0, 1.5, 0.8), 123)]:
        g[f"shino_{tag}_Np"] = np.array(Np)
        g[f"shino_{tag}_xRange"] = np.array(xr)
        g[f"shino_{tag}_corrL"] = np.array(cl)
        g[f"shino_{tag}_seed"] = np.array(seed)
        g[f"shino_{tag}_out"] = shino(Np, xr, cl, seed)
    # padded periodic method with injected normals
    for tag, Np, P, dx, cl, cm, nu in [("g", (12, 10, 9), (32, 32, 16), (1.0, 0.5, 1.0), (4.0, 3.0, 2.5), 1, 0.5),
                                       ("e", (10, 12, 8), (32, 32, 16), (1.0, 1.0, 2.0), (3.0, 5.0, 4.0), 3, 0.5),
                                       ("v", (9, 9, 14), (32, 16, 32), (1.0, 1.0, 1.0), (4.0, 2.0, 6.0), 2, 1.5)]:
        Hx = P[0] // 2 + 1
        xi = rng.standard_normal((Hx, P[1], P[2], 2))
        out, norm = padded(Np, P, dx, cl, cm, nu, xi)
        g[f"pad_{tag}_Np"] = np.array(Np)
        g[f"pad_{tag}_P"] = np.array(P)
        g[f"pad_{tag}_dx"] = np.array(dx)
        g[f"pad_{tag}_corrL"] = np.array(cl)
        g[f"pad_{tag}_cm"] = np.array(cm)
        g[f"pad_{tag}_nu"] = np.array(nu)
        # mode index kx fastest: pairs laid out (kz, ky, kx, 2) in C order
        g[f"pad_{tag}_xi"] = np.ascontiguousarray(xi.transpose(2, 1, 0, 3))
        g[f"pad_{tag}_norm"] = np.array(norm)
        g[f"pad_{tag}_out"] = out
    # partition of unity
    for tag, Np, No, pos, shape in [("a", (9, 8, 7), (4, 3, 2), (1, 0, 1), (3, 2, 2)),
                                    ("b", (6, 6, 6), (3, 1, 3), (0, 1, 1), (2, 2, 2))]:
        g[f"pou_{tag}_Np"] = np.array(Np)
        g[f"pou_{tag}_No"] = np.array(No)
        g[f"pou_{tag}_pos"] = np.array(pos)
        g[f"pou_{tag}_shape"] = np.array(shape)
        g[f"pou_{tag}_w"] = pou_weights(Np, No, pos, shape)
    # overlap add over simulated ranks
    for tag, Np, No, shape in [("a", (7, 6, 5), (3, 2, 2), (2, 2, 2)),
                               ("b", (6, 5, 5), (2, 1, 3), (3, 2, 1))]:
        nb = int(np.prod(shape))
        RF = [np.asfortranarray(rng.standard_normal(Np)) for _ in range(nb)]
        g[f"ovl_{tag}_Np"] = np.array(Np)
        g[f"ovl_{tag}_No"] = np.array(No)
        g[f"ovl_{tag}_shape"] = np.array(shape)
        g[f"ovl_{tag}_in"] = np.stack(RF)
        g[f"ovl_{tag}_out"] = np.stack(add_overlap(RF, Np, No, shape))
    # covariance estimator
    f = np.asfortranarray(rng.standard_normal((12, 10, 14)))
    avg, sd = f.mean(), f.std()
    g["sk_field"] = f
    g["sk_avg"] = np.array(avg)
    g["sk_sd"] = np.array(sd)
    for d in range(3):
        g[f"sk_dir{d}"] = rebuild_sk(f, d, avg, sd)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **g)
    print("wrote", os.path.join(HERE, "golden.npz"), len(g), "arrays")


if __name__ == "__main__":
    main()
