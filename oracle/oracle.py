"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Arrays follow the reference's column-major layout: a field of
shape (nx, ny, nz) is a numpy array in Fortran order.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build.build()
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_i32 = C.POINTER(C.c_int32)
_u32 = C.POINTER(C.c_uint32)


def _declare(L):
    L.so_pm_step.restype = C.c_int32
    L.so_pm_step.argtypes = [C.c_int32]
    L.so_r8vec_uniform_01.argtypes = [C.c_int, _i32, _d]
    L.so_r8vec_normal_01.argtypes = [C.c_int, _i32, _d]
    L.so_pm_jump.restype = C.c_int32
    L.so_pm_jump.argtypes = [C.c_int32, C.c_uint64]
    L.so_philox4x32_10.argtypes = [_u32, _u32, _u32]
    L.so_normals.argtypes = [C.c_uint64, C.c_uint32, _i, _d]
    L.so_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, _d]
    L.so_ensemble_draw.argtypes = [C.c_uint64, C.c_int64, C.c_int, _i, C.c_int, C.c_double,
                                   C.c_double, _i, _d]
    L.so_verify_inputs.restype = C.c_int
    L.so_verify_inputs.argtypes = [_d, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int, _i, C.c_int]
    L.so_find_factors.argtypes = [C.c_int, _i]
    L.so_decide_topo_shape.argtypes = [C.c_int, _i, _i, C.c_int64, _i]
    L.so_get_topo_pos.argtypes = [C.c_int, _i, _i]
    L.so_get_topo_rank.restype = C.c_int
    L.so_get_topo_rank.argtypes = [_i, _i]
    L.so_sample_layout.restype = C.c_int
    L.so_sample_layout.argtypes = [_d, _d, _d, _d, _i, C.c_int, C.c_int, _i, _i, _i, _i, _i, _d]
    L.so_tile_geometry.argtypes = [_i, _i, _i, _d, _d, _i, _i, _d, _d, _d]
    L.so_unity_partition_weights.argtypes = [_i, _i, C.c_int, _i, _i, _d]
    L.so_apply_unity_partition.argtypes = [_i, _i, C.c_int, _i, _i, _d]
    L.so_add_overlap.argtypes = [C.POINTER(_d), _i, _i, _i]
    L.so_normalize_field.argtypes = [C.POINTER(_d), _i, _i, _i, _d, _d]
    L.so_multivariate_transformation.restype = C.c_int
    L.so_multivariate_transformation.argtypes = [C.c_double, C.c_double, C.c_int, _d, C.c_int64]
    L.so_assemble_global.argtypes = [C.POINTER(_d), _i, _i, _i, _i, _d]
    L.so_fft1d.argtypes = [_d, C.c_int, C.c_int]
    L.so_dct3_1d.argtypes = [_d, _d, C.c_int]
    L.so_dct3_3d.argtypes = [_d, _d, _i]
    L.so_c2c_3d.argtypes = [_d, _i, C.c_int]
    L.so_c2r_3d_crop.argtypes = [_d, _i, _i, _d]
    L.so_gen_std_gauss_fft.argtypes = [_d, _i, _d, _d, _d, _d]
    L.so_gen_std_gauss_fft_mpi.argtypes = [_d, _i, _d, _d, _d, _d]
    L.so_padded_size_literal.restype = C.c_int
    L.so_padded_size_literal.argtypes = [C.c_int]
    L.so_shino_sizes.restype = C.c_int
    L.so_shino_sizes.argtypes = [_i, _d, _d, _i, _i, _d]
    L.so_build_sk_mtx.argtypes = [C.c_int32, _i, _d, _d]
    L.so_gen_std_gauss_shino_fft.argtypes = [_d, _i, _d, _d, C.c_int32, C.c_int]
    L.so_spectrum.restype = C.c_double
    L.so_spectrum.argtypes = [C.c_int, C.c_double, _d, _d]
    L.so_spectrum_sum.restype = C.c_double
    L.so_spectrum_sum.argtypes = [C.c_int, C.c_double, _i, _d, _d]
    L.so_padded_spectrum.argtypes = [C.c_int, C.c_double, _i, _d, _d, C.c_int, C.c_uint64,
                                     C.c_uint32, _d, _d]
    L.so_gen_padded.argtypes = [_d, _i, _i, _d, _d, C.c_int, C.c_double, C.c_int, C.c_uint64,
                                C.c_uint32, _d]
    L.so_gen_padded_stream.argtypes = [_d, _i, _i, _d, _d, C.c_int, C.c_double, C.c_double,
                                       C.c_uint64, C.c_uint32, C.c_int]
    L.so_generate_sample.restype = C.c_int
    L.so_generate_sample.argtypes = [C.c_int, _d, _d, _d, _d, _i, C.c_int, C.c_double, C.c_int,
                                     C.c_double, C.c_double, C.c_int, C.c_int, _i, _i, C.c_int,
                                     C.c_int, _d, _d]
    L.so_moments.argtypes = [_d, C.c_int64, C.c_int, _d, _d, _d, _d]
    L.so_tukey.argtypes = [C.c_int, C.c_int, _d]
    L.so_axis_cov.argtypes = [_d, _i, C.c_int, _d, _d]
    L.so_rebuild_sk_fft.argtypes = [_d, _i, C.c_int, C.c_double, C.c_double, C.c_int, _d]
    L.so_rebuild_corrL.argtypes = [_d, _i, _d, _d]


def _dp(a):
    return a.ctypes.data_as(_d)


def _ia(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    return a, a.ctypes.data_as(_i)


def _da(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
    return a, a.ctypes.data_as(_d)


# ---------------- random numbers ----------------
def pm_step(seed):
    return int(lib().so_pm_step(int(np.int32(seed))))


def r8vec_uniform_01(n, seed):
    s = C.c_int32(int(np.int32(seed)))
    r = np.empty(n)
    lib().so_r8vec_uniform_01(n, C.byref(s), _dp(r))
    return r, s.value


def r8vec_normal_01(n, seed):
    s = C.c_int32(int(np.int32(seed)))
    x = np.empty(max(n, 1))
    lib().so_r8vec_normal_01(n, C.byref(s), _dp(x))
    return x[:n], s.value


def pm_jump(state, n):
    return int(lib().so_pm_jump(int(state), int(n)))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) & 0xFFFFFFFF for v in key])
    o = (C.c_uint32 * 4)()
    lib().so_philox4x32_10(c, k, o)
    return [int(v) for v in o]


def normals(seed, stream, P):
    """Canonical normals of padded grid P as (P2, P1, P0/2+1, 2) in C order."""
    p, pp = _ia(P)
    Hx = int(P[0]) // 2 + 1
    out = np.empty((int(P[2]), int(P[1]), Hx, 2))
    lib().so_normals(seed, stream, pp, _dp(out))
    return out


def uniforms(seed, stream, first, n):
    out = np.empty(max(n, 1))
    lib().so_uniforms(seed, stream, first, n, _dp(out))
    return out[:n]


def ensemble_draw(seed, first, n, choices, lmin, lmax):
    ch = np.ascontiguousarray(choices, dtype=np.int32)
    Np = np.zeros((max(n, 1), 3), dtype=np.int32)
    cl = np.zeros((max(n, 1), 3))
    lib().so_ensemble_draw(seed, first, n, ch.ctypes.data_as(_i), len(ch), lmin, lmax,
                           Np.ctypes.data_as(_i), _dp(cl))
    return Np[:n], cl[:n]


# ---------------- index maps ----------------
def verify_inputs(xMin, xMax, corrL, overlap, avg, std_dev, corrMod, margiFirst, ppcl, gen_meth=1):
    a, pa = _da(xMin); b, pb = _da(xMax); c, pc = _da(corrL); o, po = _da(overlap)
    p, pp = _ia(ppcl)
    return lib().so_verify_inputs(pa, pb, pc, po, avg, std_dev, corrMod, margiFirst, pp, gen_meth)


def decide_topo_shape(nb_procs, L, ovlp, ppbi=1):
    l, pl = _ia(L); o, po = _ia(ovlp)
    t = np.zeros(3, np.int32)
    lib().so_decide_topo_shape(nb_procs, pl, po, ppbi, t.ctypes.data_as(_i))
    return t


def find_factors(n):
    d = np.zeros(100, np.int32)
    lib().so_find_factors(n, d.ctypes.data_as(_i))
    return [int(v) for v in d if v]


def get_topo_pos(rank, shape):
    s, ps = _ia(shape)
    p = np.zeros(3, np.int32)
    lib().so_get_topo_pos(rank, ps, p.ctypes.data_as(_i))
    return p


def sample_layout(xMin, xMax, corrL, overlap, ppcl, gen_meth=1, nb_procs=1, topo=None):
    a, pa = _da(xMin); b, pb = _da(xMax); c, pc = _da(corrL); o, po = _da(overlap)
    p, pp = _ia(ppcl)
    if topo is not None:
        t_in, pt_in = _ia(topo)
    else:
        pt_in = None
    L = np.zeros(3, np.int32); Np = np.zeros(3, np.int32); No = np.zeros(3, np.int32)
    T = np.zeros(3, np.int32); xs = np.zeros(3)
    rc = lib().so_sample_layout(pa, pb, pc, po, pp, gen_meth, nb_procs, pt_in,
                                L.ctypes.data_as(_i), Np.ctypes.data_as(_i), No.ctypes.data_as(_i),
                                T.ctypes.data_as(_i), _dp(xs))
    if rc:
        raise ValueError("topology does not match nb_procs")
    return dict(L=L, Np=Np, Np_ovlp=No, topo=T, xStep=xs)


def tile_geometry(Np, Np_ovlp, topo_pos, xStep, xMin):
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); t, pt = _ia(topo_pos)
    x, px = _da(xStep); m, pm = _da(xMin)
    p0 = np.zeros(3, np.int32); pN = np.zeros(3, np.int32)
    c0 = np.zeros(3); cN = np.zeros(3); xr = np.zeros(3)
    lib().so_tile_geometry(pn, po, pt, px, pm, p0.ctypes.data_as(_i), pN.ctypes.data_as(_i),
                           _dp(c0), _dp(cN), _dp(xr))
    return dict(pos_0=p0, pos_N=pN, coord_0=c0, coord_N=cN, xRange=xr)


# ---------------- post steps ----------------
def unity_partition_weights(Np, Np_ovlp, topo_pos, topo_shape, partitionType=1):
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); t, pt = _ia(topo_pos); s, ps = _ia(topo_shape)
    w = np.empty(tuple(int(v) for v in Np), order="F")
    lib().so_unity_partition_weights(pn, po, partitionType, pt, ps, _dp(w))
    return w


def apply_unity_partition(field, Np, Np_ovlp, topo_pos, topo_shape, partitionType=1):
    f = np.array(field, dtype=np.float64, order="F", copy=True)
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); t, pt = _ia(topo_pos); s, ps = _ia(topo_shape)
    lib().so_apply_unity_partition(pn, po, partitionType, pt, ps, _dp(f))
    return f


def add_overlap(fields, Np, Np_ovlp, topo_shape):
    fs = [np.asfortranarray(f, dtype=np.float64).copy(order="F") for f in fields]
    arr = (_d * len(fs))(*[_dp(f) for f in fs])
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); s, ps = _ia(topo_shape)
    lib().so_add_overlap(arr, pn, po, ps)
    return fs


def normalize_field(fields, Np, Np_ovlp, topo_shape):
    fs = [np.asfortranarray(f, dtype=np.float64).copy(order="F") for f in fields]
    arr = (_d * len(fs))(*[_dp(f) for f in fs])
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); s, ps = _ia(topo_shape)
    a = C.c_double(); sd = C.c_double()
    lib().so_normalize_field(arr, pn, po, ps, C.byref(a), C.byref(sd))
    return fs, a.value, sd.value


def multivariate_transformation(avg, std_dev, margiFirst, field):
    f = np.array(field, dtype=np.float64, order="F", copy=True)
    rc = lib().so_multivariate_transformation(avg, std_dev, margiFirst, _dp(f), f.size)
    if rc:
        raise ValueError("marginal transform rejected the inputs")
    return f


def assemble_global(fields, Np, Np_ovlp, topo_shape, L):
    fs = [np.asfortranarray(f, dtype=np.float64) for f in fields]
    arr = (_d * len(fs))(*[_dp(f) for f in fs])
    n, pn = _ia(Np); o, po = _ia(Np_ovlp); s, ps = _ia(topo_shape); l, pl = _ia(L)
    g = np.zeros(tuple(int(v) for v in L), order="F")
    lib().so_assemble_global(arr, pn, po, ps, pl, _dp(g))
    return g


# ---------------- transforms ----------------
def fft1d(x, sign):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).copy()
    lib().so_fft1d(a.view(np.float64).ctypes.data_as(_d), a.size, sign)
    return a


def dct3_1d(x):
    a = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(a)
    lib().so_dct3_1d(_dp(a), _dp(y), a.size)
    return y


def dct3_3d(x):
    a = np.asfortranarray(x, dtype=np.float64)
    y = np.empty_like(a, order="F")
    n, pn = _ia(a.shape)
    lib().so_dct3_3d(_dp(a), _dp(y), pn)
    return y


def c2c_3d(x, sign):
    a = np.array(x, dtype=np.complex128, order="F", copy=True)
    n, pn = _ia(a.shape)
    lib().so_c2c_3d(a.reshape(-1, order="F").view(np.float64).ctypes.data_as(_d) if False else
                    a.ctypes.data_as(_d), pn, sign)
    return a


def c2r_3d_crop(H, P, Nout):
    h = np.asfortranarray(H, dtype=np.complex128)
    p, pp = _ia(P); n, pn = _ia(Nout)
    out = np.empty(tuple(int(v) for v in Nout), order="F")
    lib().so_c2r_3d_crop(h.ctypes.data_as(_d), pp, pn, _dp(out))
    return out


# ---------------- generators ----------------
def gen_std_gauss_fft(Np, xRange, corrL, phiK, gammaK=None):
    n, pn = _ia(Np); x, px = _da(xRange); c, pc = _da(corrL)
    ph = np.asfortranarray(phiK, dtype=np.float64)
    g = None if gammaK is None else np.asfortranarray(gammaK, dtype=np.float64)
    out = np.empty(tuple(int(v) for v in Np), order="F")
    lib().so_gen_std_gauss_fft(_dp(out), pn, px, pc, _dp(ph), None if g is None else _dp(g))
    return out


def gen_std_gauss_fft_mpi(L, xRange, corrL, phiK, gammaK=None):
    n, pn = _ia(L); x, px = _da(xRange); c, pc = _da(corrL)
    ph = np.asfortranarray(phiK, dtype=np.float64)
    g = None if gammaK is None else np.asfortranarray(gammaK, dtype=np.float64)
    out = np.empty(tuple(int(v) for v in L), order="F")
    lib().so_gen_std_gauss_fft_mpi(_dp(out), pn, px, pc, _dp(ph), None if g is None else _dp(g))
    return out


def padded_size_literal(n):
    return int(lib().so_padded_size_literal(int(n)))


def shino_sizes(Np, xRange, corrL):
    n, pn = _ia(Np); x, px = _da(xRange); c, pc = _da(corrL)
    sc = np.zeros(3, np.int32); sz = np.zeros(3, np.int32); dk = np.zeros(3)
    cl = lib().so_shino_sizes(pn, px, pc, sc.ctypes.data_as(_i), sz.ctypes.data_as(_i), _dp(dk))
    return dict(sz_c=sc, sz_Sk=sz, delta_k=dk, clamped=bool(cl))


def build_sk_mtx(seed, sz_Sk, delta_k):
    s, ps = _ia(sz_Sk); d, pd = _da(delta_k)
    Sk = np.zeros((int(sz_Sk[0]), 2 * int(sz_Sk[1]), 2 * int(sz_Sk[2])), np.complex128, order="F")
    lib().so_build_sk_mtx(int(np.int32(seed)), ps, pd, Sk.ctypes.data_as(_d))
    return Sk


def gen_std_gauss_shino_fft(Np, xRange, corrL, seed, via_c2c=0):
    n, pn = _ia(Np); x, px = _da(xRange); c, pc = _da(corrL)
    out = np.empty(tuple(int(v) for v in Np), order="F")
    lib().so_gen_std_gauss_shino_fft(_dp(out), pn, px, pc, int(np.int32(seed)), via_c2c)
    return out


def spectrum(corrMod, nu, corrL, f):
    c, pc = _da(corrL); ff, pf = _da(f)
    return float(lib().so_spectrum(corrMod, nu, pc, pf))


def spectrum_sum(corrMod, nu, P, dx, corrL):
    p, pp = _ia(P); d, pd = _da(dx); c, pc = _da(corrL)
    return float(lib().so_spectrum_sum(corrMod, nu, pp, pd, pc))


def padded_spectrum(corrMod, nu, P, dx, corrL, normalise=1, seed=0, stream=0, xi=None):
    p, pp = _ia(P); d, pd = _da(dx); c, pc = _da(corrL)
    Hx = int(P[0]) // 2 + 1
    H = np.zeros((Hx, int(P[1]), int(P[2])), np.complex128, order="F")
    x = None if xi is None else np.ascontiguousarray(xi, dtype=np.float64)
    lib().so_padded_spectrum(corrMod, nu, pp, pd, pc, normalise, seed, stream,
                             None if x is None else _dp(x), H.ctypes.data_as(_d))
    return H


def gen_padded(Np, P, dx, corrL, corrMod, nu=0.5, normalise=1, seed=0, stream=0, xi=None):
    n, pn = _ia(Np); p, pp = _ia(P); d, pd = _da(dx); c, pc = _da(corrL)
    out = np.empty(tuple(int(v) for v in Np), order="F")
    x = None if xi is None else np.ascontiguousarray(xi, dtype=np.float64)
    lib().so_gen_padded(_dp(out), pn, pp, pd, pc, corrMod, nu, normalise, seed, stream,
                        None if x is None else _dp(x))
    return out


def gen_padded_stream(Np, P, dx, corrL, corrMod, nu=0.5, norm=None, seed=0, stream=0,
                      line_stride=1, out=None):
    n, pn = _ia(Np); p, pp = _ia(P); d, pd = _da(dx); c, pc = _da(corrL)
    if norm is None:
        norm = spectrum_sum(corrMod, nu, P, dx, corrL)
    if out is None:
        out = np.zeros(tuple(int(v) for v in Np), order="F")
    lib().so_gen_padded_stream(_dp(out), pn, pp, pd, pc, corrMod, nu, norm, seed, stream,
                               line_stride)
    return out


def generate_sample(generator, xMin, xMax, corrL, overlap, ppcl, corrMod=1, nu=0.5, margiFirst=1,
                    avg=0.0, std_dev=1.0, seedBase=0, nb_procs=1, topo=None, pad=None,
                    normalise_spectrum=1, normalize_field=0, phiK_all=None):
    lay = sample_layout(xMin, xMax, corrL, overlap, ppcl, 1, nb_procs, topo)
    a, pa = _da(xMin); b, pb = _da(xMax); c, pc = _da(corrL); o, po = _da(overlap)
    p, pp = _ia(ppcl)
    pt = _ia(topo)[1] if topo is not None else None
    if topo is not None:
        tkeep = _ia(topo)
        pt = tkeep[1]
    if pad is not None:
        padkeep = _ia(pad)
        ppad = padkeep[1]
    else:
        ppad = None
    ph = None if phiK_all is None else np.ascontiguousarray(phiK_all, dtype=np.float64)
    g = np.zeros(tuple(int(v) for v in lay["L"]), order="F")
    rc = lib().so_generate_sample(generator, pa, pb, pc, po, pp, corrMod, nu, margiFirst, avg,
                                  std_dev, seedBase, nb_procs, pt, ppad, normalise_spectrum,
                                  normalize_field, None if ph is None else _dp(ph), _dp(g))
    if rc:
        raise ValueError(f"generate_sample rejected the inputs (code {rc})")
    return g, lay


# ---------------- estimators ----------------
def moments(field2d):
    f = np.asfortranarray(field2d, dtype=np.float64)
    xN, nmc = f.shape
    ea = np.empty(nmc); es = np.empty(nmc); ga = C.c_double(); gs = C.c_double()
    lib().so_moments(_dp(f), xN, nmc, _dp(ea), _dp(es), C.byref(ga), C.byref(gs))
    return ea, es, ga.value, gs.value


def tukey(n, literal=1):
    w = np.empty(n)
    lib().so_tukey(n, literal, _dp(w))
    return w


def rebuild_sk_fft(field, dir, avg, stdDev, tukey_literal=1):
    f = np.asfortranarray(field, dtype=np.float64)
    L, pL = _ia(f.shape)
    Sk = np.empty(f.shape[dir])
    lib().so_rebuild_sk_fft(_dp(f), pL, dir, avg, stdDev, tukey_literal, _dp(Sk))
    return Sk


def rebuild_corrL(SkTot, nkeep, xStep):
    s = np.ascontiguousarray(SkTot, dtype=np.float64)
    n, pn = _ia(nkeep); x, px = _da(xStep)
    out = np.zeros(3)
    lib().so_rebuild_corrL(_dp(s), pn, px, _dp(out))
    return out


def axis_cov(f, maxlag):
    """Mean and (3, maxlag + 1) linear axis covariance of a Fortran-order field."""
    f = np.asfortranarray(f, dtype=np.float64)
    L, pL = _ia(f.shape)
    cov = np.zeros(3 * (maxlag + 1))
    m = C.c_double()
    lib().so_axis_cov(f.ctypes.data_as(_d), pL, int(maxlag), C.byref(m), _dp(cov))
    return m.value, cov.reshape(3, maxlag + 1)


# ---------------- padded grid policies ----------------
def _axis_correlation(corrMod, l, r):
    if r <= 0.0:
        return 1.0
    if corrMod == 1:
        return float(np.exp(-np.pi * r * r / (l * l)))
    if corrMod == 3:
        return float(np.exp(-2.0 * r / l))
    raise ValueError("closed-form axis correlation only for the Gaussian and exponential models")


def fft_length_supported(n):
    """Powers of two and 3, 5, 7 times a power of two >= 16, from 8 to 2048."""
    if n < 8 or n > 2048:
        return False
    m = n
    while m % 2 == 0:
        m //= 2
    return m == 1 or (m in (3, 5, 7) and n // m >= 16)


def pad_size(policy, corrMod, corrL, xStep, Np, tol=1e-3):
    """Padded grid per axis.  policy 0: 2^ceil(log2 2 Np) (SRC_F/fftw_ScaRL.f90:194);
    1: smallest power of two P >= Np with C((P - Np + 1) dx) <= tol; 3: the
    same rule over every supported length.  Gaussian and exponential models."""
    P = []
    for d in range(3):
        n, l, dx = int(Np[d]), float(corrL[d]), float(xStep[d])
        p = 8
        if policy == 0:
            while p < 2 * n:
                p <<= 1
        elif policy == 1:
            while p < n or _axis_correlation(corrMod, l, (p - n + 1) * dx) > tol:
                p <<= 1
        elif policy == 3:
            p = max(n, 8)
            while not fft_length_supported(p) or _axis_correlation(corrMod, l, (p - n + 1) * dx) > tol:
                p += 1
                if p > 2048:
                    raise ValueError("beyond the largest supported length")
        else:
            raise ValueError("unknown padding policy")
        P.append(p)
    return P
