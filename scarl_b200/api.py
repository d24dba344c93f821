"""Python front end of scarl_b200, named after the ScaRL routines it replaces.

Every numerical routine calls the CUDA library through the C ABI; host-side
routines (index maps, decks) call its C++ host code.  Fields are numpy arrays
in Fortran (column-major) order of shape (nx, ny, nz), or torch CUDA tensors
whose memory already holds that layout (pass `out=` to write in place).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import (CM_EXPONENTIAL, F32, F64, GEN_DCT, GEN_PADDED, GEN_SHINO, PAD_AUTO, PAD_FULL,
                   GenOpts, Layout,
                   Sample, ScarlError, Tile, lib)


def _check(rc, ctx=None):
    if rc != _lib.OK:
        msg = lib().scarl_last_error(ctx.handle if ctx is not None else None)
        raise ScarlError(rc, msg.decode() if msg else "")


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _np_dtype(dtype):
    return np.float64 if (dtype & 0xFF) == F64 else np.float32


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor."""
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class Context:
    """A scarl_ctx: one GPU, one CUDA stream, owned device workspace."""

    def __init__(self, device=0, budget_bytes=0):
        h = C.c_void_p()
        rc = lib().scarl_ctx_create(int(device), int(budget_bytes), C.byref(h))
        if rc != _lib.OK:
            raise ScarlError(rc, "scarl_ctx_create failed (is a GPU visible?)")
        self.handle = h

    def close(self):
        if self.handle:
            lib().scarl_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _check(lib().scarl_ctx_set_stream(self.handle, C.c_void_p(int(stream_ptr or 0))), self)

    def sync(self):
        _check(lib().scarl_sync(self.handle), self)

    def tc_wait_test(self, enable=True):
        """Test hook: the tensor-core pass's waits run out (SCARL_ETIMEOUT)."""
        _check(lib().scarl_tc_wait_test(self.handle, int(bool(enable))), self)

    def profile(self, enable=True):
        _check(lib().scarl_profile(self.handle, int(enable)), self)

    def profile_reset(self):
        _check(lib().scarl_profile(self.handle, 2), self)

    def autotune(self, dtype, corrMod, P, Np, xStep, corrL, nu=0.5, cache_path=None):
        _check(lib().scarl_autotune(self.handle, dtype, corrMod, nu, _i3(P), _i3(Np), _d3(xStep),
                                    _d3(corrL), cache_path.encode() if cache_path else None), self)

    def tune_get(self, dtype, pass_, N):
        v = C.c_int()
        _check(lib().scarl_tune_get(self.handle, dtype, pass_, N, C.byref(v)), self)
        return v.value

    def tune_set(self, dtype, pass_, N, variant):
        _check(lib().scarl_tune_set(self.handle, dtype, pass_, N, variant), self)

    def counters(self):
        n = C.c_longlong(); h = C.c_ulonglong(); d = C.c_ulonglong()
        _check(lib().scarl_counters(self.handle, C.byref(n), C.byref(h), C.byref(d)), self)
        return dict(launches=n.value, h2d_bytes=h.value, d2h_bytes=d.value)

    def profile_stats(self):
        out = {}
        i = 0
        name = C.create_string_buffer(128)
        ms = C.c_double()
        n = C.c_longlong()
        while lib().scarl_profile_read(self.handle, i, name, 128, C.byref(ms), C.byref(n)) == _lib.OK:
            out[name.value.decode()] = (ms.value, n.value)
            i += 1
        return out


# ---------------------------------------------------------------------------
# Samples and index maps (host)
# ---------------------------------------------------------------------------
def make_sample(xMinGlob=(0, 0, 0), xMaxGlob=(1, 1, 1), corrL=(1, 1, 1), overlap=(0, 0, 0),
                pointsPerCorrL=(5, 5, 5), corrMod=1, margiFirst=1, avg=0.0, std_dev=1.0,
                seedBase=0, nu=0.5, name="sample"):
    s = Sample()
    s.name = name.encode()[:255]
    s.xMinGlob = _d3(xMinGlob)
    s.xMaxGlob = _d3(xMaxGlob)
    s.corrL = _d3(corrL)
    s.overlap = _d3(overlap)
    s.pointsPerCorrL = _i3(pointsPerCorrL)
    s.corrMod, s.margiFirst = int(corrMod), int(margiFirst)
    s.avg, s.std_dev, s.seedBase, s.nu = float(avg), float(std_dev), int(seedBase), float(nu)
    return s


def sample_dict(s):
    return dict(name=s.name.decode(), xMinGlob=list(s.xMinGlob), xMaxGlob=list(s.xMaxGlob),
                corrL=list(s.corrL), overlap=list(s.overlap),
                pointsPerCorrL=list(s.pointsPerCorrL), corrMod=s.corrMod,
                margiFirst=s.margiFirst, avg=s.avg, std_dev=s.std_dev, seedBase=s.seedBase,
                nu=s.nu)


def verify_inputs(sample, gen_meth=1):
    """SRC_F/main_ScaRL.f90:271-340; raises ScarlError(SCARL_EINVAL) with the
    reference's message."""
    msg = C.create_string_buffer(256)
    rc = lib().scarl_verify_inputs(C.byref(sample), gen_meth, msg, 256)
    if rc != _lib.OK:
        raise ScarlError(rc, msg.value.decode())


def decide_topo_shape(nb_procs, L, Np_ovlp, pointsPerBlockIdeal=1):
    t = (C.c_int * 3)()
    _check(lib().scarl_decide_topo_shape(nb_procs, _i3(L), _i3(Np_ovlp), pointsPerBlockIdeal, t))
    return np.array(t[:], dtype=np.int32)


def get_topo_pos(rank, topo_shape):
    p = (C.c_int * 3)()
    _check(lib().scarl_get_topo_pos(rank, _i3(topo_shape), p))
    return np.array(p[:], dtype=np.int32)


def get_topo_rank(topo_shape, topo_pos):
    return int(lib().scarl_get_topo_rank(_i3(topo_shape), _i3(topo_pos)))


def _layout_dict(lay):
    return dict(L=np.array(lay.L[:], np.int32), Np=np.array(lay.Np[:], np.int32),
                Np_ovlp=np.array(lay.Np_ovlp[:], np.int32),
                topo=np.array(lay.topo_shape[:], np.int32), nb_tiles=lay.nb_tiles,
                xStep=np.array(lay.xStep[:]))


def sample_layout(sample, gen_meth=1, nb_procs=1, topo=None):
    lay = Layout()
    rc = lib().scarl_sample_layout(C.byref(sample), gen_meth, nb_procs,
                                   _i3(topo) if topo is not None else None, C.byref(lay))
    _check(rc)
    return _layout_dict(lay)


def tile_geometry(layout, xMinGlob, rank):
    lay = Layout()
    lay.L = _i3(layout["L"]); lay.Np = _i3(layout["Np"]); lay.Np_ovlp = _i3(layout["Np_ovlp"])
    lay.topo_shape = _i3(layout["topo"]); lay.nb_tiles = int(layout["nb_tiles"])
    lay.xStep = _d3(layout["xStep"])
    t = Tile()
    _check(lib().scarl_tile_geometry(C.byref(lay), _d3(xMinGlob), rank, C.byref(t)))
    return dict(topo_pos=np.array(t.topo_pos[:], np.int32), pos_0=np.array(t.pos_0[:], np.int32),
                pos_N=np.array(t.pos_N[:], np.int32), coord_0=np.array(t.coord_0[:]),
                coord_N=np.array(t.coord_N[:]), xRange=np.array(t.xRange[:]))


def unity_partition_weights(Np, Np_ovlp, topo_pos, topo_shape, partitionType=1):
    w = np.empty(tuple(int(v) for v in Np), order="F")
    _check(lib().scarl_unity_partition_weights(_i3(Np), _i3(Np_ovlp), partitionType,
                                               _i3(topo_pos), _i3(topo_shape),
                                               w.ctypes.data_as(C.POINTER(C.c_double))))
    return w


def shino_sizes(Np, xRange, corrL):
    sc = (C.c_int * 3)(); sz = (C.c_int * 3)(); dk = (C.c_double * 3)()
    _check(lib().scarl_shino_sizes(_i3(Np), _d3(xRange), _d3(corrL), sc, sz, dk))
    return dict(sz_c=np.array(sc[:]), sz_Sk=np.array(sz[:]), delta_k=np.array(dk[:]))


# ---------------------------------------------------------------------------
# Decks (host)
# ---------------------------------------------------------------------------
def read_config_ScaRL(path):
    v = [C.c_int() for _ in range(5)]
    buf = C.create_string_buffer(1024)
    _check(lib().scarl_read_config(str(path).encode(), *[C.byref(x) for x in v], buf, 1024))
    return dict(gen_meth=v[0].value, c_info_file=bool(v[1].value), d_sample=bool(v[2].value),
                one_file=bool(v[3].value), one_hdf_ds=bool(v[4].value),
                input_file=buf.value.decode())


def read_extra_config_ScaRL(path):
    found = C.c_int()
    t = (C.c_int * 3)()
    _check(lib().scarl_read_extra_config(str(path).encode(), C.byref(found), t))
    return bool(found.value), np.array(t[:], np.int32)


def _read_samples(fn, arg):
    folder = C.create_string_buffer(1024)
    n = C.c_int()
    _check(fn(arg, folder, 1024, C.byref(n), None, 0))
    arr = (Sample * max(n.value, 1))()
    _check(fn(arg, folder, 1024, C.byref(n), arr, n.value))
    return folder.value.decode(), [arr[i] for i in range(n.value)]


def read_input_ScaRL(path):
    return _read_samples(lib().scarl_read_input, str(path).encode())


def read_input_SEM(folder):
    return _read_samples(lib().scarl_read_input_sem, str(folder).encode())


# ---------------------------------------------------------------------------
# Generation (GPU)
# ---------------------------------------------------------------------------
def _alloc_out(out, shape, dtype):
    if out is not None:
        return out
    return np.empty(shape, dtype=_np_dtype(dtype), order="F")


def gen_std_gauss_FFT(ctx, Np, xRange, corrL, corrMod=1, seed=0, rank=0, phiK=None,
                      gammaK=None, out=None):
    """Drop-in for gen_std_gauss_FFT (SRC_F/fftw_ScaRL.f90:261-418), FP64."""
    out = _alloc_out(out, tuple(int(v) for v in Np), F64)
    ph = None if phiK is None else np.asfortranarray(phiK, dtype=np.float64)
    ga = None if gammaK is None else np.asfortranarray(gammaK, dtype=np.float64)
    _check(lib().scarl_gen_std_gauss_fft(ctx.handle, _ptr(out), _i3(Np), _d3(xRange), _d3(corrL),
                                         corrMod, seed, rank,
                                         None if ph is None else _ptr(ph),
                                         None if ga is None else _ptr(ga)), ctx)
    return out


def gen_std_gauss_FFT_MPI(ctx, xRange, corrL, corrMod=1, seed=0, rank=0, L=None, Np=None,
                          phiK=None, gammaK=None, out=None):
    """Drop-in for gen_Std_Gauss_FFT_MPI (SRC_F/fftw_ScaRL.f90:424-583) on one
    GPU: global DCT-III over L (Np == L), FP64."""
    L = tuple(int(v) for v in L)
    Np = L if Np is None else tuple(int(v) for v in Np)
    out = _alloc_out(out, L, F64)
    ph = None if phiK is None else np.asfortranarray(phiK, dtype=np.float64)
    ga = None if gammaK is None else np.asfortranarray(gammaK, dtype=np.float64)
    _check(lib().scarl_gen_std_gauss_fft_mpi(ctx.handle, _ptr(out), _d3(xRange), _d3(corrL),
                                             corrMod, seed, rank, _i3(L), _i3(Np),
                                             None if ph is None else _ptr(ph),
                                             None if ga is None else _ptr(ga)), ctx)
    return out


def gen_std_gauss_Shino_FFT(ctx, Np, xRange, corrL, pointsPerCorrL=(5, 5, 5), corrMod=1, seed=0,
                            rank=0, out=None):
    """Drop-in for gen_std_gauss_Shino_FFT (SRC_F/fftw_ScaRL.f90:157-255), FP64."""
    out = _alloc_out(out, tuple(int(v) for v in Np), F64)
    _check(lib().scarl_gen_std_gauss_shino_fft(ctx.handle, _ptr(out), _i3(Np), _d3(xRange),
                                               _d3(corrL), _i3(pointsPerCorrL), corrMod, seed,
                                               rank), ctx)
    return out


def gen_padded(ctx, Np, xStep, corrL, corrMod=1, nu=0.5, pad=None, normalise=True, seed=0,
               stream=0, xi=None, dtype=F32, out=None):
    """One tile of the padded periodic method (no blending)."""
    out = _alloc_out(out, tuple(int(v) for v in Np), dtype)
    x = None
    if xi is not None:
        x = xi if hasattr(xi, "data_ptr") else np.ascontiguousarray(xi, dtype=_np_dtype(dtype))
    _check(lib().scarl_gen_padded(ctx.handle, _ptr(out), dtype, _i3(Np),
                                  _i3(pad) if pad is not None else None, _d3(xStep), _d3(corrL),
                                  corrMod, float(nu), int(bool(normalise)), int(seed),
                                  int(stream), None if x is None else _ptr(x)), ctx)
    return out


ENS_AUTOTUNE = 1
ENS_NO_GRAPH = 2
ENSEMBLE_AXES = (64, 96, 128, 160, 192, 256)


def ensemble_draw(seed, first, n, choices=ENSEMBLE_AXES, lmin=4.0, lmax=32.0):
    """Shapes (n, 3) and isotropic correlation lengths (n, 3) of realisations
    first..first+n-1 (Philox4x32-10 at counter {r, r >> 32, 0, 2})."""
    ch = np.ascontiguousarray(choices, dtype=np.int32)
    Np = np.zeros((max(n, 1), 3), dtype=np.int32)
    cl = np.zeros((max(n, 1), 3))
    _check(lib().scarl_ensemble_draw(int(seed), int(first), int(n),
                                     ch.ctypes.data_as(C.POINTER(C.c_int)), len(ch), float(lmin),
                                     float(lmax), Np.ctypes.data_as(C.POINTER(C.c_int)),
                                     cl.ctypes.data_as(C.POINTER(C.c_double))))
    return Np[:n], cl[:n]


def ensemble_offsets(Np):
    """First element of each realisation's field in the packed output."""
    sizes = np.prod(np.asarray(Np, dtype=np.int64).reshape(-1, 3), axis=1)
    return np.concatenate([[0], np.cumsum(sizes)])


def ensemble_fields(out, Np):
    """Views of the packed ensemble output, one Fortran-order array each."""
    off = ensemble_offsets(Np)
    Np = np.asarray(Np).reshape(-1, 3)
    return [out[off[i]:off[i + 1]].reshape(tuple(int(v) for v in Np[i]), order="F")
            for i in range(len(Np))]


def gen_ensemble(ctx, Np, corrL, xStep=None, corrMod=CM_EXPONENTIAL, nu=0.5, pad_policy=PAD_AUTO,
                 pad_tol=1e-3, seeds=None, streams=None, dtype=F32, margiFirst=0, avg=0.0,
                 std_dev=1.0, autotune=False, graph=True, out=None):
    """n independent realisations of uneven grids in batched launches (one
    CUDA graph).  Returns the packed output (realisation i at
    ensemble_offsets(Np)[i], column-major)."""
    Np = np.ascontiguousarray(np.asarray(Np, dtype=np.int32).reshape(-1, 3))
    n = Np.shape[0]
    cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(n, 3))
    dx = np.ones((n, 3)) if xStep is None else np.broadcast_to(
        np.asarray(xStep, dtype=np.float64), (n, 3))
    dx = np.ascontiguousarray(dx, dtype=np.float64)
    total = int(ensemble_offsets(Np)[-1])
    if out is None:
        out = np.empty(total, dtype=_np_dtype(dtype))
    sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.uint64)
    st = None if streams is None else np.ascontiguousarray(streams, dtype=np.uint32)
    flags = (ENS_AUTOTUNE if autotune else 0) | (0 if graph else ENS_NO_GRAPH)
    _check(lib().scarl_gen_ensemble(
        ctx.handle, _ptr(out), dtype, n, Np.ctypes.data_as(C.POINTER(C.c_int)),
        dx.ctypes.data_as(C.POINTER(C.c_double)), cl.ctypes.data_as(C.POINTER(C.c_double)),
        corrMod, float(nu), int(pad_policy), float(pad_tol),
        None if sd is None else sd.ctypes.data_as(C.POINTER(C.c_uint64)),
        None if st is None else st.ctypes.data_as(C.POINTER(C.c_uint32)),
        int(margiFirst), float(avg), float(std_dev), flags), ctx)
    return out


def pad_size(policy, corrMod, corrL, xStep, Np, nu=0.5, tol=1e-3):
    P = (C.c_int * 3)()
    _check(lib().scarl_pad_size(policy, corrMod, nu, _d3(corrL), _d3(xStep), _i3(Np), tol, P))
    return np.array(P[:], dtype=np.int32)


def axis_correlation(corrMod, l, r, nu=0.5):
    return float(lib().scarl_axis_correlation(corrMod, nu, l, r))


def generate_sample(ctx, sample, generator=GEN_PADDED, dtype=F32, nb_procs=1, topo=None,
                    pad=None, pad_policy=PAD_FULL, pad_tol=1e-3, normalise_spectrum=True,
                    normalize_field=False, stream=0, phiK=None, autotune=False, out=None,
                    gen_meth=1, moments=None):
    """One deck sample end to end (layout, tiles, PoU blend, marginal).
    gen_meth 2 (FFT_MPI): the whole re-fitted grid as one global transform.
    moments: a float64 array of 2 that receives sum f and sum f^2 over the
    output field, accumulated inside the C2R pass."""
    lay = sample_layout(sample, gen_meth, nb_procs, topo)
    out = _alloc_out(out, tuple(int(v) for v in lay["L"]), dtype)
    o = GenOpts()
    o.generator, o.dtype, o.nb_procs = generator, dtype, nb_procs
    if topo is not None:
        o.topo_shape = _i3(topo)
    if pad is not None:
        o.pad = _i3(pad)
    o.pad_policy, o.pad_tol = int(pad_policy), float(pad_tol)
    o.no_spectral_normalisation = 0 if normalise_spectrum else 1
    o.normalize_field = int(bool(normalize_field))
    o.stream = int(stream)
    o.autotune = int(bool(autotune))
    o.gen_meth = int(gen_meth)
    keep = None
    if phiK is not None:
        keep = np.ascontiguousarray(phiK, dtype=np.float64)
        o.phiK = keep.ctypes.data_as(C.POINTER(C.c_double))
    if moments is not None:
        assert moments.dtype == np.float64 and moments.size >= 2 and moments.flags.c_contiguous
        o.moments = moments.ctypes.data_as(C.POINTER(C.c_double))
    _check(lib().scarl_generate_sample(ctx.handle, C.byref(sample), C.byref(o), _ptr(out)), ctx)
    return out, lay


# ---------------------------------------------------------------------------
# Post steps (GPU)
# ---------------------------------------------------------------------------
def apply_UnityPartition_mtx(ctx, field, Np, Np_ovlp, partitionType, topo_pos, topo_shape):
    """In place on an FP64 tile (SRC_F/main_ScaRL.f90:1216-1301)."""
    _check(lib().scarl_apply_unity_partition(ctx.handle, _ptr(field), _i3(Np), _i3(Np_ovlp),
                                             partitionType, _i3(topo_pos), _i3(topo_shape)), ctx)
    return field


def add_overlap(ctx, tiles, Np, Np_ovlp, topo_shape):
    """In place on nb consecutive FP64 tiles (SRC_F/main_ScaRL.f90:984-1210)."""
    _check(lib().scarl_add_overlap(ctx.handle, _ptr(tiles), _i3(Np), _i3(Np_ovlp),
                                   _i3(topo_shape)), ctx)
    return tiles


def multiVariateTransformation(ctx, avg, std_dev, margiFirst, field):
    dtype = F32 if field.dtype in (np.float32,) or str(field.dtype).endswith("float32") else F64
    _check(lib().scarl_multivariate_transformation(ctx.handle, _ptr(field), dtype,
                                                   _numel(field), avg, std_dev, margiFirst), ctx)
    return field


def _numel(a):
    return int(a.numel()) if hasattr(a, "numel") else int(a.size)


def _dtype_of(a):
    return F32 if str(a.dtype).endswith("float32") else F64


def normalize_field(ctx, field):
    a = C.c_double(); s = C.c_double()
    _check(lib().scarl_normalize_field(ctx.handle, _ptr(field), _dtype_of(field), _numel(field),
                                       C.byref(a), C.byref(s)), ctx)
    return a.value, s.value


# ---------------------------------------------------------------------------
# Estimators (GPU, FP64 accumulation)
# ---------------------------------------------------------------------------
def calculate_average_and_stdVar(ctx, field, Nmc=1):
    """calculate_average_and_stdVar_MPI (statistics_RF.f90:18-174) for a field
    of xNTotal * Nmc values (realisation-major)."""
    xN = _numel(field) // Nmc
    ea = np.empty(Nmc); es = np.empty(Nmc); ga = C.c_double(); gs = C.c_double()
    _check(lib().scarl_moments(ctx.handle, _ptr(field), _dtype_of(field), xN, Nmc,
                               ea.ctypes.data_as(C.POINTER(C.c_double)),
                               es.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ga),
                               C.byref(gs)), ctx)
    return ea, es, ga.value, gs.value


def rebuild_Sk(ctx, field, L, avg, stdDev, tukey_literal=True):
    """rebuild_Sk_FFT + rebuild_Sk (statistics_RF.f90:180-462): the kept lags
    of the three directional covariances, concatenated."""
    n = sum(int(v) // 2 for v in L)
    out = np.empty(n)
    _check(lib().scarl_rebuild_sk(ctx.handle, _ptr(field), _dtype_of(field), _i3(L), avg, stdDev,
                                  int(bool(tukey_literal)),
                                  out.ctypes.data_as(C.POINTER(C.c_double))), ctx)
    return out


def axis_cov(ctx, field, L, maxlag, known_mean=None, sums=None):
    """Mean, variance and covariance (3, maxlag + 1) along each axis of one
    field (numpy array or device tensor, column-major L), FP64 sums; the
    lag products are centred by known_mean when given, else the sample mean.
    sums: (sum f, sum f^2) streamed from generate_sample(moments=...), which
    spares the moment pass (known_mean must then be None)."""
    L = [int(v) for v in L]
    cov = np.zeros(3 * (maxlag + 1))
    m, v = C.c_double(), C.c_double()
    if sums is not None:
        assert known_mean is None
        sm = np.ascontiguousarray(sums, dtype=np.float64)
        _check(lib().scarl_axis_cov_sums(ctx.handle, _ptr(field), _dtype_of(field), _i3(L), int(maxlag),
                                         sm.ctypes.data_as(C.POINTER(C.c_double)), C.byref(m), C.byref(v),
                                         cov.ctypes.data_as(C.POINTER(C.c_double))), ctx)
        return m.value, v.value, cov.reshape(3, maxlag + 1)
    km = None if known_mean is None else C.byref(C.c_double(float(known_mean)))
    _check(lib().scarl_axis_cov(ctx.handle, _ptr(field), _dtype_of(field), _i3(L), int(maxlag),
                                km, C.byref(m), C.byref(v),
                                cov.ctypes.data_as(C.POINTER(C.c_double))), ctx)
    return m.value, v.value, cov.reshape(3, maxlag + 1)


# ---------------------------------------------------------------------------
# Output files (HDF5 + XDMF, self-written classic-format encoder)
# ---------------------------------------------------------------------------
def _layout_struct(layout):
    lay = Layout()
    lay.L = _i3(layout["L"])
    lay.Np = _i3(layout["Np"])
    lay.Np_ovlp = _i3(layout["Np_ovlp"])
    lay.topo_shape = _i3(layout["topo"])
    lay.nb_tiles = int(layout["nb_tiles"])
    lay.xStep = _d3(layout["xStep"])
    return lay


def write_sample_h5(ctx, folder, output_name, field, sample, layout, one_file=True,
                    one_hdf_ds=True, times=None, time_labels=None):
    """HDF5 + XDMF files of one generated field (write_hdf5_multi_proc_3D_1ds,
    write_hdf5_multi_proc_3D or write_hdf5_single_proc_3D by one_file /
    one_hdf_ds).  field: the column-major global field (numpy or device
    tensor); ctx may be None for host fields."""
    lay = _layout_struct(layout)
    nt = 0 if times is None else len(times)
    tv = None if times is None else np.ascontiguousarray(times, dtype=np.float64)
    lab = None
    if nt:
        labels = list(time_labels or [""] * nt)
        lab = "".join(str(x)[:20].ljust(20) for x in labels).encode()
    f = field if hasattr(field, "data_ptr") else np.asfortranarray(field)
    _check(lib().scarl_write_sample_h5(None if ctx is None else ctx.handle, str(folder).encode(),
                                       str(output_name).encode(), _ptr(f), _dtype_of(f),
                                       C.byref(sample), C.byref(lay), int(bool(one_file)),
                                       int(bool(one_hdf_ds)), lab,
                                       None if tv is None else tv.ctypes.data_as(C.POINTER(C.c_double)),
                                       nt), ctx)


def write_constant_field_h5(folder, output_name, xMinGlob, xMaxGlob, avg):
    """write_constant_field: the file of a sample with std_dev = 0."""
    _check(lib().scarl_write_constant_field_h5(str(folder).encode(), str(output_name).encode(),
                                               _d3(xMinGlob), _d3(xMaxGlob), float(avg)))


def stat_file(ctx, res_path, dset_name="samples", calculate_corrL=True):
    """Stat_ScaRL's step for one result file on the GPU: FP64 moments, with
    calculate_corrL the spectra and correlation lengths written back to the
    file; always writes STAT_<file> beside it.  Returns (avg, std, corrL)."""
    a, s = C.c_double(), C.c_double()
    cl = (C.c_double * 3)()
    _check(lib().scarl_stat_file(ctx.handle, str(res_path).encode(), dset_name.encode(),
                                 int(bool(calculate_corrL)), C.byref(a), C.byref(s), cl), ctx)
    return a.value, s.value, np.array(cl[:]) if calculate_corrL else None


def _h5_check(rc, msg):
    if rc != _lib.OK:
        raise ScarlError(rc, msg.value.decode(errors="replace"))


def h5_list(path):
    buf = C.create_string_buffer(1 << 16)
    msg = C.create_string_buffer(512)
    _h5_check(lib().scarl_h5_list(str(path).encode(), buf, len(buf), msg, len(msg)), msg)
    return [n for n in buf.value.decode().split("\n") if n]


def h5_overwrite_dataset(path, name, data):
    """Overwrites a dataset's raw bytes in place (same size)."""
    a = np.ascontiguousarray(data)
    msg = C.create_string_buffer(512)
    _h5_check(lib().scarl_h5_overwrite_dataset(str(path).encode(), name.encode(),
                                               C.c_void_p(a.ctypes.data), a.nbytes, msg, len(msg)),
              msg)


def h5_read_dataset(path, name, dtype=F64):
    """A numeric dataset as a column-major numpy array (HDF5 dims reversed)."""
    dims = (C.c_longlong * 3)()
    rank = C.c_int()
    msg = C.create_string_buffer(512)
    _h5_check(lib().scarl_h5_read_dataset(str(path).encode(), name.encode(), None, dtype, dims,
                                          C.byref(rank), msg, len(msg)), msg)
    shape = tuple(int(d) for d in dims[:max(rank.value, 1)])
    out = np.empty(shape, dtype=_np_dtype(dtype), order="F")
    _h5_check(lib().scarl_h5_read_dataset(str(path).encode(), name.encode(), _ptr(out), dtype, dims,
                                          C.byref(rank), msg, len(msg)), msg)
    return out


def h5_read_attr(path, name, obj=None):
    """A numeric attribute of the root group (obj None) or a dataset."""
    cnt = C.c_int()
    msg = C.create_string_buffer(512)
    o = b"" if obj is None else obj.encode()
    _h5_check(lib().scarl_h5_read_attr(str(path).encode(), o, name.encode(), None, 0, C.byref(cnt),
                                       msg, len(msg)), msg)
    out = np.empty(max(cnt.value, 1))
    _h5_check(lib().scarl_h5_read_attr(str(path).encode(), o, name.encode(),
                                       out.ctypes.data_as(C.POINTER(C.c_double)), cnt.value,
                                       C.byref(cnt), msg, len(msg)), msg)
    return out[:cnt.value]


def rebuild_corrL(SkTot, L, xStep):
    out = (C.c_double * 3)()
    s = np.ascontiguousarray(SkTot, dtype=np.float64)
    _check(lib().scarl_rebuild_corrL(s.ctypes.data_as(C.POINTER(C.c_double)), _i3(L),
                                     _d3(xStep), out))
    return np.array(out[:])
