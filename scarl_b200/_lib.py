"""ctypes binding of libscarl_b200.so (the C ABI declared in include/scarl.h).

The shared library is built in-tree (scarl_b200/libscarl_b200.so).  Importing
this module without it raises ImportError: there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscarl_b200.so")

# status codes (include/scarl.h)
OK, EINVAL, ENOMEM, EDEVICE, ETIMEOUT, EUNSUPPORTED, EIO = range(7)
STATUS_NAMES = {0: "SCARL_OK", 1: "SCARL_EINVAL", 2: "SCARL_ENOMEM", 3: "SCARL_EDEVICE",
                4: "SCARL_ETIMEOUT", 5: "SCARL_EUNSUPPORTED", 6: "SCARL_EIO"}
FFT, FFT_MPI = 1, 2
CM_GAUSSIAN, CM_VON_KARMAN, CM_EXPONENTIAL = 1, 2, 3
MLP_PARAMS = 5378
MLP_IN = 16
FOM_GAUSSIAN, FOM_LOGNORMAL = 1, 2
F32, F64 = 4, 8
# flag on F32: pass 1's z DFT as split-BF16 tensor-core products
SPLIT_BF16 = 0x100
SPLIT_BF16_X = 0x200
GEN_DCT, GEN_SHINO, GEN_PADDED = 1, 2, 3
PAD_FULL, PAD_AUTO, PAD_LEARNED, PAD_SMOOTH = 0, 1, 2, 3


class Sample(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("xMinGlob", C.c_double * 3),
                ("xMaxGlob", C.c_double * 3), ("corrL", C.c_double * 3),
                ("overlap", C.c_double * 3), ("pointsPerCorrL", C.c_int * 3),
                ("corrMod", C.c_int), ("margiFirst", C.c_int), ("avg", C.c_double),
                ("std_dev", C.c_double), ("seedBase", C.c_int), ("nu", C.c_double)]


class Layout(C.Structure):
    _fields_ = [("L", C.c_int * 3), ("Np", C.c_int * 3), ("Np_ovlp", C.c_int * 3),
                ("topo_shape", C.c_int * 3), ("nb_tiles", C.c_int), ("xStep", C.c_double * 3)]


class Tile(C.Structure):
    _fields_ = [("topo_pos", C.c_int * 3), ("pos_0", C.c_int * 3), ("pos_N", C.c_int * 3),
                ("coord_0", C.c_double * 3), ("coord_N", C.c_double * 3),
                ("xRange", C.c_double * 3)]


class GenOpts(C.Structure):
    _fields_ = [("generator", C.c_int), ("dtype", C.c_int), ("nb_procs", C.c_int),
                ("topo_shape", C.c_int * 3), ("pad", C.c_int * 3),
                ("pad_policy", C.c_int), ("pad_tol", C.c_double),
                ("no_spectral_normalisation", C.c_int), ("normalize_field", C.c_int),
                ("stream", C.c_uint32), ("autotune", C.c_int), ("phiK", C.POINTER(C.c_double)),
                ("gen_meth", C.c_int), ("moments", C.POINTER(C.c_double))]


_vp = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes); every function of include/scarl.h
SIGNATURES = {
    "scarl_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(_vp)]),
    "scarl_ctx_destroy": (C.c_int, [_vp]),
    "scarl_last_error": (C.c_char_p, [_vp]),
    "scarl_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "scarl_sync": (C.c_int, [_vp]),
    "scarl_tc_wait_test": (C.c_int, [_vp, C.c_int]),
    "scarl_counters": (C.c_int, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong),
                                 C.POINTER(C.c_ulonglong)]),
    "scarl_autotune": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, _ip, _ip, _dp, _dp,
                                 C.c_char_p]),
    "scarl_tune_get": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _ip]),
    "scarl_tune_set": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "scarl_profile": (C.c_int, [_vp, C.c_int]),
    "scarl_profile_read": (C.c_int, [_vp, C.c_int, C.c_char_p, C.c_size_t, _dp,
                                     C.POINTER(C.c_longlong)]),
    "scarl_version": (C.c_char_p, []),
    "scarl_verify_inputs": (C.c_int, [C.POINTER(Sample), C.c_int, C.c_char_p, C.c_size_t]),
    "scarl_decide_topo_shape": (C.c_int, [C.c_int, _ip, _ip, C.c_longlong, _ip]),
    "scarl_get_topo_pos": (C.c_int, [C.c_int, _ip, _ip]),
    "scarl_get_topo_rank": (C.c_int, [_ip, _ip]),
    "scarl_sample_layout": (C.c_int, [C.POINTER(Sample), C.c_int, C.c_int, _ip,
                                      C.POINTER(Layout)]),
    "scarl_tile_geometry": (C.c_int, [C.POINTER(Layout), _dp, C.c_int, C.POINTER(Tile)]),
    "scarl_unity_partition_weights": (C.c_int, [_ip, _ip, C.c_int, _ip, _ip, _dp]),
    "scarl_shino_sizes": (C.c_int, [_ip, _dp, _dp, _ip, _ip, _dp]),
    "scarl_pad_size": (C.c_int, [C.c_int, C.c_int, C.c_double, _dp, _dp, _ip, C.c_double, _ip]),
    "scarl_axis_correlation": (C.c_double, [C.c_int, C.c_double, C.c_double, C.c_double]),
    "scarl_read_config": (C.c_int, [C.c_char_p, _ip, _ip, _ip, _ip, _ip, C.c_char_p,
                                    C.c_size_t]),
    "scarl_read_extra_config": (C.c_int, [C.c_char_p, _ip, _ip]),
    "scarl_read_input": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, _ip,
                                   C.POINTER(Sample), C.c_int]),
    "scarl_read_input_sem": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, _ip,
                                       C.POINTER(Sample), C.c_int]),
    "scarl_gen_std_gauss_fft": (C.c_int, [_vp, _vp, _ip, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                          _vp, _vp]),
    "scarl_gen_std_gauss_fft_mpi": (C.c_int, [_vp, _vp, _dp, _dp, C.c_int, C.c_int, C.c_int, _ip,
                                              _ip, _vp, _vp]),
    "scarl_gen_std_gauss_shino_fft": (C.c_int, [_vp, _vp, _ip, _dp, _dp, _ip, C.c_int,
                                                C.c_int, C.c_int]),
    "scarl_gen_padded": (C.c_int, [_vp, _vp, C.c_int, _ip, _ip, _dp, _dp, C.c_int, C.c_double,
                                   C.c_int, C.c_uint64, C.c_uint32, _vp]),
    "scarl_gen_padded_noalloc": (C.c_int, [_vp, C.c_int, _ip, _ip, _dp, _dp, C.c_int, C.c_double,
                                           C.c_int, C.c_uint64, C.c_uint32, _vp, C.c_char_p,
                                           C.c_size_t]),
    "scarl_generate_sample": (C.c_int, [_vp, C.POINTER(Sample), C.POINTER(GenOpts), _vp]),
    "scarl_pad_labels": (C.c_int, [_vp, C.c_int, _ip, _dp, _dp, _ip, _ip, _ip, _ip]),
    "scarl_pad_error": (C.c_int, [_vp, C.c_int, _ip, _dp, _dp, _ip, _ip, _dp]),
    "scarl_mlp_features": (C.c_int, [C.c_int, _ip, _dp, _dp, _ip, C.POINTER(C.c_float)]),
    "scarl_mlp_targets": (C.c_int, [C.c_int, _dp, _ip, _ip, _ip, C.POINTER(C.c_float)]),
    "scarl_mlp_init": (C.c_int, [_vp, C.c_uint64]),
    "scarl_mlp_params": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "scarl_mlp_grad": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                                 C.POINTER(C.c_float), _dp]),
    "scarl_mlp_train": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                                  C.c_int, C.c_float, _dp]),
    "scarl_mlp_predict": (C.c_int, [_vp, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float)]),
    "scarl_pad_size_learned": (C.c_int, [_vp, C.c_int, C.c_double, _dp, _dp, _ip, _ip, _ip, _ip]),
    "scarl_write_sample_h5": (C.c_int, [_vp, C.c_char_p, C.c_char_p, _vp, C.c_int,
                                        C.POINTER(Sample), C.POINTER(Layout), C.c_int, C.c_int,
                                        C.c_char_p, _dp, C.c_int]),
    "scarl_write_constant_field_h5": (C.c_int, [C.c_char_p, C.c_char_p, _dp, _dp, C.c_double]),
    "scarl_stat_file": (C.c_int, [_vp, C.c_char_p, C.c_char_p, C.c_int, _dp, _dp, _dp]),
    "scarl_h5_overwrite_dataset": (C.c_int, [C.c_char_p, C.c_char_p, _vp, C.c_ulonglong,
                                             C.c_char_p, C.c_size_t]),
    "scarl_h5_list": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]),
    "scarl_h5_read_dataset": (C.c_int, [C.c_char_p, C.c_char_p, _vp, C.c_int,
                                        C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.c_char_p,
                                        C.c_size_t]),
    "scarl_h5_read_attr": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, _dp, C.c_int,
                                     C.POINTER(C.c_int), C.c_char_p, C.c_size_t]),
    "scarl_axis_cov": (C.c_int, [_vp, _vp, C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp]),
    "scarl_axis_cov_sums": (C.c_int, [_vp, _vp, C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp]),
    "scarl_ensemble_draw": (C.c_int, [C.c_uint64, C.c_longlong, C.c_int, _ip, C.c_int, C.c_double,
                                      C.c_double, _ip, _dp]),
    "scarl_gen_ensemble": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _ip, _dp, _dp, C.c_int,
                                     C.c_double, C.c_int, C.c_double,
                                     C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.c_int,
                                     C.c_double, C.c_double, C.c_int]),
    "scarl_apply_unity_partition": (C.c_int, [_vp, _vp, _ip, _ip, C.c_int, _ip, _ip]),
    "scarl_add_overlap": (C.c_int, [_vp, _vp, _ip, _ip, _ip]),
    "scarl_multivariate_transformation": (C.c_int, [_vp, _vp, C.c_int, C.c_longlong, C.c_double,
                                                    C.c_double, C.c_int]),
    "scarl_normalize_field": (C.c_int, [_vp, _vp, C.c_int, C.c_longlong, _dp, _dp]),
    "scarl_moments": (C.c_int, [_vp, _vp, C.c_int, C.c_longlong, C.c_int, _dp, _dp, _dp, _dp]),
    "scarl_rebuild_sk": (C.c_int, [_vp, _vp, C.c_int, _ip, C.c_double, C.c_double, C.c_int,
                                   _dp]),
    "scarl_rebuild_corrL": (C.c_int, [_dp, _ip, _dp, _dp]),
}

_LIB = None


def lib():
    """Load the in-tree library (raises ImportError when it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python scarl_b200/build.py` "
                "(scarl_b200 has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class ScarlError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
