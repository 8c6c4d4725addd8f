"""ctypes binding of the C ABI in include/apirl_b200.h.

The shared library is built in-tree (apirl_b200/_build/libapirl_b200.so) by
``apirl_b200.build.build()``.  Loading fails loudly when it is missing: there
is no CPU fallback for any operation of this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libapirl_b200.so")

APIRL_OK = 0
APIRL_ERR_INVALID = 1
APIRL_ERR_CUDA = 2
APIRL_ERR_OOM = 3
APIRL_ERR_NOT_SUPPORTED = 4
APIRL_ERR_ABORTED = 5

APIRL_OPT_DUAL_LAYOUT = 1
APIRL_OPT_KERNEL_TIMING = 2
APIRL_OPT_EM_BLOCK = 3
APIRL_OPT_PERSISTENT = 4
APIRL_OPT_SPARSE_IMAGE = 5
APIRL_OPT_ACCUMULATE = 6
APIRL_OPT_L2_PERSIST = 7
APIRL_OPT_LIST_ORDER = 8
APIRL_OPT_GATHER_UNROLL = 9
APIRL_SPARSE_ZERO_COUNT = 0
APIRL_SPARSE_GEOMETRY = 1
APIRL_ACC_ATOMIC = 0
APIRL_ACC_WARP = 1
APIRL_ACC_COMPENSATED = 2

APIRL_ALPHA_F32 = 0
APIRL_ALPHA_F64 = 1
APIRL_SCANNER_CYLINDRICAL = 0
APIRL_SCANNER_MMR = 1
APIRL_MAX_SAMPLES = 64

APIRL_F32 = 0
APIRL_U32 = 1
APIRL_U16 = 2

_i = ctypes.c_int
_i64 = ctypes.c_int64
_f = ctypes.c_float
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)


class ImageGeomC(ctypes.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("nz", _i), ("dx", _f), ("dy", _f), ("dz", _f)]


class Sino2DGeomC(ctypes.Structure):
    _fields_ = [("n_proj", _i), ("n_r", _i), ("r_fov", _f), ("r_scanner", _f)]


class Sino3DGeomC(ctypes.Structure):
    _fields_ = [("n_proj", _i), ("n_r", _i), ("n_rings", _i), ("n_segments", _i),
                ("r_fov", _f), ("axial_fov", _f), ("r_scanner", _f),
                ("min_ring_diff", ctypes.POINTER(_i)), ("max_ring_diff", ctypes.POINTER(_i)), ("scanner", _i)]


class SamplingC(ctypes.Structure):
    """apirl_sampling: rays per bin (numSamplesOnDetector, numAxialSamplesOnDetector, useMultipleLorsPerBin)."""
    _fields_ = [("n_samples", _i), ("n_axial_samples", _i), ("multiple_lors_per_bin", _i)]


class ReconOptionsC(ctypes.Structure):
    """apirl_recon_options: rays per bin, given / returned sensitivity images."""
    _fields_ = [("sampling", ctypes.POINTER(SamplingC)), ("h_sens_in", _vp), ("h_sens_out", _vp),
                ("update_positive_sens", _i), ("n_sens_out", _i)]


class TuneC(ctypes.Structure):
    """apirl_tune: the fused pass's launch shape picked by apirl_projector_autotune_ex."""
    _fields_ = [("block", _i), ("unroll", _i), ("ms", ctypes.c_double)]


class JobDescC(ctypes.Structure):
    _fields_ = [("img", ImageGeomC), ("sino", Sino3DGeomC), ("h_counts", _vp), ("counts_dtype", _i),
                ("h_mult", _vp), ("h_add", _vp), ("h_init", _vp), ("iters", _i), ("nsubsets", _i),
                ("update_positive_sens", _i)]


# name -> (restype, argtypes)
SIGNATURES = {
    "apirl_last_error": (ctypes.c_char_p, []),
    "apirl_version": (ctypes.c_char_p, []),
    "apirl_lor_table": (_i, [_i, _i, _f, _f, _vp]),
    "apirl_mmr_lor_table": (_i, [_i, _i, _vp]),
    "apirl_projector_create_3d_mmr": (_i, [ctypes.POINTER(ImageGeomC), _i, _i, _i, _i, _vp, _vp, _i,
                                           ctypes.POINTER(_vp)]),
    "apirl_sino3d_ring_z": (_i, [ctypes.POINTER(Sino3DGeomC), _vp]),
    "apirl_projector_create_2d": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino2DGeomC), _i,
                                       ctypes.POINTER(_vp)]),
    "apirl_projector_create_3d": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino3DGeomC), _i,
                                       ctypes.POINTER(_vp)]),
    "apirl_projector_destroy": (None, [_vp]),
    "apirl_projector_num_bins": (_i64, [_vp, _i, _i]),
    "apirl_projector_num_sinograms": (_i, [_vp]),
    "apirl_projector_tables": (_i, [_vp, _vp, _vp]),
    "apirl_projector_set_alpha_precision": (_i, [_vp, _i]),
    "apirl_projector_set_option": (_i, [_vp, _i, _i]),
    "apirl_projector_kernel_ms": (_i, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "apirl_projector_autotune": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, ctypes.POINTER(_i), _vp]),
    "apirl_projector_autotune_ex": (_i, [_vp, _vp, _i, _vp, _vp, _i, _i, _i, ctypes.POINTER(TuneC), _vp]),
    "apirl_count_steps": (_i, [_vp, _i, _i, _vp, _vp]),
    "apirl_project": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "apirl_backproject": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "apirl_divide_and_backproject": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "apirl_generate_acf": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "apirl_inverse_divide": (_i, [_i64, _vp, _vp, _vp]),
    "apirl_add_bins": (_i, [_i64, _vp, _vp, _vp]),
    "apirl_likelihood": (_i, [_i64, _vp, _vp, _i, _vp, _vp]),
    "apirl_likelihood_noalloc": (_i, [_i64, _vp, _vp, _i, _vp, _vp]),
    "apirl_mlem_threshold": (_i, [_i64, _vp, _vp, _vp]),
    "apirl_update_pixels": (_i, [_i64, _vp, _vp, _vp, _vp, _f, _i, _i, _vp]),
    "apirl_force_positive": (_i, [_i64, _vp, _vp]),
    "apirl_em_pass": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp, _vp]),
    "apirl_zero_count_image": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _i, _i, _vp]),
    "apirl_em_pass_sparse": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp, _vp]),
    "apirl_em_project_backproject": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "apirl_stage_counts": (_i, [_vp, _vp, _i, _vp, _i, _i, _vp]),
    "apirl_em_pass_host": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp, _vp, _vp]),
    "apirl_em_pass_host_async": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp, _vp, _vp]),
    "apirl_set_iteration_hook": (_i, [_vp, _i, _vp]),
    "apirl_backproject_ones": (_i, [_vp, _vp, _i, _i, _vp]),
    "apirl_backproject_and_ones": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "apirl_em_project_backproject_sparse": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "apirl_osem_3d": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino3DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                           _i, _vp, _vp, _vp, ctypes.POINTER(SamplingC)]),
    "apirl_mlem_3d": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino3DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                           _vp, _vp, _vp, ctypes.POINTER(SamplingC)]),
    "apirl_osem_3d_ex": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino3DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                              _i, _vp, _vp, ctypes.POINTER(ReconOptionsC)]),
    "apirl_mlem_3d_ex": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino3DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                              _vp, _vp, ctypes.POINTER(ReconOptionsC)]),
    "apirl_mlem_2d_ex": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino2DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                              _vp, _vp, ctypes.POINTER(ReconOptionsC)]),
    "apirl_projector_set_sampling": (_i, [_vp, _i, _i, _i]),
    "apirl_projector_set_shard": (_i, [_vp, _i, _i]),
    "apirl_job_footprint": (_i64, [ctypes.POINTER(JobDescC)]),
    "apirl_batch_create": (_i, [_i, _i64, ctypes.POINTER(_vp)]),
    "apirl_batch_destroy": (None, [_vp]),
    "apirl_batch_submit": (_i, [_vp, ctypes.POINTER(JobDescC), ctypes.POINTER(_i64)]),
    "apirl_batch_step": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "apirl_batch_result": (_i, [_vp, _i64, _vp, _vp, ctypes.POINTER(_i)]),
    "apirl_mlem_2d": (_i, [ctypes.POINTER(ImageGeomC), ctypes.POINTER(Sino2DGeomC), _vp, _vp, _vp, _vp, _i, _i,
                           _vp, _vp, _vp]),
}

_lib = None


class ApirlError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"apirl error {code}: {msg}")
        self.code = code


def load(path=LIB_PATH):
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with apirl_b200.build.build() "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != APIRL_OK:
        raise ApirlError(status, _lib.apirl_last_error().decode(errors="replace"))
    return status
