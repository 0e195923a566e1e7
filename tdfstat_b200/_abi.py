"""ctypes mirror of include/tdfcuda.h (the C ABI of libtdfcuda).

The structure layouts here must match the header field for field;
tests/test_abi.py compares their sizes with what a C compiler gives.
"""
import ctypes as C
import os

TDF_MAX_DETECTORS = 8
TDF_MAX_LINES = 512
TDF_NAVFSTAT = 4096

TDF_OK = 0
TDF_ERR_INVALID = 1
TDF_ERR_CUDA = 2
TDF_ERR_TRIGGER_OVERFLOW = 3
TDF_ERR_OUT_OF_MEMORY = 4
TDF_ERR_CAPACITY = 5
TDF_ERR_UNSUPPORTED = 6
TDF_ERR_NO_DEVICE = 7
TDF_ERR_NOT_BUILT = 8

TDF_FORM_SPLIT = 0
TDF_FORM_FP64 = 1

FORMS = {"split": TDF_FORM_SPLIT, "fp64": TDF_FORM_FP64}


class TdfDetector(C.Structure):
    _fields_ = [
        ("xdat", C.POINTER(C.c_float)),
        ("detssb", C.POINTER(C.c_double)),
        ("sig2", C.c_double),
        ("sphir", C.c_double),
        ("cphir", C.c_double),
        ("amod", C.c_double * 9),
    ]


class TdfSegment(C.Structure):
    _fields_ = [
        ("N", C.c_int32),
        ("nfft", C.c_int32),
        ("nfftf", C.c_int32),
        ("Ninterp", C.c_int32),
        ("interpftpad", C.c_int32),
        ("nifo", C.c_int32),
        ("dt", C.c_double),
        ("oms", C.c_double),
        ("sepsm", C.c_double),
        ("cepsm", C.c_double),
        ("Smin", C.c_double),
        ("Smax", C.c_double),
        ("M", C.c_double * 16),
        ("cosmodf", C.POINTER(C.c_double)),
        ("sinmodf", C.POINTER(C.c_double)),
        ("det", TdfDetector * TDF_MAX_DETECTORS),
    ]


class TdfSearchOpts(C.Structure):
    _fields_ = [
        ("thr", C.c_double),
        ("fr", C.c_int32 * 2),
        ("allsky", C.c_int32),
        ("blocks_avg", C.c_int32),
        ("spndr", C.c_float * 2),
        ("sstep", C.c_float),
        ("bufsize", C.c_int32),
        ("numlines", C.c_int32),
        ("lines", C.POINTER(C.c_double)),
    ]


class TdfRecord(C.Structure):
    _fields_ = [
        ("m", C.c_float),
        ("n", C.c_float),
        ("s", C.c_float),
        ("ra", C.c_float),
        ("dec", C.c_float),
        ("fdot", C.c_float),
        ("len", C.c_uint32),
        ("pad", C.c_uint32),
        ("offset", C.c_int64),
    ]


class TdfSignal(C.Structure):
    _fields_ = [
        ("h0", C.c_double),
        ("snr", C.c_double),
        ("freq", C.c_double),
        ("fdot", C.c_double),
        ("ra", C.c_double),
        ("dec", C.c_double),
        ("iota", C.c_double),
        ("psi", C.c_double),
        ("phase", C.c_double),
        ("fpo", C.c_double),
        ("B", C.c_double),
        ("reffr", C.c_int32),
        ("seg", C.c_int32),
    ]


class TdfCoincOpts(C.Structure):
    _fields_ = [
        ("refr", C.c_int32),
        ("cthr", C.c_double),
        ("scalef", C.c_int32),
        ("scales", C.c_int32),
        ("scalem", C.c_int32),
        ("scalen", C.c_int32),
        ("mincoin", C.c_int32),
        ("shift", C.c_int32),
    ]


class TdfCoincSegment(C.Structure):
    _fields_ = [
        ("seg", C.c_int32),
        ("N", C.c_int32),
        ("nfftf", C.c_int32),
        ("dt", C.c_double),
        ("narrowdown", C.c_double),
        ("nlines", C.c_int32),
        ("lines", C.POINTER(C.c_double)),
        ("nrec", C.c_int64),
        ("recs", C.POINTER(TdfRecord)),
        ("pairs", C.POINTER(C.c_float)),
    ]


class TdfCoincidence(C.Structure):
    _fields_ = [
        ("shift", C.c_int32),
        ("w", C.c_int32),
        ("avg_snr", C.c_float),
        ("avg_f", C.c_float),
        ("avg_fdot", C.c_float),
        ("avg_ra", C.c_float),
        ("avg_dec", C.c_float),
        ("member", C.c_int64),
    ]


class TdfKernelTimes(C.Structure):
    _fields_ = [
        ("colpass_ms", C.c_double),
        ("rowpass_ms", C.c_double),
        ("threshold_ms", C.c_double),
        ("sky_ms", C.c_double),
        ("colpass_launches", C.c_int64),
        ("rowpass_launches", C.c_int64),
        ("threshold_launches", C.c_int64),
        ("sky_batches", C.c_int64),
        ("colpass_templates", C.c_int64),
    ]


# (name, restype, argtypes) of every function include/tdfcuda.h declares
P = C.c_void_p
I32P = C.POINTER(C.c_int32)
F32P = C.POINTER(C.c_float)
F64P = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)
RECP = C.POINTER(TdfRecord)

ABI_FUNCTIONS = [
    ("tdf_check_bounded_wait", C.c_int, [C.c_int, C.c_int32, C.POINTER(C.c_uint32)]),
    ("tdf_spin_order_item", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint32, C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("tdf_status_string", C.c_char_p, [C.c_int]),
    ("tdf_last_error", C.c_char_p, []),
    ("tdf_device_count", C.c_int, [I32P]),
    ("tdf_engine_create", C.c_int,
     [C.POINTER(TdfSegment), C.POINTER(TdfSearchOpts), C.c_int, C.c_int, C.c_int, C.POINTER(P)]),
    ("tdf_engine_upload", C.c_int, [P, C.POINTER(TdfSegment)]),
    ("tdf_engine_destroy", C.c_int, [P]),
    ("tdf_search_points", C.c_int,
     [P, C.c_int, I32P, F32P, F32P, F32P, RECP, C.c_int64, I64P, F32P, C.c_int64, I64P, I32P]),
    ("tdf_count_templates", C.c_int, [P, C.c_int, I32P, F32P, F32P, F32P, I64P, I32P]),
    ("tdf_last_results", C.c_int, [P, RECP, C.c_int64, I64P, F32P, C.c_int64, I64P, I32P]),
    ("tdf_search_points_device", C.c_int,
     [P, C.c_int, I32P, F32P, F32P, F32P, I64P, I64P]),
    ("tdf_engine_add_segment", C.c_int, [P, C.POINTER(TdfSegment), I32P]),
    ("tdf_engine_get_tuning", C.c_int, [P, I32P, I32P, I32P]),
    ("tdf_engine_upload_segment", C.c_int, [P, C.c_int32, C.POINTER(TdfSegment)]),
    ("tdf_engine_segment_count", C.c_int, [P, I32P]),
    ("tdf_search_segments_device", C.c_int, [P, C.c_int32, I32P, I32P, I32P, F32P, F32P, I64P, I64P]),
    ("tdf_fstat_spectrum", C.c_int,
     [P, C.c_int32, C.c_float, C.c_float, C.c_float, F64P, C.c_int64]),
    ("tdf_engine_add_signal", C.c_int, [P, C.POINTER(TdfSignal), F64P, I32P]),
    ("tdf_engine_get_signal", C.c_int, [P, C.c_int32, F64P, C.c_int64]),
    ("tdf_engine_get_xdat", C.c_int, [P, C.c_int32, F32P, C.c_int64]),
    ("tdf_coincidences", C.c_int,
     [C.POINTER(TdfCoincOpts), C.c_int32, C.POINTER(TdfCoincSegment), C.POINTER(TdfCoincidence), C.c_int64, I64P,
      C.POINTER(C.c_int16), I32P, C.POINTER(C.c_int16), C.c_int64, I64P, I32P]),
    ("tdf_fstat_operands_static", C.c_int,
     [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_float, C.c_float,
      C.c_int32, C.c_int32, P, P]),
    ("tdf_engine_get_stream", C.c_int, [P, C.POINTER(P)]),
    ("tdf_engine_set_stream", C.c_int, [P, P]),
    ("tdf_engine_autotune", C.c_int, [P, C.c_int, I32P, F32P, F32P, I32P]),
    ("tdf_engine_get_templates_per_chunk", C.c_int, [P, I32P]),
    ("tdf_engine_set_templates_per_chunk", C.c_int, [P, C.c_int32]),
    ("tdf_engine_launch_count", C.c_int, [P, I64P]),
    ("tdf_engine_set_kernel_timing", C.c_int, [P, C.c_int]),
    ("tdf_engine_get_kernel_times", C.c_int, [P, C.POINTER(TdfKernelTimes)]),
]

# include/tdfcuda_refabi.h
REFABI_FUNCTIONS = [
    ("job_core", C.c_int, [C.c_int, C.c_float, C.c_float, P, P, P, P, P, P, I32P, P, I32P]),
    ("tdf_job_core_ref", C.c_int, [C.c_int, C.c_float, C.c_float, P, P, P, P, P, P, I32P, P, I32P]),
    ("tdf_job_core_release", None, []),
    ("tdf_ref_struct_size", C.c_size_t, [C.c_int]),
]

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libtdfcuda.so")


def bind(lib):
    """Attach restype/argtypes of every ABI function to a loaded CDLL."""
    for name, res, args in ABI_FUNCTIONS + REFABI_FUNCTIONS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
