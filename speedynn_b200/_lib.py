"""ctypes binding of libspeedynn_b200.so (C ABI: include/speedynn_b200.h).

The shared library is the only implementation: if it is missing, importing
this module's :func:`lib` raises; there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# SNN_LIBRARY may name another build of the same library (e.g. a debug build).
LIB_PATH = os.environ.get("SNN_LIBRARY") or os.path.join(HERE, "libspeedynn_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "speedynn_b200.h")

SNN_OK = 0
SNN_ERR_ARG = -1
SNN_ERR_CUDA = -2
SNN_ERR_NOMEM = -3
SNN_ERR_UNSUPPORTED = -4
SNN_ERR_NO_WINNER = -5
SNN_ERR_STATE = -6
SNN_ERR_TIMEOUT = -7

SNN_OPT_KERNEL = 2
SNN_OPT_COUNTERS = 3
SNN_OPT_SEED_STEP = 4
SNN_OPT_SORTED_START = 5

_i32p = ctypes.POINTER(ctypes.c_int)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


class SnnDesc(ctypes.Structure):
    _fields_ = [
        ("n_train", ctypes.c_int),
        ("n_val", ctypes.c_int),
        ("p", ctypes.c_int),
        ("k_vals", _i32p),
        ("num_k_vals", ctypes.c_int),
        ("backward", ctypes.c_int),
        ("num_features", ctypes.c_int),
        ("k_fold", ctypes.c_int),
        ("auto_feature", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class SnnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"speedynn_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m speedynn_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sigs = {
            "snn_create": (ctypes.c_int, [ctypes.POINTER(SnnDesc), ctypes.POINTER(vp)]),
            "snn_load": (ctypes.c_int, [vp, _f32p, _f32p, _f32p, _f32p]),
            "snn_run": (ctypes.c_int, [vp]),
            "snn_reset": (ctypes.c_int, [vp]),
            "snn_step": (ctypes.c_int, [vp]),
            "snn_commit_sequence": (ctypes.c_int, [vp, _i32p, ctypes.c_int]),
            "snn_get_results": (ctypes.c_int, [vp, _i32p, _i32p, _f32p, _f64p, _i32p, _i32p, _i32p]),
            "snn_keep_neighbours": (ctypes.c_int, [vp, ctypes.c_int]),
            "snn_get_neighbours": (ctypes.c_int, [vp, _i32p, _i32p, _i32p, _i32p, _f32p]),
            "snn_get_timing": (ctypes.c_int, [vp, _f64p, _i32p, _f64p, _i32p, _f64p, _i32p]),
            "snn_destroy": (ctypes.c_int, [vp]),
            "snn_set_option": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
            "snn_get_neighbours_rows": (ctypes.c_int, [vp, _i32p, ctypes.c_int, _i32p, _f32p]),
            "snn_get_predictions": (ctypes.c_int, [vp, _i32p, ctypes.c_int, _i32p, _i32p, _f32p]),
            "snn_set_model": (ctypes.c_int, [vp, _i32p, ctypes.c_int, ctypes.c_int]),
            "snn_get_errors_all": (ctypes.c_int, [vp, _f32p, ctypes.c_int]),
            "snn_get_filter_counters": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_ulonglong),
                                                       ctypes.POINTER(ctypes.c_ulonglong),
                                                       ctypes.POINTER(ctypes.c_ulonglong)]),
            "snn_get_step_timing": (ctypes.c_int, [vp, _f32p, _f32p, ctypes.c_int]),
            "snn_get_setup_timing": (ctypes.c_int, [vp, _f32p]),
            "snn_batch_create": (ctypes.c_int, [ctypes.POINTER(SnnDesc), ctypes.c_int, ctypes.c_ulonglong,
                                                ctypes.POINTER(vp)]),
            "snn_batch_load": (ctypes.c_int, [vp, ctypes.c_int, _f32p, _f32p, _f32p, _f32p]),
            "snn_batch_set_model": (ctypes.c_int, [vp, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int]),
            "snn_batch_get_errors_all": (ctypes.c_int, [vp, ctypes.c_int, _f32p, ctypes.c_int]),
            "snn_batch_run": (ctypes.c_int, [vp]),
            "snn_batch_get_results": (ctypes.c_int, [vp, ctypes.c_int, _i32p, _i32p, _f32p, _f64p, _i32p, _i32p,
                                                     _i32p]),
            "snn_batch_get_timing": (ctypes.c_int, [vp, _f64p, _i32p]),
            "snn_batch_destroy": (ctypes.c_int, [vp]),
            "snn_last_error": (ctypes.c_char_p, []),
            "snn_version": (ctypes.c_char_p, []),
            "train_forward_selection": (ctypes.c_int, [_f32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int, _i32p,
                                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int,
                                                       ctypes.c_int, ctypes.c_int]),
            "train_backward_selection": (ctypes.c_int, [_f32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int, _i32p,
                                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int,
                                                        ctypes.c_int, ctypes.c_int]),
            "snn_score_step_noalloc": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int,
                                                      ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, _i32p,
                                                      ctypes.c_int, ctypes.c_int, vp, vp, vp]),
            "get_selected_dimensions": (None, [_i32p, ctypes.c_int]),
            "get_selected_ordering": (None, [_i32p, ctypes.c_int]),
            "get_selected_errors": (None, [_f32p, ctypes.c_int]),
            "get_final_optimal_model_k": (ctypes.c_int, []),
            "get_loss_all": (ctypes.c_float, [_f32p, ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_int]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().snn_last_error().decode(errors="replace")


def check(code):
    if code < 0:
        raise SnnError(code, last_error())
    return code


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)
