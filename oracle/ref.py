"""ctypes driver for speedynn's own CPU backend, compiled from the reference
sources by ``oracle/Makefile`` into ``oracle/_ref/libspeedynn_ref.so``.

TEST INFRASTRUCTURE ONLY: used by ``tests/golden/make_golden.py`` to produce
golden vectors, by the tests to pin the restatement, and by ``bench.py
--impl reference`` as the timed CPU reference.  Never imported by the product.

The reference keeps one problem in process-global state
(speedynn/lib/nearest_neighbors_feature_selection.c:6-35), so every call here
is serialised on one library handle.  It exits the process for n > 15000
(nearest_neighbors_feature_selection.c:84-87, :251-254); the exported
``large_scale_threshold`` (same file :35) is raised before each call.
"""
import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libspeedynn_ref.so")

_lock = threading.Lock()
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int)
_f32p = ctypes.POINTER(ctypes.c_float)


def available():
    return os.path.exists(REF_SO)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{REF_SO} is not built (make -C oracle REF=<speedynn checkout>)")
        lib = ctypes.CDLL(REF_SO)
        for name in ("train_forward_selection", "train_backward_selection"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int, _i32p, ctypes.c_int,
                           ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.get_selected_dimensions.argtypes = [_i32p, ctypes.c_int]
        lib.get_selected_ordering.argtypes = [_i32p, ctypes.c_int]
        lib.get_selected_errors.argtypes = [_f32p, ctypes.c_int]
        lib.get_final_optimal_model_k.restype = ctypes.c_int
        lib.get_loss_all.restype = ctypes.c_float
        lib.get_loss_all.argtypes = [_f32p, ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_int]
        lib.init_memory_cpu.argtypes = [ctypes.c_int]
        lib.free_memory_cpu.argtypes = [ctypes.c_int]
        lib.compute_distance_matrix_cpu.argtypes = [_i32p, ctypes.c_int]
        lib.update_current_dist_matrix_cpu.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.get_k_nearest_neighbors_cpu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p, _f32p,
                                                    ctypes.c_int, ctypes.c_int]
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def train(X, y, k_vals, num_features, k_fold, method, auto_feature=False, loss_functions=(0,), model_type=0):
    """Run the reference selector (CV mode). Returns a dict of its outputs."""
    lib = load()
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    kv = np.ascontiguousarray(k_vals, dtype=np.int32)
    lf = np.ascontiguousarray(loss_functions, dtype=np.int32)
    n, d = X.shape
    fn = {"forward": lib.train_forward_selection, "backward": lib.train_backward_selection}[method]
    with _lock:
        ctypes.c_int.in_dll(lib, "large_scale_threshold").value = max(15000, n)
        nfinal = fn(_p(X, _f32p), n, d, _p(y, _f32p), n, _p(kv, _i32p), len(kv), int(num_features),
                    int(k_fold), _p(lf, _i32p), len(lf), int(bool(auto_feature)), int(model_type))
        mask = np.zeros(d, np.int32)
        order = np.zeros(d, np.int32)
        errs = np.zeros(d * len(lf), np.float32)
        lib.get_selected_dimensions(_p(mask, _i32p), d)
        lib.get_selected_ordering(_p(order, _i32p), d)
        lib.get_selected_errors(_p(errs, _f32p), errs.size)
        best_k = lib.get_final_optimal_model_k()
    return {"num_final": int(nfinal), "mask": mask, "ordering": order,
            "errors": errs.reshape(len(lf), d), "best_k": int(best_k)}


def loss(labels, preds, loss_function):
    lib = load()
    a = np.ascontiguousarray(labels, dtype=np.float32)
    b = np.ascontiguousarray(preds, dtype=np.float32)
    with _lock:
        return float(lib.get_loss_all(_p(a, _f32p), a.size, _p(b, _f32p), b.size, int(loss_function)))


def neighbours(X, k_max, k_fold, committed, backward, candidates):
    """Neighbour lists from the reference's own get_k_nearest_neighbors_cpu
    (speedynn/lib/cpu.c:128-168) after committing ``committed`` into its
    distance matrix with update_current_dist_matrix_cpu (cpu.c:217-231).

    Returns (idx, dist) of shape [len(candidates), n, k_max].
    """
    lib = load()
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    mult = -1 if backward else 1
    npf = n // k_fold
    idx = np.zeros((len(candidates), n, k_max), np.int32)
    dist = np.zeros((len(candidates), n, k_max), np.float32)
    ib = np.zeros(k_max, np.int32)
    db = np.zeros(k_max, np.float32)
    with _lock:
        ctypes.c_int.in_dll(lib, "dim").value = d
        ctypes.c_int.in_dll(lib, "num_training_patterns").value = n
        ctypes.c_int.in_dll(lib, "k_max").value = k_max
        ctypes.c_void_p.in_dll(lib, "training_patterns").value = X.ctypes.data
        lib.init_memory_cpu(0)
        try:
            if backward:
                lib.compute_distance_matrix_cpu(None, 0)
            else:
                lib.empty_distance_matrix_cpu()
            for w in committed:
                lib.update_current_dist_matrix_cpu(int(w), mult)
            for ci, c in enumerate(candidates):
                for r in range(n):
                    lib.get_k_nearest_neighbors_cpu(r, r // npf, npf, _p(ib, _i32p), _p(db, _f32p), int(c), mult)
                    idx[ci, r] = ib
                    dist[ci, r] = db
        finally:
            lib.free_memory_cpu(0)
            ctypes.c_void_p.in_dll(lib, "training_patterns").value = None
    return idx, dist
