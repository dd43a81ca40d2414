"""C-ABI checks that need no GPU: the library builds, loads, exports every
symbol the public header declares, validates arguments, and its host-side
loss utility matches speedynn's own loss functions bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from speedynn_b200 import _lib
from speedynn_b200._lib import _f32p, _i32p, ptr

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def _declared():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        names |= set(re.findall(r"SNN_API\s+[\w\s\*]+?\b(\w+)\s*\(", src))
    return sorted(names)


@pytest.fixture(scope="module")
def L():
    from speedynn_b200 import build
    build.build()
    return _lib.lib()


def test_header_declares_reference_entry_points():
    names = _declared()
    for n in ("train_forward_selection", "train_backward_selection", "get_selected_dimensions",
              "get_selected_ordering", "get_selected_errors", "get_final_optimal_model_k", "get_loss_all",
              "snn_create", "snn_load", "snn_run", "snn_step", "snn_get_results", "snn_destroy", "snn_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(L):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string(L):
    assert b"sm_100a" in L.snn_version()


def test_loss_utility_matches_reference_losses(L):
    g = np.load(os.path.join(ROOT, "tests", "golden", "losses.npz"))
    lab = np.ascontiguousarray(g["labels"], np.float32)
    pre = np.ascontiguousarray(g["preds"], np.float32)
    got = np.array([L.get_loss_all(ptr(lab, _f32p), lab.size, ptr(pre, _f32p), pre.size, i) for i in range(9)],
                   np.float32)
    np.testing.assert_array_equal(got, g["values"])


def test_loss_utility_rejects_bad_input(L):
    a = np.ones(4, np.float32)
    b = np.ones(5, np.float32)
    assert np.isnan(L.get_loss_all(ptr(a, _f32p), 4, ptr(b, _f32p), 5, 0))
    assert np.isnan(L.get_loss_all(ptr(a, _f32p), 4, ptr(a, _f32p), 4, 42))


def _desc(**kw):
    kv = np.array(kw.pop("k_vals", [3]), np.int32)
    d = _lib.SnnDesc()
    d.n_train, d.n_val, d.p = kw.get("n_train", 100), kw.get("n_val", 0), kw.get("p", 5)
    d.k_vals = ptr(kv, _i32p)
    d.num_k_vals = kv.size
    d.backward = kw.get("backward", 0)
    d.num_features = kw.get("num_features", 2)
    d.k_fold = kw.get("k_fold", 10)
    d.auto_feature = 0
    d.device = kw.get("device", 0)
    return d, kv


@pytest.mark.parametrize("kw", [dict(n_train=0), dict(p=0), dict(k_vals=[0]), dict(k_vals=[3, -1]),
                                dict(num_features=6), dict(k_fold=0), dict(k_fold=101), dict(n_val=-3)])
def test_create_rejects_bad_descriptors(L, kw):
    d, _kv = _desc(**kw)
    h = ctypes.c_void_p()
    assert L.snn_create(ctypes.byref(d), ctypes.byref(h)) == _lib.SNN_ERR_ARG
    assert not h.value
    assert L.snn_last_error()


def test_null_handle_calls_fail_cleanly(L):
    assert L.snn_run(None) == _lib.SNN_ERR_ARG
    assert L.snn_step(None) == _lib.SNN_ERR_ARG
    assert L.snn_destroy(None) == 0


def test_dropin_rejects_unsupported_options(L):
    """Loss ids outside the reference's 0..8 and model types other than
    regression (0) / classification (1) are refused before any device work."""
    X = np.zeros((10, 3), np.float32)
    y = np.zeros(10, np.float32)
    kv = np.array([2], np.int32)
    lf = np.array([0, 9], np.int32)  # 9 is no reference loss
    rc = L.train_forward_selection(ptr(X, _f32p), 10, 3, ptr(y, _f32p), 10, ptr(kv, _i32p), 1, 2, 2, ptr(lf, _i32p),
                                   2, 0, 0)
    assert rc == _lib.SNN_ERR_UNSUPPORTED
    lf[1] = 2
    rc = L.train_forward_selection(ptr(X, _f32p), 10, 3, ptr(y, _f32p), 10, ptr(kv, _i32p), 1, 2, 2, ptr(lf, _i32p),
                                   2, 0, 2)  # model type 2 does not exist
    assert rc == _lib.SNN_ERR_UNSUPPORTED


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present")
def test_no_gpu_means_error_not_fallback(L):
    """Without a GPU the library reports an error: there is no CPU path."""
    d, _kv = _desc()
    h = ctypes.c_void_p()
    rc = L.snn_create(ctypes.byref(d), ctypes.byref(h))
    if rc == 0:
        L.snn_destroy(h)
        pytest.skip("a usable GPU is visible")
    assert rc == _lib.SNN_ERR_CUDA
    assert b"device" in L.snn_last_error() or b"CUDA" in L.snn_last_error()


def test_batch_rejects_bad_descriptors_without_a_gpu():
    """snn_batch_create validates every descriptor before touching a device."""
    import numpy as np
    from speedynn_b200 import _lib
    from speedynn_b200.batch import Batch
    good = dict(Xtrain=np.zeros((50, 4), np.float32), ytrain=np.zeros(50, np.float32), k_vals=[3], num_features=2,
                k_fold=5)
    bad = dict(good, k_vals=[0])
    with pytest.raises(Exception) as e:
        Batch([good, bad])
    assert "problem 1" in str(e.value)
    L = _lib.lib()
    assert L.snn_batch_create(None, 0, 0, None) == _lib.SNN_ERR_ARG


def test_batch_model_arguments_are_checked_without_a_gpu():
    """snn_batch_set_model checks the problem index, loss ids and model type
    before anything runs; snn_batch_get_errors_all refuses a problem that has
    not run.  None of it touches a device."""
    import numpy as np
    from speedynn_b200 import _lib
    from speedynn_b200._lib import _f32p, _i32p, ptr
    L = _lib.lib()
    kv = np.array([3], np.int32)
    d = (_lib.SnnDesc * 1)()
    d[0].n_train, d[0].n_val, d[0].p = 50, 0, 4
    d[0].k_vals, d[0].num_k_vals = ptr(kv, _i32p), 1
    d[0].num_features, d[0].k_fold = 2, 5
    h = ctypes.c_void_p()
    assert L.snn_batch_create(d, 1, 0, ctypes.byref(h)) == _lib.SNN_OK
    try:
        ok = np.array([4, 0], np.int32)
        assert L.snn_batch_set_model(h, 0, ptr(ok, _i32p), 2, 1) == _lib.SNN_OK
        assert L.snn_batch_set_model(h, 1, ptr(ok, _i32p), 2, 0) == _lib.SNN_ERR_ARG  # no problem 1
        bad = np.array([0, 9], np.int32)
        assert L.snn_batch_set_model(h, 0, ptr(bad, _i32p), 2, 0) == _lib.SNN_ERR_ARG
        assert b"loss id 9" in L.snn_last_error()
        assert L.snn_batch_set_model(h, 0, ptr(ok, _i32p), 2, 2) == _lib.SNN_ERR_ARG
        assert L.snn_batch_set_model(h, 0, None, 0, 0) == _lib.SNN_ERR_ARG
        out = np.zeros(8, np.float32)
        assert L.snn_batch_get_errors_all(h, 0, ptr(out, _f32p), out.size) == _lib.SNN_ERR_STATE
    finally:
        L.snn_batch_destroy(h)
