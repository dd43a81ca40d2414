"""Failure detection without a GPU fault (fault injection, each fires once).

* A device pipeline wait that runs out: block 0 of a scoring launch never
  receives one stage's copies, its bounded waits give up after about a
  second, the call returns SNN_ERR_TIMEOUT, and the same handle then runs to
  the same results as a clean one (the context stays usable).
* Host-side failures: an injected allocation failure in snn_create and an
  injected launch failure at a greedy step come back as status codes, and the
  handle recovers with snn_reset.
"""
import os
import time

import numpy as np
import pytest

from speedynn_b200 import _lib, datagen
from speedynn_b200.selector import Selector

pytestmark = pytest.mark.gpu

KEYS = ("ordering", "mask", "errors", "errors64", "step_best_k", "best_k", "num_final")


def _data():
    return datagen.generate(3000, 1200, 12, n_mag=5, seed=81)


def _make(s, **env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=[5, 9], num_features=4, method="forward")
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _same(a, b):
    for k in KEYS:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


def test_bounded_wait_runs_out_and_the_handle_recovers():
    s = _data()
    with _make(s) as sel:
        clean = sel.run()
    with _make(s, SNN_INJECT_STALL=3) as sel:
        t0 = time.perf_counter()
        with pytest.raises(_lib.SnnError) as e:
            sel.run()
        assert e.value.code == _lib.SNN_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 30.0
        sel.reset()
        _same(sel.run(), clean)


def test_injected_allocation_failure_is_reported():
    s = _data()
    with pytest.raises(_lib.SnnError) as e:
        _make(s, SNN_INJECT_FAIL="alloc:4")
    assert e.value.code == _lib.SNN_ERR_NOMEM
    assert "injected" in str(e.value)
    with _make(s) as sel:  # nothing left over
        sel.run()


def test_injected_launch_failure_then_reset_recovers():
    s = _data()
    with _make(s) as sel:
        clean = sel.run()
    with _make(s, SNN_INJECT_FAIL="launch:2") as sel:
        with pytest.raises(_lib.SnnError) as e:
            sel.run()
        assert e.value.code == _lib.SNN_ERR_CUDA
        sel.reset()
        _same(sel.run(), clean)
