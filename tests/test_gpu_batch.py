"""Batches (snn_batch_*): each problem's results equal a Selector run of
that problem alone -- bit for bit, as the batch reuses the same handles --
whether the batch runs in one wave or in one wave per problem."""
import numpy as np
import pytest

from speedynn_b200 import datagen
from speedynn_b200.batch import Batch
from speedynn_b200.selector import Selector

pytestmark = pytest.mark.gpu

KEYS = ("ordering", "mask", "errors", "errors64", "step_best_k", "best_k", "num_final")


def _problems():
    probs = []
    shapes = [(1500, 700, 12, [10], 4, "forward"), (900, 0, 10, [1, 5], 3, "forward"),
              (1200, 500, 14, [5, 20], 9, "backward"), (700, 300, 9, [3], 5, "forward"),
              (2100, 0, 11, [7, 2], 6, "backward"), (1000, 450, 13, [40], 3, "forward")]
    for i, (nt, nv, p, kv, nf, method) in enumerate(shapes):
        s = datagen.generate(nt, max(nv, 32), p, n_mag=5, seed=500 + i)
        pr = dict(Xtrain=s.Xtrain, ytrain=s.ytrain, k_vals=kv, num_features=nf, method=method, k_fold=4)
        if nv:
            pr.update(Xval=s.Xval, yval=s.yval)
        probs.append(pr)
    probs[3]["auto_feature"] = True
    return probs


def _alone(pr):
    kw = {k: v for k, v in pr.items() if k not in ("Xtrain", "ytrain", "Xval", "yval")}
    with Selector(pr["Xtrain"], pr["ytrain"], pr.get("Xval"), pr.get("yval"), **kw) as sel:
        return sel.run()


@pytest.mark.parametrize("max_bytes", [0, 1])
def test_batch_matches_single_runs(max_bytes):
    probs = _problems()
    want = [_alone(pr) for pr in probs]
    with Batch(probs, max_device_bytes=max_bytes) as b:
        got = b.run()
        tm = b.timing()
    assert tm["waves"] == (1 if max_bytes == 0 else len(probs))
    assert tm["run_ms"] > 0
    for w, g in zip(want, got):
        for k in KEYS:
            np.testing.assert_array_equal(np.asarray(g[k]), np.asarray(w[k]), err_msg=k)


def test_many_concurrent_problems_match_single_runs():
    """64 problems issued while later ones are still being created and loaded,
    so early selections run on a busy GPU: every problem still equals its own
    single-handle run (each handle's k values reach the device before its
    first step)."""
    rng = np.random.default_rng(9)
    probs = []
    for i in range(64):
        nt = int(rng.integers(1500, 12000))
        s = datagen.generate(nt, nt // 2, 20, n_mag=5, seed=900 + i)
        probs.append(dict(Xtrain=s.Xtrain, ytrain=s.ytrain, Xval=s.Xval, yval=s.yval,
                          k_vals=[[1, 5, 10, 20][i % 4]], num_features=6, method="forward"))
    with Batch(probs) as b:
        got = b.run()
    for i, (pr, g) in enumerate(zip(probs, got)):
        w = _alone(pr)
        for k in KEYS:
            np.testing.assert_array_equal(np.asarray(g[k]), np.asarray(w[k]), err_msg=f"problem {i}: {k}")


def _model_problems():
    """Problems with loss lists and the classification model: (n_train, n_val,
    p, k values, features, method, loss ids, model type)."""
    shapes = [(1400, 600, 11, [5, 1], 4, "forward", (4, 0), 1),   # classification, zero-one loss decides
              (1000, 0, 10, [3, 9], 3, "backward", (0,), 1),      # classification, CV mode
              (1200, 500, 12, [7], 5, "forward", (2, 0, 5), 0),   # MAD decides, RMSE and std kept
              (800, 400, 9, [4, 20], 6, "backward", (1, 8), 0)]   # normalised RMSE decides
    probs = []
    for i, (nt, nv, p, kv, nf, method, lf, mt) in enumerate(shapes):
        s = datagen.generate(nt, max(nv, 32), p, n_mag=5, seed=700 + i)
        yt, yv = s.ytrain, s.yval
        if mt == 1:  # class labels
            yt = np.floor(3.0 * yt).astype(np.float32)
            yv = np.floor(3.0 * yv).astype(np.float32)
        pr = dict(Xtrain=s.Xtrain, ytrain=yt, k_vals=kv, num_features=nf, method=method, k_fold=4,
                  loss_functions=lf, model_type=mt)
        if nv:
            pr.update(Xval=s.Xval, yval=yv)
        probs.append(pr)
    return probs


@pytest.mark.parametrize("max_bytes", [0, 1])
def test_batch_losses_and_classification_match_single_runs(max_bytes):
    """snn_batch_set_model: each problem's selection, FP32 and FP64 errors and
    the errors of every loss equal a Selector run with the same losses and
    model, in one wave and in one wave per problem (the arena then holds
    exactly one problem's buffers, the loss and neighbour arrays included)."""
    probs = _model_problems()
    want = [_alone(pr) for pr in probs]
    with Batch(probs, max_device_bytes=max_bytes) as b:
        got = b.run()
    for w, g in zip(want, got):
        for k in KEYS:
            np.testing.assert_array_equal(np.asarray(g[k]), np.asarray(w[k]))
        np.testing.assert_array_equal(g["errors_all"], w["errors_all"])
