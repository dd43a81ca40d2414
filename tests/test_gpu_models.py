"""GPU parity for loss lists (the first loss decides) and the classification
model: CV mode against speedynn's own outputs (golden vectors), holdout mode
against the NumPy restatement that those vectors pin."""
import os

import numpy as np
import pytest

from conftest import ROOT, golden_cases
from oracle import oracle
from speedynn_b200 import _lib, datagen
from speedynn_b200._lib import _f32p, _i32p, ptr
from speedynn_b200.base import IncrementalNNFeatureSelection
from speedynn_b200.selector import Selector

pytestmark = pytest.mark.gpu

GDIR = os.path.join(ROOT, "tests", "golden")
MODEL_CASES = golden_cases("model_")
ID2NAME = {v: k for k, v in IncrementalNNFeatureSelection.loss_dict.items()}


def _g(name):
    return dict(np.load(os.path.join(GDIR, name + ".npz")))


@pytest.mark.parametrize("name", MODEL_CASES)
def test_dropin_class_matches_reference_models(name):
    g = _g(name)
    sel = IncrementalNNFeatureSelection(g["X"], g["y"], k_vals=list(g["k_vals"]), auto_feature=bool(g["auto_feature"]),
                                        num_features=int(g["num_features"]), k_fold=int(g["k_fold"]),
                                        method=str(g["method"]),
                                        loss_functions=[ID2NAME[int(i)] for i in g["loss_functions"]],
                                        model_type="classification" if int(g["model_type"]) else "regression")
    sel.train()
    np.testing.assert_array_equal(sel.get_selected_ordering(), g["ordering"])
    np.testing.assert_array_equal(sel.get_selected_dimensions(), g["mask"])
    np.testing.assert_array_equal(sel.get_selected_errors(), g["errors_all"].T)  # (p, num_losses)
    assert sel.get_optimal_model_k() == int(g["best_k"])
    assert sel.num_final_features == int(g["num_final"])


@pytest.mark.parametrize("name", ["model_losses_fwd", "model_classif_bwd", "model_classif_auto"])
def test_c_abi_entry_points_with_losses(name):
    """train_*_selection with a loss list and model type, read back through get_selected_errors."""
    g = _g(name)
    L = _lib.lib()
    X = np.ascontiguousarray(g["X"], np.float32)
    y = np.ascontiguousarray(g["y"], np.float32)
    kv = np.ascontiguousarray(g["k_vals"], np.int32)
    lf = np.ascontiguousarray(g["loss_functions"], np.int32)
    n, d = X.shape
    fn = L.train_forward_selection if str(g["method"]) == "forward" else L.train_backward_selection
    nf = d if int(g["auto_feature"]) else int(g["num_features"])
    rc = fn(ptr(X, _f32p), n, d, ptr(y, _f32p), n, ptr(kv, _i32p), kv.size, nf, int(g["k_fold"]), ptr(lf, _i32p),
            lf.size, int(g["auto_feature"]), int(g["model_type"]))
    assert rc == int(g["num_final"]), _lib.last_error()
    errs = np.zeros(lf.size * d, np.float32)
    L.get_selected_errors(ptr(errs, _f32p), errs.size)
    np.testing.assert_array_equal(errs.reshape(lf.size, d), g["errors_all"])
    assert L.get_final_optimal_model_k() == int(g["best_k"])


def _classify(y):
    return np.digitize(y, np.quantile(y, [0.33, 0.66])).astype(np.float32)


@pytest.mark.parametrize("variant", ["lanes", "tma", "tma_seeded"])
@pytest.mark.parametrize("case", [
    dict(losses=[2, 0, 4, 6], model=0, kv=[3, 8], method="forward", nf=4),
    dict(losses=[1, 5, 8], model=0, kv=[5], method="backward", nf=5),
    dict(losses=[4, 3], model=1, kv=[1, 4, 7], method="forward", nf=4),
    dict(losses=[4], model=1, kv=[2, 6], method="backward", nf=4),
])
def test_holdout_models_match_restatement(case, variant):
    s = datagen.generate(320, 110, 9, n_mag=5, seed=90 + len(case["losses"]) + case["model"])
    yt, yv = s.ytrain, s.yval
    if case["model"] == 1:
        yt, yv = _classify(yt), _classify(yv)
    prob = oracle.Problem(s.Xtrain, yt, s.Xval, yv)
    o = oracle.np_select(prob, case["kv"], case["nf"], case["method"], loss_functions=case["losses"],
                         model_type=case["model"])
    with Selector(s.Xtrain, yt, s.Xval, yv, k_vals=case["kv"], num_features=case["nf"], method=case["method"],
                  loss_functions=case["losses"], model_type=case["model"]) as sel:
        sel.set_kernel(1 if variant == "lanes" else 3)
        if variant == "tma_seeded":
            sel.set_seed_step(1)
        r = sel.run()
    np.testing.assert_array_equal(r["ordering"], o["ordering"])
    np.testing.assert_array_equal(r["mask"], o["mask"])
    np.testing.assert_array_equal(r["errors_all"], o["errors_all"])
    assert r["best_k"] == o["best_k"] and r["num_final"] == o["num_final"]
