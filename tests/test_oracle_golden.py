"""Pin the CPU oracle against golden vectors from speedynn's own CPU backend."""
import os

import numpy as np
import pytest

from conftest import ROOT, golden_cases
from oracle import oracle, ref

GDIR = os.path.join(ROOT, "tests", "golden")
SELECT_CASES = [n for n in golden_cases() if not n.startswith(("nn_", "model_", "config_")) and n != "losses"]
NN_CASES = golden_cases("nn_")


def _load(name):
    return dict(np.load(os.path.join(GDIR, name + ".npz")))


@pytest.mark.parametrize("name", SELECT_CASES)
def test_c_oracle_matches_reference_golden(name):
    g = _load(name)
    method = str(g["method"])
    prob = oracle.Problem(g["X"], g["y"], k_fold=int(g["k_fold"]))
    o = oracle.select(prob, g["k_vals"], int(g["num_features"]), method, auto_feature=bool(g["auto_feature"]))
    np.testing.assert_array_equal(o["ordering"], g["ordering"])
    np.testing.assert_array_equal(o["mask"], g["mask"])
    np.testing.assert_array_equal(o["errors"], g["errors"])  # bit-exact FP32
    assert o["best_k"] == int(g["best_k"])
    assert o["num_final"] == int(g["num_final"])


@pytest.mark.parametrize("name", [n for n in SELECT_CASES if n not in ("pooled_fwd_3000",)])
def test_numpy_restatement_matches_reference_golden(name):
    g = _load(name)
    if bool(g["auto_feature"]):
        pytest.skip("the NumPy restatement has no auto_feature stop")
    if g["X"].shape[0] > 150:
        pytest.skip("NumPy restatement is for tiny inputs")
    prob = oracle.Problem(g["X"], g["y"], k_fold=int(g["k_fold"]))
    o = oracle.np_select(prob, g["k_vals"], int(g["num_features"]), str(g["method"]))
    np.testing.assert_array_equal(o["ordering"], g["ordering"])
    np.testing.assert_array_equal(o["errors"], g["errors"])
    assert o["best_k"] == int(g["best_k"])


@pytest.mark.parametrize("name", NN_CASES)
def test_oracle_neighbours_match_reference(name):
    g = _load(name)
    kmax = int(g["k_max"])
    prob = oracle.Problem(g["X"], g["y"], k_fold=int(g["k_fold"]))
    s = oracle.step(prob, [kmax], list(g["committed"]), list(g["candidates"]), method=str(g["method"]))
    np.testing.assert_array_equal(s["nn_idx"], g["nn_idx"])
    np.testing.assert_array_equal(s["nn_dist"], g["nn_dist"])


def test_fp64_pipeline_close_to_fp32():
    g = _load("pooled_fwd_3000")
    prob = oracle.Problem(g["X"], g["y"], k_fold=int(g["k_fold"]))
    committed = list(g["ordering"][:3])
    s32 = oracle.step(prob, [10], committed, [g["ordering"][3]], want_neighbours=False)
    s64 = oracle.step(prob, [10], committed, [g["ordering"][3]], precision=1, want_neighbours=False)
    e32 = oracle.rmse32(s32["sq32"][0, 0])
    e64 = np.sqrt(s64["sq64"][0, 0].mean())
    assert e32 == g["errors"][3]
    assert abs(float(e32) - e64) / e64 < 1e-3


@pytest.mark.skipif(not ref.available(), reason="reference library not built here")
def test_live_reference_random_case():
    """Fresh seeded case against the reference library itself (where it is built)."""
    from speedynn_b200 import datagen
    s = datagen.generate(257, 1, 11, n_mag=5, seed=99)
    for method, nf, kv, kf in [("forward", 4, [2, 9, 5], 7), ("backward", 6, [3], 4)]:
        r = ref.train(s.Xtrain, s.ytrain, kv, nf, kf, method)
        o = oracle.select(oracle.Problem(s.Xtrain, s.ytrain, k_fold=kf), kv, nf, method)
        np.testing.assert_array_equal(o["ordering"], r["ordering"])
        np.testing.assert_array_equal(o["errors"], r["errors"][0])
        assert o["best_k"] == r["best_k"]


MODEL_CASES = golden_cases("model_")


@pytest.mark.parametrize("name", MODEL_CASES)
def test_numpy_restatement_matches_reference_models(name):
    """Loss lists (first decides) and the classification model: the NumPy
    restatement reproduces speedynn's own outputs, every loss of every step."""
    g = dict(np.load(os.path.join(GDIR, name + ".npz")))
    prob = oracle.Problem(g["X"], g["y"], k_fold=int(g["k_fold"]))
    o = oracle.np_select(prob, list(g["k_vals"]), int(g["num_features"]), str(g["method"]),
                         loss_functions=list(g["loss_functions"]), model_type=int(g["model_type"]),
                         auto_feature=bool(g["auto_feature"]))
    np.testing.assert_array_equal(o["ordering"], g["ordering"])
    np.testing.assert_array_equal(o["mask"], g["mask"])
    np.testing.assert_array_equal(o["errors_all"], g["errors_all"])
    assert o["best_k"] == int(g["best_k"])
    assert o["num_final"] == int(g["num_final"])
