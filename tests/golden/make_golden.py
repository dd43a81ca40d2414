"""Generate golden vectors from speedynn's own CPU backend.

Runs the reference library built by ``oracle/Makefile`` from the reference
sources (``oracle/_ref/libspeedynn_ref.so``) on seeded inputs and stores
inputs + outputs as ``tests/golden/<case>.npz``.  Needs the reference sources
(only this generator does); the committed .npz files are what the tests use.

    python tests/golden/make_golden.py                 # every fixture
    python tests/golden/make_golden.py --only models   # the model_* cases (losses, classification)

Each case stores: X, y, method, k_vals, num_features, k_fold, auto_feature and
the reference outputs ordering, mask, errors (loss 0), best_k, num_final.
Neighbour cases additionally store the lists returned by the reference's
get_k_nearest_neighbors_cpu (speedynn/lib/cpu.c:128-168) after committing
``committed`` with update_current_dist_matrix_cpu (cpu.c:217-231).  Model
cases (``model_*``) run the reference with a list of loss ids (the first
decides) and the regression or classification model, and store every loss of
every step (``errors_all``, the reference's [loss][p] layout).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from speedynn_b200 import datagen  # noqa: E402


def _gen(n, p, seed, n_mag=5):
    s = datagen.generate(n, 1, p, n_mag=n_mag, seed=seed)
    return s.Xtrain, s.ytrain


def cases():
    out = []
    # the reference's own example (examples/simple.py:8-31): sklearn make_regression, forward,
    # k in 2..50, 3 features, 10 folds
    from sklearn.datasets import make_regression
    X, y = make_regression(n_samples=100, n_features=10, n_informative=3, noise=0.5, coef=False, bias=0.0,
                           random_state=0)
    out.append(("simple_example", X, y, "forward", list(range(2, 51)), 3, 10, False))

    # pooled CPU workload: [X_val; X_train] of the 2k/1k/20 generator, k_fold=3 puts the
    # validation block in fold 0; k=10, 8 features
    s = datagen.generate(2000, 1000, 20, n_mag=5, seed=0)
    Xp = np.concatenate([s.Xval, s.Xtrain])
    yp = np.concatenate([s.yval, s.ytrain])
    out.append(("pooled_fwd_3000", Xp, yp, "forward", [10], 8, 3, False))

    X, y = _gen(150, 12, 11)
    out.append(("bwd_default_k", X, y, "backward", list(range(1, 10)), 4, 10, False))

    X, y = _gen(103, 9, 12)
    out.append(("extra_partial_fold", X, y, "forward", [3, 5], 4, 10, False))

    # duplicated rows -> exact distance ties resolved by index
    X, y = _gen(60, 9, 13)
    X = np.concatenate([X, X])
    y = np.concatenate([y, y])
    rng = np.random.default_rng(13)
    perm = rng.permutation(X.shape[0])
    out.append(("duplicate_rows", X[perm], y[perm], "forward", [4, 1], 4, 5, False))

    # integer-valued features: massive distance ties
    rng = np.random.default_rng(14)
    X = rng.integers(0, 4, size=(90, 7)).astype(np.float32)
    y = (X[:, 2] - 0.5 * X[:, 5] + rng.normal(0, 0.1, 90)).astype(np.float32)
    out.append(("quantized_ties", X, y, "forward", [3, 6], 5, 6, False))
    out.append(("quantized_ties_bwd", X, y, "backward", [3, 6], 2, 6, False))

    # k larger than the available neighbours (k_fold=2, 10 valid columns): padding index 0
    X, y = _gen(20, 9, 15)
    out.append(("k_exceeds_neighbours", X, y, "forward", [12, 3], 3, 2, False))

    # a constant feature and a duplicated feature (candidate-error exact tie -> lower index)
    X, y = _gen(120, 10, 16)
    X = X.copy()
    X[:, 3] = 1.25
    X[:, 6] = X[:, 1]
    out.append(("const_and_dup_feature", X, y, "forward", [5], 6, 4, False))
    out.append(("const_and_dup_feature_bwd", X, y, "backward", [5], 2, 4, False))

    X, y = _gen(200, 10, 17)
    out.append(("auto_forward", X, y, "forward", [4, 8], 2, 10, True))
    out.append(("auto_backward", X, y, "backward", [4, 8], 2, 10, True))
    return out


def _classes(n, p, seed, n_cls=3):
    """Integer class labels from a noisy linear rule on two features."""
    X, _ = _gen(n, p, seed)
    rng = np.random.default_rng(seed)
    score = X[:, 0] - 0.7 * X[:, 2] + rng.normal(0, 0.4, n)
    y = np.digitize(score, np.quantile(score, np.linspace(0, 1, n_cls + 1)[1:-1])).astype(np.float32)
    return X, y


def model_cases():
    """(name, X, y, method, k_vals, num_features, k_fold, auto, loss ids, model type)."""
    out = []
    X, y = _gen(140, 9, 21)
    out.append(("model_losses_fwd", X, y, "forward", [3, 7], 4, 5, False, [1, 0, 2, 3, 4, 5, 6, 7, 8], 0))
    X, y = _gen(120, 10, 22)
    out.append(("model_mad_bwd", X, y, "backward", [2, 5], 3, 4, False, [2, 0], 0))
    X, y = _gen(90, 9, 23)
    out.append(("model_std_fwd", X, y, "forward", [4], 3, 3, False, [5, 8, 0], 0))
    X, y = _gen(110, 9, 27)
    out.append(("model_rmse_norm_bwd_auto", X, y, "backward", [3], 2, 5, True, [1], 0))
    X, y = _classes(150, 9, 24)
    out.append(("model_classif_fwd", X, y, "forward", [1, 4, 6], 4, 5, False, [4, 0], 1))
    X, y = _classes(130, 10, 25)
    out.append(("model_classif_bwd", X, y, "backward", [3, 6], 2, 5, False, [4], 1))
    X, y = _classes(160, 9, 26)
    out.append(("model_classif_auto", X, y, "forward", [2, 5], 2, 4, True, [4, 2], 1))
    return out


def make_model_cases():
    for name, X, y, method, kv, nf, kf, auto, losses, model in model_cases():
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        r = ref.train(X, y, kv, nf, kf, method, auto_feature=auto, loss_functions=losses, model_type=model)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, y=y, method=method,
                            k_vals=np.asarray(kv, np.int32), num_features=nf, k_fold=kf, auto_feature=int(auto),
                            loss_functions=np.asarray(losses, np.int32), model_type=model,
                            ordering=r["ordering"], mask=r["mask"], errors_all=r["errors"], best_k=r["best_k"],
                            num_final=r["num_final"])
        print(f"{name}: n={X.shape[0]} p={X.shape[1]} {method} losses={losses} model={model} -> "
              f"{r['ordering']} k*={r['best_k']}")


NEIGHBOUR_CASES = [
    # (case, k_max, committed, method, candidates)
    ("extra_partial_fold", 5, [2], "forward", [0, 1, 3, 8]),
    ("duplicate_rows", 4, [1, 4], "forward", [0, 2, 3, 7]),
    ("quantized_ties", 6, [2], "forward", [0, 1, 3, 4, 5, 6]),
    ("quantized_ties_bwd", 6, [0, 4], "backward", [1, 2, 3, 5, 6]),
    ("k_exceeds_neighbours", 12, [0], "forward", [1, 2, 5]),
]


def main():
    made = {}
    for name, X, y, method, kv, nf, kf, auto in cases():
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        r = ref.train(X, y, kv, nf, kf, method, auto_feature=auto)
        made[name] = (X, y)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, y=y, method=method,
                            k_vals=np.asarray(kv, np.int32), num_features=nf, k_fold=kf, auto_feature=int(auto),
                            ordering=r["ordering"], mask=r["mask"], errors=r["errors"][0], best_k=r["best_k"],
                            num_final=r["num_final"])
        print(f"{name}: n={X.shape[0]} p={X.shape[1]} {method} -> {r['ordering']} k*={r['best_k']}")
    for name, kmax, committed, method, cands in NEIGHBOUR_CASES:
        X, y = made[name]
        kf = int(np.load(os.path.join(HERE, name + ".npz"))["k_fold"])
        idx, dist = ref.neighbours(X, kmax, kf, committed, method == "backward", cands)
        np.savez_compressed(os.path.join(HERE, f"nn_{name}.npz"), X=X, y=y, k_fold=kf, k_max=kmax,
                            committed=np.asarray(committed, np.int32), method=method,
                            candidates=np.asarray(cands, np.int32), nn_idx=idx, nn_dist=dist)
        print(f"nn_{name}: {idx.shape}")
    # loss utility (speedynn/lib/loss_functions.c:6-38) on fixed vectors, all nine ids
    rng = np.random.default_rng(18)
    lab = rng.uniform(0, 3, 257).astype(np.float32)
    pre = (lab + rng.normal(0, 0.3, 257)).astype(np.float32)
    vals = np.array([ref.loss(lab, pre, i) for i in range(9)], np.float32)
    np.savez_compressed(os.path.join(HERE, "losses.npz"), labels=lab, preds=pre, values=vals)
    print("losses:", vals)


if __name__ == "__main__":
    if sys.argv[1:] == ["--only", "models"]:
        make_model_cases()
    else:
        main()
        make_model_cases()
