"""GPU parity: the CUDA path against the reference's golden vectors and the
CPU oracle.  Bar: ordering, mask, best k and neighbour indices bit-exact;
FP32 errors bit-exact (the reference's own FP32 RMSE); FP64 errors within
1e-9 relative of the oracle's FP64 sum of the same residuals."""
import ctypes
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
SELECT_CASES = [n for n in golden_cases() if not n.startswith(("nn_", "model_", "config_")) and n != "losses"]
# scoring variants: rows-per-lane kernel; TMA-fed kernel with the default seed
# step; TMA-fed kernel with seeded bounds from the second forward step on
VARIANTS = ["lanes", "tma", "tma_seeded"]
NN_CASES = golden_cases("nn_")
ERR64_RTOL = 1e-9


def _g(name):
    return dict(np.load(os.path.join(GDIR, name + ".npz")))


@pytest.mark.parametrize("name", SELECT_CASES)
def test_dropin_api_matches_reference_golden(name):
    g = _g(name)
    sel = IncrementalNNFeatureSelection(g["X"], g["y"], k_vals=list(g["k_vals"]), auto_feature=bool(g["auto_feature"]),
                                        num_features=int(g["num_features"]), k_fold=int(g["k_fold"]),
                                        method=str(g["method"]))
    sel.train()
    np.testing.assert_array_equal(sel.get_selected_ordering(), g["ordering"])
    np.testing.assert_array_equal(sel.get_selected_dimensions(), g["mask"])
    np.testing.assert_array_equal(sel.get_selected_errors()[:, 0], g["errors"])
    assert sel.get_optimal_model_k() == int(g["best_k"])
    assert sel.num_final_features == int(g["num_final"])


@pytest.mark.parametrize("name", ["pooled_fwd_3000", "bwd_default_k", "quantized_ties_bwd", "auto_backward"])
def test_c_abi_reference_entry_points(name):
    """The SWIG-level names, called through ctypes exactly as the reference's wrapper would."""
    g = _g(name)
    L = _lib.lib()
    X = np.ascontiguousarray(g["X"], np.float32)
    y = np.ascontiguousarray(g["y"], np.float32)
    kv = np.ascontiguousarray(g["k_vals"], np.int32)
    lf = np.zeros(1, np.int32)
    n, d = X.shape
    fn = L.train_forward_selection if str(g["method"]) == "forward" else L.train_backward_selection
    nf = int(g["num_features"]) if not int(g["auto_feature"]) else d
    rc = fn(ptr(X, _f32p), n, d, ptr(y, _f32p), n, ptr(kv, _i32p), kv.size, nf, int(g["k_fold"]), ptr(lf, _i32p), 1,
            int(g["auto_feature"]), 0)
    assert rc == int(g["num_final"]), _lib.last_error()
    mask = np.zeros(d, np.int32)
    order = np.zeros(d, np.int32)
    errs = np.zeros(d, np.float32)
    L.get_selected_dimensions(ptr(mask, _i32p), d)
    L.get_selected_ordering(ptr(order, _i32p), d)
    L.get_selected_errors(ptr(errs, _f32p), d)
    np.testing.assert_array_equal(order, g["ordering"])
    np.testing.assert_array_equal(mask, g["mask"])
    np.testing.assert_array_equal(errs, g["errors"])
    assert L.get_final_optimal_model_k() == int(g["best_k"])


@pytest.mark.parametrize("name", NN_CASES)
def test_neighbour_lists_match_reference(name):
    g = _g(name)
    committed = list(g["committed"])
    method = str(g["method"])
    kmax = int(g["k_max"])
    X, y = g["X"], g["y"]
    p = X.shape[1]
    # drive the selector to the committed state, then score once with lists kept
    with Selector(X, y, k_vals=[kmax], num_features=p if method == "forward" else 0, method=method,
                  k_fold=int(g["k_fold"])) as s:
        s.commit_sequence(committed)
        s.keep_neighbours(True)
        assert s.step()
        cands, idx, dist = s.neighbours()
    want = list(g["candidates"])
    for ci, c in enumerate(want):
        j = list(cands).index(c)
        np.testing.assert_array_equal(idx[j], g["nn_idx"][ci])
        np.testing.assert_array_equal(dist[j], g["nn_dist"][ci])


def configure(sel, variant):
    """Select a scoring variant on a Selector (results must not depend on it)."""
    if variant == "lanes":
        sel.set_kernel(1)
    elif variant in ("tma", "tma_seeded"):
        sel.set_kernel(3)
        if variant == "tma_seeded":
            sel.set_seed_step(1)


def _tma_skip(variant, k_vals):
    if variant.startswith("tma") and max(k_vals) > 64:
        pytest.skip("the TMA-fed kernel handles k_max <= 64")


def _holdout_case(n_train, n_val, p, seed, k_vals, nf, method, variant="auto", **kw):
    s = datagen.generate(n_train, n_val, p, n_mag=kw.pop("n_mag", 5), seed=seed, **kw)
    prob = oracle.Problem(s.Xtrain, s.ytrain, s.Xval, s.yval)
    o = oracle.select(prob, k_vals, nf, method)
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=k_vals, num_features=nf, method=method) as sel:
        configure(sel, variant)
        r = sel.run()
    return o, r


@pytest.mark.parametrize("args", [
    (2000, 1000, 20, 0, [10], 8, "forward"),          # the CPU-size forward workload
    (1500, 700, 16, 7, [1, 4, 9], 5, "forward"),
    (1200, 601, 18, 8, [5], 12, "backward"),
    (999, 333, 12, 9, [3, 30], 4, "forward"),          # k_max 30 -> 4 candidates per thread
    (700, 257, 10, 10, [64], 3, "forward"),            # k_max 64 -> 2 per thread
    (400, 130, 9, 11, [150, 2], 2, "backward"),        # k_max 150 -> 1 per thread
    (1290, 410, 11, 12, [17, 2], 5, "forward"),        # 32-slot lists; last 256-column stage holds one chunk
    (830, 300, 10, 13, [20], 6, "backward"),           # backward with 32-slot lists
    (1100, 333, 13, 14, [50, 33, 3], 5, "forward"),    # 64-slot lists, k_max 50
    (900, 250, 11, 15, [40], 5, "backward"),           # backward with 64-slot lists
])
@pytest.mark.parametrize("variant", VARIANTS)
def test_holdout_matches_oracle(args, variant):
    n_train, n_val, p, seed, kv, nf, method = args
    _tma_skip(variant, kv)
    o, r = _holdout_case(n_train, n_val, p, seed, kv, nf, method, variant=variant)
    np.testing.assert_array_equal(r["ordering"], o["ordering"])
    np.testing.assert_array_equal(r["mask"], o["mask"])
    np.testing.assert_array_equal(r["errors"], o["errors"])
    np.testing.assert_array_equal(r["step_best_k"], o["step_best_k"])
    np.testing.assert_allclose(r["errors64"], o["errors64"], rtol=ERR64_RTOL, atol=0)
    assert r["best_k"] == o["best_k"] and r["num_final"] == o["num_final"]


def test_holdout_neighbours_match_oracle():
    s = datagen.generate(3000, 1100, 24, n_mag=6, n_heavy=4, seed=21)
    kv = [7, 2]
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=kv, num_features=4, method="forward") as sel:
        for _ in range(2):
            assert sel.step()
        committed = list(sel.results()["ordering"][:2])
        sel.keep_neighbours(True)
        assert sel.step()
        cands, idx, dist = sel.neighbours()
    prob = oracle.Problem(s.Xtrain, s.ytrain, s.Xval, s.yval)
    o = oracle.step(prob, kv, committed, list(cands))
    np.testing.assert_array_equal(idx, o["nn_idx"])
    np.testing.assert_array_equal(dist, o["nn_dist"])


def test_duplicate_training_rows_tie_rule():
    """2 % duplicated training rows (exact distance ties) on the mixture generator."""
    s = datagen.generate(2500, 800, 14, n_mag=6, seed=31, mixture=True, dup_frac=0.02)
    o, r = None, None
    prob = oracle.Problem(s.Xtrain, s.ytrain, s.Xval, s.yval)
    o = oracle.select(prob, [5, 50], 5, "forward")
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=[5, 50], num_features=5, method="forward") as sel:
        r = sel.run()
    np.testing.assert_array_equal(r["ordering"], o["ordering"])
    np.testing.assert_array_equal(r["errors"], o["errors"])


def test_step_api_equals_run_and_is_deterministic():
    s = datagen.generate(4096, 2048, 30, n_mag=8, n_heavy=5, seed=41)
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=[10], num_features=6, method="forward") as sel:
        a = sel.run()
        b = sel.run()
        sel.reset()
        n = 0
        while sel.step():
            n += 1
        c = sel.results()
    assert n == 6
    for k in ("ordering", "mask", "errors", "errors64", "step_best_k"):
        np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(a[k], c[k])


def test_nan_labels_report_no_winner():
    s = datagen.generate(300, 100, 9, n_mag=5, seed=51)
    yv = s.yval.copy()
    yv[:] = np.nan
    with Selector(s.Xtrain, s.ytrain, s.Xval, yv, k_vals=[3], num_features=2) as sel:
        with pytest.raises(_lib.SnnError) as e:
            sel.run()
    assert e.value.code == _lib.SNN_ERR_NO_WINNER


def test_headline_shape_subset_rows_against_oracle():
    """The 64k x 32k x 60 forward workload at a reduced row count: neighbour
    lists and errors against the oracle for the first two steps."""
    s = datagen.generate(16384, 1024, 60, n_mag=8, n_heavy=10, seed=2)
    kv = [10]
    prob = oracle.Problem(s.Xtrain, s.ytrain, s.Xval, s.yval)
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=kv, num_features=3, method="forward") as sel:
        sel.keep_neighbours(True)
        assert sel.step()
        cands, idx, dist = sel.neighbours()
        r = sel.results()
    o = oracle.step(prob, kv, [], list(cands))
    np.testing.assert_array_equal(idx, o["nn_idx"])
    errs = np.array([oracle.rmse32(o["sq32"][ci, 0]) for ci in range(len(cands))])
    w = min(range(len(cands)), key=lambda ci: (errs[ci], cands[ci]))  # ties: smallest feature id
    assert r["ordering"][0] == cands[w]
    assert r["errors"][0] == errs[w]


@pytest.mark.parametrize("args", [
    (8192, 2048, 40, 61, [10], 9, dict(n_heavy=6)),
    (6000, 1500, 24, 62, [5, 50], 7, dict(mixture=True, dup_frac=0.02)),
    (3000, 0, 20, 63, [3, 7], 6, dict()),          # CV mode (n_val=0 -> rows are the training points)
    (2500, 700, 18, 64, [17, 31], 6, dict()),      # 32-slot lists
])
def test_seeded_bounds_equal_first_pass(args):
    """Forward steps whose starting bounds come from the commit's seed columns
    (from the second step on) against steps that always run the first pass:
    identical orderings, errors and neighbour lists."""
    n_train, n_val, p, seed, kv, nf, kw = args
    s = datagen.generate(n_train, max(n_val, 1), p, n_mag=6, seed=seed, **kw)
    Xv, yv = (s.Xval, s.yval) if n_val else (None, None)
    out = {}
    for seed_step in (1, 10 ** 6):
        with Selector(s.Xtrain, s.ytrain, Xv, yv, k_vals=kv, num_features=nf, method="forward", k_fold=5) as sel:
            sel.set_seed_step(seed_step)
            r = sel.run()
            sel.reset()
            for _ in range(4):
                sel.step()
            sel.keep_neighbours(True)
            sel.step()
            out[seed_step] = (r, sel.neighbours())
    (ra, na), (rb, nb) = out[1], out[10 ** 6]
    for k in ("ordering", "mask", "errors", "errors64", "step_best_k"):
        np.testing.assert_array_equal(ra[k], rb[k])
    for a, b in zip(na, nb):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("kv", [[10], [50, 7]])
def test_large_problem_sampled_rows_match_oracle(kv):
    """At a size the oracle cannot hold whole (120,000 training x 30,000
    validation rows, mixture features, 2 % duplicated training rows): after
    three committed steps, the fourth step's neighbour lists of 96 sampled
    validation rows equal the oracle's, which recomputes those rows'
    distances from X in commit order.  Both k = 10 (16-slot lists) and
    k = 50 (64-slot lists) run the TMA-fed kernel, the fourth step from seed
    bounds when the seed step is 3."""
    s = datagen.generate(120000, 30000, 24, n_mag=8, seed=55, mixture=True, dup_frac=0.02)
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=kv, num_features=4, method="forward") as sel:
        sel.set_seed_step(3)
        for _ in range(3):
            assert sel.step()
        committed = [int(c) for c in sel.results()["ordering"][:3]]
        sel.keep_neighbours(True)
        assert sel.step()
        cands, idx, dist = sel.neighbours()
    rows = np.sort(np.random.default_rng(5).choice(s.Xval.shape[0], 96, replace=False)).astype(np.int32)
    prob = oracle.Problem(s.Xtrain, s.ytrain, s.Xval, s.yval)
    o = oracle.step(prob, kv, committed, list(cands), rows=rows)
    np.testing.assert_array_equal(idx[:, rows], o["nn_idx"])
    np.testing.assert_array_equal(dist[:, rows], o["nn_dist"])


def test_noalloc_backward_step_matches_handle():
    """The allocation-free entry point on a backward step (it has no per-row
    distance maxima, so its backward filter flags every chunk and scores it
    exactly): same winner, best k and FP32 error as a handle's first step."""
    import ctypes

    import torch

    s = datagen.generate(1500, 400, 11, n_mag=5, seed=73)
    k_vals = np.array([4, 9], np.int32)
    n_tr, n_val, p = s.Xtrain.shape[0], s.Xval.shape[0], s.Xtrain.shape[1]
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, k_vals=k_vals, num_features=p - 1, method="backward") as sel:
        ref = sel.run()
    want = (int(ref["ordering"][p - 1]), int(ref["step_best_k"][p - 1]), ref["errors"][p - 1])
    ld = (n_tr + 63) // 64 * 64
    Dh = np.zeros((n_val, ld), np.float32)
    for k in range(p - 1, -1, -1):  # full distance, dims in descending order
        diff = s.Xval[:, k][:, None] - s.Xtrain[:, k][None, :]
        Dh[:, :n_tr] = Dh[:, :n_tr] + diff * diff
    Dh[:, n_tr:] = np.inf
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(Dh).to(dev)
    XT = torch.zeros((p, ld), dtype=torch.float32, device=dev)
    XT[:, :n_tr] = torch.from_numpy(np.ascontiguousarray(s.Xtrain.T)).to(dev)
    XV = torch.from_numpy(np.ascontiguousarray(s.Xval.T)).to(dev)
    yt = torch.from_numpy(s.ytrain).to(dev)
    yv = torch.from_numpy(s.yval).to(dev)
    cands = np.arange(p, dtype=np.int32)
    e32 = torch.zeros((p, k_vals.size), dtype=torch.float32, device=dev)
    e64 = torch.zeros((p, k_vals.size), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    L = _lib.lib()
    rc = L.snn_score_step_noalloc(D.data_ptr(), ld, XT.data_ptr(), XV.data_ptr(), n_val, yt.data_ptr(), yv.data_ptr(),
                                  n_val, n_tr, p, ptr(cands, _i32p), p, ptr(k_vals, _i32p), k_vals.size, 1,
                                  e32.data_ptr(), e64.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert rc == 0, _lib.last_error()
    err = e32.cpu().numpy()
    best = [(err[c].min(), c, int(k_vals[int(np.argmin(err[c]))])) for c in range(p)]
    e, c, k = min(best, key=lambda t: (t[0], t[1]))
    assert (c, k) == want[:2] and e == want[2]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("case", [
    dict(n_train=300, n_val=70, p=2, kv=[3], nf=2, method="forward"),       # fewer candidates than a warp's four
    dict(n_train=260, n_val=50, p=3, kv=[2, 5], nf=1, method="backward"),
    dict(n_train=37, n_val=29, p=4, kv=[6, 1], nf=3, method="forward"),      # less than one 64-column chunk
    dict(n_train=20, n_val=13, p=5, kv=[30, 3], nf=2, method="forward"),     # k > training rows: padded lists
    dict(n_train=25, n_val=9, p=4, kv=[28], nf=2, method="backward"),
    dict(n_train=45, n_val=11, p=4, kv=[50, 2], nf=2, method="forward"),     # 64-slot lists, k > training rows
    dict(n_train=70, n_val=17, p=3, kv=[33], nf=2, method="backward"),
])
def test_edge_shapes_match_oracle(case, variant):
    rng = np.random.default_rng(case["n_train"] * 7 + case["p"])
    Xt = rng.normal(size=(case["n_train"], case["p"])).astype(np.float32)
    Xv = rng.normal(size=(case["n_val"], case["p"])).astype(np.float32)
    yt = (Xt[:, 0] - 0.5 * Xt[:, -1] + rng.normal(0, 0.1, case["n_train"])).astype(np.float32)
    yv = (Xv[:, 0] - 0.5 * Xv[:, -1] + rng.normal(0, 0.1, case["n_val"])).astype(np.float32)
    _tma_skip(variant, case["kv"])
    prob = oracle.Problem(Xt, yt, Xv, yv)
    o = oracle.select(prob, case["kv"], case["nf"], case["method"])
    with Selector(Xt, yt, Xv, yv, k_vals=case["kv"], num_features=case["nf"], method=case["method"]) as sel:
        configure(sel, variant)
        r = sel.run()
    np.testing.assert_array_equal(r["ordering"], o["ordering"])
    np.testing.assert_array_equal(r["mask"], o["mask"])
    np.testing.assert_array_equal(r["errors"], o["errors"])
    np.testing.assert_array_equal(r["step_best_k"], o["step_best_k"])
    assert r["best_k"] == o["best_k"] and r["num_final"] == o["num_final"]


@pytest.mark.parametrize("variant", ["auto", "lanes", "tma_seeded"])
def test_forward_bound_overflow_and_ties(variant):
    """A dominant feature whose squared differences overflow to inf (selected
    first) leaves the committed distances non-finite, so first-pass and seed
    bounds are +inf (no bound); quantized values give ties at the bound."""
    rng = np.random.default_rng(77)
    n_train, n_val, p = 900, 260, 7
    Xt = rng.integers(-3, 4, size=(n_train, p)).astype(np.float32)
    Xv = rng.integers(-3, 4, size=(n_val, p)).astype(np.float32)
    Xt[:, 2] *= np.float32(1e19)
    Xv[:, 2] *= np.float32(1e19)
    yt = (np.sign(Xt[:, 2]) + 0.3 * Xt[:, 0] + rng.normal(0, 0.05, n_train)).astype(np.float32)
    yv = (np.sign(Xv[:, 2]) + 0.3 * Xv[:, 0] + rng.normal(0, 0.05, n_val)).astype(np.float32)
    prob = oracle.Problem(Xt, yt, Xv, yv)
    o = oracle.select(prob, [1, 6, 21], 4, "forward")
    with Selector(Xt, yt, Xv, yv, k_vals=[1, 6, 21], num_features=4, method="forward") as sel:
        configure(sel, variant)
        r = sel.run()
    assert o["ordering"][0] == 2
    np.testing.assert_array_equal(r["ordering"], o["ordering"])
    np.testing.assert_array_equal(r["errors"], o["errors"])
    np.testing.assert_array_equal(r["step_best_k"], o["step_best_k"])
    assert r["best_k"] == o["best_k"] and r["num_final"] == o["num_final"]


@pytest.mark.parametrize("method", ["forward", "backward"])
def test_resume_from_committed_prefix_equals_uninterrupted_run(method):
    """Checkpoint / resume: committing the first winners of a run (warm start)
    and stepping on reproduces the rest of that run bit for bit."""
    s = datagen.generate(3000, 1200, 16, n_mag=6, n_heavy=3, seed=61)
    kw = dict(k_vals=[3, 9], num_features=7 if method == "forward" else 4, method=method)
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, **kw) as sel:
        full = sel.run()
    p = s.Xtrain.shape[1]
    n_steps = kw["num_features"] if method == "forward" else p - kw["num_features"]
    # winners in commit order: forward fills slots from the front, backward from the back
    slots = list(range(n_steps)) if method == "forward" else [p - 1 - t for t in range(n_steps)]
    winners = [int(full["ordering"][i]) for i in slots]
    cut = 3
    with Selector(s.Xtrain, s.ytrain, s.Xval, s.yval, **kw) as sel:
        sel.commit_sequence(winners[:cut])
        while sel.step():
            pass
        res = sel.results()
    for i in slots[cut:]:
        assert res["ordering"][i] == full["ordering"][i]
        assert res["errors"][i] == full["errors"][i]
        assert res["errors64"][i] == full["errors64"][i]
        assert res["step_best_k"][i] == full["step_best_k"][i]
    np.testing.assert_array_equal(res["mask"], full["mask"])


def _first_step_data(kind, rng):
    n_train, n_val, p = 3000, 700, 9
    Xt = rng.normal(size=(n_train, p)).astype(np.float32)
    Xv = rng.normal(size=(n_val, p)).astype(np.float32)
    if kind == "duplicates":  # repeated training rows: tie groups of two and three
        Xt[1000:1300] = Xt[:300]
        Xt[2000:2100] = Xt[:100]
    elif kind == "quantized":  # integer values: tie groups far larger than a thread orders
        Xt = np.round(Xt * 2).astype(np.float32)
        Xv = np.round(Xv * 2).astype(np.float32)
    elif kind == "nonfinite":  # NaN and inf values never enter a list
        Xt[::17, 2] = np.nan
        Xt[::29, 4] = np.inf
        Xv[::13, 4] = -np.inf
        Xv[::31, 6] = np.nan
    elif kind == "few_rows":  # k above the training rows: padded lists
        Xt, n_train = Xt[:40], 40
    yt = (Xt[:, 0] - 0.5 * np.nan_to_num(Xt[:, 1], posinf=0.0) + rng.normal(0, 0.1, n_train)).astype(np.float32)
    yv = (Xv[:, 0] - 0.5 * Xv[:, 1] + rng.normal(0, 0.1, n_val)).astype(np.float32)
    return Xt, yt, Xv, yv


@pytest.mark.parametrize("kind", ["plain", "duplicates", "quantized", "nonfinite", "few_rows"])
@pytest.mark.parametrize("kv", [[10], [3, 45], [64, 1], [33]])
def test_sorted_first_steps_equal_scan(kind, kv):
    """The first two forward steps from sorted feature columns (a window
    around each row's value, then a walk of the first winner's values) against
    the scan of every column: identical neighbour lists of every candidate and
    row at both steps, and identical selections (quantized values exercise the
    hand-back to the scan).  k above 32 takes the walk whose first 64 columns
    fill the list at once (k = 64 exactly, k = 33 and 45 odd)."""
    rng = np.random.default_rng(101)
    Xt, yt, Xv, yv = _first_step_data(kind, rng)
    out = {}
    for sorted_start in (True, False):
        with Selector(Xt, yt, Xv, yv, k_vals=kv, num_features=3, method="forward") as sel:
            sel.set_sorted_start(sorted_start)
            r = sel.run()
            sel.reset()
            sel.keep_neighbours(True)
            lists = []
            for _ in range(2):
                assert sel.step()
                lists.append(sel.neighbours())
            out[sorted_start] = (r, lists)
    (ra, la), (rb, lb) = out[True], out[False]
    for k in ("ordering", "mask", "errors", "errors64", "step_best_k"):
        np.testing.assert_array_equal(ra[k], rb[k])
    for na, nb in zip(la, lb):
        for a, b in zip(na, nb):
            np.testing.assert_array_equal(a, b)
    if kind != "nonfinite":
        prob = oracle.Problem(Xt, yt, Xv, yv)
        o = oracle.select(prob, kv, 3, "forward")
        np.testing.assert_array_equal(ra["ordering"], o["ordering"])
        np.testing.assert_array_equal(ra["errors"], o["errors"])
