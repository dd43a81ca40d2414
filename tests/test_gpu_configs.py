"""Parity at the benchmark workloads' own shapes.

Each workload is generated at full size and run on the GPU with the library's
default options.  Two checks per workload:

* the whole selection (for bwd-50k its first 10 removals, for fwd-200k its
  first 4 steps) against the oracle's run of the same inputs, stored by
  tests/golden/make_config_golden.py
  (ordering, mask, best k per step and FP32 errors bit for bit; FP64 errors
  within 1e-9 relative);
* at a later step, the neighbour lists of 256 seeded validation rows for
  EVERY candidate, and those rows' kNN predictions, against the oracle, which
  rebuilds the rows' distances from X in the committed order
  (speedynn/lib/cpu.c:217-231) and scans them as speedynn/lib/cpu.c:128-168.

Workloads: fwd-64k (65,536 x 32,768 rows, p=60, k=10, 15 steps), bwd-50k
(50,000 x 25,000 rows, p=120 -> 20, k=5, 100 removals) and fwd-200k
(200,000 x 100,000 rows, p=100, k=50, 2 % duplicated training rows; an 80 GB
distance matrix).
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle
from speedynn_b200 import datagen
from speedynn_b200.selector import Selector

pytestmark = pytest.mark.gpu

ERR64_RTOL = 1e-9
N_SAMPLE = 256


def _fixture(name):
    path = os.path.join(ROOT, "tests", "golden", f"config_{name.replace('-', '')}.npz")
    return dict(np.load(path))


def _sha(split):
    h = hashlib.sha256()
    for a in (split.Xtrain, split.ytrain, split.Xval, split.yval):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _sample_rows(n, seed):
    return np.sort(np.random.default_rng(seed).choice(n, N_SAMPLE, replace=False)).astype(np.int32)


def _check_sampled_step(split, k, method, committed, sel, rows):
    """After ``committed`` is in the selector's distances and one more step ran
    with lists kept: lists and predictions of ``rows`` for every candidate."""
    cands, _ = sel.predictions(rows[:1])
    idx, dist = sel.neighbours_rows(rows)
    _, pred = sel.predictions(rows)
    prob = oracle.Problem(split.Xtrain, split.ytrain, split.Xval, split.yval)
    o = oracle.step(prob, [k], committed, list(cands), method=method, rows=rows)
    np.testing.assert_array_equal(idx, o["nn_idx"])
    np.testing.assert_array_equal(dist, o["nn_dist"])
    e = (split.yval[rows][None, None, :] - pred).astype(np.float32)
    np.testing.assert_array_equal((e * e).astype(np.float32), o["sq32"])


def _check_selection(res, g):
    """The fixture's steps bit for bit; the final mask, best k and feature
    count when the fixture covers the whole run."""
    slots = [int(i) for i in g["slots"]]
    for key in ("ordering", "errors", "step_best_k"):
        np.testing.assert_array_equal(np.asarray(res[key])[slots], g[key][slots], err_msg=key)
    np.testing.assert_allclose(np.asarray(res["errors64"])[slots], g["errors64"][slots], rtol=ERR64_RTOL, atol=0)
    if int(g["steps"]) == int(g["run_steps"]):
        np.testing.assert_array_equal(res["mask"], g["mask"])
        assert res["best_k"] == int(g["best_k"]) and res["num_final"] == int(g["num_final"])


def test_fwd64k_selection_and_last_step_lists():
    split, k, select = datagen.workload("fwd-64k")
    g = _fixture("fwd-64k")
    assert str(g["data_sha256"]) == _sha(split), "generator output differs from the fixture's inputs"
    with Selector(split.Xtrain, split.ytrain, split.Xval, split.yval, k_vals=[k], num_features=select,
                  method="forward") as sel:
        res = sel.run()
        _check_selection(res, g)
        # the last step again, its 46 candidates' lists kept (a seeded step)
        committed = [int(c) for c in g["commit_order"][:select - 1]]
        sel.commit_sequence(committed)
        sel.keep_neighbours(True)
        assert sel.step()
        _check_sampled_step(split, k, "forward", committed, sel, _sample_rows(split.Xval.shape[0], 64))


def test_bwd50k_first_removals_and_eleventh_removal_lists():
    split, k, select = datagen.workload("bwd-50k")
    g = _fixture("bwd-50k")
    assert str(g["data_sha256"]) == _sha(split), "generator output differs from the fixture's inputs"
    with Selector(split.Xtrain, split.ytrain, split.Xval, split.yval, k_vals=[k], num_features=select,
                  method="backward") as sel:
        res = sel.run()
        _check_selection(res, g)
        # the eleventh removal (110 candidates) after the first ten, lists kept
        committed = [int(c) for c in g["commit_order"][:10]]
        sel.commit_sequence(committed)
        sel.keep_neighbours(True)
        assert sel.step()
        _check_sampled_step(split, k, "backward", committed, sel, _sample_rows(split.Xval.shape[0], 65))


def test_fwd200k_first_steps_and_fifth_step_lists():
    split, k, select = datagen.workload("fwd-200k")
    g = _fixture("fwd-200k")
    assert str(g["data_sha256"]) == _sha(split), "generator output differs from the fixture's inputs"
    steps = int(g["steps"])
    with Selector(split.Xtrain, split.ytrain, split.Xval, split.yval, k_vals=[k], num_features=select,
                  method="forward") as sel:
        for _ in range(steps):
            assert sel.step()
        _check_selection(sel.results(), g)
        # on to the fifth step (four features committed: a seeded step), lists kept
        for _ in range(4 - steps):
            assert sel.step()
        committed = [int(c) for c in sel.results()["ordering"][:4]]
        sel.keep_neighbours(True)
        assert sel.step()
        _check_sampled_step(split, k, "forward", committed, sel, _sample_rows(split.Xval.shape[0], 66))
