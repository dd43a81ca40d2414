"""Full-size golden vectors for the benchmark workloads, from the CPU oracle.

The reference's own CPU backend cannot run these shapes (it has no holdout
mode and would take hours to days single-threaded), so the oracle
(``oracle/snn_oracle.c``, pinned bit for bit against the reference by
``tests/test_oracle_golden.py``) runs each whole greedy selection here, on all
host cores, and this script stores the result:

    fwd-64k   forward, 65,536 train x 32,768 validation rows, p=60, k=10, all 15 steps
    bwd-50k   backward, 50,000 x 25,000 rows, p=120 -> 20, k=5, the first STEPS_BWD
              removals (the restatement rebuilds each row's 120-feature distance every
              removal, so all 100 would take it most of a day)
    fwd-200k  forward, 200,000 x 100,000 rows, p=100, k=50, 2 % duplicated rows,
              the first STEPS_200K steps (the whole run would take the oracle days)

Each ``config_<name>.npz`` holds the selection outputs of the oracle's FP32
path (ordering, mask, FP32 errors, FP64 sums of the same residuals, best k per
step) and, for every step's winner, the RMSE of the all-FP64 pipeline (FP64
distances, FP64 neighbour order, FP64 predictions), so that each reported FP32
error can be stated against an FP64 computation.  ``data_sha256`` fingerprints
the generated inputs, so a test that regenerates the workload can tell a
generator change from a selection mismatch.

    python tests/golden/make_config_golden.py [fwd-64k] [bwd-50k] [fwd-200k] [--threads N]

Minutes to hours of CPU time per workload (fwd-64k about 20 minutes on 8 cores).  A fixture
that covers only the first steps of a run stores ``steps`` below the run's; its tests compare
those steps.
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from speedynn_b200 import datagen  # noqa: E402

STEPS_200K = 4
STEPS_BWD = 10


def data_sha256(split):
    h = hashlib.sha256()
    for a in (split.Xtrain, split.ytrain, split.Xval, split.yval):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def commit_order(ordering, p, steps, backward):
    """Winners in the order they were committed (backward fills from the end)."""
    slots = [p - 1 - t for t in range(steps)] if backward else list(range(steps))
    return [int(ordering[i]) for i in slots], slots


def make(name, threads):
    split, k, select = datagen.workload(name)
    backward = name.startswith("bwd")
    p = split.Xtrain.shape[1]
    if backward:
        steps = min(STEPS_BWD, p - select)
        nf = p - steps
    else:
        steps = STEPS_200K if name == "fwd-200k" else select
        nf = steps
    prob = oracle.Problem(split.Xtrain, split.ytrain, split.Xval, split.yval)
    t0 = time.time()
    o = oracle.select(prob, [k], nf, "backward" if backward else "forward", nthreads=threads)
    t_sel = time.time() - t0
    seq, slots = commit_order(o["ordering"], p, steps, backward)
    # the all-FP64 pipeline for each step's winner, in the committed state of that step
    full64 = np.zeros(steps, np.float64)
    t0 = time.time()
    for t in range(steps):
        r = oracle.step(prob, [k], seq[:t], [seq[t]], method="backward" if backward else "forward", precision=1,
                        want_neighbours=False, nthreads=threads)
        sq = r["sq64"][0, 0]
        full64[t] = np.sqrt(sq.sum() / sq.size)
    t_64 = time.time() - t0
    out = os.path.join(HERE, f"config_{name.replace('-', '')}.npz")
    full_steps = p - select if backward else select
    np.savez_compressed(out, workload=name, data_sha256=data_sha256(split), k=k, steps=steps,
                        run_steps=full_steps,
                        method="backward" if backward else "forward", num_features=nf,
                        ordering=o["ordering"], mask=o["mask"], errors=o["errors"], errors64=o["errors64"],
                        step_best_k=o["step_best_k"], best_k=o["best_k"], num_final=o["num_final"],
                        commit_order=np.asarray(seq, np.int32), slots=np.asarray(slots, np.int32),
                        errors_fp64_pipeline=full64)
    print(f"{name}: {steps} steps, selection {t_sel:.0f} s, FP64 pipeline {t_64:.0f} s -> {out}", flush=True)
    print("  commit order", seq, flush=True)
    print("  FP32 errors ", [float(o["errors"][s]) for s in slots], flush=True)
    print("  FP64 pipe   ", [float(x) for x in full64], flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=["fwd-64k", "bwd-50k", "fwd-200k"])
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    for n in a.names:
        make(n, a.threads)


if __name__ == "__main__":
    main()
