"""Python face of the CPU oracle (``oracle/snn_oracle.c`` -> ``libsnn_oracle.so``)
plus a tiny independent NumPy restatement used to cross-check it.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg, always as the checker, never as the
thing measured for the GPU arms or shipped.  The product library never calls
anything in this directory.

Parity pin: ``tests/test_oracle_golden.py`` checks both restatements against
golden vectors written by speedynn's own CPU backend (``tests/golden``).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsnn_oracle.so")

_lib = None
_i32p = ctypes.POINTER(ctypes.c_int)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
FLT_MAX = np.float32(np.finfo(np.float32).max)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise FileNotFoundError(f"{ORACLE_SO} not built (make -C oracle)")
        lib = ctypes.CDLL(ORACLE_SO)
        lib.snn_oracle_step.restype = ctypes.c_int
        lib.snn_oracle_step.argtypes = [
            _f32p, _f32p, ctypes.c_int, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int,
            ctypes.c_int, _i32p, ctypes.c_int,
            _i32p, ctypes.c_int,
            _i32p, ctypes.c_int,
            ctypes.c_int, ctypes.c_int,
            _i32p, _f32p, _f32p, _f64p]
        lib.snn_oracle_select.restype = ctypes.c_int
        lib.snn_oracle_select.argtypes = [
            _f32p, _f32p, ctypes.c_int, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            _i32p, _i32p, _f32p, _f64p, _i32p, _i32p, _i32p]
        _lib = lib
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Problem:
    """Rows scored against neighbour columns.  CV mode: ``Xval is None``
    (rows == columns == Xtrain, same-fold pairs excluded, reference fold rule);
    holdout mode: validation rows against training columns, no folds."""

    def __init__(self, Xtrain, ytrain, Xval=None, yval=None, k_fold=10):
        self.Xc = _f32(Xtrain)
        self.yc = _f32(ytrain)
        self.cv = Xval is None
        self.Xr = self.Xc if self.cv else _f32(Xval)
        self.yr = self.yc if self.cv else _f32(yval)
        self.k_fold = int(k_fold) if self.cv else 0
        self.p = self.Xc.shape[1]

    def _args(self):
        return (_p(self.Xr, _f32p), _p(self.yr, _f32p), self.Xr.shape[0],
                _p(self.Xc, _f32p), _p(self.yc, _f32p), self.Xc.shape[0], self.p,
                int(self.cv), self.k_fold)


def select(prob, k_vals, num_features, method="forward", auto_feature=False, nthreads=0):
    lib = load()
    kv = _i32(k_vals)
    p = prob.p
    out = {k: np.zeros(p, np.int32) for k in ("ordering", "mask", "step_best_k")}
    out["errors"] = np.zeros(p, np.float32)
    out["errors64"] = np.zeros(p, np.float64)
    bk = np.zeros(1, np.int32)
    nf = np.zeros(1, np.int32)
    st = lib.snn_oracle_select(*prob._args(), _p(kv, _i32p), kv.size, int(method == "backward"),
                               int(num_features), int(bool(auto_feature)), int(nthreads),
                               _p(out["ordering"], _i32p), _p(out["mask"], _i32p), _p(out["errors"], _f32p),
                               _p(out["errors64"], _f64p), _p(out["step_best_k"], _i32p),
                               _p(bk, _i32p), _p(nf, _i32p))
    if st != 0:
        raise RuntimeError(f"snn_oracle_select failed with status {st}")
    out["best_k"] = int(bk[0])
    out["num_final"] = int(nf[0])
    return out


def step(prob, k_vals, committed, candidates, method="forward", rows=None, precision=0,
         want_neighbours=True, nthreads=0):
    """One greedy step: neighbour lists and per-row squared residuals.

    Returns dict with ``nn_idx``/``nn_dist`` [ncand, nrows, kmax] (if asked),
    ``sq32`` [ncand, nk, nrows] (precision 0) and ``sq64`` [ncand, nk, nrows].
    """
    lib = load()
    kv = _i32(k_vals)
    kmax = int(kv.max())
    seq = _i32(committed if len(committed) else [0])
    cands = _i32(candidates)
    rws = None if rows is None else _i32(rows)
    nrows = prob.Xr.shape[0] if rws is None else rws.size
    nn_idx = np.zeros((cands.size, nrows, kmax), np.int32) if want_neighbours else None
    nn_dist = np.zeros((cands.size, nrows, kmax), np.float32) if want_neighbours else None
    sq32 = np.zeros((cands.size, kv.size, nrows), np.float32) if precision == 0 else None
    sq64 = np.zeros((cands.size, kv.size, nrows), np.float64)
    st = lib.snn_oracle_step(*prob._args(), _p(kv, _i32p), kv.size, int(method == "backward"),
                             _p(seq, _i32p), len(committed), _p(cands, _i32p), cands.size,
                             _p(rws, _i32p), 0 if rws is None else rws.size, int(precision), int(nthreads),
                             _p(nn_idx, _i32p), _p(nn_dist, _f32p), _p(sq32, _f32p), _p(sq64, _f64p))
    if st != 0:
        raise RuntimeError(f"snn_oracle_step failed with status {st}")
    return {"nn_idx": nn_idx, "nn_dist": nn_dist, "sq32": sq32, "sq64": sq64}


def rmse32(sq):
    """speedynn/lib/loss_functions.c:41-50: sequential FP32 sum, / n, sqrt in double."""
    s = np.add.accumulate(np.asarray(sq, np.float32), dtype=np.float32)[-1]
    s = np.float32(s / np.float32(len(sq)))
    return np.float32(np.sqrt(np.float64(s)))


# --------------------------------------------------------------------------
# Independent NumPy restatement (tiny inputs only), used to cross-check the C
# oracle.  Same rules, written vector-wise: neighbour lists are a stable sort
# of (distance, index) restricted to distance < FLT_MAX, padded with
# (FLT_MAX, 0) (speedynn/lib/cpu.c:212-252).
# --------------------------------------------------------------------------
def np_select(prob, k_vals, num_features, method="forward"):
    kv = np.asarray(k_vals, np.int32)
    kmax = int(kv.max())
    Xr, Xc, yr, yc = prob.Xr, prob.Xc, prob.yr, prob.yc
    nr, nc, p = Xr.shape[0], Xc.shape[0], prob.p
    back = method == "backward"
    diff = Xr[:, None, :] - Xc[None, :, :]          # float32, exact per element
    sq = diff * diff                                 # float32
    if back:
        D = np.zeros((nr, nc), np.float32)
        for k in range(p - 1, -1, -1):
            D = D + sq[:, :, k]
    else:
        D = np.zeros((nr, nc), np.float32)
    if prob.cv:
        npf = nr // prob.k_fold
        fr = np.arange(nr) // npf
        excl = fr[:, None] == fr[None, :]
    else:
        excl = np.zeros((nr, nc), bool)
    mask = np.ones(p, np.int32) if back else np.zeros(p, np.int32)
    ordering = np.zeros(p, np.int32)
    errors = np.zeros(p, np.float32)
    best_k_last = 0
    its = range(p - 1, num_features - 1, -1) if back else range(num_features)
    for it in its:
        cands = [j for j in range(p) if mask[j] == (1 if back else 0)]
        min_err, min_dim, min_k = FLT_MAX, -1, 0
        for c in cands:
            d = (D - sq[:, :, c]) if back else (D + sq[:, :, c])
            errs = []
            preds = np.zeros((len(kv), nr), np.float32)
            for r in range(nr):
                ok = (~excl[r]) & (d[r] < FLT_MAX)
                cols = np.nonzero(ok)[0]
                order = cols[np.lexsort((cols, d[r, cols]))][:kmax]
                lst = np.zeros(kmax, np.int64)
                lst[:order.size] = order
                csum = np.add.accumulate(yc[lst], dtype=np.float32)
                for m, k in enumerate(kv):
                    preds[m, r] = np.float32(csum[k - 1] / np.float32(k))
            best, bk = FLT_MAX, -1
            for m, k in enumerate(kv):
                e = yr - preds[m]
                rm = rmse32(e * e)
                if rm < best:
                    best, bk = rm, int(k)
            if bk >= 0 and best < min_err:
                min_err, min_dim, min_k = best, c, bk
        mask[min_dim] = 0 if back else 1
        ordering[it] = min_dim
        errors[it] = min_err
        best_k_last = min_k
        D = (D - sq[:, :, min_dim]) if back else (D + sq[:, :, min_dim])
    return {"ordering": ordering, "mask": mask, "errors": errors, "best_k": best_k_last}
