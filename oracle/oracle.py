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
# (FLT_MAX, 0) (speedynn/lib/cpu.c:128-168).
# --------------------------------------------------------------------------
def np_loss(labels, preds, lid):
    """speedynn/lib/loss_functions.c:6-183 with the reference's float/double
    operation order (sequential FP32 sums, double divisions where C promotes)."""
    y = np.asarray(labels, np.float32)
    pr = np.asarray(preds, np.float32)
    n = y.size
    f32, f64 = np.float32, np.float64

    def rmse():
        e = y - pr
        return rmse32(e * e)

    def rmse_norm():  # :52-62, descending index order
        tmp = ((y - pr).astype(f64) / (1.0 + y.astype(f64))).astype(f32)
        s = np.add.accumulate((tmp * tmp)[::-1], dtype=f32)[-1]
        return f32(np.sqrt(f64(f32(s / f32(n)))))

    def mad(norm):  # :66-111, find_median = sorted[n / 2] (:173-183)
        e = ((y - pr).astype(f64) / (1.0 + y.astype(f64))).astype(f32) if norm else (y - pr)
        m1 = np.sort(e)[n // 2]
        return np.sort(np.abs(e - m1))[n // 2]

    def zero_one():  # :113-127, int abs() of the truncated difference
        a = np.abs(y - pr)
        miss = np.count_nonzero((a >= 1.0) & (a < 2147483648.0))
        return f32(f32(miss) / f32(n))

    def std():  # :129-143, the loop assigns: only the last row's term remains
        mean = np.add.accumulate(y - pr, dtype=f32)[-1]
        mean = f32(mean / f32(n))
        a = f32(f32(y[-1] - pr[-1]) - mean)
        return f32(np.sqrt(f64(f32(f32(a * a) / f32(n - 1)))))

    if lid == 0:
        return rmse()
    if lid == 1:
        return rmse_norm()
    if lid == 2:
        return mad(False)
    if lid == 3:
        return mad(True)
    if lid == 4:
        return zero_one()
    if lid == 5:
        return std()
    if lid == 6:
        return f32(f64(rmse_norm()) / 0.19 + f64(mad(True)) / 0.041 + f64(std()) / 0.16)
    if lid == 7:
        return f32(f64(rmse_norm()) / 0.019 + f64(mad(True)) / 0.009)
    if lid == 8:
        return f32(rmse() + std())
    raise ValueError(lid)


def np_mode(labels):
    """speedynn/lib/util.c:165-188: each label counts at its first occurrence;
    the first position with the strictly largest count wins."""
    k = len(labels)
    rep = np.zeros(k, np.int64)
    for i in range(k):
        j = 0
        while j < i and labels[i] != labels[j]:
            j += 1
        rep[j] += 1
    best = 0
    for i in range(1, k):
        if rep[i] > rep[best]:
            best = i
    return labels[best]


def np_select(prob, k_vals, num_features, method="forward", loss_functions=(0,), model_type=0, auto_feature=False):
    kv = np.asarray(k_vals, np.int32)
    kmax = int(kv.max())
    lids = [int(x) for x in loss_functions]
    nl = len(lids)
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
    errors_all = np.zeros((nl, p), np.float32)
    best_k_last = 0
    total = p if auto_feature else (p - num_features if back else num_features)
    num_final = p if back else 0
    for t in range(total):
        it = p - 1 - t if back else t
        cands = [j for j in range(p) if mask[j] == (1 if back else 0)]
        min_err, min_dim, min_k, min_all = FLT_MAX, -1, 0, None
        for c in cands:
            d = (D - sq[:, :, c]) if back else (D + sq[:, :, c])
            preds = np.zeros((len(kv), nr), np.float32)
            for r in range(nr):
                ok = (~excl[r]) & (d[r] < FLT_MAX)
                cols = np.nonzero(ok)[0]
                order = cols[np.lexsort((cols, d[r, cols]))][:kmax]
                lst = np.zeros(kmax, np.int64)
                lst[:order.size] = order
                if model_type == 1:
                    for m, k in enumerate(kv):
                        preds[m, r] = np_mode(list(yc[lst[:k]]))
                else:
                    csum = np.add.accumulate(yc[lst], dtype=np.float32)
                    for m, k in enumerate(kv):
                        preds[m, r] = np.float32(csum[k - 1] / np.float32(k))
            vals = np.array([[np_loss(yr, preds[m], lid) for m in range(len(kv))] for lid in lids], np.float32)
            best, bm = FLT_MAX, -1
            for m in range(len(kv)):
                if vals[0, m] < best:
                    best, bm = vals[0, m], m
            if bm >= 0 and best < min_err:
                min_err, min_dim, min_k, min_all = best, c, int(kv[bm]), vals[:, bm]
        mask[min_dim] = 0 if back else 1
        ordering[it] = min_dim
        errors[it] = min_err
        errors_all[:, it] = min_all
        best_k_last = min_k
        num_final = p - (t + 1) if back else t + 1
        D = (D - sq[:, :, min_dim]) if back else (D + sq[:, :, min_dim])
        if auto_feature:
            if not back and it > 0 and errors[it - 1] < errors[it]:
                break
            if back and 0 < it < p - 1 and errors[it + 1] < errors[it]:
                break
    return {"ordering": ordering, "mask": mask, "errors": errors, "errors_all": errors_all, "best_k": best_k_last,
            "num_final": num_final}
