"""Handle-level Python interface: one selection problem on one GPU.

Adds to the reference selector a train/validation holdout mode, step-wise
execution, FP64 errors, neighbour-list inspection and kernel timings.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import _f32p, _f64p, _i32p, check, ptr


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Selector:
    """Greedy kNN wrapper feature selection on one CUDA device.

    CV mode (``Xval is None``): every training point is scored against the
    others outside its fold (folds are contiguous blocks of n // k_fold rows,
    a remainder forms an extra fold), exactly as speedynn does.  Holdout mode:
    validation points are scored against all training points.
    """

    def __init__(self, Xtrain, ytrain, Xval=None, yval=None, k_vals=(1, 2, 3, 4, 5, 6, 7, 8, 9), num_features=2,
                 method="forward", k_fold=10, auto_feature=False, device=0, loss_functions=(0,), model_type=0):
        if method not in ("forward", "backward"):
            raise ValueError(f"unknown feature selection method {method!r}")
        L = _lib.lib()
        self.Xtrain = _f32(Xtrain)
        self.ytrain = _f32(ytrain).reshape(-1)
        if self.Xtrain.ndim != 2 or self.ytrain.shape[0] != self.Xtrain.shape[0]:
            raise ValueError("Xtrain must be [n, p] and ytrain [n]")
        self.holdout = Xval is not None
        if self.holdout:
            self.Xval = _f32(Xval)
            self.yval = _f32(yval).reshape(-1)
            if self.Xval.ndim != 2 or self.Xval.shape[1] != self.Xtrain.shape[1] or self.yval.shape[0] != self.Xval.shape[0]:
                raise ValueError("Xval must be [m, p] and yval [m]")
        else:
            self.Xval = self.yval = None
        self.p = self.Xtrain.shape[1]
        self.method = method
        self.k_vals = np.ascontiguousarray(k_vals, dtype=np.int32).reshape(-1)
        d = _lib.SnnDesc()
        d.n_train = self.Xtrain.shape[0]
        d.n_val = self.Xval.shape[0] if self.holdout else 0
        d.p = self.p
        d.k_vals = ptr(self.k_vals, _i32p)
        d.num_k_vals = self.k_vals.size
        d.backward = int(method == "backward")
        d.num_features = int(num_features)
        d.k_fold = int(k_fold)
        d.auto_feature = int(bool(auto_feature))
        d.device = int(device)
        h = ctypes.c_void_p()
        check(L.snn_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.loss_ids = np.ascontiguousarray(loss_functions, dtype=np.int32).reshape(-1)
        try:
            if list(self.loss_ids) != [0] or int(model_type) != 0:
                check(L.snn_set_model(h, ptr(self.loss_ids, _i32p), self.loss_ids.size, int(model_type)))
            check(L.snn_load(h, ptr(self.Xtrain, _f32p), ptr(self.ytrain, _f32p),
                             ptr(self.Xval, _f32p) if self.holdout else None,
                             ptr(self.yval, _f32p) if self.holdout else None))
        except Exception:
            self.close()
            raise

    # -- execution -------------------------------------------------------
    def run(self):
        check(_lib.lib().snn_run(self._h))
        return self.results()

    def reset(self):
        check(_lib.lib().snn_reset(self._h))

    def step(self):
        """Run one greedy step; False when the selection had finished."""
        return bool(check(_lib.lib().snn_step(self._h)))

    def commit_sequence(self, seq):
        """Warm start: restart and commit ``seq`` in order without scoring it."""
        a = np.ascontiguousarray(seq, dtype=np.int32).reshape(-1)
        check(_lib.lib().snn_commit_sequence(self._h, ptr(a, _i32p) if a.size else None, a.size))

    def results(self):
        p = self.p
        out = {"ordering": np.zeros(p, np.int32), "mask": np.zeros(p, np.int32), "errors": np.zeros(p, np.float32),
               "errors64": np.zeros(p, np.float64), "step_best_k": np.zeros(p, np.int32)}
        bk = ctypes.c_int()
        nf = ctypes.c_int()
        check(_lib.lib().snn_get_results(self._h, ptr(out["ordering"], _i32p), ptr(out["mask"], _i32p),
                                         ptr(out["errors"], _f32p), ptr(out["errors64"], _f64p),
                                         ptr(out["step_best_k"], _i32p), ctypes.byref(bk), ctypes.byref(nf)))
        out["best_k"] = bk.value
        out["num_final"] = nf.value
        ea = np.zeros(self.loss_ids.size * p, np.float32)
        check(_lib.lib().snn_get_errors_all(self._h, ptr(ea, _f32p), ea.size))
        out["errors_all"] = ea.reshape(self.loss_ids.size, p)  # [loss][step slot], the reference's layout
        return out

    # -- inspection ------------------------------------------------------
    def keep_neighbours(self, enable=True):
        check(_lib.lib().snn_keep_neighbours(self._h, int(bool(enable))))

    def neighbours(self):
        """(candidates, idx, dist) of the last step: idx/dist [n_cand, n_rows, k_max]."""
        L = _lib.lib()
        nc = ctypes.c_int()
        km = ctypes.c_int()
        check(L.snn_get_neighbours(self._h, None, ctypes.byref(nc), ctypes.byref(km), None, None))
        n_rows = self.Xval.shape[0] if self.holdout else self.Xtrain.shape[0]
        cands = np.zeros(nc.value, np.int32)
        idx = np.zeros((nc.value, n_rows, km.value), np.int32)
        dist = np.zeros((nc.value, n_rows, km.value), np.float32)
        check(L.snn_get_neighbours(self._h, ptr(cands, _i32p), ctypes.byref(nc), ctypes.byref(km), ptr(idx, _i32p),
                                   ptr(dist, _f32p)))
        return cands, idx, dist

    def neighbours_rows(self, rows):
        """idx/dist [n_cand, len(rows), k_max] of the last kept step for the given scored rows."""
        L = _lib.lib()
        nc = ctypes.c_int()
        km = ctypes.c_int()
        check(L.snn_get_neighbours(self._h, None, ctypes.byref(nc), ctypes.byref(km), None, None))
        r = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1)
        idx = np.zeros((nc.value, r.size, km.value), np.int32)
        dist = np.zeros((nc.value, r.size, km.value), np.float32)
        check(L.snn_get_neighbours_rows(self._h, ptr(r, _i32p), r.size, ptr(idx, _i32p), ptr(dist, _f32p)))
        return idx, dist

    def predictions(self, rows):
        """(candidates, pred [n_cand, num_k_vals, len(rows)]) of the most recent scored step."""
        L = _lib.lib()
        r = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1)
        nc = ctypes.c_int()
        check(L.snn_get_predictions(self._h, ptr(r, _i32p), 0, None, ctypes.byref(nc), None))
        cands = np.zeros(nc.value, np.int32)
        pred = np.zeros((nc.value, self.k_vals.size, r.size), np.float32)
        check(L.snn_get_predictions(self._h, ptr(r, _i32p), r.size, ptr(cands, _i32p), ctypes.byref(nc),
                                    ptr(pred, _f32p)))
        return cands, pred

    def set_kernel(self, which):
        """Scoring kernel: 0 automatic, 1 rows per lane (any k), 3 TMA-fed row tiles (k <= 64)."""
        check(_lib.lib().snn_set_option(self._h, _lib.SNN_OPT_KERNEL, int(which)))

    def set_sorted_start(self, enable):
        """First forward holdout step from sorted feature columns (default on).  Results do not depend on it."""
        check(_lib.lib().snn_set_option(self._h, _lib.SNN_OPT_SORTED_START, int(bool(enable))))

    def set_seed_step(self, step):
        """First forward step whose starting bounds come from seed columns (default 2, 3 for k > 16;
        a large value turns seeded steps off).  Results do not depend on it."""
        check(_lib.lib().snn_set_option(self._h, _lib.SNN_OPT_SEED_STEP, int(step)))

    def set_counters(self, enable):
        """Keep the TMA-fed scorer's filter counters (off by default: a little slower)."""
        check(_lib.lib().snn_set_option(self._h, _lib.SNN_OPT_COUNTERS, int(bool(enable))))

    def filter_counters(self):
        """(row, chunk) pairs of the TMA-fed scorer's full passes, how many its
        filter flagged, and how many of those held a passing column."""
        a, b, c = ctypes.c_ulonglong(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
        check(_lib.lib().snn_get_filter_counters(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"row_chunks": a.value, "flagged": b.value, "passed": c.value}

    def step_timing(self):
        """Per greedy step of the last run: (score_ms, commit_ms) arrays."""
        n = self.p
        sc, cm = np.zeros(n, np.float32), np.zeros(n, np.float32)
        k = check(_lib.lib().snn_get_step_timing(self._h, ptr(sc, _f32p), ptr(cm, _f32p), n))
        return sc[:k], cm[:k]

    def setup_ms(self):
        """CUDA-event time of the last reset's initial distance matrix (backward: the full distance)."""
        ms = ctypes.c_float()
        check(_lib.lib().snn_get_setup_timing(self._h, ctypes.byref(ms)))
        return ms.value

    def timing(self):
        s, c, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        ns, nc, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_lib.lib().snn_get_timing(self._h, ctypes.byref(s), ctypes.byref(ns), ctypes.byref(c), ctypes.byref(nc),
                                        ctypes.byref(t), ctypes.byref(nt)))
        return {"score_ms": s.value, "score_launches": ns.value, "commit_ms": c.value, "commit_launches": nc.value,
                "total_ms": t.value, "launches": nt.value}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().snn_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
