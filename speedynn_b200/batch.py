"""Many independent selection problems in one call (snn_batch_* of the C ABI).

Each problem is a dict with the Selector keywords: ``Xtrain``, ``ytrain``,
optional ``Xval``/``yval`` (holdout; CV mode without them), ``k_vals``,
``num_features``, ``method``, ``k_fold``, ``auto_feature``, ``device``,
``loss_functions`` (reference loss ids, the first decides) and
``model_type`` (0 regression, 1 classification).
Problems run on their own CUDA streams so that small ones overlap on the
GPU; the library groups them into waves that fit the device memory.  Each
problem's results equal a Selector run of that problem alone.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import _f32p, _f64p, _i32p, check, ptr


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Batch:
    def __init__(self, problems, max_device_bytes=0):
        L = _lib.lib()
        self._keep = []
        descs = (_lib.SnnDesc * len(problems))()
        self.p = []
        self.models = []  # (loss ids, model type) per problem
        for i, pr in enumerate(problems):
            Xt = _f32(pr["Xtrain"])
            yt = _f32(pr["ytrain"]).reshape(-1)
            Xv = pr.get("Xval")
            yv = pr.get("yval")
            Xv = None if Xv is None else _f32(Xv)
            yv = None if yv is None else _f32(yv).reshape(-1)
            method = pr.get("method", "forward")
            if method not in ("forward", "backward"):
                raise ValueError(f"unknown feature selection method {method!r}")
            kv = np.ascontiguousarray(pr.get("k_vals", (1, 2, 3, 4, 5, 6, 7, 8, 9)), dtype=np.int32).reshape(-1)
            d = descs[i]
            d.n_train = Xt.shape[0]
            d.n_val = 0 if Xv is None else Xv.shape[0]
            d.p = Xt.shape[1]
            d.k_vals = ptr(kv, _i32p)
            d.num_k_vals = kv.size
            d.backward = int(method == "backward")
            d.num_features = int(pr.get("num_features", 2))
            d.k_fold = int(pr.get("k_fold", 10))
            d.auto_feature = int(bool(pr.get("auto_feature", False)))
            d.device = int(pr.get("device", 0))
            lf = np.ascontiguousarray(pr.get("loss_functions", (0,)), dtype=np.int32).reshape(-1)
            self._keep.append((Xt, yt, Xv, yv, kv))
            self.p.append(Xt.shape[1])
            self.models.append((lf, int(pr.get("model_type", 0))))
        h = ctypes.c_void_p()
        check(L.snn_batch_create(descs, len(problems), int(max_device_bytes), ctypes.byref(h)))
        self._h = h
        try:
            for i, (lf, mt) in enumerate(self.models):
                if list(lf) != [0] or mt != 0:
                    check(L.snn_batch_set_model(h, i, ptr(lf, _i32p), lf.size, mt))
            for i, (Xt, yt, Xv, yv, _) in enumerate(self._keep):
                check(L.snn_batch_load(h, i, ptr(Xt, _f32p), ptr(yt, _f32p), None if Xv is None else ptr(Xv, _f32p),
                                       None if yv is None else ptr(yv, _f32p)))
        except Exception:
            self.close()
            raise

    def run(self):
        """Run every problem; returns one result dict per problem (as Selector.results)."""
        check(_lib.lib().snn_batch_run(self._h))
        return [self.results(i) for i in range(len(self.p))]

    def results(self, i):
        p = self.p[i]
        out = {"ordering": np.zeros(p, np.int32), "mask": np.zeros(p, np.int32), "errors": np.zeros(p, np.float32),
               "errors64": np.zeros(p, np.float64), "step_best_k": np.zeros(p, np.int32)}
        bk, nf = ctypes.c_int(), ctypes.c_int()
        check(_lib.lib().snn_batch_get_results(self._h, i, ptr(out["ordering"], _i32p), ptr(out["mask"], _i32p),
                                               ptr(out["errors"], _f32p), ptr(out["errors64"], _f64p),
                                               ptr(out["step_best_k"], _i32p), ctypes.byref(bk), ctypes.byref(nf)))
        out["best_k"] = bk.value
        out["num_final"] = nf.value
        nl = self.models[i][0].size
        ea = np.zeros(nl * p, np.float32)
        check(_lib.lib().snn_batch_get_errors_all(self._h, i, ptr(ea, _f32p), ea.size))
        out["errors_all"] = ea.reshape(nl, p)  # [loss][step slot], as Selector.results
        return out

    def timing(self):
        ms, w = ctypes.c_double(), ctypes.c_int()
        check(_lib.lib().snn_batch_get_timing(self._h, ctypes.byref(ms), ctypes.byref(w)))
        return {"run_ms": ms.value, "waves": w.value}

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().snn_batch_destroy(h)
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
