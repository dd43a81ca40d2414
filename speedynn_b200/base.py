"""Drop-in selector API of speedynn (speedynn/base.py:9-121), Python 3.

Same class name, constructor keywords, methods and result shapes as the
reference; the SWIG modules it imported (speedynn/base.py:61-64) are replaced
by the CUDA library through :mod:`speedynn_b200.selector`.  Additions:
optional ``Xval``/``Yval`` (train on X/Y, score on the validation split
instead of k-fold CV) and ``device``.  Differences: errors raise exceptions
instead of ``sys.exit(0)``; ``use_gpu`` is accepted for compatibility, but
there is no CPU path (the library always runs on the GPU).  Every reference
loss (``loss_functions``, the first one decides) and both model types
(``"regression"``: kNN mean, ``"classification"``: the reference's mode rule)
are supported.
"""
import logging

import numpy as np

from . import _lib
from ._lib import _f32p, ptr
from .selector import Selector

log = logging.getLogger("speedynn_b200")


class IncrementalNNFeatureSelection:
    """Efficient implementation for nearest neighbor feature selection."""

    loss_dict = {
        "rmse": 0,
        "rmse_norm": 1,
        "mad": 2,
        "mad_norm": 3,
        "zero_one": 4,
        "std": 5,
        "rmse_norm_mad_norm_std": 6,
        "rmse_norm_mad_norm_galaxies": 7,
        "rmse_std": 8,
    }
    model_types = {"regression": 0, "classification": 1}

    def __init__(self, Xtrain, Ytrain, k_vals=None, auto_feature=False, num_features=2, k_fold=10, method="backward",
                 loss_functions=["rmse"], model_type="regression", use_gpu=True, Xval=None, Yval=None, device=0):
        self.Xtrain = np.array(Xtrain)
        self.Ytrain = np.asarray(Ytrain)
        self.dim = len(Xtrain[0])
        self.auto_feature = int(auto_feature)
        if k_vals is None:
            self.k_vals = np.array(range(1, 10))
        else:
            self.k_vals = np.array(k_vals)
        self.num_desired_features = num_features
        assert self.num_desired_features <= self.dim
        assert self.num_desired_features > 0
        if auto_feature:
            self.num_desired_features = self.dim
        self.dtype_int = np.int32
        self.dtype_float = np.float32
        self.Xtrain = self.Xtrain.astype(self.dtype_float)
        self.Ytrain = self.Ytrain.astype(self.dtype_float)
        self.k_vals = self.k_vals.astype(self.dtype_int)
        self.k_fold = k_fold
        self.method = method
        self.loss_functions = np.array([self.loss_dict[name] for name in loss_functions]).astype(self.dtype_int)
        self.model_type = self.model_types[model_type]
        self.use_gpu = use_gpu
        self.device = device
        self.Xval = None if Xval is None else np.asarray(Xval, dtype=self.dtype_float)
        self.Yval = None if Yval is None else np.asarray(Yval, dtype=self.dtype_float)
        if not use_gpu:
            log.info("use_gpu=False: speedynn_b200 has no CPU path; running on the GPU")
        log.debug("loss_functions: %s", loss_functions)

    def train(self):
        if self.method not in ("forward", "backward"):
            raise ValueError("Unknown feature selection method: %r" % (self.method,))
        sel = Selector(self.Xtrain, self.Ytrain, self.Xval, self.Yval, k_vals=self.k_vals,
                       num_features=self.num_desired_features, method=self.method, k_fold=self.k_fold,
                       auto_feature=bool(self.auto_feature), device=self.device,
                       loss_functions=self.loss_functions, model_type=self.model_type)
        try:
            r = sel.run()
        finally:
            sel.close()
        self.num_final_features = r["num_final"]
        self.selected_dimensions = r["mask"].astype(self.dtype_int)
        self.selected_ordering = r["ordering"].astype(self.dtype_int)
        # speedynn/base.py:79-84 reshapes the flat [loss][p] array to (p, num_losses)
        self.selected_errors = np.ascontiguousarray(r["errors_all"].T, dtype=self.dtype_float)
        self.selected_errors64 = r["errors64"]
        self.optimal_model_k = r["best_k"]

    def get_selected_dimensions(self):
        return self.selected_dimensions

    def get_selected_ordering(self):
        return self.selected_ordering

    def get_feature_ranks(self):
        if self.method == "backward":
            ranks = np.zeros(self.dim)
            for i in range(self.dim - self.num_final_features):
                ranks[self.selected_ordering[self.dim - i - 1]] = -(self.dim - self.num_final_features) + i
            return ranks
        elif self.method == "forward":
            ranks = np.zeros(self.dim)
            for i in range(self.num_final_features):
                ranks[self.selected_ordering[i]] = self.num_final_features - i
            return ranks
        raise ValueError("Unknown feature selection method: %r" % (self.method,))

    def get_selected_errors(self):
        return self.selected_errors

    def get_optimal_model_k(self):
        return self.optimal_model_k

    def get_loss(self, labels, predictions, loss_func="rmse"):
        loss_id = self.loss_dict[loss_func]
        a = np.ascontiguousarray(labels, dtype=self.dtype_float)
        b = np.ascontiguousarray(predictions, dtype=self.dtype_float)
        return float(_lib.lib().get_loss_all(ptr(a, _f32p), a.size, ptr(b, _f32p), b.size, loss_id))
