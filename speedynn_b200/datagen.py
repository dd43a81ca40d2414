"""Seeded synthetic regression data for the selection workloads.

The generator family: ``n_mag`` correlated "magnitude" columns
m_i ~ N(20, 1.5^2) with pairwise correlation 0.8 (one shared factor),
adjacent-difference "colour" columns c_i = m_i - m_{i+1}, and pure-noise
columns N(0, 1) (``n_heavy`` of them Student-t with 3 degrees of freedom).
Target y = 0.6*tanh(c1) + 0.3*c2^2 - 0.2*c3*c4 + 0.05*(m5 - 20) + N(0, 0.02^2),
clipped to [0, 3].  Columns are permuted by the seed so that informative
features do not sit at the lowest indices.

No public dataset is involved; these stand in for the workload shapes the
benchmarks are quoted on.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class Split:
    Xtrain: np.ndarray
    ytrain: np.ndarray
    Xval: np.ndarray
    yval: np.ndarray
    informative: np.ndarray  # column indices of magnitudes and colours


def _draw(rng, n, p, n_mag, n_col, n_heavy, mixture):
    rho = 0.8
    z0 = rng.standard_normal(n)
    if mixture:
        # 3-component Gaussian mixture on the shared factor
        comp = rng.choice(3, size=n, p=[0.5, 0.3, 0.2])
        z0 = z0 * np.array([1.0, 0.6, 0.8])[comp] + np.array([0.0, 3.0, -2.5])[comp]
    mags = 20.0 + 1.5 * (np.sqrt(rho) * z0[:, None] + np.sqrt(1 - rho) * rng.standard_normal((n, n_mag)))
    cols = mags[:, :n_col] - mags[:, 1:n_col + 1]
    n_noise = p - n_mag - n_col
    noise = rng.standard_normal((n, n_noise))
    if n_heavy:
        noise[:, :n_heavy] = rng.standard_t(3, size=(n, n_heavy))
    c = cols
    m5 = mags[:, 4] if n_mag >= 5 else mags[:, -1]
    y = 0.6 * np.tanh(c[:, 0]) + 0.3 * c[:, 1] ** 2 - 0.2 * c[:, 2] * c[:, 3] + 0.05 * (m5 - 20.0)
    y = y + rng.normal(0.0, 0.02, size=n)
    y = np.clip(y, 0.0, 3.0)
    X = np.concatenate([mags, cols, noise], axis=1)
    return X, y


def generate(n_train, n_val, p, n_mag, n_heavy=0, seed=0, mixture=False, standardize=False,
             dup_frac=0.0, n_col=None):
    """Return a float32 :class:`Split` (train and validation drawn i.i.d.)."""
    if n_col is None:
        n_col = n_mag - 1
    assert n_col <= n_mag - 1 and n_col >= 4 and n_mag + n_col <= p
    rng = np.random.default_rng(seed)
    X, y = _draw(rng, n_train + n_val, p, n_mag, n_col, n_heavy, mixture)
    perm = rng.permutation(p)
    X = X[:, perm]
    informative = np.sort(np.nonzero(perm < n_mag + n_col)[0]).astype(np.int32)
    Xt, yt = X[:n_train], y[:n_train]
    Xv, yv = X[n_train:], y[n_train:]
    if dup_frac > 0:
        nd = int(round(dup_frac * n_train))
        src = rng.choice(n_train, size=nd, replace=False)
        dst = rng.choice(n_train, size=nd, replace=False)
        Xt = Xt.copy()
        yt = yt.copy()
        Xt[dst] = Xt[src]
        yt[dst] = yt[src]
    if standardize:
        mu = Xt.mean(axis=0)
        sd = Xt.std(axis=0)
        sd[sd == 0] = 1.0
        Xt = (Xt - mu) / sd
        Xv = (Xv - mu) / sd
    f = np.float32
    return Split(np.ascontiguousarray(Xt, f), np.ascontiguousarray(yt, f),
                 np.ascontiguousarray(Xv, f), np.ascontiguousarray(yv, f), informative)


# Named workloads ----------------------------------------------------------

WORKLOADS = {
    # plain forward selection, CPU-runnable size
    "fwd-2k": dict(n_train=2000, n_val=1000, p=20, n_mag=5, seed=0, k=10, select=8),
    # plain forward selection on one GPU (the headline workload)
    "fwd-64k": dict(n_train=65536, n_val=32768, p=60, n_mag=8, n_heavy=10, seed=2, k=10, select=15),
    # backward elimination, standardized, 12 informative of 120
    "bwd-50k": dict(n_train=50000, n_val=25000, p=120, n_mag=7, n_col=5, seed=3, standardize=True, k=5,
                    select=20),
    # large forward selection with mixture structure and 2 % duplicated rows
    "fwd-200k": dict(n_train=200000, n_val=100000, p=100, n_mag=8, seed=5, mixture=True, dup_frac=0.02, k=50,
                     select=20),
}


def workload(name, scale_rows=1.0):
    """Generate a named workload; ``scale_rows`` shrinks n_train and n_val."""
    w = dict(WORKLOADS[name])
    k = w.pop("k")
    sel = w.pop("select")
    w["n_train"] = max(64, int(w["n_train"] * scale_rows))
    w["n_val"] = max(32, int(w["n_val"] * scale_rows))
    return generate(**w), k, sel


def batch_workload(seed0=4000, n_pools=64, n_splits=5, p=40, lo=1024, hi=40000, steps=15, scale_rows=1.0):
    """The batched workload: ``n_pools`` problems with n_train log-uniform in
    [lo, hi] (seeded per pool: seed0 + i), a pool of 1.5 * n_train rows each,
    and ``n_splits`` seeded train / validation splits of every pool (n_val =
    n_train / 2), so n_pools * n_splits holdout forward selections; pool i uses
    k = (1, 5, 10, 20)[i % 4] and ``steps`` greedy steps.  Returns a list of
    problem dicts for :class:`speedynn_b200.batch.Batch`."""
    probs = []
    for i in range(n_pools):
        rng = np.random.default_rng(seed0 + i)
        n = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))) * scale_rows))
        n = max(64, n)
        pool = generate(n, n // 2, p, n_mag=6, seed=seed0 + i)
        X = np.concatenate([pool.Xtrain, pool.Xval])
        y = np.concatenate([pool.ytrain, pool.yval])
        k = (1, 5, 10, 20)[i % 4]
        for s in range(n_splits):
            perm = np.random.default_rng((seed0 + i) * 31 + s).permutation(X.shape[0])
            tr, va = perm[:n], perm[n:n + n // 2]
            probs.append(dict(Xtrain=np.ascontiguousarray(X[tr]), ytrain=np.ascontiguousarray(y[tr]),
                              Xval=np.ascontiguousarray(X[va]), yval=np.ascontiguousarray(y[va]), k_vals=[k],
                              num_features=steps, method="forward"))
    return probs
