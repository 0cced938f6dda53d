"""Learned storage-format selector.

A small multilayer perceptron predicts, from features of a projection's
connectivity matrix (annarchy_b200.tuning.features), the log10 time of the
weighted sum under every candidate schedule; the selector takes the schedule
with the smallest prediction among the feasible ones. It is trained on the
GPU by the kernels of csrc/selector.cu (forward, masked-MSE backward, Adam)
on timings the simulator collects itself (tuning.Autotuner); the exhaustive
autotuner is its fallback and the measure of its regret. The reference picks
formats with a fixed rule (ANNarchy/core/Projection.py:691-789),
tuning.heuristic here.

`reference_loss_grad` restates the network's forward and backward pass in
numpy (float64): the CPU check of the GPU gradients.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import tuning
from .runtime import lib as L

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
SCHEDULE_NAMES = [tuning.schedule_name(s) for s in tuning.SCHEDULES]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def param_count(n_in, hidden, n_out) -> int:
    return n_in * hidden + hidden + hidden * hidden + hidden + n_out * hidden + n_out


def unpack(p, n_in, hidden, n_out):
    i = 0
    out = []
    for shape in ((hidden, n_in), (hidden,), (hidden, hidden), (hidden,), (n_out, hidden), (n_out,)):
        n = int(np.prod(shape))
        out.append(p[i:i + n].reshape(shape))
        i += n
    return out


def init_params(n_in, hidden, n_out, seed=0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((n_in, hidden), (hidden, hidden), (hidden, n_out)):
        parts.append(rng.normal(0, np.sqrt(2.0 / fan_in), (fan_out, fan_in)).ravel())
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)


def reference_loss_grad(params, x, target, mask, n_in, hidden, n_out):
    """Masked MSE and its gradient, in float64 numpy (CPU restatement of the
    GPU kernels)."""
    W1, b1, W2, b2, W3, b3 = [a.astype(np.float64) for a in
                              unpack(np.asarray(params, np.float64), n_in, hidden, n_out)]
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3.T + b3
    cnt = mask.sum()
    e = (y - target) * mask
    loss = float((e * e).sum() / cnt)
    d3 = 2 * e / cnt
    gW3, gb3 = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ W3) * (h2 > 0)
    gW2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1, gb1 = d1.T @ x, d1.sum(0)
    return loss, np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])


def gpu_loss_grad(params, x, target, mask, n_in, hidden, n_out):
    lib = L.load()
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    m = np.ascontiguousarray(mask, np.float32)
    g = np.zeros_like(p)
    loss = np.zeros(1, np.float32)
    L.check_selector("anb_mlp_loss_grad", lib.anb_mlp_loss_grad(
        _p(p), _p(x), _p(t), _p(m), x.shape[0], n_in, hidden, n_out, _p(loss), _p(g)))
    return float(loss[0]), g


class Selector:
    def __init__(self, hidden: int = 64, seed: int = 0):
        self.hidden = hidden
        self.n_in = len(tuning.FEATURE_NAMES)
        self.n_out = len(SCHEDULE_NAMES)
        self.params = init_params(self.n_in, hidden, self.n_out, seed)
        self.mu = np.zeros(self.n_in)
        self.sd = np.ones(self.n_in)

    # -- data ------------------------------------------------------------------
    @staticmethod
    def table(records):
        """Records of the autotuner -> (features, log10 times, mask) per
        matrix (grouped by tag and feature vector)."""
        groups = {}
        for r in records:
            key = (r.get("tag", ""), tuple(np.round(r["features"], 9)))
            groups.setdefault(key, {"features": r["features"], "ms": {}})
            groups[key]["ms"][r["schedule"]] = r["ms"]
        X, Y, M, T = [], [], [], []
        for key, g in groups.items():
            y = np.zeros(len(SCHEDULE_NAMES))
            m = np.zeros(len(SCHEDULE_NAMES))
            for name, ms in g["ms"].items():
                if name in SCHEDULE_NAMES:
                    j = SCHEDULE_NAMES.index(name)
                    y[j] = np.log10(ms)
                    m[j] = 1.0
            X.append(g["features"])
            Y.append(y)
            M.append(m)
            T.append(key[0])
        return np.array(X), np.array(Y), np.array(M), T

    def _norm(self, X):
        return ((X - self.mu) / self.sd).astype(np.float32)

    # -- training / inference ----------------------------------------------------
    def fit(self, X, Y, M, epochs: int = 3000, lr: float = 3e-3, weight_decay: float = 1e-4):
        X, Y, M = np.atleast_2d(X), np.atleast_2d(Y), np.atleast_2d(M)
        if X.shape[1] != self.n_in or Y.shape != (X.shape[0], self.n_out) or M.shape != Y.shape:
            raise ValueError(f"fit(): expected X (n, {self.n_in}), Y and M (n, {self.n_out}); got "
                             f"{X.shape}, {Y.shape}, {M.shape}")
        self.mu = X.mean(0)
        self.sd = X.std(0) + 1e-6
        lib = L.load()
        p = np.ascontiguousarray(self.params, np.float32)
        x = np.ascontiguousarray(self._norm(X))
        y = np.ascontiguousarray(Y, np.float32)
        m = np.ascontiguousarray(M, np.float32)
        loss = np.zeros(1, np.float32)
        L.check_selector("anb_mlp_train", lib.anb_mlp_train(
            _p(p), _p(x), _p(y), _p(m), x.shape[0], self.n_in, self.hidden, self.n_out, epochs,
            C.c_float(lr), C.c_float(weight_decay), _p(loss)))
        self.params = p
        return float(loss[0])

    def predict(self, X):
        lib = L.load()
        if np.atleast_2d(X).shape[1] != self.n_in:
            raise ValueError(f"predict(): expected {self.n_in} features per row")
        x = np.ascontiguousarray(self._norm(np.atleast_2d(X)))
        y = np.zeros((x.shape[0], self.n_out), np.float32)
        p = np.ascontiguousarray(self.params, np.float32)
        L.check_selector("anb_mlp_predict", lib.anb_mlp_predict(
            _p(p), _p(x), x.shape[0], self.n_in, self.hidden, self.n_out, _p(y)))
        return y

    def choose_index(self, X, feasible_mask):
        pred = self.predict(X)
        pred = np.where(feasible_mask > 0, pred, np.inf)
        return pred.argmin(axis=1)

    def choose(self, m) -> dict:
        """Schedule for matrix m (post, pre) among the feasible ones."""
        feat = tuning.features(m)
        feas = np.array([1.0 if tuning.feasible(m, s) else 0.0 for s in tuning.SCHEDULES])
        return dict(tuning.SCHEDULES[int(self.choose_index(feat[None], feas[None])[0])])

    # -- persistence -------------------------------------------------------------
    def save(self, path):
        with open(path, "w") as f:
            json.dump({"hidden": self.hidden, "params": self.params.tolist(), "mu": self.mu.tolist(),
                       "sd": self.sd.tolist(), "schedules": SCHEDULE_NAMES,
                       "features": tuning.FEATURE_NAMES}, f)

    @classmethod
    def load(cls, path):
        """The model saved at `path`; ValueError if it was trained for another
        list of schedules or features."""
        with open(path) as f:
            d = json.load(f)
        if d.get("schedules") != SCHEDULE_NAMES or d.get("features") != tuning.FEATURE_NAMES:
            raise ValueError(f"{path}: trained for other schedules or features")
        s = cls(hidden=d["hidden"])
        s.params = np.array(d["params"], np.float32)
        s.mu, s.sd = np.array(d["mu"]), np.array(d["sd"])
        return s


def regret(choice_idx, Y, M):
    """time(chosen) / time(best measured) per sample (inf if the chosen
    schedule was not measured)."""
    best = np.where(M > 0, Y, np.inf).min(axis=1)
    chosen = Y[np.arange(len(Y)), choice_idx]
    ok = M[np.arange(len(Y)), choice_idx] > 0
    return np.where(ok, 10.0 ** (chosen - best), np.inf)


def training_matrices(seed: int = 0, count: int = 48):
    """Synthetic connectivity matrices spanning the feature space: random
    (uniform in-degree), power-law row lengths, local neighbourhoods on a grid
    and dense blocks, at several sizes and densities."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = ["uniform", "powerlaw", "local", "blocks"][i % 4]
        n = int(rng.choice([4096, 8192, 16384, 32768]))
        if kind == "uniform":
            k = int(rng.choice([8, 24, 64, 150, 400]))
            rows = np.repeat(np.arange(n), k)
            cols = rng.integers(0, n, n * k)
            m = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n))
        elif kind == "powerlaw":
            mean = float(rng.choice([20, 60, 150]))
            lengths = np.minimum((rng.pareto(float(rng.choice([1.1, 1.5, 2.5])), n) + 1) * mean / 3,
                                 n // 2).astype(np.int64) + 1
            rows = np.repeat(np.arange(n), lengths)
            cols = rng.integers(0, n, rows.size)
            m = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n))
        elif kind == "local":
            side = int(np.sqrt(n))
            n = side * side
            radius = int(rng.choice([2, 4, 7]))
            offs = np.array([(a, b) for a in range(-radius, radius + 1)
                             for b in range(-radius, radius + 1)])
            ys, xs = np.divmod(np.arange(n), side)
            ty = (ys[:, None] + offs[None, :, 0]) % side
            tx = (xs[:, None] + offs[None, :, 1]) % side
            keep = rng.random(ty.shape) < float(rng.choice([0.3, 0.7, 1.0]))
            rr, kk = np.nonzero(keep)
            m = sp.csr_matrix((np.ones(rr.size), (rr, ty[rr, kk] * side + tx[rr, kk])), shape=(n, n))
        else:
            bs = int(rng.choice([16, 32, 64]))
            nb = n // bs
            dens = float(rng.choice([0.005, 0.01, 0.03]))
            bmask = rng.random((nb, nb)) < dens
            brow, bcol = np.nonzero(bmask)
            rr = (brow[:, None] * bs + np.arange(bs)[None, :])
            cc = (bcol[:, None] * bs + np.arange(bs)[None, :])
            rows = np.repeat(rr, bs, axis=1).ravel()
            cols = np.tile(cc, (1, bs)).ravel()
            m = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(nb * bs, nb * bs))
        m.sum_duplicates()
        m.data = rng.normal(0, 0.01, m.nnz)
        m.sort_indices()
        out.append((f"{kind}_{i}", m))
    return out


def collect(path: str, count: int = 48, seed: int = 0, reps: int = 3, dtypes=("float32",)):
    """Time every feasible schedule of every training matrix on the device
    and write the records (features, schedule, ms) to `path`."""
    tuner = tuning.Autotuner(path)
    done = {r["tag"] for r in tuner.records}
    for tag, m in training_matrices(seed, count):
        for dt in dtypes:
            t = f"{tag}/{dt}"
            if t in done:
                continue
            # the reference rule's own choice is always measured, so its
            # regret can be computed even where SELL pads heavily
            tuner.tune(m, "float", dt, reps, tag=t, extra=[{"format": "sell", "sell_sigma": 1}])
            tuner.save()
    return tuner.records


_DEFAULT = None
MODEL = os.path.join(DATA, "selector_model.json")


def default_model():
    """The shipped trained selector (None if it has not been trained)."""
    global _DEFAULT
    if _DEFAULT is None and os.path.exists(MODEL):
        _DEFAULT = Selector.load(MODEL)
    return _DEFAULT


def train_default(dataset: str = os.path.join(DATA, "selector_dataset.json"),
                  out: str = MODEL, epochs: int = 3000):
    """Train the shipped model on the whole timing dataset (GPU)."""
    X, Y, M, _ = Selector.table(json.load(open(dataset)))
    sel = Selector(hidden=64, seed=0)
    loss = sel.fit(X, Y, M, epochs=epochs, lr=3e-3)
    sel.save(out)
    return loss
