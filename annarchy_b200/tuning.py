"""Storage-format schedules of rate-coded projections: features, timing
collector and exhaustive autotuner.

The reference chooses a format with a fixed heuristic
(ANNarchy/core/Projection.py:691-789: dense above 60 % density; on the GPU
SELL for mean row length <= 128, else CSR). Here every candidate schedule
(format plus its parameter: SELL window sigma, BSR tile) is timed on the
device for the projection's actual matrix, with the L2 cache flushed before
every repetition, and the fastest is kept. The measurements form the
training set of the learned selector (annarchy_b200.selector).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np
import scipy.sparse as sp

SCHEDULES = [
    {"format": "csr"},
    {"format": "ell"},
    {"format": "ellr"},
    {"format": "sell", "sell_sigma": 1},
    {"format": "sell", "sell_sigma": 1024},
    {"format": "hyb"},
    {"format": "bsr", "bsr_tile": 16},
    {"format": "bsr", "bsr_tile": 32},
    {"format": "bsr", "bsr_tile": 64},
    # this backend's own schedule (no counterpart among the reference's formats)
    {"format": "pcsr"},
]


def schedule_name(s: dict) -> str:
    extra = "".join(f"_{v}" for k, v in sorted(s.items()) if k != "format")
    return s["format"] + extra


def block_fill(m: sp.csr_matrix, tile: int, max_nnz: int = 20_000_000) -> float:
    """nnz / (number of non-empty tile x tile blocks * tile^2), estimated on
    a band of block rows for very large matrices."""
    if m.nnz == 0:
        return 0.0
    if m.nnz > max_nnz:
        rows = int(m.shape[0] * max_nnz / m.nnz) // tile * tile
        m = m[:max(rows, tile)]
    rows = np.repeat(np.arange(m.shape[0], dtype=np.int64), np.diff(m.indptr))
    key = (rows // tile) * ((m.shape[1] + tile - 1) // tile) + m.indices // tile
    nblocks = np.unique(key).size
    return float(m.nnz / (nblocks * tile * tile))


FEATURE_NAMES = ["log_rows", "log_cols", "log_nnz", "log_mean_row", "cv_row", "max_over_mean",
                 "gini_row", "frac_empty", "log_density", "fill16", "fill32", "fill64",
                 "weight_bytes"]


def features(m: sp.csr_matrix, weight_bytes: int = 4) -> np.ndarray:
    """Row-length statistics, density and block fill of a (post, pre) matrix."""
    rl = np.diff(m.indptr).astype(np.float64)
    n_rows, n_cols = m.shape
    mean = rl.mean() if rl.size else 0.0
    srt = np.sort(rl)
    gini = 0.0
    if rl.sum() > 0:
        cum = np.cumsum(srt)
        gini = float(1.0 - 2.0 * (cum.sum() / cum[-1]) / rl.size + 1.0 / rl.size)
    return np.array([
        math.log10(max(n_rows, 1)), math.log10(max(n_cols, 1)), math.log10(max(m.nnz, 1)),
        math.log10(max(mean, 1e-3)), float(rl.std() / mean) if mean > 0 else 0.0,
        float(rl.max() / mean) if mean > 0 else 0.0, gini, float((rl == 0).mean()),
        math.log10(max(m.nnz / max(n_rows * n_cols, 1), 1e-12)),
        block_fill(m, 16), block_fill(m, 32), block_fill(m, 64), float(weight_bytes)],
        dtype=np.float64)


def stored_entries(m: sp.csr_matrix, sched: dict) -> float:
    """Slots a format stores for the matrix (padding included)."""
    rl = np.diff(m.indptr)
    fmt = sched["format"]
    if fmt in ("csr", "hyb"):
        return float(m.nnz)
    if fmt in ("ell", "ellr"):
        return float(rl.max() * m.shape[0]) if rl.size else 0.0
    if fmt == "sell":
        sigma = sched.get("sell_sigma", 1)
        C = 32
        r = rl.copy()
        if sigma > 1:
            for s0 in range(0, r.size, sigma):
                r[s0:s0 + sigma] = -np.sort(-r[s0:s0 + sigma])
        pad = np.resize(r, ((r.size + C - 1) // C) * C)
        pad[r.size:] = 0
        return float(pad.reshape(-1, C).max(axis=1).sum() * C)
    if fmt == "bsr":
        t = sched["bsr_tile"]
        fill = block_fill(m, t)
        return float(m.nnz / fill) if fill > 0 else 0.0
    return float(m.nnz)


def feasible(m: sp.csr_matrix, sched: dict, max_blowup: float = 4.0) -> bool:
    return stored_entries(m, sched) <= max_blowup * max(m.nnz, 1)


def algorithmic_bytes(m: sp.csr_matrix, weight_bytes: int) -> float:
    """Bytes one weighted sum must move: every synapse's column index and
    weight, the row pointers, the pre-synaptic rates and the sums (read and
    written)."""
    n_post, n_pre = m.shape
    return float(m.nnz * (4 + weight_bytes) + (n_post + 1) * 4 + n_pre * 4 + 2 * n_post * 4)


def measure(m: sp.csr_matrix, sched: dict, precision: str = "float",
            weight_dtype: str = "float32", reps: int = 5, seed: int = 0, flush: bool = True):
    """Device time (ms, median of `reps` repetitions) of the weighted sum of
    matrix m (post, pre) stored with schedule `sched`: with a clean L2 flush
    before each repetition (cold), or back to back (`flush=False`: the steady
    state of a running simulation, where a matrix smaller than the L2 stays
    there)."""
    from . import Network, Neuron
    n_post, n_pre = m.shape
    net = Network(dt=1.0, seed=seed)
    cfg = {k: v for k, v in sched.items() if k != "format"}
    net.config(precision=precision, engine="grid", graph_steps=0,
               **({"weight_dtype": weight_dtype} if precision == "float" else {}), **cfg)
    inp = net.create(n_pre, Neuron(parameters="r = 0.0"))
    out = net.create(n_post, Neuron(equations="r = sum(exc)"))
    net.connect(inp, out, "exc").from_sparse(m.T.tocsr(), storage_format=sched["format"])
    inp.r = np.random.default_rng(seed).uniform(0.0, 1.0, n_pre)
    net.compile()
    nat = net._backend.native
    net.simulate_steps(1)
    times = []
    for _ in range(reps):
        if flush:
            nat.flush_l2()
        nat.kernel_timing(True)
        net.simulate_steps(1)
        nat.synchronize()
        kt = nat.kernel_times()
        nat.kernel_timing(False)
        times.append(sum(t for name, (t, _) in kt.items() if name.startswith("proj0_psp")))
    net.close()
    return float(np.median(times))


class Autotuner:
    """Exhaustive search over the feasible schedules; every measurement is
    appended to `dataset` (features, schedule, time)."""

    def __init__(self, dataset_path: str | None = None):
        self.dataset_path = dataset_path
        self.records = []
        if dataset_path and os.path.exists(dataset_path):
            with open(dataset_path) as f:
                self.records = json.load(f)

    def tune(self, m: sp.csr_matrix, precision="float", weight_dtype="float32", reps=5,
             schedules=None, tag: str = "", extra=()):
        """Time every feasible schedule (and every schedule in `extra` whose
        storage stays within 64x the synapse count); returns (best, {name: ms})."""
        wb = {"float32": 4, "bfloat16": 2, "float64": 8}[weight_dtype if precision == "float"
                                                         else "float64"]
        feat = features(m, wb)
        table = {}
        cands = list(schedules or SCHEDULES)
        for e in extra:
            if e not in cands and feasible(m, e, 64.0):
                cands.append(e)
        for s in cands:
            if not (feasible(m, s) or s in extra):
                continue
            ms = measure(m, s, precision, weight_dtype, reps)
            table[schedule_name(s)] = ms
            self.records.append({"tag": tag, "features": feat.tolist(), "schedule": schedule_name(s),
                                 "ms": ms, "bytes": algorithmic_bytes(m, wb)})
        best = min(table, key=table.get)
        return best, table

    def save(self):
        if self.dataset_path:
            with open(self.dataset_path, "w") as f:
                json.dump(self.records, f)


def heuristic(m: sp.csr_matrix, plastic: bool = False) -> str:
    """The reference's GPU format choice for rate-coded projections
    (ANNarchy/core/Projection.py:691-789)."""
    n_post, n_pre = m.shape
    if m.nnz / max(n_post * n_pre, 1) >= 0.6:
        return "dense"
    mean = m.nnz / max(1, (np.diff(m.indptr) > 0).sum())
    if mean <= 128:
        return "ellr" if plastic else "sell_1"
    return "csr"


def heuristic_schedule(m: sp.csr_matrix, plastic: bool = False) -> dict:
    """The reference's choice (heuristic) as a schedule: its GPU SELL has no
    row sorting (sell_sigma = 1)."""
    name = heuristic(m, plastic)
    return {"format": "sell", "sell_sigma": 1} if name == "sell_1" else {"format": name}
