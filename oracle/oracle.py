"""Python driver of the CPU oracle (anb_oracle.c) — TEST INFRASTRUCTURE ONLY.

Only the test suite, ``__graft_entry__.smoke()`` (as the checker) and
``bench.py`` (the CPU baseline and the reference arm) use this module; the
backend never does.

Builds the CSR / column-view arrays the C restatement expects from the
``annarchy_b200.workloads`` networks and runs them. See anb_oracle.c for the
reference files and lines each part follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libanb_oracle.so")
SRC = os.path.join(HERE, "anb_oracle.c")
CFLAGS = ["-O3", "-ffp-contract=off", "-fopenmp", "-shared", "-fPIC", "-std=c11"]


def build(force: bool = False) -> str:
    """Compile anb_oracle.c with gcc (no contraction of multiply-adds)."""
    os.makedirs(BUILD, exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", *CFLAGS, "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def max_threads() -> int:
    return int(lib().orc_max_threads())


class _RateProj(C.Structure):
    _fields_ = [("pre", C.c_int), ("row_ptr", C.c_void_p), ("col", C.c_void_p), ("w", C.c_void_p),
                ("delay", C.c_int), ("syn_delay", C.c_void_p)]


class _CobaParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("El", "Vr", "Erev_exc", "Erev_inh", "Vt", "tau",
                                          "tau_exc", "tau_inh", "I")]


class _StdpParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("tau_plus", "tau_minus", "A_plus", "A_minus", "w_min",
                                          "w_max")]


class _SpikeProj(C.Structure):
    _fields_ = [("n_rows", C.c_int), ("post_rank", C.c_void_p), ("row_ptr", C.c_void_p),
                ("col", C.c_void_p), ("w", C.c_void_p), ("col_ptr", C.c_void_p),
                ("row_idx", C.c_void_p), ("inv_idx", C.c_void_p), ("target", C.c_int),
                ("stdp", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p),
                ("last_event", C.c_void_p), ("delay", C.c_int), ("syn_delay", C.c_void_p)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _delay_args(d, keep):
    """(uniform steps, per-synapse steps pointer) of a delay spec: an int
    (steps) or an array of steps per synapse in CSR order."""
    if d is None or np.ndim(d) == 0:
        return int(d or 1), None
    a = np.ascontiguousarray(d, dtype=np.int32)
    keep.append(a)
    return 1, _p(a).value


def rate_run(rn, steps: int | None = None, threads: int = 1, trace: bool = False,
             delays=(None, None)):
    """Runs the rate-coded network ``rn`` (workloads.RateNet) for ``steps``
    steps. ``delays``: (input projection, recurrent projection), each None,
    a uniform delay in steps or per-synapse steps in CSR order. Returns
    (r_final, r_trace or None)."""
    steps = rn.steps if steps is None else steps
    keep = []
    projs = (_RateProj * 2)()
    for k, (pre, m) in enumerate(((0, rn.w_in), (1, rn.w_rec))):
        rp = np.ascontiguousarray(m.indptr, dtype=np.int32)
        col = np.ascontiguousarray(m.indices, dtype=np.int32)
        w = np.ascontiguousarray(m.data, dtype=np.float64)
        keep += [rp, col, w]
        d, sd = _delay_args(delays[k], keep)
        projs[k] = _RateProj(pre, _p(rp).value, _p(col).value, _p(w).value, d, sd)
    r_in = np.ascontiguousarray(rn.r_in, dtype=np.float64)
    r = np.zeros(rn.n_out, dtype=np.float64)
    tr = np.zeros((steps, rn.n_out), dtype=np.float64) if trace else None
    rc = lib().orc_rate_run(C.c_int(rn.n_in), C.c_int(rn.n_out), _p(r_in), _p(r), C.c_int(2),
                            projs, C.c_double(rn.tau), C.c_double(rn.dt), C.c_double(0.0),
                            C.c_int(steps), _p(tr) if trace else None, C.c_int(threads))
    if rc:
        raise MemoryError("oracle allocation failed")
    return r, tr


class SpikeProjection:
    """Arrays of one spiking projection inside a population of n neurons.

    w_post_pre: (n_rows, n_pre_view) CSR; rows are post ranks post_ranks[r],
    columns are pre ranks pre_ranks[c] of the same population."""

    def __init__(self, n: int, w_post_pre: sp.csr_matrix, post_ranks, pre_ranks, target: int,
                 stdp: dict | None = None, delay=None):
        m = w_post_pre.tocsr()
        m.sort_indices()
        pre_ranks = np.asarray(pre_ranks, dtype=np.int32)
        self.post_rank = np.ascontiguousarray(post_ranks, dtype=np.int32)
        self.row_ptr = np.ascontiguousarray(m.indptr, dtype=np.int32)
        self.col = np.ascontiguousarray(pre_ranks[m.indices], dtype=np.int32)
        self.w = np.ascontiguousarray(m.data, dtype=np.float64).copy()
        nnz = self.col.size
        rows = np.repeat(np.arange(m.shape[0], dtype=np.int32), np.diff(m.indptr))
        order = np.lexsort((rows, self.col))            # by pre rank, then by row
        self.inv_idx = np.ascontiguousarray(order, dtype=np.int32)
        self.row_idx = np.ascontiguousarray(rows[order], dtype=np.int32)
        self.col_ptr = np.zeros(n + 1, dtype=np.int32)
        np.cumsum(np.bincount(self.col, minlength=n), out=self.col_ptr[1:])
        self.target = target
        self._keep = []
        self.delay, self.syn_delay = _delay_args(delay, self._keep)
        self.stdp = None
        self.x = self.y = self.last_event = None
        if stdp is not None:
            self.stdp = _StdpParams(**stdp)
            self.x = np.zeros(nnz, dtype=np.float64)
            self.y = np.zeros(nnz, dtype=np.float64)
            self.last_event = np.full(nnz, -10000, dtype=np.int64)

    def struct(self):
        return _SpikeProj(
            int(self.post_rank.size), _p(self.post_rank).value, _p(self.row_ptr).value,
            _p(self.col).value, _p(self.w).value, _p(self.col_ptr).value, _p(self.row_idx).value,
            _p(self.inv_idx).value, int(self.target),
            C.cast(C.pointer(self.stdp), C.c_void_p).value if self.stdp is not None else None,
            _p(self.x).value if self.x is not None else None,
            _p(self.y).value if self.y is not None else None,
            _p(self.last_event).value if self.last_event is not None else None,
            int(self.delay), self.syn_delay)


def coba_projections(cn, stdp_w_ee: sp.csr_matrix | None = None, stdp: dict | None = None,
                     delays=(None, None)):
    """Projections of a workloads.CobaNet: E->all (exc) and I->all (inh), or,
    with a plastic E->E matrix, E->E (STDP, exc), E->I (exc), I->all (inh).
    ``delays`` (exc, inh) of the E->all / I->all projections: None, uniform
    steps or per-synapse steps in CSR order."""
    n, ne = cn.n, cn.n_exc
    if stdp_w_ee is None:
        return [SpikeProjection(n, cn.w_exc, np.arange(n), np.arange(ne), 0, delay=delays[0]),
                SpikeProjection(n, cn.w_inh, np.arange(n), np.arange(ne, n), 1, delay=delays[1])]
    return [SpikeProjection(n, stdp_w_ee, np.arange(ne), np.arange(ne), 0, stdp=stdp),
            SpikeProjection(n, cn.w_exc[ne:], np.arange(ne, n), np.arange(ne), 0),
            SpikeProjection(n, cn.w_inh, np.arange(n), np.arange(ne, n), 1)]


def coba_run(cn, projections=None, steps: int | None = None, threads: int = 1,
             max_spikes: int | None = None):
    """Runs a workloads.CobaNet. Returns a dict with the spike raster (steps,
    ranks; sorted by step then rank) and the final states."""
    steps = cn.steps if steps is None else steps
    projections = projections if projections is not None else coba_projections(cn)
    n = cn.n
    prm = _CobaParams(**{f[0]: float(cn.params[f[0]]) for f in _CobaParams._fields_})
    v = np.ascontiguousarray(cn.v0, dtype=np.float64).copy()
    ge = np.zeros(n)
    gi = np.zeros(n)
    rr = np.zeros(n, dtype=np.int32)
    last = np.full(n, -10000, dtype=np.int64)
    spiked = np.zeros(n, dtype=np.int32)
    nsp = C.c_int(0)
    cap = int(max_spikes if max_spikes is not None else max(1024, n * steps // 20))
    st = np.zeros(cap, dtype=np.int32)
    si = np.zeros(cap, dtype=np.int32)
    total = C.c_int64(0)
    structs = (_SpikeProj * len(projections))(*[p.struct() for p in projections])
    refr = int(cn.refractory / cn.dt)
    rc = lib().orc_coba_run(C.c_int(n), C.byref(prm), C.c_int(refr), C.c_double(cn.dt),
                            C.c_int64(0), C.c_int(steps), _p(v), _p(ge), _p(gi), _p(rr), _p(last),
                            C.c_int(len(projections)), structs, _p(spiked), C.byref(nsp), _p(st),
                            _p(si), C.c_int64(cap), C.byref(total), C.c_int(threads))
    if rc:
        raise MemoryError("oracle allocation failed")
    if total.value > cap:
        raise RuntimeError(f"spike buffer too small ({total.value} > {cap})")
    k = total.value
    return dict(spike_steps=st[:k].copy(), spike_idx=si[:k].copy(), v=v, g_exc=ge, g_inh=gi,
                refractory_remaining=rr, last_spike=last, n_spikes=k)


def csr_rowsum(m: sp.csr_matrix, x: np.ndarray) -> np.ndarray:
    """Sequential per-row sum of w*x in CSR order (the reference's order)."""
    m = m.tocsr()
    rp = np.ascontiguousarray(m.indptr, dtype=np.int64)
    col = np.ascontiguousarray(m.indices, dtype=np.int32)
    w = np.ascontiguousarray(m.data, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(m.shape[0])
    lib().orc_csr_rowsum(C.c_int(m.shape[0]), _p(rp), _p(col), _p(w), _p(x), _p(out), C.c_int(0))
    return out


def poisson_run(rates, dt: float, seed, stream: int, steps: int, t0: int = 0, max_spikes: int | None = None):
    """Spike raster (steps, ranks) of Poisson neurons in double precision with
    the backend's Philox draws (orc_poisson_run)."""
    rates = np.ascontiguousarray(rates, dtype=np.float64)
    seed = np.ascontiguousarray(seed, dtype=np.uint32)
    cap = int(max_spikes if max_spikes is not None else max(1024, 2 * rates.size * steps * float(rates.max()) * dt / 1000 + 1024))
    st = np.zeros(cap, dtype=np.int32)
    si = np.zeros(cap, dtype=np.int32)
    lib().orc_poisson_run.restype = C.c_int64
    total = lib().orc_poisson_run(C.c_int(rates.size), _p(rates), C.c_double(dt), _p(seed),
                                  C.c_uint32(stream), C.c_int64(t0), C.c_int(steps), _p(st), _p(si),
                                  C.c_int64(cap))
    if total > cap:
        raise RuntimeError(f"spike buffer too small ({total} > {cap})")
    return st[:total].copy(), si[:total].copy()
