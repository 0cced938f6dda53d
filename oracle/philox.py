"""Philox4x32-10 on the host — TEST INFRASTRUCTURE ONLY.

A numpy restatement of the counter-based generator of Salmon, Moraes, Dror
and Shaw ("Parallel random numbers: as easy as 1, 2, 3", SC'11) as the
backend draws it on the device for random distributions inside neuron
equations: counter (neuron index, step low word, step high word, stream),
key = the network's two seed words; uniform floats from the top 24 bits of
the first word, doubles from 53 bits of the first two. The reference draws
from std::mt19937 (ANNarchy/generator/Population/SingleThreadGenerator.py,
update_rng), whose stream this backend does not reproduce: parity of the
draws is pinned here (published known-answer vectors, then device = host bit
for bit), parity of the simulated statistics in the tests.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10: counters and keys as uint32 arrays (or
    scalars); returns the four output words."""
    c = [np.asarray(x, dtype=np.uint32).copy() for x in (c0, c1, c2, c3)]
    k0 = np.asarray(k0, dtype=np.uint32).copy()
    k1 = np.asarray(k1, dtype=np.uint32).copy()
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = M0 * c[0].astype(np.uint64)
            p1 = M1 * c[2].astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), p0.astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), p1.astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
            k0 = k0 + W0
            k1 = k1 + W1
    return c


def words(seed, stream: int, t: int, idx):
    idx = np.asarray(idx, dtype=np.uint64)
    t = np.uint64(t)
    return philox4x32_10(idx.astype(np.uint32), np.full(idx.shape, t & np.uint64(0xFFFFFFFF), np.uint32),
                         np.full(idx.shape, t >> np.uint64(32), np.uint32),
                         np.full(idx.shape, stream, np.uint32), seed[0], seed[1])


def uniform(seed, stream: int, t: int, idx, double: bool):
    """The device's anb_unit of draw (seed, stream, t, idx): [0, 1)."""
    w = words(seed, stream, t, idx)
    if double:
        hi = (w[0] >> np.uint32(6)).astype(np.uint64) << np.uint64(27)
        return (hi | (w[1] >> np.uint32(5)).astype(np.uint64)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (w[0] >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
