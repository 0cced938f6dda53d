"""Host restatement of the device connectors' random draws (test
infrastructure): the SplitMix64-finalised counter hash and the geometric
skipping of anb_connect_fixed_probability_rows, vectorised over rows, so a
device-built projection can be checked synapse by synapse."""
import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def u01(seed, row, slot, stream):
    """53-bit uniform in [0, 1) of (seed, row, slot, stream)."""
    row = np.asarray(row, dtype=np.int64).astype(np.uint64)
    slot = np.asarray(slot, dtype=np.int64).astype(np.uint64)
    with np.errstate(over="ignore"):
        inner = row * np.uint64(0x100000001B3) + slot * np.uint64(4) + np.uint64(stream)
    h = mix64(np.uint64(seed) ^ mix64(inner))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def weights(seed, grow, slot, wkind, a, b):
    if wkind == 1:
        return a + (b - a) * u01(seed, grow, slot, 1)
    if wkind == 2:
        u1 = 1.0 - u01(seed, grow, slot, 1)
        u2 = u01(seed, grow, slot, 2)
        return a + b * np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
    return np.full(np.shape(grow), float(a))


def fixed_probability(n_post, post_base, row_offset, pre_lo, pre_hi, p, seed, exclude_self,
                      wkind=0, a=1.0, b=0.0):
    """(row_ptr, col, w) of the device's fixed-probability rows."""
    n = pre_hi - pre_lo
    with np.errstate(divide="ignore"):
        lq = np.log1p(-p)
    rows = np.arange(n_post, dtype=np.int64)
    grow = row_offset + rows
    post = post_base + rows
    pos = np.full(n_post, pre_lo - 1, dtype=np.int64)
    active = np.ones(n_post, dtype=bool)
    out_r, out_c = [], []
    k = 0
    while active.any():
        idx = np.nonzero(active)[0]
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.floor(np.log1p(-u01(seed, grow[idx], k, 3)) / lq)
        g = np.where(g <= n, g, n)
        pos[idx] += 1 + np.maximum(g, 0).astype(np.int64)
        done = pos[idx] >= pre_hi
        active[idx[done]] = False
        keep = idx[~done]
        if exclude_self:
            keep = keep[pos[keep] != post[keep]]
        out_r.append(keep)
        out_c.append(pos[keep].copy())
        k += 1
    r = np.concatenate(out_r) if out_r else np.zeros(0, np.int64)
    c = np.concatenate(out_c) if out_c else np.zeros(0, np.int64)
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    counts = np.bincount(r, minlength=n_post)
    row_ptr = np.concatenate([[0], np.cumsum(counts)])
    slot = np.arange(r.size) - row_ptr[r]
    w = weights(seed, grow[r], slot, wkind, a, b)
    return row_ptr, c, w
