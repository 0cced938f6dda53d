"""Storage-format conversions on the CPU: every format holds exactly the
matrix it was built from."""
import numpy as np
import scipy.sparse as sp

from annarchy_b200 import workloads as wl
from annarchy_b200.generator.formats import PCSR_HEADER, pcsr_arrays, pcsr_weights


def _step_panels(d):
    """Panel of every step, from the CTA table (CTAs cover the steps in order)."""
    panel = np.full(d["n_steps"], -1)
    wt = d["warp_tab"].reshape(d["cta_panel"].size, -1, 3)
    for c, p in enumerate(d["cta_panel"]):
        for sb, se, _ in wt[c]:
            assert np.all(panel[sb:se] == -1)       # every step belongs to one warp
            panel[sb:se] = p
    assert np.all(panel >= 0)
    return panel


def _decode(d, bf16=False):
    """Walk the steps as the kernel does: a header step (column >= 0xF000)
    names the rows of the slice, the steps after it hold their elements."""
    col = d["col"][: d["padded"]].reshape(-1, 32).astype(np.int64)
    is_head = col[:, 0] >= PCSR_HEADER
    assert np.all((col >= PCSR_HEADER) == is_head[:, None])   # warp-uniform
    assert np.array_equal(np.nonzero(is_head)[0], d["header"])
    slice_of = np.cumsum(is_head) - 1
    v = d["header_val"].reshape(-1, 32)
    if bf16:       # the column carries the high bits, the weight slot the low 16
        hi = (col[d["header"]] & 0xFFF) << 16
        assert np.array_equal(hi | (v & 0xFFFF), v)
    return is_head, v[slice_of] - 1


def _from_pcsr(d, shape):
    """Rebuild the matrix from the sliced panels (padding has weight 0)."""
    is_head, rows = _decode(d)
    e = 32 * np.arange(d["n_steps"])[:, None] + np.arange(32)[None, :]
    cols = d["col"][e].astype(np.int64) + _step_panels(d)[:, None] * d["panel_width"]
    keep = (rows >= 0) & (d["w"][e] != 0) & ~is_head[:, None]
    return sp.csr_matrix((d["w"][e][keep], (rows[keep], cols[keep])), shape=shape)


def test_pcsr_roundtrip_and_work_split():
    rng = np.random.default_rng(3)
    m = wl.bernoulli_csr_skip(rng, 2000, 9000, 0.01, lambda k: rng.normal(0, 1, k))
    d = pcsr_arrays(m.indptr, m.indices, m.data, 9000, panel_width=2048, ctas=37, warps=4)
    assert d["n_panels"] == 5 and d["col"].dtype == np.uint16
    assert (_from_pcsr(d, m.shape) != m).nnz == 0
    assert d["padded"] == 32 * d["n_steps"] and d["col"].size == d["padded"] + 8
    # every (panel, row) with synapses is one lane of exactly one slice
    panel = _step_panels(d)
    lanes = d["header_val"].reshape(-1, 32) - 1
    seen = set()
    for s_, p in enumerate(panel[d["header"]]):
        for r in lanes[s_][lanes[s_] >= 0]:
            assert (p, r) not in seen
            seen.add((int(p), int(r)))
    rows = np.repeat(np.arange(2000), np.diff(m.indptr))
    assert seen == set(zip((m.indices // 2048).tolist(), rows.tolist()))
    # warps name the header of the slice holding their first step; CTAs
    # carry about equal numbers of steps
    wt = d["warp_tab"]
    busy = wt[:, 1] > wt[:, 0]
    at = np.searchsorted(d["header"], wt[busy, 0], side="right") - 1
    assert np.array_equal(wt[busy, 2], d["header"][at])
    n = wt.reshape(d["cta_panel"].size, -1, 3)
    n = n[:, -1, 1] - n[:, 0, 0]
    assert n.max() <= 2.5 * n.mean()


def test_pcsr_header_weights():
    """Header rows survive the conversion of the weights to the device type:
    all 32 bits in float32, the low 16 (with 12 more in the column) in
    bfloat16."""
    from annarchy_b200.core.backend import to_bf16
    rng = np.random.default_rng(6)
    m = wl.bernoulli_csr_skip(rng, 400, 300, 0.05, lambda k: rng.normal(0, 1, k))
    post = 70000 + rng.permutation(400)             # indices above 16 bits
    d = pcsr_arrays(m.indptr, m.indices, m.data, 300, post_rank=post, warps=8)
    idx = (32 * d["header"][:, None] + np.arange(32)).reshape(-1)
    w32 = pcsr_weights(d, lambda x: np.asarray(x, np.float32))
    assert np.array_equal(w32.view(np.uint32)[idx], d["header_val"].astype(np.uint32))
    data = np.ones(w32.size, bool)
    data[idx] = False
    assert np.array_equal(w32[:d["padded"]][data[:d["padded"]]],
                          d["w"][:d["padded"]][data[:d["padded"]]].astype(np.float32))
    w16 = pcsr_weights(d, to_bf16)
    col = d["col"][idx].astype(np.int64)
    got = ((col & 0xFFF) << 16) | w16[idx].astype(np.int64)
    assert np.array_equal(got, d["header_val"])
    _decode(d, bf16=True)


def test_pcsr_post_ranks_and_empty():
    rng = np.random.default_rng(5)
    m = wl.bernoulli_csr_skip(rng, 300, 400, 0.02, 1.0)
    post = rng.permutation(1000)[:300]
    d = pcsr_arrays(m.indptr, m.indices, m.data, 400, post_rank=post, warps=8)
    ref = sp.csr_matrix((m.data, m.indices, m.indptr), shape=m.shape).tocoo()
    full = sp.csr_matrix((ref.data, (post[ref.row], ref.col)), shape=(1000, 400))
    assert (_from_pcsr(d, (1000, 400)) != full).nnz == 0
    e = pcsr_arrays(np.zeros(11, np.int64), np.zeros(0, np.int64), np.zeros(0), 64, warps=8)
    assert e["n_steps"] == 0 and e["cta_panel"].size == 1
    assert np.all(e["warp_tab"][:, 1] == e["warp_tab"][:, 0])


def test_pcsr_slices_sorted_by_length():
    """Rows of a panel are sorted by length (longest first), so a slice pads
    little; a uniform matrix stores little more than its synapses and one
    header per 32 rows."""
    rng = np.random.default_rng(4)
    m = wl.bernoulli_csr_skip(rng, 500, 700, 0.05, 1.0)
    d = pcsr_arrays(m.indptr, m.indices, m.data, 700)
    assert d["n_panels"] == 1 and (_from_pcsr(d, m.shape) != m).nnz == 0
    lens = np.diff(m.indptr)
    lanes = d["header_val"].reshape(-1, 32) - 1
    got = np.where(lanes >= 0, lens[np.maximum(lanes, 0)], -1).reshape(-1)
    got = got[got >= 0]
    assert np.all(np.diff(got) <= 0) and got.size == np.count_nonzero(lens)
    assert d["padded"] <= 1.15 * m.nnz
    # columns within a row keep their CSR order (after the slice's header)
    r = lanes[0, 0]
    e = 32 * (1 + np.arange(lens[r]))
    assert np.array_equal(d["col"][e].astype(np.int64), m.indices[m.indptr[r]:m.indptr[r + 1]])
