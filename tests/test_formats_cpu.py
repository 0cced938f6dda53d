"""Storage-format conversions on the CPU: every format holds exactly the
matrix it was built from."""
import numpy as np
import scipy.sparse as sp

from annarchy_b200 import workloads as wl
from annarchy_b200.generator.formats import pcsr_arrays


def _from_pcsr(d, shape):
    P, pw = d["n_panels"], d["panel_width"]
    rp = d["row_ptr"].reshape(P, -1)
    rows, cols, vals = [], [], []
    for p in range(P):
        lens = np.diff(rp[p])
        r = np.repeat(np.arange(shape[0]), lens)
        idx = np.concatenate([np.arange(a, b) for a, b in zip(rp[p][:-1], rp[p][1:])]) \
            if lens.sum() else np.zeros(0, int)
        rows.append(r)
        cols.append(d["col"][idx].astype(np.int64) + p * pw)
        vals.append(d["w"][idx])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=shape)


def test_pcsr_roundtrip_and_cta_table():
    rng = np.random.default_rng(3)
    m = wl.bernoulli_csr_skip(rng, 2000, 9000, 0.01, lambda k: rng.normal(0, 1, k))
    d = pcsr_arrays(m.indptr, m.indices, m.data, 9000, panel_width=2048, ctas=37, max_rows=300)
    assert d["n_panels"] == 5 and d["col"].dtype == np.uint16
    assert (_from_pcsr(d, m.shape) != m).nnz == 0
    # synapse arrays padded past a multiple of 8
    assert d["col"].size % 8 == 0 and d["col"].size >= m.nnz + 8
    # every (panel, row) with synapses belongs to exactly one CTA, at most 300 rows each
    rp = d["row_ptr"].reshape(5, -1)
    cover = np.zeros((5, 2000), int)
    for p, r0, r1, c in d["cta_tab"]:
        assert 0 < r1 - r0 <= 300
        cover[p, r0:r1] += 1
        # chunk row table: row of the first synapse of each 8-synapse chunk
        seg = rp[p, r0:r1 + 1]
        for i, j in enumerate(range(seg[0] & ~7, seg[-1], 8)):
            jj = max(j, seg[0])
            r = d["crow"][c + i]
            assert seg[r] <= jj < seg[r + 1]
    has = np.diff(rp, axis=1) > 0
    assert np.all(cover[has] == 1)
    # CTAs carry about the same number of synapses
    n = np.array([rp[p, r1] - rp[p, r0] for p, r0, r1, _ in d["cta_tab"]])
    assert n.max() <= 2.5 * n.mean()


def test_pcsr_single_panel_is_csr_order():
    rng = np.random.default_rng(4)
    m = wl.bernoulli_csr_skip(rng, 500, 700, 0.05, 1.0)
    d = pcsr_arrays(m.indptr, m.indices, m.data, 700)
    assert d["n_panels"] == 1
    assert np.array_equal(d["row_ptr"], m.indptr.astype(np.int32))
    assert np.array_equal(d["col"][: m.nnz], m.indices.astype(np.uint16))
