"""Batched block-sparse weighted sums on the tensor cores (tcgen05) and on the
CUDA cores, against a float64 product of the same bfloat16 operands."""
import numpy as np
import pytest
import scipy.sparse as sp

from annarchy_b200 import spmm


def _blocks(n_post, n_pre, density, seed):
    rng = np.random.default_rng(seed)
    nbr, nbc = -(-n_post // 64), -(-n_pre // 64)
    mask = rng.random((nbr, nbc)) < density
    dense = np.kron(mask, np.ones((64, 64)))[:n_post, :n_pre] * rng.normal(0, 0.05, (n_post, n_pre))
    return sp.csr_matrix(dense)


def test_canonical_layout():
    t = np.arange(64 * 64).reshape(1, 64, 64)          # [block][row][k]
    c = spmm.canonical_tiles(t)
    for r, k in [(0, 0), (7, 7), (8, 0), (0, 8), (13, 42), (63, 63)]:
        assert c[((r // 8) * 8 + k // 8) * 64 + (r % 8) * 8 + k % 8] == t[0, r, k]


def test_pack_x_reference_layout():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(16, 100)).astype(np.float32)
    xt = spmm.pack_x_reference(x)
    assert xt.size == 2 * 16 * 64
    from annarchy_b200.core.backend import from_bf16, to_bf16
    q = from_bf16(to_bf16(x))
    # instance 9, neuron 70 -> tile 1, k 6
    assert from_bf16(xt[1 * 16 * 64 + ((9 // 8) * 8 + 6 // 8) * 64 + (9 % 8) * 8 + 6]) == q[9, 70]
    # padding past n_pre is zero
    assert from_bf16(xt[1 * 16 * 64 + (0 * 8 + 5) * 64 + 0]) == 0.0   # neuron 104


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [16, 64, 128, 144, 256])
def test_tc_matches_reference(batch):
    w = _blocks(300, 200, 0.35, batch)                  # partial last block row and column
    bsb = spmm.BlockSparseBatch(w, batch)
    rng = np.random.default_rng(batch + 1)
    x = rng.uniform(0, 1, (batch, 200)).astype(np.float32)
    ref = bsb.reference(x)
    for _ in range(2):                                  # two calls in a row
        y = bsb(x, "tc")
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err <= 1e-5, err
    bsb.close()


def _blocks_sparse(n_post, n_pre, density, seed):
    """Dense 64 x 64 blocks at `density` without forming the dense matrix."""
    rng = np.random.default_rng(seed)
    nbr, nbc = -(-n_post // 64), -(-n_pre // 64)
    br, bc = np.nonzero(rng.random((nbr, nbc)) < density)
    r = (br[:, None, None] * 64 + np.arange(64)[None, :, None]).repeat(64, axis=2).ravel()
    c = (bc[:, None, None] * 64 + np.arange(64)[None, None, :]).repeat(64, axis=1).ravel()
    keep = (r < n_post) & (c < n_pre)
    v = rng.normal(0, 0.05, r.size)
    return sp.csr_matrix((v[keep], (r[keep], c[keep])), shape=(n_post, n_pre))


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [48, 64, 128, 192, 256])
def test_tc_many_block_rows(batch):
    """More block rows than resident CTAs (each CTA takes several rows and
    alternates its two accumulators), empty block rows, an odd n_post."""
    from annarchy_b200.core.backend import from_bf16, to_bf16
    w = _blocks_sparse(60001, 2000, 0.04, batch)
    bsb = spmm.BlockSparseBatch(w, batch)
    assert bsb.n_block_rows > 2 * 148
    x = np.random.default_rng(batch).uniform(0, 1, (batch, 2000)).astype(np.float32)
    wq = sp.csr_matrix((from_bf16(to_bf16(w.data.astype(np.float32))), w.indices, w.indptr), shape=w.shape)
    ref = np.asarray(wq @ from_bf16(to_bf16(x)).T.astype(np.float64)).T
    for _ in range(2):
        y = bsb(x, "tc")
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err <= 1e-5, err
    assert np.all(y[:, np.diff(w.indptr) == 0] == 0)
    bsb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [64, 128, 256])
def test_simt_matches_reference(batch):
    w = _blocks(300, 200, 0.35, batch + 7)
    bsb = spmm.BlockSparseBatch(w, batch)
    x = np.random.default_rng(3).uniform(0, 1, (batch, 200)).astype(np.float32)
    y = bsb(x, "simt")
    ref = bsb.reference(x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-5
    bsb.close()


@pytest.mark.gpu
def test_tc_empty_block_rows_and_accumulation():
    """Block rows without blocks leave y untouched; run() accumulates."""
    w = _blocks(256, 256, 0.0, 1).tolil()
    w[70, 10] = 0.5                                     # one block in block row 1
    w = w.tocsr()
    bsb = spmm.BlockSparseBatch(w, 64)
    x = np.ones((64, 256), np.float32)
    bsb.load(x)
    bsb.run("tc")
    bsb.run("tc")
    y = bsb.result()
    assert np.allclose(y[:, 70], 1.0) and np.count_nonzero(y) == 64
    bsb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("batch,n_pre", [(16, 100), (64, 200), (256, 131)])
def test_pack_x_device_matches_host(batch, n_pre):
    w = _blocks(64, n_pre, 1.0, 0)
    bsb = spmm.BlockSparseBatch(w, batch)
    x = np.random.default_rng(batch).normal(size=(batch, n_pre)).astype(np.float32)
    bsb.load(x)
    bsb.run("tc")
    bsb.result()
    assert np.array_equal(bsb.nat.read("xt"), spmm.pack_x_reference(x))
    bsb.close()
