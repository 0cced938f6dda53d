"""The C ABI entry points shaped like the reference module's set_seed,
estimate_record_size and proj<k>_wrapper.init_from_lil
(ANNarchy/generator/NanoBind/BaseTemplate.py:1-45, NanoBind/Projection.py:
20-60), called through ctypes on cuda:0 and checked against numpy."""
import numpy as np
import pytest

from annarchy_b200.core.backend import to_bf16
from annarchy_b200.runtime import lib as L

pytestmark = pytest.mark.gpu


def _lil(rng, n_rows, n_pre):
    post = rng.permutation(n_rows * 3)[:n_rows].astype(np.int32)
    pre, w, d = [], [], []
    for _ in range(n_rows):
        k = int(rng.integers(0, 9))
        pre.append(rng.choice(n_pre, k, replace=False).astype(np.int32))
        w.append(rng.normal(0.0, 1.0, k))
        d.append(rng.integers(1, 5, k).astype(np.int32))
    return post, pre, w, d


@pytest.mark.parametrize("weight_bytes", [8, 4, 2])
def test_init_from_lil_builds_the_csr_arrays(weight_bytes):
    rng = np.random.default_rng(3)
    post, pre, w, d = _lil(rng, 40, 100)
    nat = L.NativeNet(0)
    try:
        nnz = nat.init_from_lil("proj0", post, pre, w, d, requires_sorting=True,
                                weight_bytes=weight_bytes)
        order = np.argsort(post, kind="stable")
        want_col = np.concatenate([pre[i] for i in order])
        want_w = np.concatenate([w[i] for i in order])
        want_d = np.concatenate([d[i] for i in order])
        sizes = np.array([len(pre[i]) for i in order])
        assert nnz == want_col.size
        assert np.array_equal(nat.read("proj0__post_rank"), post[order])
        assert np.array_equal(nat.read("proj0__row_ptr"), np.concatenate([[0], np.cumsum(sizes)]))
        assert np.array_equal(nat.read("proj0__col"), want_col)
        got_w = nat.read("proj0__w")
        if weight_bytes == 8:
            assert np.array_equal(got_w, want_w)
        elif weight_bytes == 4:
            assert np.array_equal(got_w, want_w.astype(np.float32))
        else:
            assert np.array_equal(got_w.view(np.uint16), to_bf16(want_w.astype(np.float32)))
        nat.arrays["proj0__dly"] = (np.dtype(np.int32), (nnz,))
        assert np.array_equal(nat.read("proj0__dly"), want_d)
    finally:
        nat.close()


def test_init_from_lil_keeps_the_given_order_and_rejects_bad_input():
    nat = L.NativeNet(0)
    try:
        post = np.array([5, 2], dtype=np.int32)
        pre = [np.array([3, 1], dtype=np.int32), np.array([0], dtype=np.int32)]
        nnz = nat.init_from_lil("p", post, pre, [np.array([1.0, 2.0]), np.array([3.0])],
                                requires_sorting=False)
        assert nnz == 3
        assert nat.read("p__post_rank").tolist() == [5, 2]
        assert nat.read("p__col").tolist() == [3, 1, 0]
        with pytest.raises(L.BackendError) as e:
            nat.init_from_lil("q", post, [np.array([-1], dtype=np.int32), np.array([0], dtype=np.int32)],
                              [np.array([1.0]), np.array([1.0])])
        assert e.value.status == 1 and "negative pre rank" in str(e.value)
        assert nat.lib.anb_array_info(nat.h, b"q__col", None, None) == 1   # not created
    finally:
        nat.close()


def test_set_seed_and_estimate_record_size():
    nat = L.NativeNet(0)
    try:
        nat.set_seed(0x0123456789ABCDEF, 4, True)
        assert nat.read("rng_seed").tolist() == [0x89ABCDEF, 0x01234567]
        nat.record_declare("mon0__v", 1000, 8, 1)
        nat.record_declare("mon1__r", 4000, 8, 10)
        # 10^5 steps: 1000 x 8 B x 10^5 + 4000 x 8 B x 10^4 = 800 MB + 320 MB
        assert nat.estimate_record_size(100_000) == (800_000_000 + 320_000_000) >> 20
        nat.record_declare("mon0__v", 1000, 8, 100)            # declared again: updated
        assert nat.estimate_record_size(100_000) == (8_000_000 + 320_000_000) >> 20
    finally:
        nat.close()
