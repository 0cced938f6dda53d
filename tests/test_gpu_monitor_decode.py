"""Device-side decoding of spike rings against the host decoder."""
import numpy as np
import pytest

from annarchy_b200.runtime import lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("steps,words,n", [(1000, 125, 4000), (37, 7, 200), (5, 1, 17), (300, 40, 1280)])
def test_monitor_decode_matches_host(steps, words, n):
    rng = np.random.default_rng(steps + words)
    ring = (rng.random((steps, words * 32)) < 0.03).astype(np.uint8)
    ring[0] = 0                       # an empty row
    ring[min(2, steps - 1)] = 1       # a full row (bits >= n must be ignored)
    buf = np.packbits(ring, axis=1, bitorder="little").view(np.uint32).reshape(steps, words)
    nat = L.NativeNet(0)
    nat.initialize(0.1)
    nat.create("ring", np.concatenate([buf, np.zeros((3, words), np.uint32)]))  # spare rows
    s_dev, r_dev = nat.monitor_decode("ring", steps, words, n)
    s_host, r_host = L.bitmap_decode(buf, n)
    assert np.array_equal(s_dev, s_host) and np.array_equal(r_dev, r_host)
    assert r_dev.max(initial=0) < n
    nat.close()


def test_monitor_decode_rejects_rows_beyond_array():
    nat = L.NativeNet(0)
    nat.initialize(0.1)
    nat.create("ring", np.zeros((4, 2), np.uint32))
    with pytest.raises(L.BackendError):
        nat.monitor_decode("ring", 5, 2, 64)
    nat.close()
