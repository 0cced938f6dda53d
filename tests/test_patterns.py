"""Distance-based connectors (gaussian, dog) against the connectivity that
the reference's own connector code built for the same geometries
(tests/golden/connect_patterns.npz, made by tests/golden/make_golden.py):
the same dendrites, pre ranks and float32-rounded weights."""
import os

import numpy as np
import pytest

from annarchy_b200 import Network, Neuron

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "connect_patterns.npz"))

PATTERNS = {
    "g2_self": ("gaussian", (12, 10), None, dict(amp=1.0, sigma=0.3, limit=0.01)),
    "g2_map": ("gaussian", (15, 9), (8, 6), dict(amp=2.5, sigma=0.2, limit=0.05)),
    "g1": ("gaussian", (40,), (30,), dict(amp=1.0, sigma=0.1, limit=0.01)),
    "g3_self": ("gaussian", (5, 4, 3), None, dict(amp=0.7, sigma=0.35, limit=0.02)),
    "dog2_self": ("dog", (12, 10), None, dict(amp_pos=1.0, sigma_pos=0.2, amp_neg=0.5,
                                              sigma_neg=0.5, limit=0.01)),
    "dog2_map": ("dog", (10, 10), (7, 9), dict(amp_pos=1.5, sigma_pos=0.15, amp_neg=1.0,
                                               sigma_neg=0.3, limit=0.02)),
}


@pytest.mark.parametrize("key", list(PATTERNS))
def test_pattern_matches_reference(key):
    kind, g_pre, g_post, kw = PATTERNS[key]
    net = Network(dt=0.1)
    neuron = Neuron(parameters="r = 0.0")
    pre = net.create(g_pre, neuron)
    post = pre if g_post is None else net.create(g_post, neuron)
    proj = net.connect(pre, post, "exc")
    getattr(proj, kind)(**kw)
    m = proj._csr
    sizes = np.diff(m.indptr)
    assert np.array_equal(np.nonzero(sizes)[0], GOLD[key + "__post"])
    assert np.array_equal(sizes[sizes > 0], GOLD[key + "__sizes"])
    assert np.array_equal(m.indices, GOLD[key + "__pre"])
    assert np.array_equal(m.data, GOLD[key + "__w"])


def test_pattern_rejects_views():
    net = Network(dt=0.1)
    p = net.create((10, 10), Neuron(parameters="r = 0.0"))
    with pytest.raises(ValueError):
        net.connect(p[:50], p, "exc").gaussian(1.0, 0.2)
