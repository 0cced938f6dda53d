"""Distance-based patterns (gaussian, difference of Gaussians) generated on
the device (anb_connect_distance_pattern) against the host construction,
which equals the reference's connector bit for bit
(tests/golden/connect_patterns.npz, tests/test_patterns.py): the same rows,
pre ranks and float32 values, for rate-coded projections (the CSR comes back
for the storage format) and spiking ones (kept on the device)."""
import numpy as np
import pytest

from annarchy_b200 import Network, Neuron
from annarchy_b200 import workloads as wl

pytestmark = pytest.mark.gpu

CASES = [
    ("gaussian", (40, 30), None, dict(amp=1.0, sigma=0.3, limit=0.01)),
    ("gaussian", (45, 27), (24, 18), dict(amp=2.5, sigma=0.2, limit=0.05)),
    ("gaussian", (400,), (300,), dict(amp=1.0, sigma=0.1, limit=0.01)),
    ("gaussian", (12, 10, 6), None, dict(amp=0.7, sigma=0.35, limit=0.02)),
    ("dog", (36, 30), None, dict(amp_pos=1.0, sigma_pos=0.2, amp_neg=0.5, sigma_neg=0.5,
                                 limit=0.01)),
    ("dog", (30, 30), (21, 27), dict(amp_pos=1.5, sigma_pos=0.15, amp_neg=1.0, sigma_neg=0.3,
                                     limit=0.02)),
]


def _rate_pattern(kind, g_pre, g_post, kw, device):
    net = Network(dt=1.0, seed=1)
    net.config(precision="double", device_connectors=device)
    neuron = Neuron(parameters="r = 0.0")
    pre = net.create(g_pre, neuron)
    post = pre if g_post is None else net.create(g_post, Neuron(
        parameters="tau = 10.0", equations="tau * dr/dt + r = sum(exc)"))
    if g_post is None:
        pre = net.create(g_pre, neuron)
        post = net.create(g_pre, Neuron(parameters="tau = 10.0",
                                        equations="tau * dr/dt + r = sum(exc)"))
    proj = getattr(net.connect(pre, post, "exc"), kind)(**kw)
    net.compile()
    out = proj.csr_population_ranks()
    net.close()
    return out


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_pattern_equals_host_pattern(case):
    kind, g_pre, g_post, kw = CASES[case]
    host = _rate_pattern(kind, g_pre, g_post, kw, False)
    dev = _rate_pattern(kind, g_pre, g_post, kw, True)
    assert host[2].size > 1000
    for a, b in zip(host, dev):
        assert np.array_equal(a, b)


def test_device_pattern_spiking_self_projection():
    """A spiking population connected to itself with a gaussian pattern (the
    self-pairs dropped), kept on the device: its rows and weights equal the
    host construction."""
    res = []
    for device in (False, True):
        net = Network(dt=0.1, seed=2)
        net.config(precision="double", engine="grid", device_connectors=device)
        P = net.create((50, 40), wl.coba_neuron(dict(wl.COBA_PARAMS)))
        proj = net.connect(P, P, "exc").gaussian(amp=0.3, sigma=0.1, limit=0.05)
        net.compile()
        nat = net._backend.native
        k = proj.id
        rp = nat.read(f"proj{k}__row_ptr").astype(np.int64)
        col = nat.read(f"proj{k}__col").astype(np.int64)
        w = nat.read(f"proj{k}__w").astype(np.float64)
        if not device:
            post, rp_h, col_h, w_h = proj.csr_population_ranks()
            full = np.zeros(P.size + 1, np.int64)
            np.add.at(full, post.astype(np.int64) + 1, np.diff(rp_h))
            rp, col, w = np.cumsum(full), col_h.astype(np.int64), w_h
        res.append((rp, col, w))
        net.close()
    (rp_h, col_h, w_h), (rp_d, col_d, w_d) = res
    assert col_h.size > 10000
    assert np.array_equal(rp_h, rp_d) and np.array_equal(col_h, col_d) and np.array_equal(w_h, w_d)
    rows = np.repeat(np.arange(rp_d.size - 1), np.diff(rp_d))
    assert not np.any(rows == col_d)                   # no self-connections
