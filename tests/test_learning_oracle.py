"""The CPU restatement of rate-coded learning against the reference's own
run of the same network (tests/golden/rate_learning.npz): weights,
post-synaptic and projection variables and the recorded rates, bit for bit."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import learning_inputs  # noqa: E402
from oracle import learning as LO  # noqa: E402

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "rate_learning.npz"))


def oracle_run():
    r_in, w = learning_inputs()
    p1 = LO.LearningProjection(w, "exc")
    p2 = LO.LearningProjection(w * 0.5, "mod")
    rec = LO.run(r_in, [p1, p2], w.shape[0], int(GOLD["steps"]),
                 events=[(7, lambda now: p2.enable_learning(now, 1.0, 3.0, 1.0))])
    return rec, p1, p2


def test_oracle_equals_reference():
    rec, p1, p2 = oracle_run()
    assert p2.offset == 1 and p2.period == 3
    np.testing.assert_array_equal(rec, GOLD["r"])
    np.testing.assert_array_equal(np.asarray(p1.w), GOLD["w1"])
    np.testing.assert_array_equal(np.asarray(p2.w), GOLD["w2"])
    np.testing.assert_array_equal(np.asarray(p1.alpha), GOLD["alpha1"])
    np.testing.assert_array_equal(np.asarray(p2.alpha), GOLD["alpha2"])
    assert p1.beta == GOLD["beta1"] and p2.beta == GOLD["beta2"]
