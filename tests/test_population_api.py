"""Population.sum(target): the weighted sum of the last step
(ANNarchy/core/Population.py, sum), as the reference's rate transmission
tests read it (tests_python/RateSynapse/test_RateTransmission.py)."""
import numpy as np
import pytest

import annarchy_b200 as ann


def test_sum_before_compile_and_errors():
    net = ann.Network()
    p = net.create((3, 3), ann.Neuron(equations="r = sum(exc)"))
    assert p.sum("exc").shape == (3, 3) and not p.sum("exc").any()
    with pytest.raises(ValueError):
        p.sum("inh")
    s = net.create(4, ann.Neuron(equations="v = 0.0", spike="v > 1"))
    with pytest.raises(NotImplementedError):
        s.sum("exc")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "float"])
def test_sum_after_steps(precision):
    """r = 1 in the pre population; all-to-all weights 0.1 from 9 neurons:
    the sum on exc is 0.9 from the second step on (the first step sums the
    initial rates, 0), and stays readable after the update consumed it."""
    net = ann.Network(dt=1.0)
    net.config(precision=precision)
    pre = net.create((3, 3), ann.Neuron(equations="r = 1"))
    post = net.create((3, 3), ann.Neuron(equations="r = sum(exc)"))
    net.connect(pre, post, "exc").all_to_all(weights=0.1)
    net.compile()
    net.simulate(1)
    np.testing.assert_allclose(post.sum("exc"), np.zeros((3, 3)))
    net.simulate(1)
    np.testing.assert_allclose(post.sum("exc"), np.full((3, 3), 0.9), rtol=1e-6)
    np.testing.assert_allclose(post.r, np.full((3, 3), 0.9), rtol=1e-6)
    net.close()
