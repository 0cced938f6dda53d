"""Known-answer cases of the reference's own test suite, run through this
backend on the GPU with the values those tests expect:

* spike transmission without delay, with a uniform and with per-synapse
  delays (ANNarchy tests_python/SpikeSynapse/test_SpikingTransmission.py:
  74-84, 154-175, 240-253): five pre-synaptic neurons spiking at t = 1 ms,
  all-to-all onto two neurons whose g_exc is reset by their equation;
* the spike condition, reset and refractory period
  (tests_python/Neuron/test_SpikingNeuron.py:73-128);
* local, global and mixed neuron updates and bounds
  (tests_python/Neuron/test_NeuronUpdate.py:81-115);
* pre- and post-spike weight updates with bounds
  (tests_python/SpikeSynapse/test_SpikingSynapse.py:60-137) and the
  time-dependent rule's compilation (:140-195);
* rate-coded connectivity patterns (tests_python/RateSynapse/
  test_RateTransmission.py:79-131).

Every case runs in double (the reference's arithmetic) and in float
precision; the expected values are small integers or tenths, exact in
both."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

from annarchy_b200 import Network, Neuron, Synapse, Uniform

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))

pytestmark = pytest.mark.gpu

PRECISIONS = ("double", "float")


def _transmission_net(precision, connect):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    emit = Neuron(spike="t==1")
    recv = Neuron(equations="g_exc = 0", spike="g_exc>30")
    pre = net.create(5, emit)
    post = net.create(2, recv)
    connect(net.connect(pre, post, "exc"))
    mon = net.monitor(post, ["g_exc"])
    net.compile()
    return net, mon


@pytest.mark.parametrize("precision", PRECISIONS)
def test_spike_transmission_no_delay(precision):
    net, mon = _transmission_net(precision, lambda p: p.all_to_all(weights=1.0))
    net.simulate(5)
    np.testing.assert_array_equal(mon.get("g_exc"),
                                  [[0, 0], [0, 0], [5, 5], [0, 0], [0, 0]])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_spike_transmission_uniform_delay(precision):
    net, mon = _transmission_net(precision, lambda p: p.all_to_all(weights=1.0, delays=3.0))
    net.simulate(6)
    np.testing.assert_array_equal(mon.get("g_exc"),
                                  [[0, 0], [0, 0], [0, 0], [0, 0], [5, 5], [0, 0]])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_spike_transmission_nonuniform_delay(precision):
    # delays per post neuron over the five pre neurons, as the reference's
    # test sets them: post 0 gets 2 events at t = 2, 2 at t = 3, 1 at t = 4;
    # post 1 gets 1, 2 and 2
    d = np.array([[1.0, 2.0, 3.0, 2.0, 1.0], [3.0, 2.0, 1.0, 2.0, 3.0]])    # (post, pre)
    w = sp.csr_matrix(np.ones((5, 2)))                                        # (pre, post)
    net, mon = _transmission_net(
        precision, lambda p: p.from_sparse(w, delays=sp.csr_matrix(d.T)))
    net.simulate(5)
    np.testing.assert_array_equal(mon.get("g_exc"),
                                  [[0, 0], [0, 0], [2, 1], [2, 2], [1, 2]])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_spike_condition_reset_refractory(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    plain = net.create(3, Neuron(equations="v = v + 1.0", spike="v == 3.0", reset="v = 1.0"))
    refr = net.create(3, Neuron(parameters="Vt = 3.0", equations="v = v + 1.0",
                                spike="v == Vt", reset="v = 1.0 ", refractory=3.0))
    glob = net.create(3, Neuron(parameters="Vt = 3.0 : population", equations="v = v + 1.0",
                                spike="v == Vt", reset="v = 1.0 "))
    net.compile()
    seen = {id(p): [float(np.asarray(p.v)[0])] for p in (plain, refr, glob)}
    for _ in range(7):
        net.simulate(1)
        for p in (plain, refr, glob):
            seen[id(p)].append(float(np.asarray(p.v)[0]))
    assert seen[id(plain)][:6] == [0, 1, 2, 1, 2, 1]
    assert seen[id(refr)] == [0, 1, 2, 1, 1, 1, 1, 2]
    assert seen[id(glob)][:6] == [0, 1, 2, 1, 2, 1]
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_neuron_update_local_global_mixed_bounds(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    local = net.create(3, Neuron(equations="""
        noise = Uniform(0,1)
        r = t
    """))
    glob = net.create(3, Neuron(equations="""
        noise = Uniform(0,1) : population
        glob_r = t : population
        r = t
    """))
    mixed = net.create(3, Neuron(parameters="glob_par = 1.0: population",
                                 equations="r = t + glob_par"))
    bound = net.create(3, Neuron(parameters="""
        min_r=1.0: population
        max_r=3.0: population
    """, equations="r = t : min=min_r, max=max_r"))
    mon = net.monitor(bound, "r")
    net.compile()
    net.simulate(5)
    np.testing.assert_array_equal(np.asarray(local.r), [4.0, 4.0, 4.0])
    np.testing.assert_array_equal(np.ravel(glob.glob_r), [4.0])
    np.testing.assert_array_equal(np.asarray(mixed.r), [5.0, 5.0, 5.0])
    np.testing.assert_array_equal(mon.get("r")[:, 0], [1, 1, 2, 3, 3])
    net.close()


def _every_step_spiking(net):
    return net.create(3, Neuron(parameters="v = 1", equations="mp = g_exc", spike="v > 0"))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pre_spike_weight_update_with_bound(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pop = _every_step_spiking(net)
    syn = Synapse(parameters="g = 1.0", pre_spike="w -= 1.0 : min=0.0")
    proj = net.connect(pop, pop, "exc", synapse=syn)
    proj.all_to_all(5.0)
    net.compile()
    np.testing.assert_array_equal(proj.dendrite(0).w, [5.0, 5.0])
    net.simulate(5)
    np.testing.assert_array_equal(proj.dendrite(0).w, [1.0, 1.0])
    net.simulate(5)
    np.testing.assert_array_equal(proj.dendrite(0).w, [0.0, 0.0])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_post_spike_weight_update_with_bound(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pop = _every_step_spiking(net)
    syn = Synapse(parameters="constant = 1.0", post_spike="w += 1.0 * constant : max=10.0")
    proj = net.connect(pop, pop, "exc", synapse=syn)
    proj.all_to_all(5.0)
    net.compile()
    np.testing.assert_array_equal(proj.dendrite(0).w, [5.0, 5.0])
    net.simulate(5)
    np.testing.assert_array_equal(proj.dendrite(0).w, [10.0, 10.0])
    net.simulate(5)
    np.testing.assert_array_equal(proj.dendrite(0).w, [10.0, 10.0])
    net.close()


def test_time_dependent_rule_compiles_and_runs():
    # Izhikevich's (2003) regular-spiking neuron with a constant drive
    izhikevich = Neuron(
        parameters="""
            a = 0.02
            b = 0.2
            c = -65.0
            d = 8.0
            I = 10.0
        """,
        equations="""
            dv/dt = 0.04 * v^2 + 5.0 * v + 140.0 - u + I + g_exc : init = -65.0
            du/dt = a * (b * v - u) : init = -13.0
        """,
        spike="v >= 30.0",
        reset="""
            v = c
            u += d
        """)
    stdp = Synapse(
        parameters="""
            tau_pre = 10.0 : projection
            tau_post = 10.0 : projection
            cApre = 0.01 : projection
            cApost = 0.0105 : projection
            wmax = 0.01 : projection
        """,
        pre_spike="""
            g_target += w
            w = clip(w - cApost * exp((t_post - t)/tau_post) , 0.0 , wmax)
        """,
        post_spike="""
            w = clip(w + cApre * exp((t_pre - t)/tau_pre) , 0.0 , wmax)
        """)
    net = Network(dt=1.0, seed=1)
    pop = net.create(100, izhikevich)
    net.connect(pop, pop, "exc", stdp).all_to_all(Uniform(-1.0, 1.0))
    net.compile()
    net.simulate(10)
    assert net._backend.native.device_error() == 0
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rate_transmission_patterns(precision):
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pop1 = net.create((3, 3), Neuron(equations="r = 1"))
    pop2 = net.create((3, 3), Neuron(equations="r = sum(exc)"))
    one = net.connect(pop1, pop2, "exc")
    one.one_to_one(weights=0.1)
    a2a = net.connect(pop1, pop2, "exc")
    a2a.all_to_all(weights=0.1)
    fnp = net.connect(pop1, pop2, "exc")
    fnp.fixed_number_pre(3, weights=0.1)
    net.compile()
    assert list(one.dendrite(3).pre_ranks) == [3]
    np.testing.assert_allclose(one.dendrite(3).w, [0.1])
    assert list(a2a.dendrite(3).pre_ranks) == list(range(9))
    np.testing.assert_allclose(a2a.dendrite(3).w, np.ones(9) * 0.1)
    assert [d.size for d in fnp.dendrites] == [3] * 9
    # after one step every post neuron sums 1 (one-to-one) + 9 + 3 rates of
    # 1.0 weighted by 0.1 (the rates of step 0 are the initial 0.0)
    net.simulate(2)
    np.testing.assert_allclose(np.ravel(pop2.r), 1.3, rtol=1e-6)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_builtin_functions(precision):
    """modulo, power and clip (tests_python/Common/test_BuiltinFunctions.py:
    52-104)."""
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pop = net.create(1, Neuron(parameters="base = 2.0", equations="""
        r = modulo(t,3)
        pr = power(base,3)
        clip_below = clip(-2, -1, 1)
        clip_within = clip(0, -1, 1)
        clip_above = clip(2, -1, 1)
    """))
    mon = net.monitor(pop, ["r", "pr", "clip_below", "clip_within", "clip_above"])
    net.compile()
    net.simulate(10)
    got = mon.get()
    np.testing.assert_array_equal(got["r"][:, 0], [0, 1, 2, 0, 1, 2, 0, 1, 2, 0])
    np.testing.assert_array_equal(got["pr"][:, 0], [8.0] * 10)
    np.testing.assert_array_equal(got["clip_below"][:, 0], [-1.0] * 10)
    np.testing.assert_array_equal(got["clip_within"][:, 0], [0.0] * 10)
    np.testing.assert_array_equal(got["clip_above"][:, 0], [1.0] * 10)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_neuron_random_variables(precision):
    """A local Uniform(0, 1) draws a different value per neuron, a
    population-level one a single value (tests_python/Common/
    test_RandomVariables.py:47-70)."""
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    loc = net.create(3, Neuron(equations="r = Uniform(0,1)"))
    glob = net.create(3, Neuron(parameters="", equations="r = Uniform(0,1) : population"))
    net.compile()
    net.simulate(1)
    r = np.asarray(loc.r)
    assert np.all((r >= 0.0) & (r <= 1.0)) and not np.allclose(r, 0.0) and r.max() != r.min()
    g = np.ravel(glob.r)
    assert g.size == 1 and 0.0 < g[0] <= 1.0
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rate_synapse_localities_psp_access_and_modified_psp(precision):
    """Synaptic, postsynaptic and projection-level parameters; pre.sum(exc)
    and post.sum(exc) in a synaptic equation; a modified psp
    (tests_python/RateSynapse/test_RateSynapse.py:15-150, which only
    compile them); here also run, with their values checked."""
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    n0 = Neuron(parameters="r = 0")
    loc = net.connect(net.create(3, n0), net.create(1, n0), "exc", synapse=Synapse(parameters="""
        a = 0.1
        b = 0.1 : postsynaptic
        c = 0.1 : projection
    """))
    loc.all_to_all(weights=1.0)
    summing = Neuron(equations="r = sum(exc)")
    syn = Synapse(equations="w = pre.sum(exc) + post.sum(exc)")
    p1, p2 = net.create(1, summing), net.create(1, summing)
    acc1 = net.connect(p1, p2, "exc", synapse=syn)
    acc1.all_to_all(weights=1.0, force_multiple_weights=True)
    net.connect(p2, p1, "exc", synapse=syn).all_to_all(weights=1.0, force_multiple_weights=True)
    q1, q2 = net.create(1, summing), net.create(1, summing)
    net.connect(q1, q2, "exc", synapse=Synapse(parameters="reversal = 1.0",
                                                 psp="w*pos(reversal-pre.r)")).all_to_all(
        weights=1.0, force_multiple_weights=True)
    net.compile()
    net.simulate(3)
    np.testing.assert_allclose(loc.get("a", flat=True), [0.1] * 3, rtol=1e-7)
    np.testing.assert_allclose(np.ravel(loc.get("b")), [0.1], rtol=1e-7)
    np.testing.assert_allclose(loc.get("c"), 0.1, rtol=1e-7)
    # nothing drives p1 / p2: all sums and weights become and stay 0
    np.testing.assert_array_equal(acc1.get("w", flat=True), [0.0])
    # q2 sums w * pos(1 - 0) = 1 from the second step on
    np.testing.assert_array_equal(np.ravel(q2.r), [1.0])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rate_learning_rules_weighted_sums(precision):
    """Hebbian, Oja and BCM learning projections with learning disabled: the
    weighted sums of one step with a pre-synaptic rate of 1.0 equal the
    weights (tests_python/RateSynapse/test_RateDefaultSynapseModels.py:
    60-90; the three rules are written out here in their textbook form)."""
    hebb = Synapse(parameters="eta = 0.01 : projection",
                   equations="dw/dt = eta * pre.r * post.r : min=0.0, explicit")
    oja = Synapse(parameters="""
        eta = 0.01 : projection
        alpha = 1.0 : projection
    """, equations="dw/dt = eta * ( pre.r * post.r - alpha * post.r^2 * w ) : min=0.0, explicit")
    bcm = Synapse(parameters="""
        eta = 0.01 : projection
        tau = 2000.0 : projection
    """, equations="""
        tau * dtheta/dt = post.r^2 - theta : postsynaptic, exponential
        dw/dt = eta * post.r * (post.r - theta) * pre.r : min=0.0, explicit
    """)
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    neuron = Neuron(equations="r=sum(Hebb)+sum(Oja)+sum(IBCM)")
    inp, out = net.create(1, neuron), net.create(1, neuron)
    for syn, target in ((hebb, "Hebb"), (oja, "Oja"), (bcm, "IBCM")):
        net.connect(inp, out, target, synapse=syn).all_to_all(weights=0.1,
                                                             force_multiple_weights=True)
    net.compile()
    net.disable_learning()
    inp.r = 1.0
    net.simulate(1)
    for target in ("Hebb", "Oja", "IBCM"):
        np.testing.assert_allclose(out.sum(target), 0.1, rtol=1e-7)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rate_continuous_update_of_all_localities(precision):
    """Projection-level, postsynaptic and synaptic variables updated every
    step (tests_python/RateSynapse/test_RateContinuousUpdate.py:15-55, which
    runs one step): after step 0, w = 0 + 0.1 + 0.2."""
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    neuron = Neuron(parameters="r=1.0")
    proj = net.connect(net.create(3, neuron), net.create(1, neuron), "exc", Synapse(equations="""
        glob_var = 0.1 : projection
        semi_glob_var = 0.2 : postsynaptic
        w = t + glob_var + semi_glob_var
    """))
    proj.all_to_all(weights=0.0)
    net.compile()
    net.simulate(1)
    np.testing.assert_allclose(proj.get("w", flat=True), [0.3] * 3, rtol=1e-7)
    np.testing.assert_allclose(proj.get("glob_var"), 0.1, rtol=1e-7)
    np.testing.assert_allclose(np.ravel(proj.get("semi_glob_var")), [0.2], rtol=1e-7)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_spiking_synapse_with_equations_every_step(golden, precision):
    """A spiking synapse whose traces are set at pre- and post-synaptic
    spikes and decay every step, w their sum (the network of
    tests_python/SpikeSynapse/test_SpikingContinuousUpdate.py:15-60): w and
    both traces after every one of 30 steps equal the reference's run
    (tests/golden/spiking_continuous.npz)."""
    g = golden("spiking_continuous")["w_pre_post"]
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    pre = net.create(1, Neuron(equations="mp=t", spike="(modulo(t,3))"))
    post = net.create(1, Neuron(equations="mp=t", spike="(modulo(t,5))"))
    proj = net.connect(pre, post, "exc", Synapse(
        pre_spike="pre_trace=pre.mp : init=0.0", post_spike="post_trace=post.mp : init=0.0",
        equations="""
            post_trace = post_trace -1 : min=0.0
            pre_trace = pre_trace -1 : min=0.0
            w = post_trace + pre_trace
        """))
    proj.all_to_all(weights=0.0)
    net.compile()
    rows = []
    for _ in range(g.shape[0]):
        net.simulate(1)
        rows.append([proj.get(n, flat=True)[0] for n in ("w", "pre_trace", "post_trace")])
    np.testing.assert_array_equal(np.asarray(rows), g)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_synapse_random_variables(precision):
    """A Normal(1.0, 0.001) draw per synapse and step in a synaptic equation
    (tests_python/Common/test_RandomVariables.py:73-115): after one step the
    weights lie within 10 sigma of 1.0 and differ."""
    from annarchy_b200 import LeakyIntegrator
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    v = net.create(5, LeakyIntegrator())
    proj = net.connect(v, v, "exc", synapse=Synapse(equations="w = Normal(1.0, 0.001)"))
    proj.fixed_number_pre(number=1, weights=0.0)
    net.compile()
    net.simulate(1)
    w = np.asarray(proj.get("w", flat=True))
    np.testing.assert_allclose(w, 1.0, atol=0.01)
    assert w.max() != w.min()
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_if_then_else(precision):
    """Conditional statements and the ite() function, nested and inside
    ODEs (tests_python/Common/test_ITE.py:15-95): r after 10 steps."""
    from models_catalog import NEURONS
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    keys = ("ite_simple", "ite_nested", "ite_ode", "ite_function", "ite_function_nested",
            "ite_function_ode")
    pops = [net.create(1, Neuron(**NEURONS[k])) for k in keys]
    net.compile()
    net.simulate(10)
    np.testing.assert_array_equal([float(np.ravel(p.r)[0]) for p in pops],
                                  [0.0, 2.0, 4.0, 0.0, 2.0, 4.0])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_global_operations(precision):
    """mean, max, min, norm1 and norm2 of a population's variable, used in
    the next step's equations (tests_python/Neuron/test_GlobalOperations.py:
    15-150): six neurons with fixed rates, and 500 with random ones."""
    from models_catalog import NEURONS
    tol = 1e-12 if precision == "double" else 1e-6
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    small = net.create(6, Neuron(**NEURONS["global_operations"]))
    large = net.create(500, Neuron(**NEURONS["global_operations"]))
    net.compile()
    small.r = [2.0, 1.0, 0.0, -5.0, -3.0, -1.0]
    vals = np.random.default_rng(3).random(500)
    large.r = vals
    net.simulate(2)
    np.testing.assert_allclose(np.asarray(small.mean_r), -1.0, rtol=tol, atol=tol)
    np.testing.assert_allclose(np.asarray(small.max_r), 2.0, rtol=tol)
    np.testing.assert_allclose(np.asarray(small.min_r), -5.0, rtol=tol)
    np.testing.assert_allclose(np.asarray(small.l1), 12.0, rtol=tol)
    np.testing.assert_allclose(np.asarray(small.l2), np.sqrt(40.0), rtol=tol)
    np.testing.assert_allclose(np.asarray(large.mean_r), vals.mean(), rtol=tol * 10)
    np.testing.assert_allclose(np.asarray(large.min_r), np.float32(vals.min()) if tol > 1e-9
                               else vals.min(), rtol=tol)
    np.testing.assert_allclose(np.asarray(large.max_r), np.float32(vals.max()) if tol > 1e-9
                               else vals.max(), rtol=tol)
    np.testing.assert_allclose(np.asarray(large.l2), np.linalg.norm(vals), rtol=tol * 10)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_user_functions_in_equations(precision):
    """A neuron's own function with nested branches and a global one from
    add_function, evaluated in the update kernel (tests_python/Common/
    test_CustomFunc.py): inputs -2, 0.5, 1.5 and 3 through one-to-one
    weights of 1."""
    from annarchy_b200 import add_function
    add_function("glob_pos(x) = pos(x)")
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    inp = net.create(4, Neuron(parameters="r = 0.0"))
    tf = net.create(4, Neuron(equations="r = transfer_function(sum(exc), 1.0)",
                              functions="transfer_function(x, t) = if x > t: if x > 2*t : "
                                        "(x - 2*t)^2 else: x - t else: 0."))
    gp = net.create(4, Neuron(equations="r = glob_pos(sum(exc))"))
    net.connect(inp, tf, "exc").one_to_one(1.0)
    net.connect(inp, gp, "exc").one_to_one(1.0)
    net.compile()
    inp.r = [-2.0, 0.5, 1.5, 3.0]
    net.simulate(1)
    np.testing.assert_allclose(np.ravel(tf.r), [0.0, 0.0, 0.5, 1.0], rtol=1e-7)
    np.testing.assert_allclose(np.ravel(gp.r), [0.0, 0.5, 1.5, 3.0], rtol=1e-7)
    np.testing.assert_allclose(tf.transfer_function([-2.0, 0.5, 1.5, 3.0], [1.0] * 4),
                               [0.0, 0.0, 0.5, 1.0])
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rate_synapse_operations(precision):
    """max, min and mean instead of the sum over a row's synapses
    (tests_python/RateSynapse/test_RateDelays.py:405-520, weights 1.0): the
    three sums equal the largest, smallest and mean pre-synaptic rate."""
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    inp = net.create((3, 3), Neuron(parameters="r=0.0"))
    out = net.create(4, Neuron(equations="r = sum(p1) + sum(p2)"))
    for target, op in (("p1", "max"), ("p2", "min"), ("p3", "mean")):
        net.connect(inp, out, target, synapse=Synapse(psp="pre.r * w", operation=op)).all_to_all(
            weights=1.0)
    net.compile()
    pre_r = np.random.default_rng(5).random((3, 3))
    inp.r = pre_r
    net.simulate(1)
    tol = 1e-12 if precision == "double" else 1e-6
    np.testing.assert_allclose(out.sum("p1"), pre_r.max(), rtol=tol)
    np.testing.assert_allclose(out.sum("p2"), pre_r.min(), rtol=tol)
    np.testing.assert_allclose(out.sum("p3"), pre_r.mean(), rtol=tol)
    net.close()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_covariance_rule_with_population_means(golden, precision):
    """mean(pre.r) and mean(post.r) in a learning rule (the covariance
    synapse of tests_python/RateSynapse/test_RateDelays.py:530-570, compiled
    there; here run): weights after each of three steps against the
    reference's own run of the same network (tests/golden/covariance.npz,
    made by make_golden.py). The means already hold the rates set before
    the first step, so each step adds dt/tau * (pre.r - mean pre) *
    (post.r - mean post)."""
    from models_catalog import SYNAPSES
    gold = golden("covariance")
    net = Network(dt=1.0, seed=1)
    net.config(precision=precision)
    neuron = Neuron(parameters="r=0")
    pre = net.create(6, neuron)
    post = net.create(2, neuron)
    proj = net.connect(pre, post, "exc", synapse=Synapse(**SYNAPSES["covariance"]))
    proj.all_to_all(weights=1.0)
    net.compile()
    pre.r, post.r = gold["pre_r"], gold["post_r"]
    for step in range(gold["w"].shape[0]):
        net.simulate(1)
        w = np.asarray(proj.get("w", flat=True)).reshape(2, 6)
        np.testing.assert_allclose(w, gold["w"][step], rtol=1e-12 if precision == "double" else 1e-6)
    net.close()
