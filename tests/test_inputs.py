"""Random distributions in neuron equations and PoissonPopulation
(ANNarchy/inputs/PoissonPopulation.py). The device's Philox4x32-10 draws are
pinned against the generator's published known-answer vectors and a host
restatement (bit for bit); the Poisson statistics against their binomial
expectations."""
import numpy as np
import pytest

import annarchy_b200 as ann
from annarchy_b200.parser.text import ParserError
from oracle import oracle as orc
from oracle import philox


# ---------------------------------------------------------------- host
def test_philox_known_answers():
    """Published known-answer vectors of Philox4x32-10 (Salmon et al., SC'11)."""
    def hexs(v):
        return [format(int(x), "08x") for x in v]
    assert hexs(philox.philox4x32_10(0, 0, 0, 0, 0, 0)) == ["6627e8d5", "e169c58d", "bc57ac4c", "9b00dbd8"]
    f = 0xFFFFFFFF
    assert hexs(philox.philox4x32_10(f, f, f, f, f, f)) == ["408f276d", "41c83b0e", "a20bc7c6", "6d5451fd"]
    assert hexs(philox.philox4x32_10(0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344,
                                     0xA4093822, 0x299F31D0)) == ["d16cfe09", "94fdcceb", "5001e420",
                                                                  "24126ea1"]


def test_random_distributions_extracted():
    n = ann.Neuron(parameters="sigma = 2.0",
                   equations="p = Uniform(0.0, 1.0) * 1000.0 / dt\nq = Normal(0.0, sigma) + Exponential(2.0)",
                   spike="p < 1.0")
    rd = n.desc["random_distributions"]
    assert [(r["name"], r["dist"], r["args"]) for r in rd] == [
        ("rand_0", "Uniform", ["0.0", "1.0"]), ("rand_1", "Normal", ["0.0", "sigma"]),
        ("rand_2", "Exponential", ["2.0"])]
    p = next(v for v in n.desc["variables"] if v["name"] == "p")
    assert "rand_0" in p["cpp"]
    with pytest.raises(ParserError):
        ann.Neuron(equations="r = Gamma(1.0, 2.0)").desc
    with pytest.raises(ParserError):
        ann.Neuron(equations="r = Uniform(1.0)").desc


def test_poisson_population_forms():
    net = ann.Network(dt=0.1, seed=1)
    a = net.create(ann.PoissonPopulation(100, rates=20.0))
    b = net.create(ann.PoissonPopulation((10, 10), rates=np.arange(100.0)))
    c = net.create(ann.PoissonPopulation(5, rates="amp * (1.0 + sin(2*pi*t/1000.0))/2.0",
                                         parameters={"amp": 50.0}))
    assert (a.name, b.name, c.name) == ("pop0", "pop1", "pop2")
    assert a.rates[0] == 20.0 and b.rates[3, 4] == 34.0
    assert c.neuron_type.type == "spike"
    with pytest.raises(ValueError):
        ann.PoissonPopulation(10)
    with pytest.raises(NotImplementedError):
        ann.PoissonPopulation(10, target="exc")


def test_oracle_poisson_matches_host_philox():
    """The C oracle's Poisson step (double) equals the numpy restatement of
    the same draws: p = 1000 * u / dt < rates."""
    seed = np.array([12345, 678], dtype=np.uint32)
    rates = np.linspace(1.0, 200.0, 300)
    s, i = orc.poisson_run(rates, 0.1, seed, 7, 50, t0=3)
    ws, wi = [], []
    for t in range(3, 53):
        u = philox.uniform(seed, 7, t, np.arange(300), True)
        hit = np.nonzero(1000.0 * (0.0 + (1.0 - 0.0) * u) / 0.1 < rates)[0]
        ws.append(np.full(hit.size, t))
        wi.append(hit)
    assert np.array_equal(s, np.concatenate(ws)) and np.array_equal(i, np.concatenate(wi))


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_poisson_double_equals_oracle():
    """Double precision: the device raster of a PoissonPopulation with
    per-neuron rates equals the oracle's, spike for spike."""
    net = ann.Network(dt=0.1, seed=21)
    net.config(precision="double", engine="grid")
    rates = np.linspace(1.0, 100.0, 5000)
    pop = net.create(ann.PoissonPopulation(5000, rates=rates))
    mon = net.monitor(pop, "spike")
    net.compile()
    net.simulate_steps(2000)
    s, r = mon.spike_arrays()
    seed = net._backend.native.read("rng_seed")
    os_, oi = orc.poisson_run(rates, 0.1, seed, (pop.id << 8) | 0, 2000)
    assert s.size > 1000
    assert np.array_equal(s, os_) and np.array_equal(r, oi)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "float"])
def test_device_draws_match_host_philox(precision):
    """r = Uniform(0, 1) drawn on the device equals the host restatement bit
    for bit at every step checked; a normal draw agrees to rounding."""
    net = ann.Network(dt=1.0, seed=5)
    net.config(precision=precision)
    pop = net.create(1000, ann.Neuron(equations="r = Uniform(0.0, 1.0)\nz = Normal(1.0, 2.0)"))
    net.compile()
    seed = net._backend.native.read("rng_seed")
    for t in range(3):
        net.step()
        want = philox.uniform(seed, (pop.id << 8) | 0, t, np.arange(1000), precision == "double")
        assert np.array_equal(pop.r.astype(want.dtype), want)
        w = philox.words(seed, (pop.id << 8) | 1, t, np.arange(1000))
        u1 = 1.0 - philox.uniform(seed, (pop.id << 8) | 1, t, np.arange(1000), True)
        v = [w[2], w[3], w[0], w[1]]
        hi = (v[0] >> np.uint32(6)).astype(np.uint64) << np.uint64(27)
        u2 = (hi | (v[1] >> np.uint32(5)).astype(np.uint64)).astype(np.float64) / 9007199254740992.0
        if precision == "float":
            u1 = 1.0 - philox.uniform(seed, (pop.id << 8) | 1, t, np.arange(1000), False).astype(np.float64)
            u2 = (v[0] >> np.uint32(8)).astype(np.float64) / 16777216.0
        z = 1.0 + 2.0 * np.sqrt(-2.0 * np.log(u1)) * np.cos(2 * np.pi * u2)
        np.testing.assert_allclose(pop.z, z, rtol=1e-4 if precision == "float" else 1e-12, atol=1e-5)
    net.close()


def _poisson_run(engine="auto", seed=11, steps=10000, precision="float"):
    net = ann.Network(dt=0.1, seed=seed)
    net.config(engine=engine, precision=precision)
    flat = net.create(ann.PoissonPopulation(10000, rates=20.0))
    ramp = net.create(ann.PoissonPopulation(1000, rates=np.repeat([5.0, 50.0], 500)))
    mf, mr = net.monitor(flat, "spike"), net.monitor(ramp, "spike")
    net.compile()
    net.simulate_steps(steps)
    out = mf.spike_arrays(), mr.spike_arrays(), net.engine
    net.close()
    return out


@pytest.mark.gpu
def test_poisson_statistics():
    """Spike counts within 5 binomial standard deviations of rate * dt / 1000
    per step; inter-spike intervals geometric (fraction of one-step
    intervals = p)."""
    (sf, rf), (sr, rr), _ = _poisson_run()
    p = 20.0 * 0.1 / 1000.0
    n_trials = 10000 * 10000
    assert abs(sf.size - n_trials * p) < 5 * np.sqrt(n_trials * p * (1 - p))
    for lo, hi, rate in ((0, 500, 5.0), (500, 1000, 50.0)):
        k = int(((rr >= lo) & (rr < hi)).sum())
        q = rate * 1e-4
        trials = 500 * 10000
        assert abs(k - trials * q) < 5 * np.sqrt(trials * q * (1 - q)), (rate, k)
    # ISIs of the flat population: P(ISI = 1 step) = p
    order = np.lexsort((sf, rf))
    s_sorted, r_sorted = sf[order], rf[order]
    same = r_sorted[1:] == r_sorted[:-1]
    isi = np.diff(s_sorted)[same]
    frac1 = np.mean(isi == 1)
    assert abs(frac1 - p) < 5 * np.sqrt(p * (1 - p) / isi.size)


@pytest.mark.gpu
def test_poisson_reproducible_across_engines_and_seeds():
    a = _poisson_run("grid", seed=3, steps=2000)
    b = _poisson_run("grid", seed=3, steps=2000)
    c = _poisson_run("local", seed=3, steps=2000)
    d = _poisson_run("grid", seed=4, steps=2000)
    for x, y in ((a, b), (a, c)):
        assert np.array_equal(x[0][0], y[0][0]) and np.array_equal(x[0][1], y[0][1])
        assert np.array_equal(x[1][0], y[1][0]) and np.array_equal(x[1][1], y[1][1])
    assert c[2] == "cluster"
    assert not (a[0][0].size == d[0][0].size and np.array_equal(a[0][1], d[0][1]))


# ---------------------------------------------------------------- TimedArray
def test_timed_array_schedule_steps():
    net = ann.Network(dt=0.5)
    a = net.create(ann.TimedArray(rates=np.eye(4)))
    b = net.create(ann.TimedArray(rates=np.eye(4), schedule=2.0, period=10.0))
    c = net.create(ann.TimedArray(geometry=4))
    c.update(np.eye(4), schedule=[1.0, 2.0, 5.0])
    assert a.steps() == ([0, 1, 2, 3], -1)
    assert b.steps() == ([0, 4, 8, 12], 20)
    assert c.steps() == ([2, 4, 10], -1) and c.rates.shape == (3, 4)
    assert a.schedule == [0.0, 0.5, 1.0, 1.5]
    with pytest.raises(ValueError):
        c.update(np.eye(4), schedule=[2.0, 1.0])
    with pytest.raises(ValueError):
        c.update(np.ones((2, 5)))


def _timed_net(late: bool):
    inputs = np.eye(10)
    net = ann.Network(dt=1.0)
    if late:
        pops = [net.create(population=ann.TimedArray(geometry=10)) for _ in range(4)]
        pops[0].update(rates=inputs)
        pops[1].update(rates=inputs, schedule=10.0)
        pops[2].update(rates=inputs, period=10.0)
        pops[3].update(rates=inputs, schedule=2.0, period=20.0)
    else:
        pops = [net.create(population=ann.TimedArray(rates=inputs)),
                net.create(population=ann.TimedArray(rates=inputs, schedule=10.0)),
                net.create(population=ann.TimedArray(rates=inputs, period=10.0)),
                net.create(population=ann.TimedArray(rates=inputs, schedule=2.0, period=20.0))]
    out = net.create(10, ann.Neuron(equations="r = sum(exc)\nr2 = sum(exc2)\nr3 = sum(exc3)\nr4 = sum(exc4)"))
    for p, tgt in zip(pops, ("exc", "exc2", "exc3", "exc4")):
        net.connect(p, out, tgt).one_to_one(1.0)
    net.compile()
    return net, out, pops


@pytest.mark.gpu
@pytest.mark.parametrize("late", [False, True])
def test_timed_array_known_answers(late):
    """tests_python/Interface/test_TimedArray.py (read as text): outputs after
    11, 12, 21, 12 and 25 ms for the four schedule/period combinations, with
    the arrays given at construction or set later with update()."""
    net, out, pops = _timed_net(late)
    e = np.eye(10)
    net.reset()
    net.simulate(11)
    np.testing.assert_allclose(out.r, e[9])
    net.reset()
    net.simulate(12)
    np.testing.assert_allclose(out.r, e[9])
    net.reset()
    net.simulate(11)
    net.simulate(10)
    np.testing.assert_allclose(out.r2, e[1])
    net.reset()
    net.simulate(12)
    np.testing.assert_allclose(out.r3, e[0])
    net.reset()
    net.simulate(25)
    np.testing.assert_allclose(out.r4, e[1])
    # update with reset: the new buffer restarts at the next step
    net.reset()
    net.simulate(5)
    pops[0].update(rates=2 * np.eye(10), reset=True)
    net.simulate(3)
    np.testing.assert_allclose(out.r, 2 * e[1])
    net.close()
