"""Spike analysis of monitors against the reference's own functions run on
the same raster (tests/golden/spike_analysis.npz, made by
tests/golden/make_golden.py), and the monitor's time bookkeeping, names and
file output on the host."""
import os

import numpy as np
import pytest

from annarchy_b200 import Network, Neuron
from annarchy_b200.core import monitor as M

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "spike_analysis.npz"))


def spikes():
    out, at = {}, 0
    for r, n in zip(GOLD["ranks"], GOLD["sizes"]):
        out[int(r)] = GOLD["steps"][at:at + n].tolist()
        at += n
    return out


def test_raster_and_histograms():
    t, r = M.raster_plot(spikes(), dt=0.1)
    assert np.array_equal(t, GOLD["raster_t"]) and np.array_equal(r, GOLD["raster_r"])
    assert np.array_equal(M.histogram(spikes(), dt=0.1), GOLD["hist_dt"])
    assert np.array_equal(M.histogram(spikes(), bins=0.5, dt=0.1), GOLD["hist_05"])
    assert np.array_equal(M.histogram(spikes(), bins=1.0, per_neuron=True, dt=0.1), GOLD["hist_pn"])
    assert np.array_equal(M.histogram(spikes(), bins=0.5, recording_window=(100, 2400), dt=0.1),
                          GOLD["hist_win"])


def test_intervals_and_rates():
    assert np.array_equal(np.asarray(M.inter_spike_interval(spikes(), dt=0.1)), GOLD["isi"])
    pn = M.inter_spike_interval(spikes(), ranks=[1, 2, 5, 9], per_neuron=True, dt=0.1)
    assert np.array_equal(sorted(pn), GOLD["isi_pn_keys"])
    assert np.array_equal(np.concatenate([pn[k] for k in sorted(pn)]), GOLD["isi_pn_vals"])
    assert np.array_equal(np.asarray(M.coefficient_of_variation(spikes(), dt=0.1)), GOLD["cv"])
    assert np.array_equal(np.asarray(M.coefficient_of_variation(spikes(), ranks=[0, 4, 8, 12],
                                                                dt=0.1)), GOLD["cv_ranks"])
    assert M.mean_fr(spikes(), dt=0.1) == GOLD["mean_fr"]
    assert M.mean_fr(spikes(), duration=2500, dt=0.1) == GOLD["mean_fr_dur"]


@pytest.mark.parametrize("smooth", [0.0, 5.0])
@pytest.mark.parametrize("start,stop", [(0, 2300), (150, 2250)])
def test_transformations(smooth, start, stop):
    key = f"{int(smooth)}_{start}"
    np.testing.assert_array_equal(M._smoothed_rate(spikes(), start, stop, smooth, 0.1),
                                  GOLD["srate_" + key])
    np.testing.assert_array_equal(M._population_rate(spikes(), start, stop, smooth, 0.1),
                                  GOLD["prate_" + key])


def _net():
    net = Network(dt=0.1)
    P = net.create((4, 5), Neuron(parameters="tau = 10.0", equations="tau * dr/dt + r = sum(exc)"))
    inp = net.create(20, Neuron(parameters="r = 1.0"))
    net.connect(inp, P, "exc").all_to_all(0.1)
    return net, P


def test_monitor_names_periods_and_getitem():
    net, P = _net()
    m = net.monitor(P, ["r", "sum(exc)"], period=0.5, period_offset=0.2)
    assert m.period == pytest.approx(0.5) and m.period_offset == pytest.approx(0.2)
    assert M.array_name("sum(exc)") == "_sum_exc" and M.array_name("r") == "r"
    m.period = 1.0
    assert m.period_steps == 10
    with pytest.raises(ValueError):
        net.monitor(P, "sum(inh)")
    with pytest.raises(ValueError):
        net.monitor(P, "spike")
    # values appended by the drain come back per variable, reshaped to the geometry
    m._append_values("r", np.arange(40.0).reshape(2, 20), [0, 10])
    m._append_values("sum(exc)", np.ones((2, 20)), [0, 10])
    assert m["r"].shape == (2, 4, 5)
    d = m.get()
    assert set(d) == {"r", "sum(exc)"} and d["r"].shape == (0, 4, 5)
    assert m.get("sum(exc)", reshape=False).shape == (0, 20)


def test_monitor_times_and_save(tmp_path):
    net, P = _net()
    m = net.monitor(P, "r")
    m._append_values("r", np.ones((3, 20)), [0, 1, 2])
    m.get("r", keep=True)
    assert m.times() == {"r": {"start": [0], "stop": [0]}}
    m.pause()
    m.resume()
    assert m._recorded["r"]["start"] == [0, 0] and m._recorded["r"]["stop"] == [0, None]
    path = str(tmp_path / "r.npy")
    m.save(path, "r", keep=True)
    assert np.load(path).shape == (3, 20)
    with pytest.raises(ValueError):
        m.save(str(tmp_path / "r.txt"))
    m.reset()
    assert m.get("r").shape == (0, 4, 5)
