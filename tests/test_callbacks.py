"""`every` callbacks: the call steps the reference computes (relative to the
start of simulate(), offset within the period, negative offsets from its
end, wait, declaration order at equal steps), and simulate() running the
steps in between (a recording stand-in for the device)."""
from annarchy_b200 import Network, Neuron, every


class _Recorder:
    def __init__(self, net):
        self.net, self.t, self.runs = net, 0, []

    def run(self, n):
        self.runs.append(n)
        self.t += n


def _net():
    net = Network(dt=1.0)
    net.create(3, Neuron(parameters="r = 0.0"))
    rec = _Recorder(net)
    # compiled state without a device: the stand-in advances the step counter
    net._compiled = True
    net._backend = rec
    return net, rec


_orig = Network.current_step


def _patched(self):
    if self._compiled and isinstance(self._backend, _Recorder):
        return self._backend.t
    return _orig.fget(self)


def test_callback_schedule_and_runs():
    Network.current_step = property(_patched)
    try:
        _schedule_and_runs()
    finally:
        Network.current_step = _orig


def _schedule_and_runs():
    net, rec = _net()
    calls = []

    @every(network=net, period=100.0, offset=-10.0)
    def a(n):
        calls.append(("a", n, net.current_step))

    @every(network=net, period=50.0, offset=20.0, wait=100.0)
    def b(n):
        calls.append(("b", n, net.current_step))

    rec.t = 150
    net.simulate(300.0)
    assert [c for c in calls if c[0] == "a"] == [("a", 0, 240), ("a", 1, 340), ("a", 2, 440)]
    assert [c for c in calls if c[0] == "b"] == [("b", 0, 270), ("b", 1, 320), ("b", 2, 370),
                                                 ("b", 3, 420)]
    assert rec.t == 450 and sum(rec.runs) == 300
    # disabled: one plain run
    net.disable_callbacks()
    rec.runs.clear()
    net.simulate(10.0)
    assert rec.runs == [10] and not net.callbacks_enabled()
    net.enable_callbacks()
    net.clear_all_callbacks()
    assert net.callback_times(0, 100.0) == []
    net._compiled, net._backend = False, None
