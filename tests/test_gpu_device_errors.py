"""Bounded device-side waits and the error path to the host.

The grid-wide barrier of the persistent engine (anb_grid_sync) gives up
after about a second and records ANB_DEVERR_BARRIER_TIMEOUT in the
network's error word; the host turns that word into ANB_ERR_TIMEOUT with a
readable message, and the context stays usable. The test makes the wait run
out: a two-CTA launch in which only CTA 0 reaches the barrier (nobody else
arrives), so its bounded wait ends with the timeout."""
import os
import time

import numpy as np
import pytest

from annarchy_b200.generator.codegen import DEVICE_HEADER
from annarchy_b200.runtime import lib as L

pytestmark = pytest.mark.gpu


def _module(body: str) -> str:
    header = open(DEVICE_HEADER).read()
    return (header + "\n__constant__ unsigned* anb_p_gbar;\n__constant__ int* anb_p_err;\n"
            + body)


def _options():
    inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    return ["-diag-suppress=177"] + (["-I" + inc] if os.path.isdir(inc) else [])


def test_grid_barrier_wait_runs_out_and_the_host_reports_it():
    nat = L.NativeNet(0)
    try:
        nat.initialize(0.1)
        nat.create("gbar", np.zeros(2, dtype=np.uint32))
        nat.load_module(_module("""
extern "C" __global__ void lone_barrier() {
    if (blockIdx.x != 0) return;                 // CTA 1 never arrives
    anb_grid_sync(anb_p_gbar, anb_p_err);
}
extern "C" __global__ void fine() {
}
"""), _options())
        nat.plan([("lone_barrier", 2, 32, 0)])
        nat.set_graph_steps(1)
        t0 = time.time()
        nat.run(1)
        with pytest.raises(L.BackendError) as e:
            nat.synchronize()
        waited = time.time() - t0
        assert e.value.status == 5                   # ANB_ERR_TIMEOUT
        assert "barrier timeout" in str(e.value)
        assert 0.2 < waited < 30.0
        assert nat.device_error() == 1
        # the context is still usable: clear the word, run another kernel
        nat.clear_device_error()
        nat.plan([("fine", 1, 32, 0)])
        nat.run(1)
        nat.synchronize()
        assert nat.device_error() == 0
    finally:
        nat.close()


def test_other_device_errors_are_named():
    nat = L.NativeNet(0)
    try:
        nat.initialize(0.1)
        nat.write("err", np.array([3, 0, 0, 0], dtype=np.int32))
        with pytest.raises(L.BackendError) as e:
            nat.synchronize()
        assert e.value.status == 6 and "monitor" in str(e.value)
        nat.clear_device_error()
        nat.synchronize()
    finally:
        nat.close()
