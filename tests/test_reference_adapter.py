"""The reference's own Python layer driving this backend: a network built
with the reference's API (ANNarchy 5.0.3, installed in baseline/_ref) is
instantiated through annarchy_b200.reference_module, which stands in for the
extension module the reference would generate (ANNarchyWrapper<id>,
ANNarchy/generator/NanoBind/BaseTemplate.py:1-45). The reference's
Compiler._instantiate, Population, Projection, Monitor and simulate() run
unchanged on top of it.

The reference cannot be imported inside pytest's process next to this
package's own Network (both define the same names), so each case runs
tests/reference_adapter_child.py in a child process with the reference and
the stand-ins of tests/golden/refshim on its path. Without baseline/_ref the
tests are skipped."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_SITE = os.path.join(REPO, "baseline", "_ref")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_SITE, "ANNarchy")),
                                reason="the reference is not installed in baseline/_ref")


def _child(mode: str) -> dict:
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([REF_SITE, os.path.join(HERE, "golden", "refshim"), REPO,
                                         env.get("PYTHONPATH", "")])
    p = subprocess.run([sys.executable, os.path.join(HERE, "reference_adapter_child.py"), mode],
                       env=env, cwd=REPO, capture_output=True, text=True, timeout=900)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert p.returncode == 0 and lines, p.stderr[-3000:]
    return json.loads(lines[-1])


def test_reference_instantiate_wires_connectivity_and_monitors():
    """init_from_lil from the reference's connector gives the projection the
    reference's rows and weights; refractory periods arrive in steps; one
    device monitor per reference monitor, recording after start."""
    out = _child("dry")
    assert out["csr_equal"]
    assert out["refractory_steps"] == 50
    assert out["variables"] == [["spike"], ["v"]] and out["recording"] == [True, True]


@pytest.mark.gpu
def test_reference_api_simulates_on_b200_bit_exact():
    """net.simulate(), P.v and Monitor.get() of the reference over this
    backend's double-precision path: the raster, the final potentials and
    the recorded v trace equal the reference's own run bit for bit
    (tests/golden/coba_small.npz)."""
    out = _child("run")
    assert out["time"] == 2000
    assert out["raster_equal"] and out["v_equal"] and out["v_trace_equal"], out
