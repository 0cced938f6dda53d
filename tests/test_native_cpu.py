"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/annarchy_b200.h declares, and every generated module compiles for
sm_100a (NVRTC) without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from annarchy_b200 import workloads as wl
from annarchy_b200.runtime import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "annarchy_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(anb_\w+)\s*\(", txt)))


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
        assert n in L.SIGNATURES, n


def test_no_device_here_reports_cleanly():
    if L.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(L.BackendError):
        L.NativeNet(0)


def _modules():
    rn = wl.rate_net(seed=7, n_in=100, n_out=200, p_in=0.1, p_rec=0.05, steps=10)
    cn = wl.coba_net(seed=7, n=400, p=0.05, steps=10)
    w_ee = wl.stdp_matrix(cn, 7, 0.05)
    yield "rate-double", wl.build_rate_network(rn, "double")[0]
    yield "rate-float", wl.build_rate_network(rn, "float")[0]
    yield "rate-bf16", wl.build_rate_network(rn, "float", weight_dtype="bfloat16")[0]
    for fmt in ("ell", "ellr", "sell", "hyb", "pcsr"):
        yield "rate-" + fmt, wl.build_rate_network(rn, "double", storage_format=fmt)[0]
        yield "rate-float-" + fmt, wl.build_rate_network(rn, "float", storage_format=fmt)[0]
    for prec in ("double", "float"):
        for eng in ("grid", "local"):
            yield f"coba-{prec}-{eng}", wl.build_coba_network(cn, prec, eng)[0]
        yield f"stdp-{prec}", wl.build_coba_network(cn, prec, stdp_w_ee=w_ee)[0]


@pytest.mark.parametrize("name,net", list(_modules()), ids=lambda x: x if isinstance(x, str) else "")
def test_generated_module_compiles_for_sm100a(name, net):
    mod = net.generate_code()
    size, log = L.nvrtc_compile(mod.source, mod.options)
    assert size > 0
    assert "error" not in log.lower()
