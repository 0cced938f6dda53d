"""The selector's forward pass without allocation (anb_mlp_predict_noalloc).

Callers that cannot allocate device memory — a simulation loop with
real-time deadlines, where an allocation's implicit device synchronisation
would stall it, or a program whose device memory belongs to another
allocator — pass device buffers they own for the parameters, inputs and
outputs; the activations go to a fixed array inside the library. This test
calls that entry point through the C ABI with device buffers (allocated here
by torch, standing in for the caller's own memory) and compares it with the
allocating anb_mlp_predict, on two calls in a row with different inputs.

This file is collected last so that a failure here stops a run only after
every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from annarchy_b200 import selector as S
from annarchy_b200.runtime import lib as L

pytestmark = pytest.mark.gpu


def _host_predict(params, x, n_in, hidden, n_out):
    lib = L.load()
    y = np.zeros((x.shape[0], n_out), np.float32)
    L.check_selector("anb_mlp_predict", lib.anb_mlp_predict(
        params.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p), x.shape[0], n_in, hidden,
        n_out, y.ctypes.data_as(C.c_void_p)))
    return y


def test_noalloc_forward_matches_allocating_forward_twice():
    import torch
    lib = L.load()
    n_in, hidden, n_out = 13, 64, 9
    params = S.init_params(n_in, hidden, n_out, seed=5)
    rng = np.random.default_rng(7)
    dev = torch.device("cuda:0")
    d_params = torch.from_numpy(params).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call, n in enumerate((300, 1000)):          # two calls, different sizes and inputs
        x = rng.normal(size=(n, n_in)).astype(np.float32)
        d_x = torch.from_numpy(x).to(dev)
        d_y = torch.full((n, n_out), float("nan"), device=dev)
        torch.cuda.synchronize()
        L.check_selector("anb_mlp_predict_noalloc", lib.anb_mlp_predict_noalloc(
            C.c_void_p(d_params.data_ptr()), C.c_void_p(d_x.data_ptr()), n, n_in, hidden, n_out,
            C.c_void_p(d_y.data_ptr()), C.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        got = d_y.cpu().numpy()
        want = _host_predict(params, x, n_in, hidden, n_out)
        assert np.all(np.isfinite(got)), call
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch
    lib = L.load()
    limit = lib.anb_mlp_noalloc_max_floats()
    n_in, hidden, n_out = 13, 64, 9
    n = limit // (2 * hidden) + 1
    dev = torch.device("cuda:0")
    d_params = torch.zeros(S.param_count(n_in, hidden, n_out), device=dev)
    d_x = torch.zeros((n, n_in), device=dev)
    d_y = torch.zeros((n, n_out), device=dev)
    status = lib.anb_mlp_predict_noalloc(C.c_void_p(d_params.data_ptr()), C.c_void_p(d_x.data_ptr()),
                                         n, n_in, hidden, n_out, C.c_void_p(d_y.data_ptr()), None)
    assert status == 1          # ANB_ERR_ARG
    assert b"exceeds the limit" in lib.anb_selector_last_error()
