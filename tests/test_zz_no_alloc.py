"""The allocation-free ray query, lam_trace_rays_static, called through the C-ABI.

It exists for callers that cannot allocate device memory while they run (for example a render
loop with a fixed frame budget, where cudaMalloc / cudaFree can synchronise the device and stall
the frame).  Its results must equal lam_trace_rays' bit for bit - the same traversal, with the
work counter and error flags in a static device array instead of a per-call allocation - on
consecutive calls (the array keeps the previous call's contents and must be cleared each time).
This file is collected last so that a failure here cannot hide the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes

pytestmark = pytest.mark.gpu


def _bind():
    L = lb.lib()
    f = L.lam_trace_rays_static
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    return f


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(-12, 12, (n, 3))
    r[:, 4:7] = rng.normal(size=(n, 3))
    r[:, 3], r[:, 7] = 1e-4, 1000.0
    return r


def test_static_trace_matches_allocating_trace_on_consecutive_calls():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    static_trace = _bind()
    s = scenes.icosphere_field(64, 64, instances=8, subdiv=3, tex_size=16, tex_layers=2, seed=21)
    g = lb.GpuScene(s)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (seed, mode) in enumerate([(1, _abi.TRACE_CLOSEST), (2, _abi.TRACE_CLOSEST), (3, _abi.TRACE_ANY)]):
        n = 300_000 + 17 * call
        rays = torch.from_numpy(_rays(n, seed)).cuda()
        ref = torch.zeros((n, 6), dtype=torch.int32, device="cuda")
        got = torch.full((n, 6), -1, dtype=torch.int32, device="cuda")
        g.trace(rays, ref, mode)
        rc = static_trace(g._h, C.c_void_p(rays.data_ptr()), n, mode, C.c_void_p(got.data_ptr()), C.c_void_p(stream))
        assert rc == 0, lb.lib().lam_last_error_message()
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"call {call}: results differ from lam_trace_rays"
        assert (ref[:, 5] != 0).any()


def test_static_trace_rejects_too_many_rays():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    static_trace = _bind()
    g = lb.GpuScene(scenes.cornell_box(16, 16))
    dummy = torch.zeros(8, dtype=torch.float32, device="cuda")
    rc = static_trace(g._h, C.c_void_p(dummy.data_ptr()), 0x80000000, _abi.TRACE_CLOSEST, C.c_void_p(dummy.data_ptr()),
                      None)
    assert rc == _abi.ERR_INVALID_ARGUMENT
    assert b"LAM_TRACE_STATIC_MAX_RAYS" in lb.lib().lam_last_error_message()
