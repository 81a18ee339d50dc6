"""Follow-up passes against the oracle on identical inputs: temporal / spatial ReSTIR-GI resampling,
end-of-frame processing (DataBuffers::advance_frame) and the frame average."""
import ctypes

import numpy as np
import pytest
import torch

import lambent_b200 as lb
from lambent_b200 import _abi, scenes
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu

_cudart = ctypes.CDLL("libcudart.so")


def d2h(ptr, nbytes, dtype, shape):
    torch.cuda.synchronize()
    host = np.empty(nbytes, np.uint8)
    assert _cudart.cudaMemcpy(host.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(ptr), ctypes.c_size_t(nbytes), 2) == 0
    return host.view(dtype).reshape(shape).copy()


def h2d(ptr, arr):
    arr = np.ascontiguousarray(arr)
    assert _cudart.cudaMemcpy(ctypes.c_void_p(ptr), arr.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(arr.nbytes), 1) == 0
    torch.cuda.synchronize()


def random_reservoirs(rng, P):
    r = np.zeros((P, 16), np.float32)
    r[:, 0:3] = rng.normal(size=(P, 3))
    r[:, 4:7] = rng.normal(size=(P, 3))
    r[:, 8:11] = np.abs(rng.normal(size=(P, 3)))
    r[:, 12] = rng.random(P) * 0.2
    r[:, 13] = np.abs(rng.normal(size=P))
    r[:, 15] = np.abs(rng.normal(size=P))
    u = r.view(np.uint32)
    n = rng.normal(size=(P, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    # a few distinct normals so the similarity tests pass for some neighbours
    n = np.round(n * 1.2) / 1.2
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-6)
    L = O.lib()
    enc = np.array([L.oracle_normalised_to_u32((ctypes.c_float * 3)(*v)) for v in n], np.uint32)
    u[:, 3] = enc[rng.permutation(P)]
    u[:, 7] = enc
    u[:, 11] = np.where(rng.random(P) < 0.1, 0xFF, rng.integers(0, 3, P))
    u[:, 14] = rng.integers(1, 200, P).astype(np.uint32) | (1 << 31)
    return r


def test_temporal_spatial_match_oracle(cuda):
    W, H = 96, 64
    P = W * H
    rng = np.random.default_rng(3)
    bufs = lb.DataBuffers(W, H, 64, _abi.BUFFER_ALL)
    cur = random_reservoirs(rng, P)
    old = random_reservoirs(rng, P)
    info = rng.random((P, 9)).astype(np.float32)
    h2d(bufs.device_buffer(lb.DataBuffers.RESERVOIRS)[0], cur)
    h2d(bufs.device_buffer(lb.DataBuffers.OLD_RESERVOIRS)[0], old)
    h2d(bufs.device_buffer(lb.DataBuffers.INFO)[0], info)
    bufs.temporal_resampling(seed_offset=7)
    got = d2h(*bufs.device_buffer(lb.DataBuffers.RESERVOIRS), np.float32, (P, 16))
    ref = cur.copy()
    O.temporal(ref, old, W, H, 7)
    np.testing.assert_array_equal(got.view(np.uint32)[:, [3, 7, 11, 14]], ref.view(np.uint32)[:, [3, 7, 11, 14]])
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)
    col = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    bufs.spatial_resampling(lb.targets_from(col), is_samples=5, is_space=61, seed_offset=9)
    torch.cuda.synchronize()
    out = O.spatial(ref, info, W, H, 5, 61, 9)
    sky = ref.view(np.uint32)[:, 11].reshape(H, W) == 0xFF
    g = col.cpu().numpy()
    np.testing.assert_allclose(g[~sky], out[~sky], rtol=1e-4, atol=1e-5)


def test_end_of_frame_matches_oracle(cuda):
    W, H, WS = 64, 32, 4096
    P = W * H
    rng = np.random.default_rng(4)
    bufs = lb.DataBuffers(W, H, WS, _abi.BUFFER_ALL)
    res = random_reservoirs(rng, P)
    world = np.zeros((WS, 14), np.uint32)
    world[:, 0] = rng.integers(0, 2 ** 32, WS, dtype=np.uint64).astype(np.uint32)
    world[:, 1] = rng.integers(0, 1000, WS)
    world[:, 2:5] = np.abs(rng.normal(size=(WS, 3))).astype(np.float32).view(np.uint32)
    world[:, 13] = rng.integers(0, 31, WS)
    chains = rng.random((P, 8)).astype(np.float32)
    h2d(bufs.device_buffer(lb.DataBuffers.RESERVOIRS)[0], res)
    h2d(bufs.device_buffer(lb.DataBuffers.WORLD)[0], world)
    h2d(bufs.device_buffer(lb.DataBuffers.CHAINS)[0], chains)
    bufs.advance_frame(_abi.BUFFER_ALL, lb.AdvanceOptions(20))
    torch.cuda.synchronize()
    ref_res = res.copy()
    O.process_gi(ref_res, 20)
    ref_world = world.copy().reshape(-1)
    O.process_world(ref_world)
    old_res = d2h(*bufs.device_buffer(lb.DataBuffers.OLD_RESERVOIRS), np.float32, (P, 16))
    np.testing.assert_array_equal(old_res.view(np.uint32), ref_res.view(np.uint32))
    cur_res = d2h(*bufs.device_buffer(lb.DataBuffers.RESERVOIRS), np.float32, (P, 16))
    assert (cur_res == 0).all()
    old_world = d2h(*bufs.device_buffer(lb.DataBuffers.OLD_WORLD), np.uint32, (WS * 14,))
    cur_world = d2h(*bufs.device_buffer(lb.DataBuffers.WORLD), np.uint32, (WS * 14,))
    np.testing.assert_array_equal(old_world, ref_world)
    np.testing.assert_array_equal(cur_world, ref_world)  # the world grid is copied, not cleared
    old_chains = d2h(*bufs.device_buffer(lb.DataBuffers.OLD_CHAINS), np.float32, (P, 8))
    np.testing.assert_array_equal(old_chains, chains)
    # non-temporal advance clears both
    bufs.advance_frame(0, lb.AdvanceOptions(20))
    torch.cuda.synchronize()
    assert (d2h(*bufs.device_buffer(lb.DataBuffers.OLD_CHAINS), np.float32, (P, 8)) == 0).all()


def test_average_frames_matches_oracle(cuda):
    rng = np.random.default_rng(5)
    frames = [rng.random((24, 40, 4)).astype(np.float32) * 10 for _ in range(70)]
    dev = [torch.from_numpy(f).cuda() for f in frames]
    out = torch.zeros(24 * 40 * 3, dtype=torch.float32, device="cuda")
    lb.average_frames(dev, out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), O.average(frames))


def test_restir_frame_sequence(cuda):
    """Render -> temporal -> spatial -> advance over a few frames, as the reference example does."""
    s = scenes.cornell_box(64, 64)
    tracer = lb.RayTracer(lb.path_tracing.Medium)
    pipe = tracer.create_pipeline(*s.layout_counts(), lb.PathTracerOpts(samples=1, guide_mode=lb.GuideMode.MARKOV))
    g = lb.GpuScene(s)
    bufs = lb.DataBuffers(64, 64, 1 << 14, _abi.BUFFER_ALL)
    col = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
    tg = lb.targets_from(col)
    for f in range(6):
        pipe.render(g, bufs, s.camera, tg, f)
        bufs.temporal_resampling(f)
        bufs.spatial_resampling(tg, 5, 61, f)
        bufs.advance_frame(_abi.BUFFER_ALL, lb.AdvanceOptions.SEMI_INTERACTIVE)
    torch.cuda.synchronize()
    c = col.cpu().numpy()
    assert np.isfinite(c).all() and c[..., :3].mean() > 0.0
    st = pipe.stats()
    assert st.error_flags == 0
