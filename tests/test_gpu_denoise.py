"""The denoiser hand-off (OidnState::denoise, examples/cornell_box/src/main.rs:797-963): the averaged
frame and the first-hit normal / albedo AOVs reach a host filter, and the filtered frame returns to the
device buffer in place."""
import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes

pytestmark = pytest.mark.gpu


def _frames(W, H, n=3):
    import torch
    s = scenes.cornell_box(W, H)
    g = lb.GpuScene(s)
    pipe = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
        samples=2, restir_temporal=_abi.RESTIR_DISABLED, max_depth=5))
    bufs = lb.DataBuffers(W, H, 1, 0)
    frames = []
    nrm, alb = (torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(2))
    for k in range(n):
        col = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        pipe.render(g, bufs, s.camera, lb.targets_from(col, nrm, alb), 17 * k)
        frames.append(col)
    rgb = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    lb.average_frames(frames, rgb)
    torch.cuda.synchronize()
    return frames, rgb, nrm, alb


def _box3(img):
    """3 x 3 box filter with edge replication: the stand-in for OIDN's RayTracing filter."""
    p = np.pad(img, ((1, 1), (1, 1), (0, 0)), mode="edge")
    return sum(p[dy:dy + img.shape[0], dx:dx + img.shape[1]] for dy in range(3) for dx in range(3)) / 9.0


def test_handoff_filters_the_averaged_frame_in_place(cuda):
    W, H = 96, 64
    frames, rgb, nrm, alb = _frames(W, H)
    before = rgb.cpu().numpy().reshape(H, W, 3).copy()
    # the averaged frame is the mean of the three renders (average_to_buf.wgsl)
    mean = np.mean([f.cpu().numpy()[..., :3] for f in frames], axis=0)
    np.testing.assert_allclose(before, mean, rtol=1e-6, atol=1e-7)
    seen = {}

    def filt(c, n, a):
        seen["rgb"], seen["normal"], seen["albedo"] = c.copy(), n.copy(), a.copy()
        c[...] = _box3(c.astype(np.float64)).astype(np.float32)

    d = lb.Denoiser(W, H)
    d.run(rgb, filt, normal=nrm, albedo=alb)
    np.testing.assert_array_equal(seen["rgb"], before)
    np.testing.assert_array_equal(seen["normal"], nrm.cpu().numpy()[..., :3])
    np.testing.assert_array_equal(seen["albedo"], alb.cpu().numpy()[..., :3])
    after = rgb.cpu().numpy().reshape(H, W, 3)
    np.testing.assert_array_equal(after, _box3(before.astype(np.float64)).astype(np.float32))
    # a second run on the same staging, colour only
    d.run(rgb, lambda c, n, a: c.__imul__(0.5) if n is None and a is None else None)
    np.testing.assert_array_equal(rgb.cpu().numpy().reshape(H, W, 3), after * np.float32(0.5))


def test_handoff_reports_a_failing_filter_and_keeps_the_frame(cuda):
    W, H = 32, 32
    _, rgb, _, _ = _frames(W, H, n=1)
    before = rgb.cpu().numpy().copy()

    def bad(c, n, a):
        c[...] = 0.0
        raise RuntimeError("filter failed")

    d = lb.Denoiser(W, H)
    with pytest.raises(lb.LambentError) as e:
        d.run(rgb, bad)
    assert e.value.code == _abi.ERR_CALLBACK
    np.testing.assert_array_equal(rgb.cpu().numpy(), before)
    with pytest.raises(ValueError):
        d.run(rgb[:-3], lambda c, n, a: None)
