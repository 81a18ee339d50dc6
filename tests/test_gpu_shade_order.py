"""Material-ordered shading (lam_pipeline_set_shade_order): sorting a bounce's hits by shading class
(sky, diffuse, metallic, transparent) changes which lanes share a warp, not what a path computes."""
import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu

QUEUE, MATERIAL = _abi.SHADE_ORDER_QUEUE, _abi.SHADE_ORDER_MATERIAL


def render(s, samples, order, quality=_abi.QUALITY_MEDIUM, restir=_abi.RESTIR_PER_PIXEL, depth=8,
           guide=_abi.GUIDE_NONE, seed=0, wave_paths=0, world=1 << 16):
    import torch
    tracer = lb.RayTracer(lb.api._Quality(quality, "q"))
    opts = lb.PathTracerOpts(samples=samples, restir_temporal=restir, max_depth=depth, guide_mode=guide)
    pipe = tracer.create_pipeline(*s.layout_counts(), opts)
    pipe.set_wave_paths(wave_paths)
    pipe.set_shade_order(order)
    g = lb.GpuScene(s)
    W, H = s.width, s.height
    bufs = lb.DataBuffers(W, H, world, _abi.BUFFER_ALL)
    col, nrm, alb = (torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(3))
    pipe.render(g, bufs, s.camera, lb.targets_from(col, nrm, alb), seed)
    torch.cuda.synchronize()
    return {"color": col.cpu().numpy(), "normal": nrm.cpu().numpy(), "albedo": alb.cpu().numpy(),
            "stats": pipe.stats()}


@pytest.mark.parametrize("quality", [_abi.QUALITY_LOW, _abi.QUALITY_MEDIUM, _abi.QUALITY_HIGH])
def test_material_order_gives_the_same_image(cuda, quality):
    """Every shading class occurs (textured walls, an emitting wall, rough glass with an IOR range,
    metal, sky through the open front); each path draws from its own seed chain, so the outputs and
    the traced segments are bit-identical in either order."""
    s = scenes.textured_cornell(96, 64)
    a = render(s, 8, QUEUE, quality)
    b = render(s, 8, MATERIAL, quality)
    c = render(s, 8, _abi.SHADE_ORDER_AUTO, quality)
    for k in ("color", "normal", "albedo"):
        np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(a[k], c[k])
    assert a["stats"].ray_segments == b["stats"].ray_segments == c["stats"].ray_segments


def test_material_order_across_waves_on_the_instanced_field(cuda):
    """The instanced, textured field in waves of 3 + 3 + 2 samples per pixel: the order buffers are
    rebuilt at every depth of every wave."""
    s = scenes.icosphere_field(96, 64, instances=8, subdiv=3, tex_size=16, tex_layers=2, seed=9)
    a = render(s, 8, QUEUE, depth=12, restir=_abi.RESTIR_DISABLED, wave_paths=96 * 64 * 3)
    b = render(s, 8, MATERIAL, depth=12, restir=_abi.RESTIR_DISABLED, wave_paths=96 * 64 * 3)
    for k in ("color", "normal", "albedo"):
        np.testing.assert_array_equal(a[k], b[k])
    assert a["stats"].ray_segments == b["stats"].ray_segments


def test_material_order_with_an_intersection_handler(cuda):
    """Procedural spheres through the run-time-linked extend kernel and the handler's normals: the
    sort classes procedural hits by their instance's material like triangle hits, and the image is
    the same either way."""
    import os
    import torch
    src = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "sphere_handler.cu")).read()
    s = scenes.with_spheres(scenes.cornell_box(64, 64), n=48, seed=3)
    g = lb.GpuScene(s)
    out = []
    for order in (QUEUE, MATERIAL):
        t = lb.RayTracer(lb.path_tracing.Medium)
        t.set_intersection_handler(src)
        pipe = t.create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
            samples=8, restir_temporal=_abi.RESTIR_DISABLED, max_depth=5))
        pipe.set_shade_order(order)
        col = torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda")
        pipe.render(g, lb.DataBuffers(s.width, s.height, 1, 0), s.camera, lb.targets_from(col), 7)
        torch.cuda.synchronize()
        assert pipe.stats().error_flags == 0
        out.append(col.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])


def test_material_order_matches_oracle(cuda):
    """The sorted render against the oracle, with the same-seed bound of the queue-ordered test."""
    s = scenes.cornell_box(64, 64)
    g = render(s, 8, MATERIAL, depth=5)
    o = O.OracleScene(s).render(s.camera, 64, 64, samples=8, restir=_abi.RESTIR_PER_PIXEL)
    diff = np.abs(g["color"] - o["color"])[..., :3].max(-1)
    close = diff <= 1e-3 * np.maximum(1.0, np.abs(o["color"][..., :3]).max(-1))
    assert close.mean() > 0.97, close.mean()
    np.testing.assert_allclose(g["normal"], o["normal"], atol=1e-5)


def test_markov_guided_material_order_keeps_the_mean(cuda):
    """Under Markov guiding the world-grid updates land in another order, so sorted and unsorted
    renders differ sample by sample; their means over independent renders agree within 3 standard
    errors of the difference."""
    s = scenes.cornell_box(32, 32)
    n = 24

    def means(order, base):
        v = np.array([render(s, 64, order, restir=_abi.RESTIR_DISABLED, depth=5, guide=_abi.GUIDE_MARKOV,
                             seed=base + r)["color"][..., :3].mean() for r in range(n)])
        return v.mean(), v.std(ddof=1) / np.sqrt(n)

    qm, qs = means(QUEUE, 0)
    mm, ms = means(MATERIAL, 500)
    assert abs(qm - mm) < 3.0 * np.hypot(qs, ms), (qm, mm, qs, ms)


def test_unknown_shade_order_is_rejected(cuda):
    s = scenes.cornell_box(16, 16)
    pipe = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(samples=1))
    with pytest.raises(lb.LambentError):
        pipe.set_shade_order(7)
