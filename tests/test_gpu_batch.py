"""Batched renders (lam_batch_render): every request of a batch renders exactly what lam_render
renders for it alone (same seeds, same arithmetic), with and without CUDA-graph replay."""
import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes

pytestmark = pytest.mark.gpu


def _pipe(s, samples=4, depth=6):
    opts = lb.PathTracerOpts(samples=samples, restir_temporal=_abi.RESTIR_DISABLED, max_depth=depth)
    return lb.RayTracer(lb.path_tracing.Medium).create_pipeline(8, 8, 8, 8, opts)


def _requests(torch):
    specs = [(scenes.cornell_box(64, 48), 5, 11), (scenes.box_field(3000, 96, 64, seed=1), 3, 22),
             (scenes.occluded_cornell(80, 80), 9, 33), (scenes.box_field(20000, 40, 120, seed=2), 1, 44),
             (scenes.cornell_box(128, 128), 16, 55), (scenes.box_field(3000, 32, 32, seed=1), 7, 66)]
    reqs = []
    for s, spp, seed in specs:
        g = lb.GpuScene(s)
        col, nrm, alb = (torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda") for _ in range(3))
        reqs.append({"scene": s, "gpu": g, "spp": spp, "seed": seed, "col": col, "nrm": nrm, "alb": alb,
                     "tg": lb.targets_from(col, nrm, alb)})
    return reqs


def _single(req, torch):
    s = req["scene"]
    p = _pipe(s, samples=req["spp"])
    col, nrm, alb = (torch.zeros_like(req["col"]) for _ in range(3))
    p.render(req["gpu"], lb.DataBuffers(s.width, s.height, 1, 0), s.camera, lb.targets_from(col, nrm, alb), req["seed"])
    torch.cuda.synchronize()
    return col.cpu().numpy(), nrm.cpu().numpy(), alb.cpu().numpy()


@pytest.mark.parametrize("graph", [0, 1])
def test_batch_matches_single_renders(cuda, graph):
    """Two calls on one pipeline, the first in material order (the default) and the second in
    queue order: a captured graph is rebuilt when the order changes, and either order renders
    each request exactly as lam_render does."""
    import torch
    reqs = _requests(torch)
    pipe = _pipe(reqs[0]["scene"])
    batch = [(r["gpu"], r["scene"].camera, r["tg"], r["spp"], r["seed"]) for r in reqs]
    # a small queue forces several waves and splits the largest request's samples across them
    tuning = _abi.BatchTuning(wave_paths=64 * 1024, use_graph=graph)
    refs = [_single(r, torch) for r in reqs]
    for call, order in enumerate((_abi.SHADE_ORDER_AUTO, _abi.SHADE_ORDER_QUEUE)):
        pipe.set_shade_order(order)
        for r in reqs:
            r["col"].zero_()
        pipe.batch_render(batch, tuning)
        torch.cuda.synchronize()
        st = pipe.stats()
        assert st.error_flags == 0
        assert st.samples == sum(r["scene"].width * r["scene"].height * r["spp"] for r in reqs)
        for r, (c, n, a) in zip(reqs, refs):
            np.testing.assert_array_equal(r["col"].cpu().numpy(), c)
            np.testing.assert_array_equal(r["nrm"].cpu().numpy(), n)
            np.testing.assert_array_equal(r["alb"].cpu().numpy(), a)
        lat = pipe.batch_latencies(len(reqs))
        assert all(0.0 < x < 60_000.0 for x in lat), lat


def test_batch_autotune_returns_a_working_tuning(cuda):
    import torch
    reqs = _requests(torch)[:4]
    pipe = _pipe(reqs[0]["scene"])
    batch = [(r["gpu"], r["scene"].camera, r["tg"], r["spp"], r["seed"]) for r in reqs]
    t = pipe.batch_autotune(batch, spp_divisor=2)
    assert t.wave_paths >= 1 << 20 and t.use_graph == 1
    refs = [_single(r, torch) for r in reqs]
    pipe.batch_render(batch, t)
    torch.cuda.synchronize()
    for r, (c, _, _) in zip(reqs, refs):
        np.testing.assert_array_equal(r["col"].cpu().numpy(), c)


def test_batch_rejects_unsupported_modes(cuda):
    import torch
    s = scenes.cornell_box(16, 16)
    g = lb.GpuScene(s)
    col = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda")
    opts = lb.PathTracerOpts(samples=1, restir_temporal=_abi.RESTIR_PER_PIXEL)
    p = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), opts)
    with pytest.raises(lb.LambentError):
        p.batch_render([(g, s.camera, lb.targets_from(col), 1, 0)])
