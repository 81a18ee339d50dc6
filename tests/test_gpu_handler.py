"""Procedural geometry with an intersection handler on the B200: lam_pipeline_trace_rays runs the
handler (tests/data/sphere_handler.cu: the sphere inscribed in each AABB) inside the BVH8 traversal.
Expected hits combine the oracle's triangles with a float64 sphere intersection; without a handler
the procedural instance is invisible (the reference's default handler misses)."""
import os

import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes
from oracle import oracle_py as O

from test_gpu_trace import compare, gpu_trace, ulp_diff

pytestmark = pytest.mark.gpu
SRC = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "sphere_handler.cu")).read()


def _scene(w=64, h=64):
    return scenes.with_spheres(scenes.cornell_box(w, h), n=48, seed=3)


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(-0.95, 1.95, (n, 3))
    r[:, 4:7] = rng.normal(size=(n, 3))
    r[:, 3], r[:, 7] = 1e-4, 1000.0
    return r


def _pipeline(handler, s):
    t = lb.RayTracer(lb.path_tracing.Medium)
    if handler:
        t.set_intersection_handler(SRC)
    return t.create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
        samples=8, restir_temporal=_abi.RESTIR_DISABLED, max_depth=5))


def _spheres(s, rays):
    """Closest sphere hit per ray in float64: (t or inf, primitive)."""
    inst = s.instances[1]
    M = np.eye(4)
    M[:3, :] = np.asarray(inst["transform"], np.float64).reshape(3, 4)
    Mi = np.linalg.inv(M)
    o = rays[:, 0:3].astype(np.float64) @ Mi[:3, :3].T + Mi[:3, 3]
    d = rays[:, 4:7].astype(np.float64) @ Mi[:3, :3].T
    box = s.blas[inst["blas"]]["aabbs"].astype(np.float64)
    c = 0.5 * (box[:, :3] + box[:, 3:])
    rad = 0.5 * (box[:, 3] - box[:, 0])
    oc = o[:, None, :] - c[None, :, :]
    a = np.sum(d * d, axis=1)[:, None]
    b = np.einsum("nk,nmk->nm", d, oc)
    cc = np.sum(oc * oc, axis=2) - rad[None, :] ** 2
    disc = b * b - a * cc
    sq = np.sqrt(np.maximum(disc, 0.0))
    t0 = (-b - sq) / a
    t1 = (-b + sq) / a
    t = np.where(t0 > 1e-4, t0, t1)
    t = np.where((disc >= 0) & (t > 1e-4) & (t < 1000.0), t, np.inf)
    k = np.argmin(t, axis=1)
    return t[np.arange(len(k)), k], k


def test_handler_trace_matches_triangles_and_spheres(cuda):
    import torch
    s = _scene()
    g = lb.GpuScene(s)
    p = _pipeline(True, s)
    rays = _rays(50_000, 5)
    h = torch.zeros((rays.shape[0], 6), dtype=torch.int32, device="cuda")
    p.trace_rays(g, torch.from_numpy(rays).cuda(), h)
    torch.cuda.synchronize()
    got = h.cpu().numpy().view(O.HIT_DTYPE).reshape(-1)
    tri = O.OracleScene(s).trace(rays)
    ts, ks = _spheres(s, rays)
    t_tri = np.where(tri["kind"] != 0, tri["t"].astype(np.float64), np.inf)
    want_sphere = ts < t_tri
    got_sphere = (got["kind"] != 0) & (got["inst"] == 1)
    agree = want_sphere == got_sphere
    assert agree.mean() > 0.998, agree.mean()
    both = want_sphere & got_sphere
    assert both.sum() > 1000
    assert (got["prim"][both] == ks[both]).mean() > 0.998
    rel = np.abs(got["t"][both] - ts[both]) / ts[both]
    assert np.median(rel) < 1e-5 and rel.max() < 1e-3
    tri_both = ~want_sphere & ~got_sphere
    np.testing.assert_array_equal(got["prim"][tri_both], tri["prim"][tri_both])
    np.testing.assert_array_equal(got["inst"][tri_both], tri["inst"][tri_both])
    hit = tri_both & (tri["kind"] != 0)
    assert ulp_diff(got["t"][hit], tri["t"][hit]).max() <= 2


def test_without_handler_procedural_geometry_misses(cuda):
    s = _scene()
    rays = _rays(50_000, 6)
    compare(gpu_trace(lb.GpuScene(s), rays), O.OracleScene(s).trace(rays))


def test_handler_render(cuda):
    import torch
    s = _scene()
    g = lb.GpuScene(s)

    def render(p):
        col = torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda")
        p.render(g, lb.DataBuffers(s.width, s.height, 1, 0), s.camera, lb.targets_from(col), 7)
        torch.cuda.synchronize()
        assert p.stats().error_flags == 0
        return col.cpu().numpy()

    with_h = render(_pipeline(True, s))
    without = render(_pipeline(False, s))
    plain = scenes.cornell_box(64, 64)
    gp = lb.GpuScene(plain)
    col = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
    _pipeline(False, s).render(gp, lb.DataBuffers(64, 64, 1, 0), plain.camera, lb.targets_from(col), 7)
    torch.cuda.synchronize()
    assert np.isfinite(with_h).all()
    np.testing.assert_array_equal(without, col.cpu().numpy())  # default handler: spheres invisible
    differs = np.abs(with_h[..., :3] - without[..., :3]).max(-1) > 1e-3
    assert differs.mean() > 0.05  # the spheres show up
