"""Ray-query parity: lam_trace_rays (BVH8 traversal on the B200) against the CPU oracle.

Closest-hit primitive / instance indices must match bit for bit; t and barycentrics are the FP64
re-evaluation rounded to f32 on both sides and must agree within 2 ulp (they are computed with the
same never-contracted operation order, so in practice they are identical)."""
import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, scenes
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def gpu_trace(gscene, rays, mode=_abi.TRACE_CLOSEST):
    import torch
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    h = torch.zeros((rays.shape[0], 6), dtype=torch.int32, device="cuda")
    gscene.trace(r, h, mode)
    torch.cuda.synchronize()
    return h.cpu().numpy().view(O.HIT_DTYPE).reshape(-1)


def compare(g, o):
    assert (g["kind"] != 0).sum() == (o["kind"] != 0).sum()
    np.testing.assert_array_equal(g["prim"], o["prim"])
    np.testing.assert_array_equal(g["inst"], o["inst"])
    np.testing.assert_array_equal(g["kind"], o["kind"])
    hit = o["kind"] != 0
    for f in ("t", "u", "v"):
        assert ulp_diff(g[f][hit], o[f][hit]).max() <= 2, f


def rays_in_box(n, rng, lo, hi, tmin=1e-4, tmax=1000.0):
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    r[:, 4:7] = rng.normal(size=(n, 3))
    r[:, 3], r[:, 7] = tmin, tmax
    return r


def test_cornell_closest_hit_matches_bruteforce(cuda):
    s = scenes.cornell_box(16, 16)
    g = lb.GpuScene(s)
    rng = np.random.default_rng(11)
    rays = rays_in_box(1 << 20, rng, -0.99, 1.99)
    compare(gpu_trace(g, rays), O.OracleScene(s).trace(rays, bruteforce=True))


def test_edge_cases(cuda):
    s = scenes.cornell_box(16, 16)
    g = lb.GpuScene(s)
    osc = O.OracleScene(s)
    rng = np.random.default_rng(12)
    verts = s.blas[0]["vertices"]
    n = 200000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.5, 0.5, (n, 3)) + np.array([0, 1, 0])
    # aim exactly at vertices and edge midpoints, axis-aligned directions, tiny/huge tmax
    tgt = verts[rng.integers(0, verts.shape[0], n)]
    mid = 0.5 * (verts[rng.integers(0, verts.shape[0], n)] + verts[rng.integers(0, verts.shape[0], n)])
    rays[:, 4:7] = np.where(rng.random((n, 1)) < 0.5, tgt, mid) - rays[:, 0:3]
    k = rng.integers(0, 3, n // 4)
    axis = np.zeros((n // 4, 3), np.float32)
    axis[np.arange(n // 4), k] = rng.choice([-1.0, 1.0], n // 4)
    rays[: n // 4, 4:7] = axis
    rays[:, 3] = rng.choice([0.0, 1e-4, 0.5], n)
    rays[:, 7] = rng.choice([1000.0, 1.0, 1e-3], n)
    rays[:10, 4:7] = 0.0  # zero direction: never hits
    compare(gpu_trace(g, rays), osc.trace(rays, bruteforce=True))


def test_any_hit_agrees_on_occupancy(cuda):
    s = scenes.icosphere_field(64, 64, instances=8, subdiv=3, tex_size=16, tex_layers=2, seed=9)
    g = lb.GpuScene(s)
    rng = np.random.default_rng(13)
    rays = rays_in_box(200000, rng, -12, 12)
    closest = gpu_trace(g, rays)
    anyh = gpu_trace(g, rays, _abi.TRACE_ANY)
    np.testing.assert_array_equal(closest["kind"] != 0, anyh["kind"] != 0)


def test_instance_mask_and_empty_scene(cuda):
    s = scenes.icosphere_field(64, 64, instances=4, subdiv=2, tex_size=16, tex_layers=2, seed=4)
    s.instances[1]["mask"] = 0
    g = lb.GpuScene(s)
    rng = np.random.default_rng(14)
    rays = rays_in_box(100000, rng, -12, 12)
    compare(gpu_trace(g, rays), O.OracleScene(s).trace(rays, bruteforce=True))
    empty = scenes.Scene()
    ge = lb.GpuScene(empty)
    h = gpu_trace(ge, rays[:1000])
    assert (h["kind"] == 0).all()


def test_alpha_tested_geometry(cuda):
    s = scenes.cornell_box(16, 16)
    s.blas[0]["flags"] = 0  # not opaque: candidates run the alpha test
    tex = np.full((64, 64, 4), 200, np.uint8)
    tex[:, :32, 3] = 0  # half of every diffuse texture transparent
    s.diffuse = [tex.copy() for _ in s.diffuse]
    g = lb.GpuScene(s)
    rng = np.random.default_rng(15)
    rays = rays_in_box(300000, rng, -0.99, 1.99)
    compare(gpu_trace(g, rays), O.OracleScene(s).trace(rays, bruteforce=True))


def test_icosphere_field_10m_rays(cuda):
    """The at-scale scene: 64 instances x 20,480 triangles, 10M seeded rays vs the oracle BVH."""
    s = scenes.icosphere_field(64, 64, tex_size=16, tex_layers=2)
    g = lb.GpuScene(s)
    st = g.stats()
    assert st.triangle_count == 64 * 20480
    rng = np.random.default_rng(2025)
    n = 10_000_000
    rays = rays_in_box(n, rng, -12.0, 12.0)
    # a third of the rays start at the camera and point into the field (coherent primary-like rays)
    rays[: n // 3, 0:3] = (0.0, 2.0, 16.0)
    rays[: n // 3, 4:7] = rng.uniform(-8, 8, (n // 3, 3)) - np.array([0.0, 2.0, 16.0])
    gh = gpu_trace(g, rays)
    oh = O.OracleScene(s).trace(rays)
    compare(gh, oh)
    assert (oh["kind"] != 0).mean() > 0.3
