"""A scene given in the no-vertex-return format renders exactly as the same scene given directly."""
import copy

import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi, api, scenes

pytestmark = pytest.mark.gpu


def _render(s):
    import torch
    p = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
        samples=4, restir_temporal=_abi.RESTIR_DISABLED, max_depth=5))
    col = torch.zeros((s.height, s.width, 4), dtype=torch.float32, device="cuda")
    p.render(lb.GpuScene(s), lb.DataBuffers(s.width, s.height, 1, 0), s.camera, lb.targets_from(col), 3)
    torch.cuda.synchronize()
    return col.cpu().numpy()


def test_vertices_format_renders_identically(cuda):
    s = scenes.cornell_box(64, 64)
    v3 = s.blas[0]["vertices"]
    v4 = np.concatenate([v3, np.zeros((v3.shape[0], 1), np.float32)], axis=1)
    tris = v3.shape[0] // 3
    blob = api.Vertices(3 * tris, v4).append_bytes()
    s2 = copy.copy(s)
    s2.blas = [dict(api.blas_from_vertices(blob, np.zeros(1, np.uint32), [tris], flags=s.blas[0]["flags"]))]
    s2.instances = [dict(s.instances[0], material_indices=api.material_table_for_geometries(
        s.instances[0]["material_indices"], [tris]))]
    np.testing.assert_array_equal(_render(s), _render(s2))
