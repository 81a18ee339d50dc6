"""The no-vertex-return scene input (Vertices / Indices records, src/lib.rs:439-454, bindings.wesl:83-113)
through lam_blas_from_vertices: slot arithmetic geometry_stride * g + 3p + j, the length-1 "no
indices" rule, bounds errors, and the per-geometry material lookup."""
import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import api


def _verts(n, seed=0):
    rng = np.random.default_rng(seed)
    v = np.zeros((n, 4), np.float32)
    v[:, :3] = rng.uniform(-1, 1, (n, 3))
    return v


def test_indexed_geometries_flatten_in_order():
    v = _verts(12)
    stride = 9  # index slots per geometry
    idx = np.arange(2 * stride, dtype=np.uint32)[::-1] % 12  # any in-range indices
    blas = api.blas_from_vertices(api.Vertices(stride, v).append_bytes(), idx, [2, 3])
    want = [idx[stride * g + 3 * p + j] for g, n in enumerate([2, 3]) for p in range(n) for j in range(3)]
    assert blas["indices"].tolist() == [int(x) for x in want]
    np.testing.assert_array_equal(blas["vertices"], v)


def test_length_one_indices_means_direct_vertex_indices():
    v = _verts(18)
    blas = api.blas_from_vertices(api.Vertices(9, v).append_bytes(), np.zeros(1, np.uint32), [2, 3])
    want = [9 * g + 3 * p + j for g, n in enumerate([2, 3]) for p in range(n) for j in range(3)]
    assert blas["indices"].tolist() == want


def test_out_of_range_is_rejected():
    v = _verts(6)
    with pytest.raises(lb.LambentError):
        api.blas_from_vertices(api.Vertices(3, v).append_bytes(), np.zeros(4, np.uint32), [2])  # slot 5 >= 4
    with pytest.raises(lb.LambentError):
        api.blas_from_vertices(api.Vertices(3, v).append_bytes(), np.full(6, 7, np.uint32), [2])  # vertex 7 >= 6
    with pytest.raises(lb.LambentError):
        api.blas_from_vertices(api.Vertices(3, v).append_bytes()[:-4], np.zeros(1, np.uint32), [1])  # ragged blob


def test_material_table_follows_the_per_geometry_primitive_index():
    table = [7, 8, 9]
    got = api.material_table_for_geometries(table, [2, 4])
    # geometry 0: primitives 0, 1; geometry 1: primitives 0..3 (3 clamps to the last entry)
    assert got.tolist() == [7, 8, 7, 8, 9, 9]
