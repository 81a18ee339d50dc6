"""Intersection handlers (RayTracer::set_intersection_handler, src/lib.rs:291-295): the handler's CUDA
source is compiled and linked into the procedural traversal kernels when a pipeline is created
(NVRTC + nvJitLink, no GPU needed); compile errors are reported with the compiler's log."""
import os

import pytest

import lambent_b200 as lb

HERE = os.path.dirname(os.path.abspath(__file__))


def _pipe(tracer):
    return tracer.create_pipeline(2, 1, 1, 1, lb.PathTracerOpts(samples=1))


def test_handler_compiles_and_links():
    t = lb.RayTracer(lb.path_tracing.Medium)
    t.set_intersection_handler(open(os.path.join(HERE, "data", "sphere_handler.cu")).read())
    assert _pipe(t) is not None


def test_handler_compile_error_is_reported():
    t = lb.RayTracer(lb.path_tracing.Medium)
    t.set_intersection_handler(
        "__device__ lam_aabb_intersection intersect(const lam_ray_intersection& i) { return no_such_name; }")
    with pytest.raises(lb.LambentError) as e:
        _pipe(t)
    assert e.value.code == lb._abi.ERR_COMPILE
    assert "no_such_name" in str(e.value)


def test_handler_without_intersect_fails_to_link():
    t = lb.RayTracer(lb.path_tracing.Medium)
    t.set_intersection_handler("__device__ int unrelated() { return 1; }")
    with pytest.raises(lb.LambentError):
        _pipe(t)


def test_null_restores_the_default_handler():
    t = lb.RayTracer(lb.path_tracing.Medium)
    t.set_intersection_handler("this is not CUDA")
    t.set_intersection_handler(None)
    assert _pipe(t) is not None
