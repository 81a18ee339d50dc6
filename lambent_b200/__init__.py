"""lambent_b200 - B200-native (sm_100a) drop-in for the Lambent path-tracing hot path.

The compute path is the C-ABI library liblambent_b200.so (include/lambent.h); this package is
its Python host mirror of the reference crate's API.
"""
from . import _abi
from .api import (AdvanceOptions, BufferType, Camera, DataBuffers, Denoiser, EmissionScale, GpuScene, Guide, GuideMode,
                  GuideOptions, LambentError,
                  Material, MaterialType, PathTracerOpts, Pipeline, RayTracer, RayTracingOptions, RestirTemporalMode,
                  TextureLoader, average_frames, check, debug, dispatch_size, lib, path_tracing, pipeline_layout,
                  refractive_indices, targets_from)

__all__ = [
    "AdvanceOptions", "BufferType", "Camera", "DataBuffers", "Denoiser", "EmissionScale", "GpuScene", "Guide", "GuideMode",
    "GuideOptions", "LambentError",
    "Material", "MaterialType", "PathTracerOpts", "Pipeline", "RayTracer", "RayTracingOptions", "RestirTemporalMode",
    "TextureLoader", "average_frames", "check", "debug", "dispatch_size", "lib", "path_tracing", "pipeline_layout",
    "refractive_indices", "targets_from",
]
