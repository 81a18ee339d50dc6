"""Python mirror of the reference crate's public API over the C-ABI library.

Names, argument meaning and error behaviour follow the Rust crate (Vecvec/Lambent):
  Material::new / EmissionScale / MaterialType / refractive_indices   src/lib.rs:30-205
  Camera::from_proj_view (README "Camera::new") / update / descriptor  src/camera.rs:6-70
  TextureLoader::{new, load, load_from_bytes, raw}                     src/textures.rs:12-91, README.md:29-45
  low_level::pipeline_layout / RayTracingOptions                       src/low_level.rs:77-343
  RayTracer::<S>::{new, set_intersection_handler, create_pipeline}     src/lib.rs:260-329
  path_tracing::{Low, Medium, High, PathTracerOpts, RestirTemporalMode} src/path_tracing/mod.rs:7-147
  DataBuffers / BufferType / AdvanceOptions                            src/data_buffer/mod.rs:18-472
  dispatch_size                                                        src/lib.rs:207-219
Errors the reference reports with Result become LambentError with the C status; the panics of the
reference (u16::MAX texture index, WESL link errors) become LambentError too.
"""
import ctypes as C
import os

from . import _abi
from ._abi import (BlasDesc, Camera as _CCamera, FrameTargets, Hit, InstanceDesc, Material as _CMaterial,
                   RawTextures, Ray, RenderStats, SceneDesc, SceneDescHolder, SceneStats, TracerOptions)

_LIB = None
_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liblambent_b200.so")


class LambentError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{_abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def _sig(lib, name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)


def lib():
    """Loads liblambent_b200.so (fails loudly when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: run __graft_entry__.build() (make -C lambent_b200/csrc)")
    L = C.CDLL(_LIB_PATH)
    i, u32, vp, f32p, u32p = C.c_int, C.c_uint32, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32)
    P = C.POINTER
    _sig(L, "lam_version", u32)
    _sig(L, "lam_last_error_message", C.c_char_p)
    _sig(L, "lam_dispatch_size", i, u32, u32, u32p)
    _sig(L, "lam_material_new", i, f32p, f32p, f32p, P(C.c_uint16), C.c_uint16, C.c_int32, C.c_int32, C.c_float,
         C.c_float, f32p, u32, P(_CMaterial))
    _sig(L, "lam_material_descriptor", i, P(_CMaterial), u32, u32, P(_abi.BufferDescriptor))
    _sig(L, "lam_refractive_index_between", i, f32p, f32p, f32p)
    _sig(L, "lam_camera_new", i, f32p, f32p, P(_CCamera))
    _sig(L, "lam_camera_from_proj_view", i, f32p, f32p, P(_CCamera))
    _sig(L, "lam_camera_update_from_proj_view", i, P(_CCamera), f32p, f32p)
    _sig(L, "lam_camera_descriptor", i, P(_CCamera), u32, P(_abi.BufferDescriptor))
    _sig(L, "lam_texture_loader_new", i, P(vp))
    _sig(L, "lam_texture_loader_load", i, vp, C.c_char_p, C.c_char_p, C.c_char_p)
    _sig(L, "lam_texture_loader_load_from_bytes", i, vp, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_char_p,
         C.c_size_t)
    _sig(L, "lam_texture_loader_load_rgba8", i, vp, u32, u32, vp, vp, vp)
    _sig(L, "lam_texture_loader_raw", i, vp, P(RawTextures))
    _sig(L, "lam_raw_textures_free", i, P(RawTextures))
    _sig(L, "lam_texture_loader_free", i, vp)
    _sig(L, "lam_pipeline_layout_create", i, u32, u32, u32, u32, P(vp))
    _sig(L, "lam_pipeline_layout_destroy", i, vp)
    _sig(L, "lam_tracer_create", i, u32, P(vp))
    _sig(L, "lam_tracer_set_intersection_handler", i, vp, C.c_char_p)
    _sig(L, "lam_tracer_destroy", i, vp)
    _sig(L, "lam_tracer_options_default", i, P(TracerOptions))
    _sig(L, "lam_tracer_create_pipeline", i, vp, vp, P(TracerOptions), P(vp))
    _sig(L, "lam_pipeline_destroy", i, vp)
    _sig(L, "lam_scene_create", i, P(SceneDesc), vp, P(vp))
    _sig(L, "lam_scene_update_materials", i, vp, P(_CMaterial), u32, vp)
    _sig(L, "lam_scene_stats_get", i, vp, P(SceneStats))
    _sig(L, "lam_scene_destroy", i, vp)
    _sig(L, "lam_trace_rays", i, vp, vp, u32, u32, vp, vp)
    _sig(L, "lam_data_buffers_new", i, u32, u32, u32, u32, P(vp))
    _sig(L, "lam_data_buffers_resize", i, vp, u32, u32)
    _sig(L, "lam_data_buffers_advance_frame", i, vp, u32, u32, vp)
    _sig(L, "lam_data_buffers_get", i, vp, u32, P(vp), P(C.c_size_t))
    _sig(L, "lam_data_buffers_destroy", i, vp)
    _sig(L, "lam_render", i, vp, vp, vp, P(_CCamera), P(FrameTargets), u32, vp)
    _sig(L, "lam_render_stats_get", i, vp, P(RenderStats))
    _sig(L, "lam_pipeline_set_profiling", i, vp, i)
    _sig(L, "lam_pipeline_set_wave_paths", i, vp, C.c_uint64)
    _sig(L, "lam_pipeline_set_shade_order", i, vp, C.c_uint32)
    _sig(L, "lam_render_profile_get", i, vp, P(_abi.StageTimes))
    _sig(L, "lam_render_profile_reset", i, vp)
    _sig(L, "lam_temporal_resampling", i, vp, u32, u32, u32, vp)
    _sig(L, "lam_spatial_resampling", i, vp, P(FrameTargets), u32, u32, u32, vp)
    _sig(L, "lam_average_frames", i, P(vp), u32, u32, u32, vp, vp)
    _sig(L, "lam_guide_options_default", i, P(_abi.GuideOptions))
    _sig(L, "lam_guide_create", i, P(_abi.GuideOptions), P(vp))
    _sig(L, "lam_guide_destroy", i, vp)
    _sig(L, "lam_guide_get_params", i, vp, f32p)
    _sig(L, "lam_guide_set_params", i, vp, f32p)
    _sig(L, "lam_guide_eval", i, vp, vp, u32, f32p, vp, vp)
    _sig(L, "lam_guide_loss_grad", i, vp, vp, u32, f32p, vp, vp, vp)
    _sig(L, "lam_guide_train", i, vp, vp, u32, u32, f32p, vp)
    _sig(L, "lam_guide_progress", i, vp, P(C.c_uint64), u32p)
    _sig(L, "lam_guide_set_wait_limit", i, vp, u32)
    _sig(L, "lam_denoiser_create", i, u32, u32, P(vp))
    _sig(L, "lam_denoiser_run", i, vp, vp, vp, vp, DenoiseFn, vp, vp)
    _sig(L, "lam_denoiser_destroy", i, vp)
    _sig(L, "lam_pipeline_set_guide", i, vp, vp)
    _sig(L, "lam_scene_bounds", i, vp, f32p)
    _sig(L, "lam_pipeline_trace_rays", i, vp, vp, vp, u32, u32, vp, vp)
    _sig(L, "lam_blas_from_vertices", i, vp, C.c_size_t, u32p, C.c_size_t, u32, u32p, u32, P(_abi.BlasDesc))
    _sig(L, "lam_blas_desc_free", i, P(_abi.BlasDesc))
    _sig(L, "lam_material_table_for_geometries", i, u32p, u32, u32, u32p, u32p)
    _sig(L, "lam_batch_render", i, vp, P(_abi.BatchRequest), u32, P(_abi.BatchTuning), vp)
    _sig(L, "lam_batch_latencies", i, vp, u32, P(C.c_double))
    _sig(L, "lam_batch_autotune", i, vp, P(_abi.BatchRequest), u32, u32, P(_abi.BatchTuning), vp)
    _LIB = L
    return L


def check(rc):
    if rc != 0:
        msg = lib().lam_last_error_message()
        raise LambentError(rc, msg.decode() if msg else "")
    return rc


def _f32(*vals):
    return (C.c_float * len(vals))(*vals)


# ---------------------------------------------------------------- materials (src/lib.rs)
class MaterialType:
    Diffuse = _abi.DIFFUSE
    Metallic = _abi.METALLIC
    Transparent = _abi.TRANSPARENT


class refractive_indices:
    """Refractive index ranges (760 nm .. 340 nm), src/lib.rs:32-56."""
    VACUUM = (1.0, 1.0)
    AIR = (1.00027531, 1.000287)
    ICE = (1.3057, 1.3267)
    WATER = (1.33, 1.3442)
    GLASS = (1.4540, 1.4787)
    DIAMOND = (2.4063, 2.4922)

    @staticmethod
    def refractive_index_between(in_front, behind):
        out = _f32(0.0, 0.0)
        check(lib().lam_refractive_index_between(_f32(*in_front), _f32(*behind), out))
        return (out[0], out[1])


class EmissionScale:
    def __init__(self, emissive_texture_scale=0.0, diffuse_texture_scale=0.0):
        self.emissive_texture_scale = float(emissive_texture_scale)
        self.diffuse_texture_scale = float(diffuse_texture_scale)

    @classmethod
    def from_emission_scale(cls, scale):
        return cls(scale, 0.0)

    @classmethod
    def from_f32(cls, emissive, diffuse):
        return cls(emissive, diffuse)


class Material:
    @staticmethod
    def new(tex_pos_1, tex_pos_2, tex_pos_3, tex_pos_recolour, tex_idx_diffuse, tex_idx_emission,
            tex_idx_attributes, emission_scale, refractive_index, ty):
        """Material::new (src/lib.rs:132-163); None for the optional indices / refractive range."""
        m = _CMaterial()
        rec = (C.c_uint16 * 2)(*tex_pos_recolour)
        ior = _f32(*refractive_index) if refractive_index is not None else None
        check(lib().lam_material_new(_f32(*tex_pos_1), _f32(*tex_pos_2), _f32(*tex_pos_3), rec, tex_idx_diffuse,
                                     -1 if tex_idx_emission is None else tex_idx_emission,
                                     -1 if tex_idx_attributes is None else tex_idx_attributes,
                                     emission_scale.emissive_texture_scale, emission_scale.diffuse_texture_scale,
                                     ior, ty, C.byref(m)))
        return m

    @staticmethod
    def descriptor(materials, further_usages=0):
        """<[Material] as Descriptor>::buffer_descriptor: (bytes, usage)."""
        arr = (_CMaterial * len(materials))(*materials)
        d = _abi.BufferDescriptor()
        check(lib().lam_material_descriptor(arr, len(materials), further_usages, C.byref(d)))
        return bytes(C.string_at(d.contents, d.size)), d.usage


# ---------------------------------------------------------------- camera (src/camera.rs)
class Camera:
    def __init__(self, c):
        self.c = c

    @classmethod
    def new(cls, proj, view):
        """Camera::new / from_proj_view: proj and view as 4x4 column-major (16 floats or [[col]]*4)."""
        return cls.from_proj_view(proj, view)

    @classmethod
    def from_proj_view(cls, proj, view):
        c = _CCamera()
        check(lib().lam_camera_from_proj_view(_f32(*_flat16(proj)), _f32(*_flat16(view)), C.byref(c)))
        return cls(c)

    def update_from_proj_view(self, proj=None, view=None):
        check(lib().lam_camera_update_from_proj_view(C.byref(self.c), None if proj is None else _f32(*_flat16(proj)),
                                                      None if view is None else _f32(*_flat16(view))))

    def descriptor(self, further_usages=0):
        d = _abi.BufferDescriptor()
        check(lib().lam_camera_descriptor(C.byref(self.c), further_usages, C.byref(d)))
        return bytes(C.string_at(d.contents, d.size)), d.usage

    @property
    def position(self):
        return tuple(self.c.view_inverse[12:15])


def _flat16(m):
    import numpy as np
    a = np.asarray(m, dtype=np.float32).reshape(-1)
    if a.size != 16:
        raise ValueError("a 4x4 matrix is required")
    return [float(x) for x in a]


# ---------------------------------------------------------------- textures (src/textures.rs, README raw)
class TextureLoader:
    def __init__(self):
        h = C.c_void_p()
        check(lib().lam_texture_loader_new(C.byref(h)))
        self._h = h

    @classmethod
    def default(cls):
        return cls()

    def load(self, diffuse, lit=None, attributes=None):
        enc = lambda p: None if p is None else os.fsencode(p)
        check(lib().lam_texture_loader_load(self._h, enc(diffuse), enc(lit), enc(attributes)))

    def load_from_bytes(self, diffuse, lit=None, attributes=None):
        ln = lambda b: 0 if b is None else len(b)
        check(lib().lam_texture_loader_load_from_bytes(self._h, diffuse, len(diffuse), lit, ln(lit), attributes,
                                                        ln(attributes)))

    def load_rgba8(self, diffuse, lit=None, attributes=None):
        import numpy as np
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.uint8) for a in (diffuse, lit, attributes)]
        h, w = arrs[0].shape[:2]
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        check(lib().lam_texture_loader_load_rgba8(self._h, w, h, ptr(arrs[0]), ptr(arrs[1]), ptr(arrs[2])))

    def raw(self):
        """Consumes the loader: {'diffuse'|'lit'|'attributes': (layers, H, W, 4) uint8, 'layer_of_entry': ...}."""
        import numpy as np
        if self._h is None:
            raise LambentError(_abi.ERR_INVALID_ARGUMENT, "texture loader already consumed")
        raw = RawTextures()
        h, self._h = self._h, None
        check(lib().lam_texture_loader_raw(h, C.byref(raw)))
        try:
            out = {"entry_count": raw.entry_count, "layer_of_entry": {}}
            for k, name in enumerate(("diffuse", "lit", "attributes")):
                L, H, W = raw.layers[k], raw.height[k], raw.width[k]
                n = L * H * W * 4
                buf = np.ctypeslib.as_array(raw.cuboid[k], shape=(max(n, 1),))[:n].copy()
                out[name] = buf.reshape(L, H, W, 4) if n else np.zeros((0, H, W, 4), np.uint8)
                out["layer_of_entry"][name] = [raw.layer_of_entry[k][i] for i in range(raw.entry_count)]
            return out
        finally:
            lib().lam_raw_textures_free(C.byref(raw))

    def __del__(self):
        if getattr(self, "_h", None) is not None and _LIB is not None:
            _LIB.lam_texture_loader_free(self._h)
            self._h = None


# ---------------------------------------------------------------- options / layout / tracer
class RestirTemporalMode:
    Disabled = _abi.RESTIR_DISABLED
    PerSample = _abi.RESTIR_PER_SAMPLE
    PerPixel = _abi.RESTIR_PER_PIXEL


class GuideMode:
    NONE = _abi.GUIDE_NONE
    MARKOV = _abi.GUIDE_MARKOV
    LEARNED = _abi.GUIDE_LEARNED
    # the Markov-chain mixture weighted by the density its direction was drawn from (unbiased); MARKOV
    # alone keeps the reference's weighting, whose cosine term is evaluated at the cosine branch's draw
    MARKOV_UNBIASED = _abi.GUIDE_MARKOV | _abi.GUIDE_PDF_AT_SAMPLE
    # cosine + Markov vMF lobes + the network in one one-sample-MIS mixture
    LEARNED_MARKOV = _abi.GUIDE_LEARNED | _abi.GUIDE_MARKOV
    # modifier of the learned modes: the learned lobes are mixed in at rough metallic vertices too
    METAL = _abi.GUIDE_METAL


DEFAULT_NUM_SAMPLES = 4
DEFAULT_T_MIN = 0.0001
DEFAULT_T_MAX = 1000.0


class RayTracingOptions:
    def __init__(self, samples=DEFAULT_NUM_SAMPLES, tmin=DEFAULT_T_MIN, tmax=DEFAULT_T_MAX):
        self.samples, self.tmin, self.tmax = samples, tmin, tmax
        self.restir_temporal = RestirTemporalMode.PerPixel  # get_non_sample returns () -> default
        self.max_depth = 5
        self.guide_mode = GuideMode.NONE

    def to_c(self):
        return TracerOptions(self.samples, self.tmin, self.tmax, self.restir_temporal, self.max_depth, self.guide_mode)


class PathTracerOpts(RayTracingOptions):
    def __init__(self, samples=DEFAULT_NUM_SAMPLES, tmin=DEFAULT_T_MIN, tmax=DEFAULT_T_MAX,
                 restir_temporal=RestirTemporalMode.PerPixel, max_depth=5, guide_mode=GuideMode.NONE):
        super().__init__(samples, tmin, tmax)
        self.restir_temporal = restir_temporal
        self.max_depth = max_depth
        self.guide_mode = guide_mode


class PipelineLayout:
    def __init__(self, blas_count, diffuse_count, emission_count, attribute_count):
        h = C.c_void_p()
        check(lib().lam_pipeline_layout_create(blas_count, diffuse_count, emission_count, attribute_count, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_pipeline_layout_destroy(self._h)
            self._h = None


def pipeline_layout(blas_count, diffuse_count, emission_count, attribute_count, extra_bgls=()):
    """low_level::pipeline_layout (src/low_level.rs:237-343).  extra_bgls are accepted and, as in the
    reference (low_level.rs:331-341), not part of the layout."""
    return PipelineLayout(blas_count, diffuse_count, emission_count, attribute_count)


class _Quality:
    def __init__(self, code, name):
        self.code, self.name = code, name

    def __repr__(self):
        return f"path_tracing.{self.name}"


class path_tracing:
    Low = _Quality(_abi.QUALITY_LOW, "Low")
    Medium = _Quality(_abi.QUALITY_MEDIUM, "Medium")
    High = _Quality(_abi.QUALITY_HIGH, "High")
    PathTracerOpts = PathTracerOpts
    RestirTemporalMode = RestirTemporalMode


class debug:
    FrontFace = _Quality(_abi.DEBUG_FRONT_FACE, "FrontFace")
    Reflectance = _Quality(_abi.DEBUG_REFLECTANCE, "Reflectance")
    Tangent = _Quality(_abi.DEBUG_TANGENT, "Tangent")


class RayTracer:
    """RayTracer::<S>::new(&device) with S = path_tracing.Low / Medium / High."""

    def __init__(self, shader=path_tracing.Medium):
        h = C.c_void_p()
        check(lib().lam_tracer_create(shader.code, C.byref(h)))
        self._h = h
        self.shader = shader

    def set_intersection_handler(self, cuda_source):
        check(lib().lam_tracer_set_intersection_handler(self._h, None if cuda_source is None else cuda_source.encode()))

    def create_pipeline(self, blas_count, diffuse_count, emission_count, attribute_count, options=None):
        layout = pipeline_layout(blas_count, diffuse_count, emission_count, attribute_count)
        opts = (options or RayTracingOptions()).to_c()
        h = C.c_void_p()
        check(lib().lam_tracer_create_pipeline(self._h, layout._h, C.byref(opts), C.byref(h)))
        return Pipeline(h, layout, opts)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_tracer_destroy(self._h)
            self._h = None


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def targets_from(color=None, normal=None, albedo=None, width=None, height=None):
    """FrameTargets from torch CUDA tensors of shape (H, W, 4) float32 (any may be None)."""
    ref = next(t for t in (color, normal, albedo) if t is not None)
    h, w = ref.shape[0], ref.shape[1]
    for t in (color, normal, albedo):
        if t is not None and (t.dtype.__str__() != "torch.float32" or not t.is_contiguous() or tuple(t.shape) != (h, w, 4)):
            raise ValueError("targets must be contiguous float32 (H, W, 4) tensors")
    p = lambda t: None if t is None else t.data_ptr()
    return FrameTargets(p(color), p(normal), p(albedo), width or w, height or h)


class Pipeline:
    def __init__(self, h, layout, opts):
        self._h, self.layout, self.options = h, layout, opts

    def render(self, scene, buffers, camera, targets, seed_offset=0, stream=None):
        check(lib().lam_render(self._h, scene._h, buffers._h, C.byref(camera.c), C.byref(targets), seed_offset,
                               _stream_ptr(stream)))

    def stats(self):
        s = RenderStats()
        check(lib().lam_render_stats_get(self._h, C.byref(s)))
        return s

    def set_profiling(self, enabled=True):
        check(lib().lam_pipeline_set_profiling(self._h, 1 if enabled else 0))

    def set_wave_paths(self, max_paths=0):
        """Bounds the paths of one wave (device memory ~220 B per path); 0 restores the default."""
        check(lib().lam_pipeline_set_wave_paths(self._h, int(max_paths)))

    def set_shade_order(self, order=_abi.SHADE_ORDER_AUTO):
        """SHADE_ORDER_MATERIAL sorts each bounce's hits by class (sky, diffuse, metallic,
        transparent) before shading; SHADE_ORDER_QUEUE shades them in traversal order;
        SHADE_ORDER_AUTO (the default) sorts except under Markov guiding."""
        check(lib().lam_pipeline_set_shade_order(self._h, int(order)))

    def profile(self):
        t = _abi.StageTimes()
        check(lib().lam_render_profile_get(self._h, C.byref(t)))
        return t

    def profile_reset(self):
        check(lib().lam_render_profile_reset(self._h))

    def trace_rays(self, scene, rays, hits, mode=_abi.TRACE_CLOSEST, stream=None):
        """lam_pipeline_trace_rays: ray queries that run the pipeline's intersection handler.
        rays / hits as for GpuScene.trace."""
        n = _check_ray_tensors(scene, rays, hits)
        check(lib().lam_pipeline_trace_rays(self._h, scene._h, C.c_void_p(rays.data_ptr()), n, mode,
                                            C.c_void_p(hits.data_ptr()), _stream_ptr(stream)))

    def batch_render(self, requests, tuning=None, stream=None):
        """requests: list of (GpuScene, Camera, FrameTargets, samples, seed_offset).  Renders all of them as
        one wavefront (lam_batch_render); tuning: a _abi.BatchTuning or None for the defaults."""
        arr = self._batch_array(requests)
        check(lib().lam_batch_render(self._h, arr, len(requests), C.byref(tuning) if tuning is not None else None,
                                     _stream_ptr(stream)))

    def batch_latencies(self, n):
        out = (C.c_double * n)()
        check(lib().lam_batch_latencies(self._h, n, out))
        return list(out)

    def batch_autotune(self, requests, spp_divisor=4, stream=None):
        arr = self._batch_array(requests)
        t = _abi.BatchTuning()
        check(lib().lam_batch_autotune(self._h, arr, len(requests), spp_divisor, C.byref(t), _stream_ptr(stream)))
        return t

    def _batch_array(self, requests):
        arr = (_abi.BatchRequest * len(requests))()
        for k, (scene, camera, targets, samples, seed) in enumerate(requests):
            arr[k] = _abi.BatchRequest(scene._h.value, camera.c, targets, samples, seed)
        self._batch_keep = (arr, requests)
        return arr

    def set_guide(self, guide):
        """Attaches a learned Guide (used when the options' guide_mode is GuideMode.LEARNED)."""
        self._guide = guide
        check(lib().lam_pipeline_set_guide(self._h, guide._h if guide is not None else None))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_pipeline_destroy(self._h)
            self._h = None


def dispatch_size(width, height):
    out = (C.c_uint32 * 2)()
    check(lib().lam_dispatch_size(width, height, out))
    return (out[0], out[1])


# ---------------------------------------------------------------- scene (BLAS/TLAS + bindings)
class GpuScene:
    """A scene built on the device (BVH8 per BLAS, TLAS over instances, materials, textures)."""

    def __init__(self, scene, stream=None):
        self.holder = SceneDescHolder(scene)
        h = C.c_void_p()
        check(lib().lam_scene_create(self.holder.ptr(), _stream_ptr(stream), C.byref(h)))
        self._h = h
        self.holder = None
        import torch
        self.device = torch.device("cuda", torch.cuda.current_device())  # the scene lives on this device

    def stats(self):
        s = SceneStats()
        check(lib().lam_scene_stats_get(self._h, C.byref(s)))
        return s

    def bounds(self):
        """World-space bounds of the geometry: (lo xyz, hi xyz)."""
        b = (C.c_float * 6)()
        check(lib().lam_scene_bounds(self._h, b))
        return list(b)

    def update_materials(self, materials, stream=None):
        arr = (_CMaterial * len(materials))(*materials)
        check(lib().lam_scene_update_materials(self._h, arr, len(materials), _stream_ptr(stream)))

    def trace(self, rays, hits, mode=_abi.TRACE_CLOSEST, stream=None):
        """rays: contiguous CUDA tensor (n, 8) float32 on the scene's device (lam_ray records); hits:
        contiguous CUDA tensor of at least n rows of 6 four-byte elements (int32 / uint32 / float32
        storage of lam_hit records).  Anything else raises ValueError before the C-ABI is called."""
        n = _check_ray_tensors(self, rays, hits)
        check(lib().lam_trace_rays(self._h, C.c_void_p(rays.data_ptr()), n, mode, C.c_void_p(hits.data_ptr()),
                                   _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_scene_destroy(self._h)
            self._h = None


def _check_ray_tensors(scene, rays, hits):
    """Validates the ray / hit tensors of a ray query and returns the ray count: the kernels read
    32-byte rays and write 24-byte hits through raw device pointers, so a host tensor, a strided view,
    a wrong element size or a short hit tensor would make them access memory out of bounds."""
    import torch
    for name, t in (("rays", rays), ("hits", hits)):
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if t.device != scene.device:
            raise ValueError(f"{name} is on {t.device}, the scene on {scene.device}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
    if rays.dtype != torch.float32 or rays.dim() != 2 or rays.shape[1] != 8:
        raise ValueError("rays must be a float32 tensor of shape (n, 8)")
    if hits.dtype not in (torch.int32, torch.float32) and str(hits.dtype) != "torch.uint32":
        raise ValueError("hits must hold 4-byte elements (int32, uint32 or float32)")
    if hits.dim() != 2 or hits.shape[1] != 6:
        raise ValueError("hits must have shape (m, 6)")
    n = rays.shape[0]
    if hits.shape[0] < n:
        raise ValueError(f"hits holds {hits.shape[0]} rows, fewer than the {n} rays")
    if n > 0xFFFFFFFF:
        raise ValueError("too many rays for one query")
    return n


# ---------------------------------------------------------------- DataBuffers (src/data_buffer/mod.rs)
class BufferType:
    MARKOV_CHAIN_SCREEN_SPACE = _abi.BUFFER_MARKOV_CHAIN_SCREEN_SPACE
    SPATIAL_RESAMPLING = _abi.BUFFER_SPATIAL_RESAMPLING
    MARKOV_CHAIN_WORLD_SPACE = _abi.BUFFER_MARKOV_CHAIN_WORLD_SPACE

    @staticmethod
    def all():
        return _abi.BUFFER_ALL


class AdvanceOptions:
    def __init__(self, confidence_cap):
        self.confidence_cap = confidence_cap


AdvanceOptions.RESPONSIVE = AdvanceOptions(2)
AdvanceOptions.SEMI_INTERACTIVE = AdvanceOptions(30)
AdvanceOptions.SLOW = AdvanceOptions(100)


class DataBuffers:
    RESERVOIRS, OLD_RESERVOIRS, INFO, CHAINS, OLD_CHAINS, WORLD, OLD_WORLD, PIXEL_SEED = range(8)

    def __init__(self, width, height, world_space_buffer_size, buffers):
        h = C.c_void_p()
        check(lib().lam_data_buffers_new(width, height, world_space_buffer_size, buffers, C.byref(h)))
        self._h = h
        self.width, self.height = max(1, width), max(1, height)

    @classmethod
    def new(cls, width, height, world_space_buffer_size, buffers):
        return cls(width, height, world_space_buffer_size, buffers)

    def resize(self, width, height):
        check(lib().lam_data_buffers_resize(self._h, width, height))
        self.width, self.height = max(1, width), max(1, height)

    def advance_frame(self, buffers_to_temporally_advance, options, stream=None):
        check(lib().lam_data_buffers_advance_frame(self._h, buffers_to_temporally_advance, options.confidence_cap,
                                                   _stream_ptr(stream)))

    def device_buffer(self, which):
        p, n = C.c_void_p(), C.c_size_t()
        check(lib().lam_data_buffers_get(self._h, which, C.byref(p), C.byref(n)))
        return p.value, n.value

    def temporal_resampling(self, seed_offset=0, stream=None):
        check(lib().lam_temporal_resampling(self._h, self.width, self.height, seed_offset, _stream_ptr(stream)))

    def spatial_resampling(self, targets, is_samples=8, is_space=61, seed_offset=0, stream=None):
        check(lib().lam_spatial_resampling(self._h, C.byref(targets), is_samples, is_space, seed_offset,
                                           _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_data_buffers_destroy(self._h)
            self._h = None


def average_frames(frames, out_rgb, stream=None):
    """average (average_to_buf.wgsl): out_rgb (H*W*3 float32 CUDA tensor) = mean of rgba32f CUDA frames."""
    f0 = frames[0]
    h, w = f0.shape[0], f0.shape[1]
    ptrs = (C.c_void_p * len(frames))(*[f.data_ptr() for f in frames])
    check(lib().lam_average_frames(ptrs, len(frames), w, h, C.c_void_p(out_rgb.data_ptr()), _stream_ptr(stream)))


# ---------------------------------------------------------------- denoiser hand-off (examples/cornell_box/src/main.rs:797-963)
DenoiseFn = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                        C.c_uint32, C.c_uint32)


class Denoiser:
    """OidnState: pinned host staging of one frame size.  run() hands the averaged frame (and the
    first-hit normal / albedo AOVs) to a host filter and uploads the filtered frame in place."""

    def __init__(self, width, height):
        h = C.c_void_p()
        check(lib().lam_denoiser_create(width, height, C.byref(h)))
        self._h, self.width, self.height = h, width, height

    def run(self, rgb, filter, normal=None, albedo=None, stream=None):
        """rgb: CUDA float32 tensor of width * height * 3 elements (lam_average_frames' layout), filtered
        in place.  normal / albedo: CUDA float32 (H, W, 4) AOVs or None.  filter(rgb, normal, albedo)
        gets numpy views, (H, W, 3) each (None where not given), and writes the result into rgb; an
        exception in it becomes LambentError(LAM_ERR_CALLBACK)."""
        import numpy as np
        import torch
        W, H = self.width, self.height
        if not (isinstance(rgb, torch.Tensor) and rgb.is_cuda and rgb.is_contiguous() and rgb.dtype == torch.float32
                and rgb.numel() == W * H * 3):
            raise ValueError("rgb must be a contiguous CUDA float32 tensor of width * height * 3 elements")
        for name, t in (("normal", normal), ("albedo", albedo)):
            if t is not None and not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()
                                      and t.dtype == torch.float32 and tuple(t.shape) == (H, W, 4)):
                raise ValueError(f"{name} must be a contiguous CUDA float32 tensor of shape ({H}, {W}, 4)")

        def view(p):
            return None if not p else np.ctypeslib.as_array(p, shape=(H, W, 3))

        def call(user, c, n, a, w, h):
            try:
                filter(view(c), view(n), view(a))
                return 0
            except Exception:
                return 1

        cb = DenoiseFn(call)
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        check(lib().lam_denoiser_run(self._h, C.c_void_p(rgb.data_ptr()), ptr(normal), ptr(albedo), cb, None,
                                     _stream_ptr(stream)))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_denoiser_destroy(self._h)
            self._h = None


# ---------------------------------------------------------------- learned path guiding (no reference counterpart)
class GuideOptions:
    """Mirror of lam_guide_options (defaults from lam_guide_options_default)."""

    def __init__(self, **kw):
        o = _abi.GuideOptions()
        check(lib().lam_guide_options_default(C.byref(o)))
        for k, v in kw.items():
            if not hasattr(o, k):
                raise AttributeError(k)
            setattr(o, k, v)
        self.c = o


def _fbox(box):
    return (C.c_float * 6)(*[float(v) for v in box])


def _check_f32(t, name, shape, min_rows=0):
    """A contiguous CUDA float32 tensor of `shape` (None: any extent) with at least min_rows rows: the
    guide kernels read and write these through raw device pointers."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous() or t.dtype != torch.float32:
        raise ValueError(f"{name} must be a contiguous CUDA float32 tensor")
    if t.dim() != len(shape) or any(w is not None and d != w for d, w in zip(t.shape, shape)):
        raise ValueError(f"{name} must have shape {tuple('n' if w is None else w for w in shape)}")
    if t.shape[0] < min_rows:
        raise ValueError(f"{name} holds {t.shape[0]} rows, fewer than {min_rows}")


class Guide:
    """The learned guiding network: 4 x 64 x 64 parameters, tcgen05 evaluation and training."""

    def __init__(self, options=None):
        self.options = options or GuideOptions()
        h = C.c_void_p()
        check(lib().lam_guide_create(C.byref(self.options.c), C.byref(h)))
        self._h = h

    def params(self):
        out = (C.c_float * _abi.GUIDE_PARAMS)()
        check(lib().lam_guide_get_params(self._h, out))
        return list(out)

    def set_params(self, params):
        arr = (C.c_float * _abi.GUIDE_PARAMS)(*[float(v) for v in params])
        check(lib().lam_guide_set_params(self._h, arr))

    def eval(self, queries, box, out, stream=None):
        """queries: CUDA float32 (n, 9) = pos, normal, wo; out: CUDA float32 (n, 40) head outputs."""
        _check_f32(queries, "queries", (None, 9))
        _check_f32(out, "out", (None, _abi.GUIDE_OUTPUTS), min_rows=queries.shape[0])
        check(lib().lam_guide_eval(self._h, C.c_void_p(queries.data_ptr()), queries.shape[0], _fbox(box),
                                   C.c_void_p(out.data_ptr()), _stream_ptr(stream)))

    def loss_grad(self, records, box, grad, loss, stream=None):
        """records: CUDA float32 (n, 13); grad: CUDA float32 (16384,); loss: CUDA float32 (1,)."""
        _check_f32(records, "records", (None, 13))
        _check_f32(grad, "grad", (_abi.GUIDE_PARAMS,))
        _check_f32(loss, "loss", (1,))
        check(lib().lam_guide_loss_grad(self._h, C.c_void_p(records.data_ptr()), records.shape[0], _fbox(box),
                                        C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()),
                                        _stream_ptr(stream)))

    def train(self, records, steps, box, stream=None):
        _check_f32(records, "records", (None, 13))
        check(lib().lam_guide_train(self._h, C.c_void_p(records.data_ptr()), records.shape[0], steps, _fbox(box),
                                    _stream_ptr(stream)))

    def set_wait_limit(self, tries):
        """Polls of a tensor-core completion barrier before a wait gives up (lam_guide_set_wait_limit);
        0 makes every wait give up at once."""
        check(lib().lam_guide_set_wait_limit(self._h, int(tries)))

    def progress(self):
        st, spp = C.c_uint64(), C.c_uint32()
        check(lib().lam_guide_progress(self._h, C.byref(st), C.byref(spp)))
        return st.value, spp.value

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.lam_guide_destroy(self._h)
            self._h = None


# ---------------------------------------------------------------- no-vertex-return input format
class Vertices:
    """The reference's Vertices record (src/lib.rs:439-454): geometry_stride and [f32; 4] vertices."""

    def __init__(self, geometry_stride, vertices):
        import numpy as np
        self.geometry_stride = int(geometry_stride)
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 4)

    def append_bytes(self, out=None):
        """Vertices::append_bytes: stride (u32), 12 zero bytes, then the vertices."""
        import numpy as np
        b = np.uint32(self.geometry_stride).tobytes() + bytes(12) + self.vertices.tobytes()
        return b if out is None else out + b


def blas_from_vertices(vertices_blob, indices, triangles_per_geometry, flags=1):
    """lam_blas_from_vertices: a BLAS dict (vertices (V, 4), indices, flags) for lambent_b200 scenes."""
    import numpy as np
    blob = np.frombuffer(bytes(vertices_blob), dtype=np.uint8).copy()
    idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    tpg = np.ascontiguousarray(triangles_per_geometry, dtype=np.uint32).reshape(-1)
    d = _abi.BlasDesc()
    check(lib().lam_blas_from_vertices(blob.ctypes.data_as(C.c_void_p), blob.size,
                                       idx.ctypes.data_as(C.POINTER(C.c_uint32)), idx.size, tpg.size,
                                       tpg.ctypes.data_as(C.POINTER(C.c_uint32)), flags, C.byref(d)))
    try:
        v = np.ctypeslib.as_array(d.vertices, shape=(d.vertex_count * 4,)).reshape(-1, 4).copy() if d.vertex_count else \
            np.zeros((0, 4), np.float32)
        ix = np.ctypeslib.as_array(d.indices, shape=(d.index_count,)).copy() if d.index_count else np.zeros(0, np.uint32)
    finally:
        check(lib().lam_blas_desc_free(C.byref(d)))
    return {"vertices": v, "indices": ix, "flags": flags}


def material_table_for_geometries(table, triangles_per_geometry):
    import numpy as np
    t = np.ascontiguousarray(table, dtype=np.uint32).reshape(-1)
    tpg = np.ascontiguousarray(triangles_per_geometry, dtype=np.uint32).reshape(-1)
    out = np.zeros(int(tpg.sum()), dtype=np.uint32)
    check(lib().lam_material_table_for_geometries(t.ctypes.data_as(C.POINTER(C.c_uint32)), t.size, tpg.size,
                                                  tpg.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                  out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out
