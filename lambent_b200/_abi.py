"""ctypes mirror of include/lambent.h (plain data types, enums, status codes).

The struct layouts are bit-identical to the reference's GPU-visible records
(Material, src/lib.rs:83-94; Camera, src/camera.rs:6-11; Reservoir, src/bindings.wesl:158-169;
MarcovChainState / WorldMarcovChainState, src/bindings.wesl:3-40).
"""
import ctypes as C

u8, u16, u32, u64, i32, f32 = C.c_uint8, C.c_uint16, C.c_uint32, C.c_uint64, C.c_int32, C.c_float

# status codes
LAM_OK = 0
STATUS_NAMES = {
    0: "LAM_OK", -1: "LAM_ERR_INVALID_ARGUMENT", -2: "LAM_ERR_OUT_OF_MEMORY", -3: "LAM_ERR_CUDA",
    -4: "LAM_ERR_NOT_BUILT", -5: "LAM_ERR_PROJECTION_UNINVERTIBLE", -6: "LAM_ERR_VIEW_UNINVERTIBLE",
    -7: "LAM_ERR_TEXTURE", -8: "LAM_ERR_COMPILE", -9: "LAM_ERR_LAYOUT_MISMATCH", -10: "LAM_ERR_UNSUPPORTED",
    -11: "LAM_ERR_DEVICE_TIMEOUT", -12: "LAM_ERR_STACK_OVERFLOW", -13: "LAM_ERR_CALLBACK",
}
ERR_INVALID_ARGUMENT = -1
ERR_PROJECTION_UNINVERTIBLE = -5
ERR_VIEW_UNINVERTIBLE = -6
ERR_TEXTURE = -7
ERR_COMPILE = -8
ERR_LAYOUT_MISMATCH = -9
ERR_UNSUPPORTED = -10
ERR_DEVICE_TIMEOUT = -11
ERR_CALLBACK = -13

DIFFUSE, METALLIC, TRANSPARENT, SKY = 0, 1, 2, 0xFF
QUALITY_LOW, QUALITY_MEDIUM, QUALITY_HIGH = 0, 1, 2
DEBUG_FRONT_FACE, DEBUG_REFLECTANCE, DEBUG_TANGENT = 16, 17, 18
RESTIR_DISABLED, RESTIR_PER_SAMPLE, RESTIR_PER_PIXEL = 0, 1, 2
GUIDE_NONE, GUIDE_MARKOV, GUIDE_LEARNED = 0, 1, 2
GUIDE_PDF_AT_SAMPLE = 4  # modifier of GUIDE_MARKOV: mixture pdf with its cosine term at the chosen direction
GUIDE_METAL = 8  # modifier of the learned modes: mix the learned lobes in at rough metallic vertices too
SHADE_ORDER_AUTO = 0      # lam_pipeline_set_shade_order: material order except under Markov guiding
SHADE_ORDER_QUEUE = 1     # traversal order
SHADE_ORDER_MATERIAL = 2  # sorted by shading class (sky, diffuse, metallic, transparent)
BUFFER_MARKOV_CHAIN_SCREEN_SPACE, BUFFER_SPATIAL_RESAMPLING, BUFFER_MARKOV_CHAIN_WORLD_SPACE = 1, 2, 4
BUFFER_ALL = 7
USAGE_COPY_DST, USAGE_UNIFORM, USAGE_STORAGE = 0x8, 0x40, 0x80
GEOMETRY_OPAQUE = 1
TRACE_CLOSEST, TRACE_ANY = 0, 1
HIT_NONE, HIT_FRONT, HIT_BACK = 0, 1, 2


class Material(C.Structure):
    _fields_ = [("tex_pos_1", u32), ("tex_pos_2", u32), ("tex_pos_3", u32), ("tex_pos_recolour", u32),
                ("tex_idx_diffuse_emission", u32), ("tex_idx_attributes_ty", u32),
                ("emission_scale", u32), ("refractive_index", u32)]


class Camera(C.Structure):
    _fields_ = [("projection_inverse", f32 * 16), ("view_inverse", f32 * 16)]


class MarkovChain(C.Structure):
    _fields_ = [("light_source", f32 * 3), ("mean_cosine", f32), ("weight_sum", f32), ("num_samples", u32),
                ("score", f32), ("_pad", u32)]


class WorldMarkovChain(C.Structure):
    _fields_ = [("secondary_hash", u32), ("num_samples", u32), ("luminance", u32 * 3), ("lock", u32),
                ("chain_light_source", u32 * 3), ("chain_mean_cosine", u32), ("chain_weight_sum", u32),
                ("chain_num_samples", u32), ("chain_score", u32), ("timeout", u32)]


class Reservoir(C.Structure):
    _fields_ = [("visible_point", f32 * 3), ("visible_normal", u32), ("sample_point", f32 * 3),
                ("sample_normal", u32), ("out_radiance", f32 * 3), ("ty", u32), ("roughness", f32), ("w", f32),
                ("packed_confidence_valid", u32), ("W", f32)]


class Info(C.Structure):
    _fields_ = [("arr", f32 * 9)]


class BufferDescriptor(C.Structure):
    _fields_ = [("contents", C.c_void_p), ("size", C.c_size_t), ("usage", u32)]


class BlasDesc(C.Structure):
    _fields_ = [("vertices", C.POINTER(f32)), ("vertex_count", u32), ("vertex_stride", u32),
                ("indices", C.POINTER(u32)), ("index_count", u32), ("flags", u32),
                ("aabbs", C.POINTER(f32)), ("aabb_count", u32)]


class InstanceDesc(C.Structure):
    _fields_ = [("transform", f32 * 12), ("blas", u32), ("custom_index", u32), ("mask", u32),
                ("material_indices", C.POINTER(u32)), ("material_index_count", u32)]


class TextureLayer(C.Structure):
    _fields_ = [("rgba8", C.POINTER(u8)), ("width", u32), ("height", u32)]


class SceneDesc(C.Structure):
    _fields_ = [("blas", C.POINTER(BlasDesc)), ("blas_count", u32),
                ("instances", C.POINTER(InstanceDesc)), ("instance_count", u32),
                ("materials", C.POINTER(Material)), ("material_count", u32),
                ("diffuse", C.POINTER(TextureLayer)), ("diffuse_count", u32),
                ("emission", C.POINTER(TextureLayer)), ("emission_count", u32),
                ("attributes", C.POINTER(TextureLayer)), ("attribute_count", u32),
                ("recolour", C.POINTER(TextureLayer)),
                ("sky_faces", C.POINTER(u8)), ("sky_size", u32)]


class SceneStats(C.Structure):
    _fields_ = [("triangle_count", u64), ("blas_node_count", u64), ("tlas_node_count", u64),
                ("device_bytes", u64), ("build_seconds", C.c_double)]


class TracerOptions(C.Structure):
    _fields_ = [("samples", u32), ("tmin", f32), ("tmax", f32), ("restir_temporal", u32), ("max_depth", u32),
                ("guide_mode", u32)]


class FrameTargets(C.Structure):
    _fields_ = [("color", C.c_void_p), ("normal", C.c_void_p), ("albedo", C.c_void_p), ("width", u32),
                ("height", u32)]


class Ray(C.Structure):
    _fields_ = [("origin", f32 * 3), ("tmin", f32), ("direction", f32 * 3), ("tmax", f32)]


class Hit(C.Structure):
    _fields_ = [("t", f32), ("u", f32), ("v", f32), ("primitive_index", u32), ("instance_index", u32),
                ("kind", u32)]


class RenderStats(C.Structure):
    _fields_ = [("ray_segments", u64), ("samples", u64), ("kernel_launches", u32), ("error_flags", u32)]


class StageTimes(C.Structure):
    _fields_ = [("generate_ms", C.c_double), ("extend_ms", C.c_double), ("shade_ms", C.c_double),
                ("accumulate_ms", C.c_double), ("extend_launches", u64), ("shade_launches", u64),
                ("ray_segments", u64), ("train_ms", C.c_double)]


class BatchRequest(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("targets", FrameTargets), ("samples", u32),
                ("seed_offset", u32)]


class BatchTuning(C.Structure):
    _fields_ = [("wave_paths", u32), ("extend_blocks_per_sm", u32), ("shade_blocks_per_sm", u32), ("use_graph", u32)]


class GuideOptions(C.Structure):
    _fields_ = [("train_spp", u32), ("steps_per_wave", u32), ("batch", u32), ("record_capacity", u32),
                ("learning_rate", C.c_float), ("guide_fraction", C.c_float), ("seed", u32)]


GUIDE_PARAMS = 16384
GUIDE_OUTPUTS = 40


class RawTextures(C.Structure):
    _fields_ = [("cuboid", C.POINTER(u8) * 3), ("width", u32 * 3), ("height", u32 * 3), ("layers", u32 * 3),
                ("layer_of_entry", C.POINTER(i32) * 3), ("entry_count", u32)]


assert C.sizeof(Material) == 32
assert C.sizeof(Camera) == 128
assert C.sizeof(MarkovChain) == 32
assert C.sizeof(WorldMarkovChain) == 56
assert C.sizeof(Reservoir) == 64
assert C.sizeof(Info) == 36
assert C.sizeof(Ray) == 32
assert C.sizeof(Hit) == 24


class SceneDescHolder:
    """Builds a SceneDesc from numpy arrays and keeps every buffer alive while in use."""

    def __init__(self, scene):
        import numpy as np
        self._keep = []
        blas = (BlasDesc * max(1, len(scene.blas)))()
        for i, b in enumerate(scene.blas):
            if b.get("aabbs") is not None:  # procedural geometry: (N, 6) boxes, min xyz / max xyz
                a = np.ascontiguousarray(b["aabbs"], dtype=np.float32).reshape(-1, 6)
                self._keep.append(a)
                blas[i].vertices = None
                blas[i].vertex_count = 0
                blas[i].vertex_stride = 3
                blas[i].indices = None
                blas[i].index_count = 0
                blas[i].aabbs = a.ctypes.data_as(C.POINTER(f32))
                blas[i].aabb_count = a.shape[0]
                blas[i].flags = b.get("flags", GEOMETRY_OPAQUE)
                continue
            v = np.ascontiguousarray(b["vertices"], dtype=np.float32)
            idx = b.get("indices")
            self._keep.append(v)
            blas[i].vertices = v.ctypes.data_as(C.POINTER(f32))
            blas[i].vertex_count = v.shape[0]
            blas[i].vertex_stride = v.shape[1]
            if idx is not None:
                idx = np.ascontiguousarray(idx, dtype=np.uint32).reshape(-1)
                self._keep.append(idx)
                blas[i].indices = idx.ctypes.data_as(C.POINTER(u32))
                blas[i].index_count = idx.size
            else:
                blas[i].indices = None
                blas[i].index_count = (v.shape[0] // 3) * 3
            blas[i].flags = b.get("flags", GEOMETRY_OPAQUE)
        inst = (InstanceDesc * max(1, len(scene.instances)))()
        for i, it in enumerate(scene.instances):
            xf = np.asarray(it["transform"], dtype=np.float32).reshape(12)
            for k in range(12):
                inst[i].transform[k] = float(xf[k])
            inst[i].blas = it["blas"]
            inst[i].custom_index = it.get("custom_index", 0)
            inst[i].mask = it.get("mask", 0xFF)
            mi = np.ascontiguousarray(it["material_indices"], dtype=np.uint32)
            self._keep.append(mi)
            inst[i].material_indices = mi.ctypes.data_as(C.POINTER(u32))
            inst[i].material_index_count = mi.size
        mats = (Material * max(1, len(scene.materials)))(*scene.materials)

        def layers(arr):
            out = (TextureLayer * max(1, len(arr)))()
            for i, t in enumerate(arr):
                t = np.ascontiguousarray(t, dtype=np.uint8)
                self._keep.append(t)
                out[i].rgba8 = t.ctypes.data_as(C.POINTER(u8))
                out[i].height, out[i].width = t.shape[0], t.shape[1]
            return out

        d = SceneDesc()
        d.blas, d.blas_count = blas, len(scene.blas)
        d.instances, d.instance_count = inst, len(scene.instances)
        d.materials, d.material_count = mats, len(scene.materials)
        d.diffuse, d.diffuse_count = layers(scene.diffuse), len(scene.diffuse)
        d.emission, d.emission_count = layers(scene.emission), len(scene.emission)
        d.attributes, d.attribute_count = layers(scene.attributes), len(scene.attributes)
        d.recolour = None
        if getattr(scene, "recolour", None) is not None:
            rc = layers([scene.recolour])
            self._keep.append(rc)
            d.recolour = rc
        if getattr(scene, "sky", None) is not None:
            sky = np.ascontiguousarray(scene.sky, dtype=np.uint8)
            self._keep.append(sky)
            d.sky_faces = sky.ctypes.data_as(C.POINTER(u8))
            d.sky_size = sky.shape[1]
        else:
            d.sky_faces = None
            d.sky_size = 0
        self._keep += [blas, inst, mats]
        self.desc = d

    def ptr(self):
        return C.byref(self.desc)
