"""ctypes wrapper of the CPU oracle (liblambent_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
leg as the checker of the CUDA product; the product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from lambent_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblambent_oracle.so")
# The same restatement built with floating-point contraction (a * b + c fused where the compiler
# chooses): it differs from LIB_PATH only in last bits, which measures how far same-seed renders
# can drift apart from last-bit arithmetic differences alone.
FMA_LIB_PATH = os.path.join(HERE, "liblambent_oracle_fma.so")
_LIB = None
_FMA_LIB = None


class RenderArgs(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("samples", C.c_uint32), ("quality", C.c_uint32),
                ("restir", C.c_uint32), ("max_depth", C.c_uint32), ("guide", C.c_uint32), ("seed_offset", C.c_uint32),
                ("tmin", C.c_float), ("tmax", C.c_float), ("camera", C.POINTER(_abi.Camera)),
                ("crop_x0", C.c_uint32), ("crop_y0", C.c_uint32), ("crop_w", C.c_uint32), ("crop_h", C.c_uint32),
                ("threads", C.c_int32),
                ("chains", C.c_void_p), ("old_chains", C.c_void_p), ("chains_len", C.c_uint64),
                ("old_chains_len", C.c_uint64), ("world", C.c_void_p), ("old_world", C.c_void_p),
                ("world_len", C.c_uint64), ("reservoirs", C.c_void_p), ("info", C.c_void_p),
                ("out_color", C.c_void_p), ("out_normal", C.c_void_p), ("out_albedo", C.c_void_p),
                ("segments_out", C.c_uint64), ("samples_out", C.c_uint64)]


def build():
    """Compiles the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def fma_available():
    """The contracted build needs the host's FMA instructions."""
    try:
        return " fma " in (" " + open("/proc/cpuinfo").read().replace("\n", " ") + " ")
    except OSError:
        return False


def lib(contracted=False):
    """The oracle library; contracted=True: the build with floating-point contraction (FMA_LIB_PATH)."""
    global _LIB, _FMA_LIB
    if contracted:
        if _FMA_LIB is None:
            if not os.path.exists(FMA_LIB_PATH):
                subprocess.run(["make", "-s", "-C", HERE, "liblambent_oracle_fma.so"], check=True)
            _FMA_LIB = _bind(C.CDLL(FMA_LIB_PATH))
        return _FMA_LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        build()
    _LIB = _bind(C.CDLL(LIB_PATH))
    return _LIB


def _bind(L):
    vp, i, u32 = C.c_void_p, C.c_int, C.c_uint32
    L.oracle_scene_create.argtypes = [C.POINTER(_abi.SceneDesc), C.POINTER(vp)]
    L.oracle_scene_create.restype = i
    L.oracle_scene_destroy.argtypes = [vp]
    L.oracle_trace.argtypes = [vp, vp, C.c_uint64, u32, vp, C.c_int32, C.c_int32]
    L.oracle_trace.restype = i
    L.oracle_render.argtypes = [vp, C.POINTER(RenderArgs)]
    L.oracle_render.restype = i
    L.oracle_temporal_resampling.argtypes = [vp, vp, u32, u32, u32]
    L.oracle_spatial_resampling.argtypes = [vp, vp, u32, u32, u32, u32, u32, vp]
    L.oracle_process_gi_reservoirs.argtypes = [vp, C.c_uint64, u32]
    L.oracle_process_world_markov_chains.argtypes = [vp, C.c_uint64]
    L.oracle_average_frames.argtypes = [C.POINTER(vp), u32, u32, u32, vp]
    L.oracle_rand_u32.argtypes = [u32]
    L.oracle_rand_u32.restype = u32
    L.oracle_rand_f32.argtypes = [u32]
    L.oracle_rand_f32.restype = C.c_float
    L.oracle_f32_to_f16.argtypes = [C.c_float]
    L.oracle_f32_to_f16.restype = C.c_uint16
    L.oracle_f16_to_f32.argtypes = [C.c_uint16]
    L.oracle_f16_to_f32.restype = C.c_float
    L.oracle_f32_to_bf16.argtypes = [C.c_float]
    L.oracle_f32_to_bf16.restype = C.c_uint16
    L.oracle_normalised_to_u32.argtypes = [C.POINTER(C.c_float)]
    L.oracle_normalised_to_u32.restype = u32
    L.oracle_u32_to_normalised.argtypes = [u32, C.POINTER(C.c_float)]
    L.oracle_material_new.argtypes = [C.POINTER(C.c_float)] * 3 + [C.POINTER(C.c_uint16), C.c_uint16, C.c_int32,
                                                                    C.c_int32, C.c_float, C.c_float,
                                                                    C.POINTER(C.c_float), u32,
                                                                    C.POINTER(_abi.Material)]
    L.oracle_material_new.restype = i
    L.oracle_camera_from_proj_view.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(_abi.Camera)]
    L.oracle_camera_from_proj_view.restype = i
    L.oracle_invert_3x4.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.oracle_invert_3x4.restype = i
    fp = C.POINTER(C.c_float)
    L.oracle_wbw.argtypes = [fp, fp, fp, fp, fp, fp, fp, fp, fp, C.POINTER(C.c_int32)]
    L.oracle_wbw.restype = i
    return L


class OracleCamera:
    """A packed camera record (`.c`, the 128-byte lam_camera) made without the product library."""

    def __init__(self, c):
        self.c = c


class OraclePacker:
    """Scene packer for lambent_b200.scenes that uses the oracle's own restatements of
    Material::new (src/lib.rs:132-163) and Camera::from_proj_view (src/camera.rs:15-24, 59-70), so
    that the CPU legs of the benchmark never load the product library."""

    @staticmethod
    def material(uv1, uv2, uv3, recolour, diffuse, emission, attributes, emission_scale, ior, ty):
        f2 = lambda p: (C.c_float * 2)(*p)
        m = _abi.Material()
        rc = lib().oracle_material_new(f2(uv1), f2(uv2), f2(uv3), (C.c_uint16 * 2)(*recolour), diffuse,
                                       -1 if emission is None else emission, -1 if attributes is None else attributes,
                                       emission_scale.emissive_texture_scale, emission_scale.diffuse_texture_scale,
                                       None if ior is None else f2(ior), ty, C.byref(m))
        if rc != 0:
            raise ValueError(f"oracle_material_new failed: {rc}")
        return m

    @staticmethod
    def camera(proj, view):
        flat = lambda m: (C.c_float * 16)(*[float(x) for x in np.asarray(m, np.float32).reshape(-1)])
        c = _abi.Camera()
        rc = lib().oracle_camera_from_proj_view(flat(proj), flat(view), C.byref(c))
        if rc != 0:
            raise ValueError(f"oracle_camera_from_proj_view failed: {rc}")
        return OracleCamera(c)


def flatten_no_vertex_return(vertices, geometry_stride, indices, triangles_per_geometry, material_table):
    """The reference's no-vertex-return lookup, restated independently of the library: triangle p of
    geometry g reads index slots geometry_stride * g + 3p + {0, 1, 2}, or uses the slot numbers
    themselves when the index array has length 1 (get_vertices, src/bindings.wesl:103-110); its
    material is material_table[p], the primitive index within its geometry, clamped to the table as
    a bounds-checked GPU load is (general.wesl:1086).

    Returns (triangle-list vertices (3T, 3) f32, per-triangle material indices (T,) u32)."""
    vertices = np.asarray(vertices, np.float32).reshape(-1, 4)
    indices = np.asarray(indices, np.uint32).reshape(-1)
    table = np.asarray(material_table, np.uint32).reshape(-1)
    tri_v, tri_m = [], []
    for g, count in enumerate(triangles_per_geometry):
        for p in range(count):
            slot = geometry_stride * g + 3 * p
            for j in range(3):
                vi = slot + j if indices.size == 1 else int(indices[slot + j])
                tri_v.append(vertices[vi, :3])
            tri_m.append(table[min(p, table.size - 1)])
    return np.asarray(tri_v, np.float32), np.asarray(tri_m, np.uint32)


HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<u4"), ("inst", "<u4"), ("kind", "<u4")])


class OracleScene:
    def __init__(self, scene, contracted=False):
        self.holder = _abi.SceneDescHolder(scene)
        self._L = lib(contracted)
        h = C.c_void_p()
        rc = self._L.oracle_scene_create(self.holder.ptr(), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle_scene_create failed: {rc}")
        self._h = h

    def trace(self, rays, mode=_abi.TRACE_CLOSEST, threads=None, bruteforce=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
        threads = threads or os.cpu_count() or 1
        rc = self._L.oracle_trace(self._h, rays.ctypes.data, rays.shape[0], mode, hits.ctypes.data, threads,
                                1 if bruteforce else 0)
        if rc != 0:
            raise RuntimeError(f"oracle_trace failed: {rc}")
        return hits

    def render(self, camera, width, height, samples=4, quality=_abi.QUALITY_MEDIUM, restir=_abi.RESTIR_PER_PIXEL,
               max_depth=5, guide=_abi.GUIDE_NONE, seed_offset=0, tmin=1e-4, tmax=1000.0, crop=None, threads=None,
               buffers=None):
        """Returns dict with color/normal/albedo (H, W, 4) and the state buffers (numpy)."""
        P = width * height
        out = {k: np.zeros((height, width, 4), np.float32) for k in ("color", "normal", "albedo")}
        b = buffers if buffers is not None else new_buffers(width, height, 1 << 16)
        a = RenderArgs()
        a.width, a.height, a.samples, a.quality = width, height, samples, quality
        a.restir, a.max_depth, a.guide, a.seed_offset = restir, max_depth, guide, seed_offset
        a.tmin, a.tmax = tmin, tmax
        cam = camera.c if hasattr(camera, "c") else camera
        a.camera = C.pointer(cam)
        if crop is not None:
            a.crop_x0, a.crop_y0, a.crop_w, a.crop_h = crop
        a.threads = threads or os.cpu_count() or 1
        a.chains = b["chains"].ctypes.data
        a.old_chains = b["old_chains"].ctypes.data
        a.chains_len = a.old_chains_len = b["chains"].shape[0]
        a.world = b["world"].ctypes.data
        a.old_world = b["old_world"].ctypes.data
        a.world_len = b["world"].shape[0] // 14
        a.reservoirs = b["reservoirs"].ctypes.data
        a.info = b["info"].ctypes.data
        a.out_color = out["color"].ctypes.data
        a.out_normal = out["normal"].ctypes.data
        a.out_albedo = out["albedo"].ctypes.data
        rc = self._L.oracle_render(self._h, C.byref(a))
        if rc != 0:
            raise RuntimeError(f"oracle_render failed: {rc}")
        out["segments"] = a.segments_out
        out["samples"] = a.samples_out
        out["buffers"] = b
        return out

    def __del__(self):
        if getattr(self, "_h", None) and getattr(self, "_L", None) is not None:
            self._L.oracle_scene_destroy(self._h)
            self._h = None


def new_buffers(width, height, world_size):
    P = width * height
    return {
        "chains": np.zeros((P, 8), np.float32), "old_chains": np.zeros((P, 8), np.float32),
        "world": np.zeros(world_size * 14, np.uint32), "old_world": np.zeros(world_size * 14, np.uint32),
        "reservoirs": np.zeros((P, 16), np.float32), "old_reservoirs": np.zeros((P, 16), np.float32),
        "info": np.zeros((P, 9), np.float32),
    }


def temporal(cur, old, width, height, seed_offset):
    lib().oracle_temporal_resampling(cur.ctypes.data, old.ctypes.data, width, height, seed_offset)


def spatial(cur, info, width, height, is_samples, is_space, seed_offset):
    out = np.zeros((height, width, 4), np.float32)
    lib().oracle_spatial_resampling(cur.ctypes.data, info.ctypes.data, width, height, is_samples, is_space,
                                    seed_offset, out.ctypes.data)
    return out


def process_gi(res, cap):
    lib().oracle_process_gi_reservoirs(res.ctypes.data, res.shape[0], cap)


def process_world(world):
    lib().oracle_process_world_markov_chains(world.ctypes.data, world.size // 14)


def average(frames):
    h, w = frames[0].shape[:2]
    arrs = [np.ascontiguousarray(f, np.float32) for f in frames]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    out = np.zeros(h * w * 3, np.float32)
    lib().oracle_average_frames(ptrs, len(arrs), w, h, out.ctypes.data)
    return out
