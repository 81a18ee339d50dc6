"""C-ABI surface: the library loads without a GPU, exports every entry point of include/lambent.h,
and its host-only functions (Material, Camera, TextureLoader, layouts) follow the reference."""
import ctypes as C
import os
import re
import struct
import zlib

import numpy as np
import pytest

import lambent_b200 as lb
from lambent_b200 import _abi
from oracle import oracle_py as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    src = open(os.path.join(ROOT, "include", "lambent.h")).read()
    return sorted(set(re.findall(r"\b(lam_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = lb.lib()
    names = declared_entry_points()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_dispatch_size():
    assert lb.lib().lam_version() == 0x00010000
    assert lb.dispatch_size(1920, 1080) == (30, 1080)
    assert lb.dispatch_size(65, 3) == (2, 3)


def test_material_matches_oracle_packing():
    rng = np.random.default_rng(1)
    for _ in range(200):
        uv = [tuple(map(float, rng.normal(0, 2, 2))) for _ in range(3)]
        rec = tuple(int(x) for x in rng.integers(0, 65535, 2))
        d = int(rng.integers(0, 65535))
        e = None if rng.random() < 0.3 else int(rng.integers(0, 65535))
        a = None if rng.random() < 0.3 else int(rng.integers(0, 65535))
        es = lb.EmissionScale.from_f32(float(rng.lognormal(0, 3)), float(rng.normal()))
        ior = None if rng.random() < 0.3 else tuple(map(float, rng.uniform(1, 3, 2)))
        ty = int(rng.integers(0, 3))
        m = lb.Material.new(uv[0], uv[1], uv[2], rec, d, e, a, es, ior, ty)
        ref = _abi.Material()
        f = lambda v: (C.c_float * 2)(*v)
        rc = O.lib().oracle_material_new(f(uv[0]), f(uv[1]), f(uv[2]), (C.c_uint16 * 2)(*rec), d,
                                         -1 if e is None else e, -1 if a is None else a, es.emissive_texture_scale,
                                         es.diffuse_texture_scale, None if ior is None else f(ior), ty, C.byref(ref))
        assert rc == 0
        assert bytes(m) == bytes(ref)


def test_material_reserved_index_is_an_error():
    with pytest.raises(lb.LambentError) as e:
        lb.Material.new((0, 0), (0, 0), (0, 0), (0, 0), 0, 0xFFFF, None, lb.EmissionScale(), None, 0)
    assert e.value.code == _abi.ERR_INVALID_ARGUMENT


def test_material_layout_fields():
    m = lb.Material.new((1.0, 1.0), (0.0, 1.0), (1.0, 0.0), (3, 4), 2, None, 7, lb.EmissionScale.from_f32(15.0, 0.5),
                        (1.5, 1.5), lb.MaterialType.Transparent)
    assert m.tex_pos_1 == 0x3C003C00 and m.tex_pos_2 == 0x3C000000 and m.tex_pos_3 == 0x00003C00
    assert m.tex_pos_recolour == (4 << 16) | 3
    assert m.tex_idx_diffuse_emission == (0xFFFF << 16) | 2
    assert m.tex_idx_attributes_ty == (2 << 16) | 7
    assert m.emission_scale == (0x3F00 << 16) | 0x4170
    assert m.refractive_index == 0x3E003E00
    data, usage = lb.Material.descriptor([m, m])
    assert len(data) == 64 and usage == _abi.USAGE_STORAGE


def test_refractive_index_between():
    r = lb.refractive_indices.refractive_index_between(lb.refractive_indices.AIR, lb.refractive_indices.DIAMOND)
    assert abs(r[0] - 2.4063 / 1.00027531) < 1e-6 and abs(r[1] - 2.4922 / 1.000287) < 1e-6


def test_camera_inverse_matches_oracle_and_errors():
    from lambent_b200 import scenes
    proj = scenes.perspective(45.0, 1.5, 0.1, 200.0)
    view = scenes.look_to_rh((0.5, 0.5, -1.0), (0.0, 0.0, 1.0), np.array([0.0, 1.0, 0.0]))
    cam = lb.Camera.new(proj, view)
    ref = _abi.Camera()
    f = lambda m: (C.c_float * 16)(*np.asarray(m, np.float32).reshape(-1))
    assert O.lib().oracle_camera_from_proj_view(f(proj), f(view), C.byref(ref)) == 0
    a = np.array(cam.c.projection_inverse[:] + cam.c.view_inverse[:], np.float32)
    b = np.array(ref.projection_inverse[:] + ref.view_inverse[:], np.float32)
    np.testing.assert_allclose(a, b, rtol=2e-7, atol=1e-7)
    data, usage = cam.descriptor()
    assert len(data) == 128 and usage == _abi.USAGE_UNIFORM
    with pytest.raises(lb.LambentError) as e:
        lb.Camera.new(np.zeros((4, 4)), view)
    assert e.value.code == _abi.ERR_PROJECTION_UNINVERTIBLE
    with pytest.raises(lb.LambentError) as e:
        lb.Camera.new(proj, np.zeros((4, 4)))
    assert e.value.code == _abi.ERR_VIEW_UNINVERTIBLE
    cam.update_from_proj_view(view=np.eye(4))
    assert list(cam.c.view_inverse) == list(np.eye(4, dtype=np.float32).reshape(-1))


def _png(img, ctype=6, filt=None, depth=8):
    h, w = img.shape[:2]
    ch = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    raw = b""
    prev = np.zeros(w * ch * (depth // 8), np.int64)
    for y in range(h):
        row = img[y].reshape(-1).astype(np.int64)
        if depth == 16:
            row = np.stack([row * 257 >> 8, row * 257 & 255], 1).reshape(-1)
        ft = (y % 5) if filt is None else filt
        bpp = ch * depth // 8
        left = np.concatenate([np.zeros(bpp, np.int64), row[:-bpp]])
        up = prev
        ul = np.concatenate([np.zeros(bpp, np.int64), prev[:-bpp]])
        if ft == 0:
            enc = row
        elif ft == 1:
            enc = row - left
        elif ft == 2:
            enc = row - up
        elif ft == 3:
            enc = row - (left + up) // 2
        else:
            p = left + up - ul
            pa, pb, pc = np.abs(p - left), np.abs(p - up), np.abs(p - ul)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, up, ul))
            enc = row - pred
        raw += bytes([ft]) + bytes((enc & 255).astype(np.uint8))
        prev = row
    chunk = lambda t, d: struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)
    ihdr = struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0)
    return b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", ihdr) + chunk(b"IDAT", zlib.compress(raw, 9)) + chunk(b"IEND", b"")


@pytest.mark.parametrize("ctype", [0, 2, 4, 6])
@pytest.mark.parametrize("depth", [8, 16])
def test_texture_loader_png_decode(ctype, depth):
    rng = np.random.default_rng(ctype + depth)
    ch = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    img = rng.integers(0, 256, (37, 23, ch), dtype=np.uint8)
    tl = lb.TextureLoader()
    tl.load_from_bytes(_png(img, ctype, depth=depth))
    raw = tl.raw()
    got = raw["diffuse"][0]
    exp = np.zeros((37, 23, 4), np.uint8)
    if ch in (1, 2):
        exp[..., 0] = exp[..., 1] = exp[..., 2] = img[..., 0]
        exp[..., 3] = img[..., 1] if ch == 2 else 255
    else:
        exp[..., :3] = img[..., :3]
        exp[..., 3] = img[..., 3] if ch == 4 else 255
    np.testing.assert_array_equal(got, exp)


def test_texture_loader_raw_cuboids_and_errors():
    a = np.full((8, 8, 4), 10, np.uint8)
    b = np.full((4, 6, 4), 20, np.uint8)
    tl = lb.TextureLoader()
    tl.load_rgba8(a, lit=a)
    tl.load_rgba8(b, attributes=b)
    raw = tl.raw()
    assert raw["diffuse"].shape == (2, 8, 8, 4) and raw["lit"].shape == (1, 8, 8, 4)
    assert raw["attributes"].shape == (1, 4, 6, 4)
    assert raw["layer_of_entry"]["lit"] == [0, -1] and raw["layer_of_entry"]["attributes"] == [-1, 0]
    assert (raw["diffuse"][1, :4, :6] == 20).all() and (raw["diffuse"][1, 4:] == 0).all()
    tl = lb.TextureLoader()
    with pytest.raises(lb.LambentError) as e:
        tl.load_from_bytes(b"not a png")
    assert e.value.code == _abi.ERR_TEXTURE
    with pytest.raises(lb.LambentError):
        tl.load("/nonexistent/texture.png")


# The reference checkout's root, when one is available (LAMBENT_REFERENCE_DIR); its 64x64 PNG
# fixtures live under src/tests.
REF_PNG = os.path.join(os.environ.get("LAMBENT_REFERENCE_DIR", ""), "src", "tests")


@pytest.mark.skipif(not os.environ.get("LAMBENT_REFERENCE_DIR") or not os.path.isdir(REF_PNG),
                    reason="set LAMBENT_REFERENCE_DIR to a reference checkout to decode its PNG fixtures")
def test_texture_loader_reads_reference_fixtures():
    # first pixels as recorded for the reference's own 64x64 RGBA8 fixtures
    tl = lb.TextureLoader()
    tl.load(os.path.join(REF_PNG, "diffuse.png"), os.path.join(REF_PNG, "emission.png"),
            os.path.join(REF_PNG, "pure_white.png"))
    raw = tl.raw()
    assert tuple(raw["diffuse"][0, 0, 0]) == (34, 177, 76, 255)
    assert tuple(raw["lit"][0, 0, 0]) == (255, 0, 0, 255)
    assert tuple(raw["attributes"][0, 0, 0]) == (250, 250, 250, 255)


def test_layout_and_options():
    with pytest.raises(lb.LambentError):
        lb.pipeline_layout(0, 1, 1, 1)
    lb.pipeline_layout(1, 4, 1, 1)
    o = _abi.TracerOptions()
    lb.check(lb.lib().lam_tracer_options_default(C.byref(o)))
    assert (o.samples, o.restir_temporal, o.max_depth) == (4, _abi.RESTIR_PER_PIXEL, 5)
    assert abs(o.tmin - 1e-4) < 1e-9 and o.tmax == 1000.0
    t = lb.RayTracer(lb.path_tracing.High)
    t.set_intersection_handler(None)
    with pytest.raises(lb.LambentError):
        lb.lib().lam_tracer_create(99, C.byref(C.c_void_p())) and lb.check(-1)


def test_pipeline_tuning_entry_points_reject_null_pipelines():
    """The host-side pipeline knobs validate their handle before anything touches the GPU."""
    L = lb.lib()
    assert L.lam_pipeline_set_wave_paths(None, C.c_uint64(1 << 20)) == _abi.ERR_INVALID_ARGUMENT
    assert L.lam_pipeline_set_profiling(None, 1) == _abi.ERR_INVALID_ARGUMENT
    assert L.lam_pipeline_set_guide(None, None) == _abi.ERR_INVALID_ARGUMENT
    assert L.lam_pipeline_set_shade_order(None, _abi.SHADE_ORDER_MATERIAL) == _abi.ERR_INVALID_ARGUMENT
