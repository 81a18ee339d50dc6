// materials.cuh - material record decode and texture fetches on the device.
//
// Material layout: src/bindings.wesl:48-57 (packed by Material::new, src/lib.rs:132-182).
// Texture sampling: textureSampleLevel with wgpu's default sampler (nearest filtering,
// clamp-to-edge) on Rgba8Unorm textures with a single mip level (src/textures.rs:41-90, 196),
// textureLoad of the recolour texture (general.wesl:1122) and the sky cube map
// (general.wesl:1180-1182; face order +X,-X,+Y,-Y,+Z,-Z with the standard cube-map (s,t) table).
#pragma once
#include "device_math.cuh"
#include "scene.h"

namespace lam {

LAM_DEV uint32_t clamp_idx(uint32_t i, uint32_t n) { return n == 0u ? 0u : (i < n ? i : n - 1u); }

LAM_DEV lam_material load_material(const DevScene& S, uint32_t inst, uint32_t prim) {
    const DevInstance& I = S.inst[inst];
    uint32_t mi = I.mat_count ? __ldg(S.mat_idx + I.mat_offset + clamp_idx(prim, I.mat_count)) : 0u;
    mi = clamp_idx(mi, S.material_count);
    const uint4* mp = reinterpret_cast<const uint4*>(S.materials + mi);
    uint4 a = __ldg(mp), b = __ldg(mp + 1);
    lam_material m;
    m.tex_pos_1 = a.x; m.tex_pos_2 = a.y; m.tex_pos_3 = a.z; m.tex_pos_recolour = a.w;
    m.tex_idx_diffuse_emission = b.x; m.tex_idx_attributes_ty = b.y; m.emission_scale = b.z; m.refractive_index = b.w;
    return m;
}

LAM_DEV float4 unpack_texel(uint32_t t) {
    const float s = 1.0f / 255.0f;
    return make_float4((float)(t & 0xFFu) / 255.0f, (float)((t >> 8) & 0xFFu) / 255.0f,
                       (float)((t >> 16) & 0xFFu) / 255.0f, (float)(t >> 24) / 255.0f);
    (void)s;
}

// Nearest, clamp-to-edge sample of layer `layer` of a texture array [first, first + count).
LAM_DEV float4 tex_sample(const DevScene& S, uint32_t first, uint32_t count, uint32_t layer, float u, float v) {
    if (layer >= count) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const DevTexLayer L = S.layers[first + layer];
    if (L.w == 0u || L.h == 0u) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    int32_t x = f2i(floorf(u * (float)L.w));
    int32_t y = f2i(floorf(v * (float)L.h));
    x = min(max(x, 0), (int32_t)L.w - 1);
    y = min(max(y, 0), (int32_t)L.h - 1);
    return unpack_texel(__ldg(S.texels + L.offset + (uint32_t)y * L.w + (uint32_t)x));
}

LAM_DEV float4 recolour_load(const DevScene& S, uint32_t x, uint32_t y) {
    const DevTexLayer L = S.layers[S.recolour_layer];
    x = clamp_idx(x, L.w);
    y = clamp_idx(y, L.h);
    return unpack_texel(__ldg(S.texels + L.offset + y * L.w + x));
}

LAM_DEV v3 sky_sample(const DevScene& S, v3 d) {
    if (S.sky == nullptr || S.sky_size == 0u) return splat(0.0f);
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    uint32_t face;
    float sc, tc, ma;
    if (ax >= ay && ax >= az) {
        ma = ax;
        if (d.x >= 0.0f) { face = 0; sc = -d.z; tc = -d.y; } else { face = 1; sc = d.z; tc = -d.y; }
    } else if (ay >= az) {
        ma = ay;
        if (d.y >= 0.0f) { face = 2; sc = d.x; tc = d.z; } else { face = 3; sc = d.x; tc = -d.z; }
    } else {
        ma = az;
        if (d.z >= 0.0f) { face = 4; sc = d.x; tc = -d.y; } else { face = 5; sc = -d.x; tc = -d.y; }
    }
    if (!(ma > 0.0f)) return splat(0.0f);
    float s = 0.5f * (sc / ma + 1.0f), t = 0.5f * (tc / ma + 1.0f);
    const int32_t n = (int32_t)S.sky_size;
    int32_t x = min(max(f2i(floorf(s * (float)S.sky_size)), 0), n - 1);
    int32_t y = min(max(f2i(floorf(t * (float)S.sky_size)), 0), n - 1);
    float4 c = unpack_texel(__ldg(S.sky + ((size_t)face * S.sky_size + (uint32_t)y) * S.sky_size + (uint32_t)x));
    return mk(c.x, c.y, c.z);
}

// UV of a hit from the material's three per-vertex UVs: uv1 * (1-u-v) + uv2 * u + uv3 * v
// (general.wesl:1061-1062, 1118-1119).
LAM_DEV float2 hit_uv(const lam_material& m, float bu, float bv) {
    float bz = (1.0f - bu) - bv;
    float2 t1 = unpack2x16float(m.tex_pos_1), t2 = unpack2x16float(m.tex_pos_2), t3 = unpack2x16float(m.tex_pos_3);
    return make_float2(fmaf(t1.x, bz, fmaf(t2.x, bu, t3.x * bv)), fmaf(t1.y, bz, fmaf(t2.y, bu, t3.y * bv)));
}

LAM_DEV bool alpha_accept(const DevScene& S, uint32_t inst, uint32_t prim, float bu, float bv, bool transparent_passes) {
    if (S.material_count == 0u) return true;
    lam_material m = load_material(S, inst, prim);
    float2 uv = hit_uv(m, bu, bv);
    uint32_t idx_d = m.tex_idx_diffuse_emission & 0xFFFFu;
    uint32_t ty = m.tex_idx_attributes_ty >> 16;
    float4 px = tex_sample(S, S.diffuse_first, S.diffuse_count, idx_d, uv.x, uv.y);
    return !near_zero(px.w) || (transparent_passes && ty == TY_TRANSPARENT);
}

}  // namespace lam
