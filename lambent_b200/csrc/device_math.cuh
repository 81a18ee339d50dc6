// device_math.cuh - WGSL built-in semantics on sm_100a for the shading kernels.
//
// Reference shader helpers restated: RNG (src/importance_sampling/shared.wesl:266-292),
// safe_div / copy_sign (shared.wesl:255-312), near_zero (src/bindings.wesl:171-175),
// strip_NaN (src/path_tracing/general.wesl:117-135), octahedral packing
// (general.wesl:1293-1305, shared.wesl:233-245).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lam {

#define LAM_DEV __device__ __forceinline__

// Cache policy of the wavefront's loads.  Scene data that every ray of a render revisits (BVH nodes,
// triangles, instances) goes through the read-only path with an L2 access policy of evict_last;
// path state that one kernel reads once by queue position goes through ld.global.cs (evict first),
// so that the gigabytes of path state streamed per step push less of the scene out of L2 (measured
// on the bench scene: 141 -> 134.5 DRAM bytes per traversal segment, +0.5% rays/s).
LAM_DEV uint64_t keep_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));  // pure: identical calls fold
    return pol;
}
LAM_DEV uint4 ld_keep(const uint4* p) {
    uint4 v;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(keep_policy()));
    return v;
}
LAM_DEV float4 ld_keep(const float4* p) {
    float4 v;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(keep_policy()));
    return v;
}
template <class T>
LAM_DEV T ld_stream(const T* p) {
    return __ldcs(p);
}

struct v3 {
    float x, y, z;
};
LAM_DEV v3 mk(float x, float y, float z) { return v3{x, y, z}; }
LAM_DEV v3 splat(float a) { return v3{a, a, a}; }
LAM_DEV v3 operator+(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
LAM_DEV v3 operator-(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
LAM_DEV v3 operator-(v3 a) { return mk(-a.x, -a.y, -a.z); }
LAM_DEV v3 operator*(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
LAM_DEV v3 operator*(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
LAM_DEV v3 operator/(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
LAM_DEV float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LAM_DEV v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
LAM_DEV float len(v3 a) { return sqrtf(dot(a, a)); }
LAM_DEV v3 normalize(v3 a) { return a / len(a); }
LAM_DEV v3 fma3(v3 a, v3 b, v3 c) { return mk(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z)); }
LAM_DEV float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
LAM_DEV v3 clamp3(v3 v, float lo, float hi) { return mk(clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi)); }
LAM_DEV float saturate(float x) { return clampf(x, 0.0f, 1.0f); }
LAM_DEV float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
LAM_DEV v3 mix3(v3 a, v3 b, float t) { return a * (1.0f - t) + b * t; }
LAM_DEV v3 reflect(v3 e1, v3 e2) { return e1 - e2 * (2.0f * dot(e2, e1)); }
LAM_DEV v3 refract(v3 e1, v3 e2, float e3) {
    float d = dot(e2, e1);
    float k = 1.0f - e3 * e3 * (1.0f - d * d);
    if (k < 0.0f) return splat(0.0f);
    return e1 * e3 - e2 * (e3 * d + sqrtf(k));
}
LAM_DEV float fractf(float x) { return x - floorf(x); }
LAM_DEV int32_t f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)f;
}
LAM_DEV uint32_t f2u(float f) {
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)f;
}

constexpr float PI_F = 3.14159265358979323846f;
constexpr float HALF_PI_F = 3.14159265358979323846f / 2.0f;
constexpr float TAU_F = 2.0f * 3.14159265358979323846f;
constexpr uint32_t TY_DIFFUSE = 0u, TY_METALLIC = 1u, TY_TRANSPARENT = 2u, TY_SKY = 0xFFu;

LAM_DEV bool near_zero(float f) { return (f < 0.0001f) && (f > -0.0001f); }
LAM_DEV bool v3_near_zero(v3 v) { return near_zero(v.x) && near_zero(v.y) && near_zero(v.z); }

// PCG-style hash, shared.wesl:266-270
LAM_DEV uint32_t rand_u32(uint32_t s) {
    uint32_t state = s * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
// fract(f32(u) * (1 / f32(0xFFFFFFFF))) with f32(0xFFFFFFFF) == 2^32
LAM_DEV float u32_to_unit(uint32_t u) { return fractf(__uint2float_rn(u) * 2.3283064365386963e-10f); }
LAM_DEV float rand_f32(uint32_t s) { return u32_to_unit(rand_u32(s)); }
LAM_DEV float rand_f32_ptr(uint32_t* s) {
    *s = rand_u32(*s);
    return u32_to_unit(*s);
}

LAM_DEV float copy_sign(float src, float dst) {
    float a = fabsf(dst);
    return src < 0.0f ? -a : a;
}
LAM_DEV float safe_div(float n, float d) { return near_zero(d) ? 0.0f : n / d; }
LAM_DEV v3 safe_div3(v3 n, float d) { return near_zero(d) ? splat(0.0f) : n / d; }
LAM_DEV float len_sqrd(v3 v) { return fmaf(v.x, v.x, fmaf(v.y, v.y, v.z * v.z)); }

LAM_DEV float strip_nan(float f) {
    uint32_t b = __float_as_uint(f);
    if ((b & 0x7F800000u) == 0x7F800000u) return (b & 0x007FFFFFu) == 0u ? 10000.0f : 0.0f;
    return f;
}
LAM_DEV v3 strip_nan3(v3 v) { return mk(strip_nan(v.x), strip_nan(v.y), strip_nan(v.z)); }

LAM_DEV uint32_t pack_snorm16(float e) {
    float c = fminf(1.0f, fmaxf(-1.0f, e));
    int32_t v = (int32_t)floorf(0.5f + 32767.0f * c);
    return (uint32_t)(uint16_t)(int16_t)v;
}
LAM_DEV float unpack_snorm16(uint32_t h) { return fmaxf((float)(int16_t)(uint16_t)h / 32767.0f, -1.0f); }
LAM_DEV uint32_t normalised_to_u32(v3 n) {
    v3 v = n / fmaxf(fabsf(n.x) + fabsf(n.y) + fabsf(n.z), 0.01f);
    if (v.y >= 0.0f) return pack_snorm16(v.x) | (pack_snorm16(v.z) << 16);
    float xx = copy_sign(v.x, 1.0f - fabsf(v.z));
    float zz = copy_sign(v.z, 1.0f - fabsf(v.x));
    return pack_snorm16(xx) | (pack_snorm16(zz) << 16);
}
LAM_DEV v3 u32_to_normalised(uint32_t u) {
    v3 v;
    v.x = unpack_snorm16(u & 0xFFFFu);
    v.z = unpack_snorm16(u >> 16);
    v.y = 1.0f - (fabsf(v.x) + fabsf(v.z));
    if (v.y < 0.0f) {
        float x = v.x;
        v.x = copy_sign(x, 1.0f - fabsf(v.z));
        v.z = copy_sign(v.z, 1.0f - fabsf(x));
    }
    return normalize(v);
}

// IEEE binary16 -> f32 (exact), used by unpack2x16float
LAM_DEV float f16_bits_to_f32(uint32_t h) {
    uint32_t sign = (h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    if (exp == 0u) {
        float v = (float)man * 5.9604644775390625e-08f;  // man * 2^-24, exact
        return __uint_as_float(__float_as_uint(v) | sign);
    }
    if (exp == 0x1Fu) return __uint_as_float(sign | 0x7F800000u | (man << 13));
    return __uint_as_float(sign | ((exp + 112u) << 23) | (man << 13));
}
LAM_DEV float2 unpack2x16float(uint32_t u) { return make_float2(f16_bits_to_f32(u & 0xFFFFu), f16_bits_to_f32(u >> 16)); }

}  // namespace lam
