// oracle_math.h - TEST INFRASTRUCTURE ONLY (the CPU oracle).  Nothing in the product
// may include or link this file; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg use the oracle library built from it.
//
// WGSL built-in semantics restated on the CPU in IEEE f32 (compiled with
// -ffp-contract=off so that every a*b+c rounds twice unless fma() is written).
// Follows the reference shader sources (Vecvec/Lambent):
//   src/importance_sampling/shared.wesl (RNG :266-292, copy_sign :255-262, safe_div :294-312,
//   octahedral decode :233-245), src/path_tracing/general.wesl (strip_NaN :117-135,
//   normalised_to_u32 :1293-1305), src/bindings.wesl (near_zero :171-175, unpack_2xu16 :152-156).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace oracle {

// Runs body(i) for i in [0, n) on `threads` std::threads with dynamic chunking.
template <class F>
void parallel_for(long long n, int threads, long long chunk, F body) {
    if (threads <= 1 || n <= chunk) {
        for (long long i = 0; i < n; ++i) body(i, 0);
        return;
    }
    std::atomic<long long> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t]() {
            for (;;) {
                long long b = next.fetch_add(chunk);
                if (b >= n) break;
                long long e = std::min(n, b + chunk);
                for (long long i = b; i < e; ++i) body(i, t);
            }
        });
    }
    for (auto& th : pool) th.join();
}

struct vec2 { float x, y; };
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit vec3(float a) : x(a), y(a), z(a) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline vec3 operator+(vec3 a, vec3 b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(vec3 a, vec3 b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator-(vec3 a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3 operator*(vec3 a, vec3 b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator*(vec3 a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, vec3 a) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(vec3 a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator/(vec3 a, vec3 b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline bool operator!=(vec3 a, vec3 b) { return a.x != b.x || a.y != b.y || a.z != b.z; }

// WGSL dot: plain sum of products, left to right.
inline float dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(vec3 a, vec3 b) {
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(vec3 a) { return std::sqrt(dot(a, a)); }
inline vec3 normalize(vec3 a) { return a / length(a); }
inline vec3 fma3(vec3 a, vec3 b, vec3 c) {
    return vec3(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y), std::fma(a.z, b.z, c.z));
}
// WGSL min/max return the non-NaN operand (IEEE minNum/maxNum as on GPUs).
inline float wmin(float a, float b) { return std::fmin(a, b); }
inline float wmax(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
inline vec3 clamp3(vec3 v, float lo, float hi) {
    return vec3(clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi));
}
inline vec3 max3(vec3 v, float lo) { return vec3(wmax(v.x, lo), wmax(v.y, lo), wmax(v.z, lo)); }
inline float saturate(float x) { return clampf(x, 0.0f, 1.0f); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline vec3 mix3(vec3 a, vec3 b, float t) { return a * (1.0f - t) + b * t; }
inline float fractf(float x) { return x - std::floor(x); }
// WGSL reflect(e1, e2) = e1 - 2 * dot(e2, e1) * e2
inline vec3 reflect(vec3 e1, vec3 e2) { return e1 - e2 * (2.0f * dot(e2, e1)); }
// WGSL refract(e1, e2, e3)
inline vec3 refract(vec3 e1, vec3 e2, float e3) {
    float d = dot(e2, e1);
    float k = 1.0f - e3 * e3 * (1.0f - d * d);
    if (k < 0.0f) return vec3(0.0f);
    return e1 * e3 - e2 * (e3 * d + std::sqrt(k));
}
inline float absf(float x) { return std::fabs(x); }

// f32 -> u32 / i32 conversions: truncate toward zero, saturate, NaN -> 0.
inline uint32_t f2u(float f) {
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)f;
}
inline int32_t f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)f;
}
inline float u2f(uint32_t u) { return (float)u; }  // round to nearest even

inline uint32_t f2bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bits2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ---------------------------------------------------------------- constants (shared.wesl:3-10)
constexpr float PI = 3.14159265358979323846f;
constexpr float HALF_PI = 3.14159265358979323846f / 2.0f;
constexpr float TAU = 2.0f * 3.14159265358979323846f;
constexpr uint32_t DIFFUSE = 0u, METALLIC = 1u, TRANSPARENT = 2u, SKY = 0xFFu;
constexpr float SMALL_VAL = 0.0001f;  // bindings.wesl:171

inline bool near_zero(float f) { return (f < SMALL_VAL) && (f > -SMALL_VAL); }
inline bool vec3_near_zero(vec3 v) { return near_zero(v.x) && near_zero(v.y) && near_zero(v.z); }

// ---------------------------------------------------------------- RNG (shared.wesl:266-292)
inline uint32_t rand_u32(uint32_t s) {
    uint32_t state = s * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
// RECIP_U32_MAX = 1 / f32(U32_MAX) = 1 / 2^32 (f32(0xFFFFFFFF) rounds to 2^32).
constexpr float RECIP_U32_MAX = 2.3283064365386963e-10f;
inline float rand_f32_ptr(uint32_t* s) {
    *s = rand_u32(*s);
    return fractf(u2f(*s) * RECIP_U32_MAX);
}
inline float rand_f32(uint32_t s) { uint32_t t = s; return rand_f32_ptr(&t); }
inline vec3 rand_xz_vec3_f32(uint32_t* s) {
    float a = rand_f32_ptr(s);
    float b = rand_f32_ptr(s);
    return vec3(a, 0.0f, b);
}

// ---------------------------------------------------------------- helpers (shared.wesl)
inline float copy_sign(float src, float dst) {
    float a = absf(dst);
    return src < 0.0f ? -a : a;
}
inline float div_or(float n, float d, float o) { return near_zero(d) ? o : n / d; }
inline float safe_div(float n, float d) { return div_or(n, d, 0.0f); }
inline vec3 safe_div_vec3(vec3 n, float d) { return near_zero(d) ? vec3(0.0f) : n / d; }
inline float len_sqrd(vec3 v) { return std::fma(v.x, v.x, std::fma(v.y, v.y, v.z * v.z)); }

// strip_NaN, general.wesl:117-135
inline float strip_NaN(float f) {
    uint32_t b = f2bits(f);
    if ((b & 0x7F800000u) == 0x7F800000u) {
        if ((b & ~(0x7F800000u | 0x80000000u)) == 0u) return 10000.0f;
        return 0.0f;
    }
    return f;
}
inline vec3 strip_NaN_vec3(vec3 v) { return vec3(strip_NaN(v.x), strip_NaN(v.y), strip_NaN(v.z)); }

// pack2x16snorm / unpack2x16snorm (WGSL)
inline uint32_t pack_snorm16(float e) {
    float c = wmin(1.0f, wmax(-1.0f, e));
    int32_t v = (int32_t)std::floor(0.5f + 32767.0f * c);
    return (uint32_t)(uint16_t)(int16_t)v;
}
inline uint32_t pack2x16snorm(float a, float b) { return pack_snorm16(a) | (pack_snorm16(b) << 16); }
inline float unpack_snorm16(uint32_t h) {
    int16_t v = (int16_t)(uint16_t)h;
    return wmax((float)v / 32767.0f, -1.0f);
}

// normalised_to_u32, general.wesl:1293-1305
inline uint32_t normalised_to_u32(vec3 n) {
    vec3 v = n / wmax(absf(n.x) + absf(n.y) + absf(n.z), 0.01f);
    if (v.y >= 0.0f) return pack2x16snorm(v.x, v.z);
    float xx = copy_sign(v.x, 1.0f - absf(v.z));
    float zz = copy_sign(v.z, 1.0f - absf(v.x));
    return pack2x16snorm(xx, zz);
}
// u32_to_normalised, shared.wesl:233-245
inline vec3 u32_to_normalised(uint32_t u) {
    vec3 v;
    v.x = unpack_snorm16(u & 0xFFFFu);
    v.z = unpack_snorm16(u >> 16);
    v.y = 1.0f - (absf(v.x) + absf(v.z));
    if (v.y < 0.0f) {
        float x = v.x;
        v.x = copy_sign(x, 1.0f - absf(v.z));
        v.z = copy_sign(v.z, 1.0f - absf(x));
    }
    return normalize(v);
}

// ---------------------------------------------------------------- f16 / bf16 (half 2.6.0 semantics)
// IEEE binary16 from f32 with round-to-nearest-even, overflow to inf, subnormals, NaN kept quiet.
inline uint16_t f32_to_f16(float f) {
    uint32_t x = f2bits(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFFu) return (uint16_t)(sign | 0x7C00u | (man ? (0x200u | (man >> 13)) : 0u));
    int32_t e = (int32_t)exp - 127 + 15;
    if (e >= 0x1F) return (uint16_t)(sign | 0x7C00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half_man = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (half_man & 1u))) half_man++;
        return (uint16_t)(sign | half_man);
    }
    uint32_t half_man = man >> 13;
    uint32_t rem = man & 0x1FFFu;
    uint32_t out = sign | ((uint32_t)e << 10) | half_man;
    if (rem > 0x1000u || (rem == 0x1000u && (half_man & 1u))) out++;
    return (uint16_t)out;
}
inline float f16_to_f32(uint16_t h) {
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t exp = ((uint32_t)h >> 10) & 0x1Fu;
    uint32_t man = (uint32_t)h & 0x3FFu;
    uint32_t out;
    if (exp == 0) {
        if (man == 0) {
            out = sign;
        } else {
            int e = -1;
            do { man <<= 1; e++; } while (!(man & 0x400u));
            man &= 0x3FFu;
            out = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 0x1F) {
        out = sign | 0x7F800000u | (man << 13);
    } else {
        out = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    return bits2f(out);
}
// bf16 from f32: round to nearest even; NaN -> quiet NaN.
inline uint16_t f32_to_bf16(float f) {
    uint32_t x = f2bits(f);
    if ((x & 0x7FFFFFFFu) > 0x7F800000u) return (uint16_t)((x >> 16) | 0x0040u);
    uint32_t round_bit = 0x00008000u;
    if ((x & round_bit) && (x & (3u * round_bit - 1u))) return (uint16_t)((x >> 16) + 1u);
    return (uint16_t)(x >> 16);
}
inline vec2 unpack2x16float(uint32_t u) {
    return vec2{f16_to_f32((uint16_t)(u & 0xFFFFu)), f16_to_f32((uint16_t)(u >> 16))};
}
inline void unpack_2xu16(uint32_t u, uint32_t* a, uint32_t* b) { *a = u & 0xFFFFu; *b = (u & 0xFFFF0000u) >> 16u; }

}  // namespace oracle
