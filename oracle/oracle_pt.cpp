// oracle_pt.cpp - TEST INFRASTRUCTURE ONLY (the CPU oracle; see oracle_math.h).
//
// CPU restatement of the reference path tracer (Vecvec/Lambent):
//   rt_main              src/path_tracing/general.wesl:506-610
//   rt_sample            general.wesl:643-975
//   ray_hit              general.wesl:1052-1137 (+ correct_tangent :1139-1156)
//   create_ray / at      general.wesl:1158-1178
//   BSDF helpers         general.wesl:1206-1289, shared.wesl:39-46, 215-231
//   quality variants     src/path_tracing/{low,medium,high}.wesl
//   Markov-chain guiding general.wesl:147-500, 984-1047
//   reservoir ops        src/importance_sampling/shared.wesl:63-168
//   temporal / spatial   src/importance_sampling/temporal_resampling.wesl:37-65,
//                        spatial_resampling.wesl:35-194
//   end of frame         src/data_buffer/end_of_frame.wesl:14-99
//   average              examples/cornell_box/src/average_to_buf.wgsl:11-21
// Subgroup semantics: a subgroup is 32 consecutive pixels of a row (workgroups of 64x1); all
// lanes fill their screen-space candidates before any lane traces (lock-step), and the chain
// shuffle after each sample moves lane (l + 1) % 32's chain into lane l.  Lanes past the
// image edge are inactive and contribute zero chains.  World-grid updates use relaxed atomics
// in the same protocol as the shader; with one thread the order is sequential and deterministic.
#include "oracle_pt.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace oracle {
namespace {

struct vec4 { float x, y, z, w; };

struct MC {
    vec3 light_source;
    float mean_cosine = 0.0f, weight_sum = 0.0f;
    uint32_t num_samples = 0;
    float score = 0.0f;
};

constexpr int NUM_RESAMPLES_SCREEN_SPACE = 4;
constexpr int NUM_RESAMPLES_SCREEN_SPACE_LAST_FRAME = 12;
constexpr int NUM_NON_PIXEL_RESAMPLES = 20;
constexpr int NUM_RESAMPLES = 21;
constexpr uint32_t RESAMPLE_SIZE = 91;
constexpr int32_t RESAMPLE_SIZE_SHIFT = 45;
constexpr float GRID_SIZE = 0.1f;
constexpr float SIZE_PER_GRID_CHANGE = 1.0f;
constexpr uint32_t CACHE_TIMEOUT = 30u;
constexpr uint32_t MAX_NUM_SAMPLES = 0x0FFFFFFFu;
constexpr uint32_t MARCOV_CHAIN_SAMPLE_CLAMP = 1024u;
constexpr float JITTER_SIZE = GRID_SIZE * 1.5f;
constexpr uint32_t SUBGROUP = 32u;

enum { W_SEC = 0, W_NUM = 1, W_LUM = 2, W_LOCK = 5, W_CL = 6, W_CMEAN = 9, W_CWS = 10, W_CNUM = 11,
       W_CSCORE = 12, W_TIMEOUT = 13, W_STRIDE = 14 };

inline uint32_t aload(const uint32_t* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void astore(uint32_t* p, uint32_t v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }

struct Ray { vec3 direction, origin; };

struct Intersection {
    vec3 color;
    float t = 0.0f;
    vec3 emission;
    uint32_t ty = 0;
    vec3 normal;
    bool front_face = false;
    vec3 tangent;
    bool hit = false;
    vec2 roughness{0.0f, 0.0f};
    vec2 roughness_transparent{0.0f, 0.0f};
    float refractive_index_low = 0.0f, refractive_index_high = 0.0f;
};

struct SampleReturn {
    vec3 color, normal, albedo, point, emission, visible_point, visible_normal, out_radiance;
    uint32_t ty = 0;
    float roughness = 0.0f;
    bool valid = false;
    float pdf = 0.0f;
};

struct Picked { float picked_idx = 0.0f; bool picked = false; };

struct Sample {
    vec3 visible_point;
    uint32_t visible_normal = 0;
    vec3 sample_point;
    uint32_t sample_normal = 0;
    vec3 out_radiance;
    uint32_t ty = 0;
    float roughness = 0.0f;
};

struct Lane {
    MC tentative;
    MC cand[NUM_RESAMPLES];
    float sum_mc = 0.0f;
    vec3 camera_loc;
};

// ---------------------------------------------------------------- reservoirs (shared.wesl:63-168)
constexpr uint32_t MAX_CONFIDANCE = 0x7FFFFFFFu;
inline uint32_t conf_of(uint32_t p) { return p & MAX_CONFIDANCE; }
inline uint32_t valid_of(uint32_t p) { return (p & ~MAX_CONFIDANCE) >> 31; }
inline uint32_t pack_conf(uint32_t c, uint32_t v) { return (c & MAX_CONFIDANCE) | (v << 31); }

inline vec3 v3(const float* a) { return vec3(a[0], a[1], a[2]); }
inline void st3(float* a, vec3 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }

inline Sample sam_from_res(const lam_reservoir& r) {
    Sample s;
    s.visible_point = v3(r.visible_point);
    s.visible_normal = r.visible_normal;
    s.sample_point = v3(r.sample_point);
    s.sample_normal = r.sample_normal;
    s.out_radiance = v3(r.out_radiance);
    s.ty = r.ty;
    s.roughness = r.roughness;
    return s;
}
inline void assign_sam_to_res(lam_reservoir* r, const Sample& s) {
    st3(r->visible_point, s.visible_point);
    r->visible_normal = s.visible_normal;
    st3(r->sample_point, s.sample_point);
    r->sample_normal = s.sample_normal;
    st3(r->out_radiance, s.out_radiance);
    r->ty = s.ty;
    r->roughness = s.roughness;
    r->packed_confidence_valid = pack_conf(conf_of(r->packed_confidence_valid), 1u);
}
inline float p_hat(const Sample& s) { return wmax(length(s.out_radiance), 0.00001f); }
inline lam_reservoir update(const Sample& s_new, float w_new, lam_reservoir r, uint32_t seed) {
    r.w = r.w + w_new;
    r.packed_confidence_valid = pack_conf(conf_of(r.packed_confidence_valid) + 1u, valid_of(r.packed_confidence_valid));
    if (rand_f32(seed) * r.w < w_new) assign_sam_to_res(&r, s_new);
    return r;
}
inline lam_reservoir merge(lam_reservoir res, const lam_reservoir& r, float p, uint32_t seed, bool* picked) {
    uint32_t c = conf_of(res.packed_confidence_valid);
    uint32_t v = valid_of(res.packed_confidence_valid);
    uint32_t oc = conf_of(r.packed_confidence_valid);
    float w_new = p * r.W * u2f(oc);
    res.packed_confidence_valid = pack_conf(c + oc, v);
    res.w = res.w + w_new;
    *picked = false;
    if (rand_f32(seed) * res.w < w_new) {
        assign_sam_to_res(&res, sam_from_res(r));
        *picked = true;
    }
    return res;
}

// ---------------------------------------------------------------- geometry helpers
inline vec3 at(const Ray& r, float t) { return fma3(r.direction, vec3(t), r.origin); }

inline vec3 to_onb(vec3 src, vec3 up, vec3 tangent) {
    vec3 s = tangent;
    vec3 t = cross(up, s);
    vec3 inv_s = cross(up, t);
    vec3 inv_up = cross(t, s);
    vec3 inv_t = cross(s, up);
    return fma3(vec3(src.x), inv_s, fma3(vec3(src.y), inv_up, inv_t * src.z));
}
inline vec3 from_onb(vec3 src, vec3 up, vec3 tangent) {
    vec3 s = tangent;
    vec3 t = cross(up, s);
    return fma3(vec3(src.x), s, fma3(vec3(src.y), up, t * src.z));
}
inline vec3 from_onb_no_tangent(vec3 src, vec3 up) {
    vec3 other = near_zero(up.x) ? vec3(1.0f, 0.0f, 0.0f) : vec3(0.0f, 1.0f, 0.0f);
    vec3 tangent = normalize(cross(up, other));
    return from_onb(src, up, tangent);
}
inline vec3 onb_cosine_weighted_hemisphere(uint32_t seed) {
    float r1 = rand_f32(seed);
    float r2 = rand_f32(seed + 1u);
    float phi = TAU * r1;
    float x = std::cos(phi) * std::sqrt(r2);
    float z = std::sin(phi) * std::sqrt(r2);
    float y = std::sqrt(1.0f - r2);
    return vec3(x, y, z);
}
inline vec3 cosine_weighted_hemisphere(uint32_t seed, vec3 normal, vec3 tangent) {
    return from_onb(onb_cosine_weighted_hemisphere(seed), normal, tangent);
}
inline vec3 sample_ggx_interal(float u1, float u2, vec3 wi) {
    float phi = TAU * u1;
    float y = std::fma(1.0f - u2, 1.0f + wi.y, -wi.y);
    float sin_theta = std::sqrt(clampf(std::fma(y, -y, 1.0f), 0.0f, 1.0f));
    float x = sin_theta * std::cos(phi);
    float z = sin_theta * std::sin(phi);
    return vec3(x, y, z) + wi;
}
inline vec3 sample_vndf_ggx(uint32_t seed, vec3 view, vec2 rough) {
    float u1 = rand_f32(seed);
    float u2 = rand_f32(seed + 1u);
    vec3 in(view.x * rough.x, view.y, view.z * rough.y);
    if (vec3_near_zero(in)) in = vec3(0.0f, -1.0f, 0.0f);
    vec3 warped = normalize(in);
    vec3 wm_std = sample_ggx_interal(u1, u2, warped);
    vec3 out(wm_std.x * rough.x, wm_std.y, wm_std.z * rough.y);
    if (vec3_near_zero(out)) out = vec3(0.0f, 1.0f, 0.0f);
    return normalize(out);
}
inline float reflectance(float cosine, float ref_idx) {
    float r0 = (1.0f - ref_idx) / (1.0f + ref_idx);
    float r0s = r0 * r0;
    return std::fma(1.0f - r0s, std::pow(1.0f - cosine, 5.0f), r0s);
}
inline vec3 oren_nayar_improved(vec3 incoming, vec3 reflected, float roughness, vec3 color) {
    float rr = roughness * HALF_PI;
    float rr2 = rr * rr;
    vec3 a = fma3(color * 0.17f, vec3(rr2 / (rr2 + 0.13f)), vec3(1.0f - (0.5f * (rr2 / (rr2 + 0.33f)))));
    float b = 0.45f * (rr2 / (rr2 + 0.09f));
    float s = std::fma(-reflected.y, incoming.y, dot(reflected, incoming));
    float t = 1.0f;
    if (s > 0.0f) {
        t = wmax(reflected.y, incoming.y);
        if (near_zero(t)) t = 0.001f;
    }
    return fma3(vec3(b), vec3(s / t), a);
}
inline vec3 correct_tangent(vec3 tangent) {
    vec3 dir = tangent;
    vec3 a(absf(dir.x), absf(dir.y), absf(dir.z));
    bool x_largest = a.x > a.y && a.x > a.z;
    bool y_largest = a.y > a.x && a.y > a.z;
    bool reverse_dir;
    if (x_largest) reverse_dir = dir.x < 0.0f;
    else if (y_largest) reverse_dir = dir.y < 0.0f;
    else reverse_dir = dir.z < 0.0f;
    if (reverse_dir) dir = -dir;
    return dir;
}

// ---------------------------------------------------------------- vMF (general.wesl:1000-1047)
inline float exp_minus_one(float x) {
    float u = std::exp(x);
    if (u == 1.0f) return x;
    float y = u - 1.0f;
    if (absf(x) < 1.0f) return (x * y) / std::log(u);
    return y;
}
inline float x_divided_by_exp_minus_one(float x) {
    float u = std::exp(x);
    if (u == 1.0f) return 1.0f;
    float y = u - 1.0f;
    if (absf(x) < 1.0f) return std::log(u) / y;
    return x / y;
}
inline bool marcov_chain_valid(const MC& s) { return s.weight_sum > 0.0f; }
inline vec3 get_light_dir(const MC& s, vec3 current) { return safe_div_vec3(s.light_source, s.weight_sum) - current; }
inline float get_kappa(const MC& s) {
    const float Np = 0.2f, rp = 0.99f;
    uint32_t N = s.num_samples;
    float N_sqrd = u2f(N * N);
    float r = ((N_sqrd * (s.mean_cosine / s.weight_sum)) + (Np * rp)) / (N_sqrd + Np);
    return clampf(((3.0f * r) - ((r * r) * r)) / (1.0f - (r * r)), 0.001f, 8.50705867e37f);
}
inline float vmf_pdf(vec3 mean, float kappa, vec3 direction) {
    float minus_2_kappa = -2.0f * kappa;
    float fraction = x_divided_by_exp_minus_one(minus_2_kappa) / (4.0f * PI);
    float cos_theta = dot(direction, mean);
    return wmax(fraction * std::exp(kappa * (cos_theta - 1.0f)), 0.0f);
}

// ---------------------------------------------------------------- High spectral weight (high.wesl:19-59)
inline float g_lobe(float x, float u, float t1, float t2) {
    float tau = x < u ? t1 : t2;
    float d = x - u;
    float d2 = d * d;
    float tau2 = tau * tau;
    return std::exp(-(d2 * tau2) * 0.5f);
}

// ---------------------------------------------------------------- the tracer
struct PT {
    const Scene& sc;
    const RenderParams& p;
    bool guide;
    uint64_t segments = 0;
    uint64_t pixels = 0;

    // pdf_at_sample: LAM_GUIDE_PDF_AT_SAMPLE, the cosine term of the mixture pdf evaluated at the
    // chosen direction instead of at the cosine branch's draw (general.wesl:793, 840)
    bool pdf_at_sample;
    PT(const Scene& s, const RenderParams& pr)
        : sc(s), p(pr), guide((pr.guide & LAM_GUIDE_MARKOV) != 0u),
          pdf_at_sample((pr.guide & LAM_GUIDE_PDF_AT_SAMPLE) != 0u) {}

    // ----- quality hooks
    vec3 get_normal(vec3 ray_dir, vec3 normal, vec3 tangent, uint32_t seed, vec2 rough) const {
        if (p.quality == LAM_QUALITY_LOW) return normal;
        vec3 ray_onb = to_onb(ray_dir, normal, tangent);
        vec3 n_onb = sample_vndf_ggx(seed, ray_onb, rough);
        return from_onb(n_onb, normal, tangent);
    }
    vec3 make_diffuse(vec3 hit_color, const Ray& ray, vec3 n, vec3 t, float rough, vec3 new_dir) const {
        if (p.quality == LAM_QUALITY_LOW) return vec3(1.0f);
        vec3 ray_onb = to_onb(ray.direction, n, t);
        return oren_nayar_improved(ray_onb, new_dir, rough, hit_color);
    }
    float conv_rough(float r) const { return p.quality == LAM_QUALITY_LOW ? 0.0f : r; }
    vec4 pick_ref_idx(Picked* picked, float low, float high, uint32_t seed) const {
        if (p.quality == LAM_QUALITY_LOW) return vec4{1.0f, 1.0f, 1.0f, low};
        if (p.quality == LAM_QUALITY_MEDIUM) {
            if (!picked->picked) { picked->picked_idx = rand_f32(seed); picked->picked = true; }
            return vec4{1.0f, 1.0f, 1.0f, mixf(low, high, picked->picked_idx)};
        }
        if (!picked->picked) {
            float pi = rand_f32(seed);
            picked->picked_idx = pi;
            picked->picked = true;
            float lambda = mixf(760.0f, 340.0f, pi);
            float x = std::fma(1.056f, g_lobe(lambda, 599.8f, 0.0264f, 0.0323f),
                               std::fma(0.362f, g_lobe(lambda, 442.0f, 0.0624f, 0.0374f),
                                        -(0.065f * g_lobe(lambda, 501.1f, 0.049f, 0.0382f))));
            float y = std::fma(0.821f, g_lobe(lambda, 568.8f, 0.0213f, 0.0248f), 0.286f * g_lobe(lambda, 530.9f, 0.0613f, 0.0322f));
            float z = std::fma(1.217f, g_lobe(lambda, 437.0f, 0.0845f, 0.0278f), 0.681f * g_lobe(lambda, 459.0f, 0.0385f, 0.0725f));
            vec3 rgb = vec3(3.2406f, -0.9689f, 0.0557f) * x + vec3(-1.5372f, 1.8758f, -0.204f) * y +
                       vec3(-0.4986f, 0.0415f, 1.057f) * z;
            vec3 w = vec3(saturate(rgb.x), saturate(rgb.y), saturate(rgb.z)) * vec3(3.910f, 4.411f, 5.511f);
            return vec4{w.x, w.y, w.z, mixf(low, high, pi)};
        }
        return vec4{1.0f, 1.0f, 1.0f, mixf(low, high, picked->picked_idx)};
    }

    // ----- camera (general.wesl:1158-1173)
    Ray create_ray(uint32_t x, uint32_t y) const {
        float hx = u2f(p.width) / 2.0f, hy = u2f(p.height) / 2.0f;
        float nx = (u2f(x) / hx) - 1.0f, ny = (u2f(y) / hy) - 1.0f;
        float v[4] = {nx, -ny, 1.0f, 1.0f};
        const float* P = p.camera.projection_inverse;
        float q[4];
        for (int i = 0; i < 4; ++i) q[i] = P[0 * 4 + i] * v[0] + P[1 * 4 + i] * v[1] + P[2 * 4 + i] * v[2] + P[3 * 4 + i] * v[3];
        float l = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        for (int i = 0; i < 4; ++i) q[i] = q[i] / l;
        const float* V = p.camera.view_inverse;
        vec3 dir(V[0] * q[0] + V[4] * q[1] + V[8] * q[2] + V[12] * 0.0f,
                 V[1] * q[0] + V[5] * q[1] + V[9] * q[2] + V[13] * 0.0f,
                 V[2] * q[0] + V[6] * q[1] + V[10] * q[2] + V[14] * 0.0f);
        vec3 pos(V[0] * 0.0f + V[4] * 0.0f + V[8] * 0.0f + V[12] * 1.0f,
                 V[1] * 0.0f + V[5] * 0.0f + V[9] * 0.0f + V[13] * 1.0f,
                 V[2] * 0.0f + V[6] * 0.0f + V[10] * 0.0f + V[14] * 1.0f);
        Ray r;
        r.direction = dir;
        r.origin = pos;
        return r;
    }

    // ----- ray_hit (general.wesl:1052-1137)
    const lam_material& material_of(uint32_t inst, uint32_t prim) const {
        static const lam_material zero{};
        if (sc.materials.empty()) return zero;
        const Instance& in = sc.inst[inst];
        uint32_t mi = in.mat.empty() ? 0u : in.mat[std::min<size_t>(prim, in.mat.size() - 1)];
        return sc.materials[std::min<size_t>(mi, sc.materials.size() - 1)];
    }
    Intersection ray_hit(const Ray& ray) {
        segments++;
        Hit h = sc.trace(ray.origin, ray.direction, p.tmin, p.tmax, false);
        Intersection r;
        if (!h.hit) return r;
        r.hit = true;
        r.t = h.t;
        r.front_face = h.front;
        const lam_material& m = material_of(h.inst, h.prim);
        uint32_t idx_d, idx_e, idx_a, ty;
        unpack_2xu16(m.tex_idx_diffuse_emission, &idx_d, &idx_e);
        unpack_2xu16(m.tex_idx_attributes_ty, &idx_a, &ty);
        r.ty = ty;
        vec2 ri = unpack2x16float(m.refractive_index);
        r.refractive_index_low = ri.x;
        r.refractive_index_high = ri.y;
        vec3 tangent = correct_tangent(normalize(h.ov0 - h.ov1));
        vec3 normal = normalize(cross(tangent, h.ov0 - h.ov2));
        r.normal = dot(ray.direction, normal) > 0.0f ? -normal : normal;
        r.tangent = tangent;
        float bx = h.u, by = h.v, bz = (1.0f - h.u) - h.v;
        vec2 t1 = unpack2x16float(m.tex_pos_1), t2 = unpack2x16float(m.tex_pos_2), t3 = unpack2x16float(m.tex_pos_3);
        float tu = std::fma(t1.x, bz, std::fma(t2.x, bx, t3.x * by));
        float tv = std::fma(t1.y, bz, std::fma(t2.y, bx, t3.y * by));
        float d4[4], rc[4];
        sc.sample(sc.diffuse, idx_d, tu, tv, d4);
        uint32_t rx, ry;
        unpack_2xu16(m.tex_pos_recolour, &rx, &ry);
        sc.load_recolour(rx, ry, rc);
        vec3 diffuse_colour = vec3(d4[0], d4[1], d4[2]) * vec3(rc[0], rc[1], rc[2]);
        r.color = diffuse_colour;
        float es_x = bits2f((m.emission_scale & 0xFFFFu) << 16);
        float es_y = bits2f(((m.emission_scale & 0xFFFF0000u) >> 16) << 16);
        if (idx_e != 0xFFFFu) {
            float e4[4];
            sc.sample(sc.emission, idx_e, tu, tv, e4);
            r.emission = vec3(e4[0], e4[1], e4[2]) * es_x;
        }
        r.emission = r.emission + diffuse_colour * es_y;
        if (idx_a != 0xFFFFu) {
            float a4[4];
            sc.sample(sc.attributes, idx_a, tu, tv, a4);
            r.roughness = vec2{a4[0], a4[1]};
            r.roughness_transparent = vec2{a4[2], a4[3]};
        }
        return r;
    }

    // ----- world grid (general.wesl:147-311)
    struct ivec3 { int32_t x, y, z; };
    ivec3 grid_loc(vec3 pos, vec3 camera_loc) const {
        vec3 diff = pos - camera_loc;
        diff = vec3(absf(diff.x), absf(diff.y), absf(diff.z));
        float len = wmax(diff.x, wmax(diff.y, diff.z));
        uint32_t num_shifts = f2u(std::log2(wmax(len / SIZE_PER_GRID_CHANGE, 1.0f)));
        uint32_t mask = 0xFFFFFFFFu << std::min(num_shifts, 30u);
        ivec3 g{f2i(pos.x / GRID_SIZE), f2i(pos.y / GRID_SIZE), f2i(pos.z / GRID_SIZE)};
        g.x &= (int32_t)mask; g.y &= (int32_t)mask; g.z &= (int32_t)mask;
        return g;
    }
    static uint32_t incoming_hash(vec3 v) {
        return (uint32_t)(v.x > 0.0f) | ((uint32_t)(v.y > 0.0f) << 1) | ((uint32_t)(v.z > 0.0f) << 2);
    }
    static uint32_t primary_hasher(ivec3 loc, vec3 normal, vec3 incoming) {
        uint32_t n = normalised_to_u32(normal) & 0xFF00FF00u;
        uint32_t inc = rand_u32(incoming_hash(incoming));
        uint32_t hx = 1u * (uint32_t)loc.x, hy = 687603047u * (uint32_t)loc.y, hz = 571899763u * (uint32_t)loc.z,
                 hw = 894271171u * n;
        return (((hx ^ hy) ^ hz) ^ hw) ^ (inc * 840057787u);
    }
    static uint32_t secondary_hasher(ivec3 loc, vec3 normal) {
        uint32_t n = normalised_to_u32(normal) & 0xFF00FF00u;
        uint32_t hx = 1699644091u * (uint32_t)loc.x, hy = 550105817u * (uint32_t)loc.y,
                 hz = 956114303u * (uint32_t)loc.z, hw = 155096983u * n;
        return ((rand_u32((hx ^ hy) ^ hz) ^ hw) ^ (0u * 284005801u)) | 1u;
    }
    uint32_t* wentry(uint64_t idx) const { return p.world + idx * W_STRIDE; }
    const uint32_t* oentry(uint64_t idx) const { return p.old_world ? p.old_world + idx * W_STRIDE : nullptr; }
    static MC read_chain(const uint32_t* e) {
        MC s;
        s.light_source = vec3(bits2f(aload(e + W_CL)), bits2f(aload(e + W_CL + 1)), bits2f(aload(e + W_CL + 2)));
        s.mean_cosine = bits2f(aload(e + W_CMEAN));
        s.weight_sum = bits2f(aload(e + W_CWS));
        s.num_samples = aload(e + W_CNUM);
        s.score = bits2f(aload(e + W_CSCORE));
        return s;
    }
    MC grid_load(const Lane& L, vec3 pos, vec3 normal, vec3 incoming, bool force_old) const {
        if (!guide || !p.world || !p.world_len) return MC();
        ivec3 g = grid_loc(pos, L.camera_loc);
        uint64_t idx = primary_hasher(g, normal, incoming) % p.world_len;
        uint32_t* e = wentry(idx);
        uint32_t sec = secondary_hasher(g, normal);
        MC s = read_chain(e);
        if (aload(e + W_SEC) != sec || force_old) {
            const uint32_t* o = oentry(idx);
            if (o && aload(o + W_SEC) == sec) s = read_chain(o);
            else s = MC();
        } else {
            astore(e + W_TIMEOUT, CACHE_TIMEOUT);
        }
        s.light_source = strip_NaN_vec3(s.light_source);
        s.mean_cosine = strip_NaN(s.mean_cosine);
        s.weight_sum = strip_NaN(s.weight_sum);
        s.score = strip_NaN(s.score);
        return s;
    }
    void grid_store_markov_chain(const Lane& L, vec3 pos, vec3 normal, vec3 incoming, const MC& st) const {
        if (!guide || !p.world || !p.world_len) return;
        ivec3 g = grid_loc(pos, L.camera_loc);
        uint64_t idx = primary_hasher(g, normal, incoming) % p.world_len;
        uint32_t* e = wentry(idx);
        uint32_t sec = secondary_hasher(g, normal);
        if (aload(e + W_SEC) != sec) {
            uint32_t expected = 0u;
            if (!__atomic_compare_exchange_n(e + W_SEC, &expected, sec, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
        }
        astore(e + W_CL, f2bits(st.light_source.x));
        astore(e + W_CL + 1, f2bits(st.light_source.y));
        astore(e + W_CL + 2, f2bits(st.light_source.z));
        astore(e + W_CMEAN, f2bits(st.mean_cosine));
        astore(e + W_CWS, f2bits(st.weight_sum));
        astore(e + W_CNUM, st.num_samples);
        astore(e + W_CSCORE, f2bits(st.score));
        astore(e + W_TIMEOUT, CACHE_TIMEOUT);
    }
    vec3 grid_load_radiance_estimate(const Lane& L, vec3 pos, vec3 normal, vec3 incoming) const {
        if (!guide || !p.world || !p.world_len) return vec3(0.0f);
        ivec3 g = grid_loc(pos, L.camera_loc);
        uint64_t idx = primary_hasher(g, normal, incoming) % p.world_len;
        uint32_t* e = wentry(idx);
        uint32_t num = aload(e + W_NUM);
        vec3 rad(bits2f(aload(e + W_LUM)), bits2f(aload(e + W_LUM + 1)), bits2f(aload(e + W_LUM + 2)));
        uint32_t sec = secondary_hasher(g, normal);
        if (aload(e + W_SEC) != sec) {
            const uint32_t* o = oentry(idx);
            if (o && aload(o + W_SEC) == sec) {
                num = aload(o + W_NUM);
                rad = vec3(bits2f(aload(o + W_LUM)), bits2f(aload(o + W_LUM + 1)), bits2f(aload(o + W_LUM + 2)));
            } else {
                return vec3(0.0f);
            }
        } else {
            astore(e + W_TIMEOUT, CACHE_TIMEOUT);
        }
        if (num == 0u) return vec3(0.0f);
        vec3 radiance = rad / u2f(num);
        return clamp3(radiance, 0.0f, 1000.0f);
    }
    void grid_add_radiance(const Lane& L, vec3 pos, vec3 normal, vec3 incoming, vec3 radiance) const {
        if (!guide || !p.world || !p.world_len) return;
        ivec3 g = grid_loc(pos, L.camera_loc);
        uint64_t idx = primary_hasher(g, normal, incoming) % p.world_len;
        uint32_t* e = wentry(idx);
        uint32_t sec = secondary_hasher(g, normal);
        vec3 c = clamp3(radiance, 0.0f, 100.0f);
        if (aload(e + W_SEC) != sec) {
            uint32_t expected = 0u;
            if (!__atomic_compare_exchange_n(e + W_SEC, &expected, sec, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
        }
        uint32_t locked = __atomic_exchange_n(e + W_LOCK, 1u, __ATOMIC_ACQUIRE);
        if (locked == 1u) return;
        uint32_t num = aload(e + W_NUM);
        if (num >= MAX_NUM_SAMPLES) {
            __atomic_store_n(e + W_LOCK, 0u, __ATOMIC_RELEASE);
            astore(e + W_TIMEOUT, CACHE_TIMEOUT);
            return;
        }
        __atomic_fetch_add(e + W_NUM, 1u, __ATOMIC_RELAXED);
        float cc[3] = {c.x, c.y, c.z};
        for (int k = 0; k < 3; ++k) {
            float r = strip_NaN(cc[k] + bits2f(aload(e + W_LUM + k)));
            astore(e + W_LUM + k, f2bits(wmax(r, 0.0f)));
        }
        __atomic_store_n(e + W_LOCK, 0u, __ATOMIC_RELEASE);
        astore(e + W_TIMEOUT, CACHE_TIMEOUT);
    }

    // ----- chain update (general.wesl:464-492)
    MC update_marcov_state(const Lane& L, vec3 x1, vec3 x2, float p_hat_v, uint32_t seed, bool not_vmf, MC state,
                           float confidence) const {
        if (not_vmf) state = MC();
        float score = p_hat_v;
        float rnd = rand_f32(seed);
        if ((rnd * L.sum_mc) < (p_hat_v * (float)NUM_RESAMPLES)) {
            if (near_zero(length(get_light_dir(state, x1)))) return state;
            state.num_samples = std::min(state.num_samples + 1u, MARCOV_CHAIN_SAMPLE_CLAMP);
            float alpha = state.num_samples == 1u ? 1.0f : wmax(1.0f / u2f(state.num_samples), 0.01f) * confidence;
            state.weight_sum = mixf(state.weight_sum, score, alpha);
            state.light_source = mix3(state.light_source, x2 * score, alpha);
            vec3 mean = normalize(get_light_dir(state, x1));
            state.mean_cosine = mixf(state.mean_cosine, score * dot(normalize(x2 - x1), mean), alpha);
        }
        return state;
    }

    // ----- candidate sets (general.wesl:367-425)
    void fill_mc_screen_space_states(Lane& L, uint32_t* own_seed, const MC* snapshot, const bool* lane_active,
                                     uint32_t px, uint32_t py) const {
        int i = 0;
        for (; i < NUM_RESAMPLES_SCREEN_SPACE; ++i) {
            uint32_t sub_id = rand_u32(*own_seed) % SUBGROUP;
            L.cand[i] = (guide && lane_active[sub_id]) ? snapshot[sub_id] : MC();
        }
        for (; i < NUM_RESAMPLES_SCREEN_SPACE_LAST_FRAME + NUM_RESAMPLES_SCREEN_SPACE; ++i) {
            uint32_t x_rand = rand_u32(*own_seed);
            *own_seed = x_rand;
            uint32_t y_rand = rand_u32(*own_seed);
            *own_seed = y_rand;
            int32_t x = (int32_t)(x_rand % RESAMPLE_SIZE) - RESAMPLE_SIZE_SHIFT;
            int32_t y = (int32_t)(y_rand % RESAMPLE_SIZE) - RESAMPLE_SIZE_SHIFT;
            uint32_t nx = (uint32_t)((int32_t)px + x), ny = (uint32_t)((int32_t)py + y);
            uint64_t idx = (uint32_t)(nx + ny * p.width);
            if (guide && p.old_chains && p.old_chains_len) {
                idx = std::min<uint64_t>(idx, p.old_chains_len - 1);
                const lam_markov_chain& c = p.old_chains[idx];
                MC s;
                s.light_source = vec3(c.light_source[0], c.light_source[1], c.light_source[2]);
                s.mean_cosine = c.mean_cosine;
                s.weight_sum = c.weight_sum;
                s.num_samples = c.num_samples;
                s.score = c.score;
                L.cand[i] = s;
            } else {
                L.cand[i] = MC();
            }
        }
    }
    void fill_mc_world_space_states(Lane& L, uint32_t* own_seed, vec3 pos, vec3 normal, vec3 incoming) const {
        for (int i = NUM_RESAMPLES_SCREEN_SPACE + NUM_RESAMPLES_SCREEN_SPACE_LAST_FRAME; i < NUM_NON_PIXEL_RESAMPLES; ++i) {
            bool rand_candidate = rand_f32(*own_seed) < 0.7f;
            float jitter_mul = rand_candidate ? 0.75f : 1.0f;
            vec3 jitter = (rand_xz_vec3_f32(own_seed) * JITTER_SIZE) * jitter_mul;
            L.cand[i] = guide ? grid_load(L, pos + from_onb_no_tangent(jitter, normal), normal, incoming, rand_candidate) : MC();
            *own_seed += 1u;
        }
        L.cand[NUM_NON_PIXEL_RESAMPLES] = L.tentative;
    }
    MC resample_mcmm(Lane& L, uint32_t* own_seed) const {
        MC s;
        L.sum_mc = 0.0f;
        for (int i = 0; i < NUM_RESAMPLES; ++i) {
            *own_seed = rand_u32(*own_seed);
            const MC& c = L.cand[i];
            L.sum_mc += c.weight_sum;
            float weight = c.weight_sum;
            float rnd = rand_f32(*own_seed);
            if (rnd * L.sum_mc < weight) s = c;
            *own_seed = rand_u32(*own_seed);
        }
        return s;
    }
    float all_vmf_pdfs(const Lane& L, vec3 hit, vec3 direction) const {
        float pdfs = 0.0f;
        if (L.sum_mc > 0.0f) {
            for (int i = 0; i < NUM_RESAMPLES; ++i) {
                const MC& s = L.cand[i];
                if (!marcov_chain_valid(s)) continue;
                pdfs += vmf_pdf(normalize(get_light_dir(s, hit)), get_kappa(s), direction) * (s.weight_sum / L.sum_mc);
            }
        }
        return pdfs;
    }

    // ----- one path (general.wesl:643-975)
    SampleReturn rt_sample(Lane& L, uint32_t px, uint32_t py, uint32_t own_seed) {
        uint32_t self_seed = own_seed;
        Ray ray = create_ray(px, py);
        vec3 color(1.0f), out_radiance_colour(1.0f);
        SampleReturn sample;
        sample.ty = SKY;
        L.camera_loc = ray.origin;
        sample.pdf = 1.0f;
        vec3 accum_emission(0.0f), accum_albedo(1.0f);
        Picked picked;
        vec3 last_normal, last_dir;
        float cached_pdf = 0.0f, cached_brdf = 0.0f;
        bool last_not_vmf = false;
        float vmf_weight = 1.0f;
        vec3 start_dir = ray.direction;
        for (uint32_t i = 0; i < p.max_depth; ++i) {
            Intersection is = ray_hit(ray);
            if (is.hit) {
                vec3 new_pos = at(ray, is.t);
                if (i != 0u) {
                    vec3 radiance_reflected = strip_NaN_vec3(
                        ((is.color * grid_load_radiance_estimate(L, new_pos, is.normal, ray.direction)) * cached_brdf) / cached_pdf);
                    vec3 radiance_out = (is.emission * cached_brdf) / cached_pdf;
                    grid_add_radiance(L, ray.origin, last_normal, last_dir, radiance_out + radiance_reflected);
                    float weight = length(radiance_out + radiance_reflected);
                    if (weight > 0.0f) {
                        if (guide) {
                            MC st = update_marcov_state(L, ray.origin, new_pos, weight, self_seed, false,
                                                        grid_load(L, ray.origin, last_normal, last_dir, false), 1.0f);
                            grid_store_markov_chain(L, ray.origin, last_normal, last_dir, st);
                            L.tentative = update_marcov_state(L, ray.origin, new_pos, length(radiance_out), self_seed,
                                                              last_not_vmf, L.tentative, i == 1u ? 1.0f : 0.5f);
                        }
                        self_seed++;
                    }
                }
                last_normal = is.normal;
                last_dir = ray.direction;
                last_not_vmf = false;
                ray.origin = new_pos;
                accum_emission = fma3(is.emission, accum_albedo, accum_emission);
                accum_albedo = accum_albedo * is.color;
                if (i == 0u) {
                    sample.point = ray.origin;
                    sample.emission = accum_emission;
                    sample.ty = is.ty;
                    sample.normal = is.normal;
                    sample.albedo = accum_albedo;
                } else if (i == 1u) {
                    sample.visible_point = ray.origin;
                    sample.visible_normal = is.normal;
                }
                sample.color = fma3(color, is.emission, sample.color);
                if (i != 0u) sample.out_radiance = fma3(out_radiance_colour, is.emission, sample.out_radiance);
                vec3 assign_normal = get_normal(ray.direction, is.normal, is.tangent, self_seed, is.roughness);
                vec3 transparent_normal = get_normal(ray.direction, is.normal, is.tangent, self_seed, is.roughness_transparent);
                vec3 normal = transparent_normal;
                bool should_reflect = false;
                self_seed = self_seed + 1u;
                vec4 cri = pick_ref_idx(&picked, is.refractive_index_low, is.refractive_index_high, self_seed);
                float refractive_index = cri.w;
                self_seed = self_seed + 1u;
                if (!(!is.front_face && is.ty == TRANSPARENT)) refractive_index = 1.0f / refractive_index;
                vec3 cw(cri.x, cri.y, cri.z);
                color = color * cw;
                out_radiance_colour = out_radiance_colour * cw;
                if (refractive_index != 1.0f) {
                    float cos_theta = wmin(dot(-ray.direction, normal), 1.0f);
                    float sin_theta = std::sqrt(1.0f - (cos_theta * cos_theta));
                    bool cannot_refract = (refractive_index * sin_theta) > 1.0f;
                    float pdf = reflectance(cos_theta, refractive_index);
                    float rnd = rand_f32(self_seed);
                    if (cannot_refract || (pdf > rnd)) should_reflect = true;
                    self_seed = self_seed + 1u;
                }
                if (!should_reflect || is.ty == TRANSPARENT) {
                    color = color * is.color;
                    if (i != 0u) out_radiance_colour = out_radiance_colour * is.color;
                }
                if (!should_reflect) {
                    normal = assign_normal;
                    self_seed = self_seed + 1u;
                }
                fill_mc_world_space_states(L, &self_seed, ray.origin, is.normal, ray.direction);
                MC s = resample_mcmm(L, &self_seed);
                bool reflecting = should_reflect || is.ty == METALLIC;
                if (!reflecting) {
                    if (is.ty == DIFFUSE) {
                        vec3 dir;
                        vec3 dir_cosine = cosine_weighted_hemisphere(self_seed, is.normal, is.tangent);
                        float cosine_pdf = wmax(dot(dir_cosine, is.normal) / PI, 0.0f);
                        float theta = rand_f32(self_seed) * TAU;
                        self_seed = self_seed + 1u;
                        float xi = rand_f32(self_seed);
                        self_seed = self_seed + 1u;
                        float conf0 = 1.0f, conf1 = 0.0f;
                        vec3 dir_markov;
                        if (guide) {
                            vec3 light_dir = get_light_dir(s, ray.origin);
                            vec3 mean = normalize(light_dir);
                            float kappa = get_kappa(s);
                            float cv = std::cos(theta), sv = std::sin(theta);
                            float minus_2_kappa = -2.0f * kappa;
                            float W_minus_1 = std::log(1.0f + (xi * exp_minus_one(minus_2_kappa))) / kappa;
                            float W = 1.0f + W_minus_1;
                            float norm_V = std::sqrt(-std::fma(W_minus_1, W_minus_1, 2.0f * W_minus_1));
                            vec3 Xs = from_onb_no_tangent(vec3(strip_NaN(cv * norm_V), W, strip_NaN(sv * norm_V)), mean);
                            dir_markov = normalize(Xs);
                            float u0 = 0.2f, u1 = 0.8f;
                            if (!marcov_chain_valid(s) || near_zero(length(light_dir)) || near_zero(s.weight_sum) ||
                                near_zero(length(Xs))) {
                                u0 = 1.0f;
                                u1 = 0.0f;
                            }
                            float csum = u0 + u1;
                            conf0 = u0 / csum;
                            conf1 = u1 / csum;
                        }
                        float rnd = rand_f32(self_seed);
                        self_seed = self_seed + 1u;
                        if (rnd < conf0) {
                            dir = dir_cosine;
                            last_not_vmf = true;
                        } else {
                            dir = dir_markov;
                        }
                        // general.wesl:840 weights by the cosine pdf of dir_cosine even when dir is the
                        // vMF draw; LAM_GUIDE_PDF_AT_SAMPLE evaluates it at dir
                        float cos_term = pdf_at_sample ? wmax(dot(dir, is.normal) / PI, 0.0f) : cosine_pdf;
                        float avg_pdf = (conf0 * cos_term) + (conf1 == 0.0f ? 0.0f : conf1 * wmax(all_vmf_pdfs(L, ray.origin, dir), 0.0f));
                        vec3 diffuse = make_diffuse(is.color, ray, is.normal, is.tangent, is.roughness.x, dir);
                        cached_pdf = avg_pdf;
                        cached_brdf = wmax(dot(dir, is.normal) / PI, 0.0f);
                        float normalization_factor = absf(cached_brdf) / wmax(avg_pdf, 0.001f);
                        color = (color * normalization_factor) * diffuse;
                        out_radiance_colour = (out_radiance_colour * normalization_factor) * diffuse;
                        ray.direction = dir;
                        if (i == 0u) sample.pdf = avg_pdf;
                    } else if (is.ty == TRANSPARENT) {
                        cached_pdf = 1.0f;
                        cached_brdf = 1.0f;
                        ray.direction = refract(ray.direction, normal, refractive_index);
                    }
                } else {
                    cached_pdf = 1.0f;
                    cached_brdf = 1.0f;
                    ray.direction = reflect(ray.direction, normal);
                    if (dot(ray.direction, is.normal) < 0.0f) ray.direction = reflect(ray.direction, is.normal);
                }
            } else {
                vec3 bg = sc.background(ray.direction);
                vec3 new_pos = at(ray, p.tmax);
                if (i == 1u) {
                    sample.visible_point = new_pos;
                    sample.visible_normal = -ray.direction;
                }
                if (i != 0u) {
                    sample.out_radiance = fma3(out_radiance_colour, bg, sample.out_radiance);
                    vec3 radiance_out = (bg * cached_brdf) / cached_pdf;
                    grid_add_radiance(L, ray.origin, last_normal, last_dir, radiance_out);
                    float weight = length(radiance_out);
                    if (weight > 0.0f) {
                        if (guide) {
                            MC st = update_marcov_state(L, ray.origin, new_pos, weight, self_seed, false,
                                                        grid_load(L, ray.origin, last_normal, last_dir, false), 1.0f);
                            grid_store_markov_chain(L, ray.origin, last_normal, last_dir, st);
                            L.tentative = update_marcov_state(L, ray.origin, new_pos, length(radiance_out), self_seed,
                                                              false, L.tentative, i == 1u ? 1.0f : 0.5f);
                        }
                        self_seed++;
                    }
                }
                sample.color = fma3(color, bg, sample.color);
                break;
            }
        }
        if (guide) {
            MC world_cache = grid_load(L, sample.point, sample.normal, start_dir, false);
            MC st = update_marcov_state(L, sample.point, sample.visible_point, length(sample.out_radiance), self_seed,
                                        false, world_cache, 1.0f);
            grid_store_markov_chain(L, sample.point, sample.normal, start_dir, st);
            grid_add_radiance(L, sample.point, sample.normal, start_dir, sample.out_radiance);
        }
        sample.color = sample.color / vmf_weight;
        sample.out_radiance = sample.out_radiance / vmf_weight;
        sample.valid = true;
        return sample;
    }

    // ----- one subgroup of 32 lanes (general.wesl:506-610)
    void rt_main_subgroup(uint32_t y, uint32_t x_base) {
        Lane lanes[SUBGROUP];
        bool active[SUBGROUP];
        uint32_t own_seed[SUBGROUP];
        vec3 pixel_color[SUBGROUP], pixel_normal[SUBGROUP], pixel_albedo[SUBGROUP], pixel_emission[SUBGROUP];
        vec3 out_radiance[SUBGROUP];
        uint32_t pixel_ty[SUBGROUP];
        Sample sample[SUBGROUP];
        bool sample_valid[SUBGROUP];
        float pdf[SUBGROUP];
        lam_reservoir R[SUBGROUP];
        uint32_t x_end = p.crop_w ? p.crop_x0 + p.crop_w : p.width;
        uint32_t x_begin = p.crop_w ? p.crop_x0 : 0u;
        for (uint32_t l = 0; l < SUBGROUP; ++l) {
            uint32_t x = x_base + l;
            active[l] = x < p.width && x >= x_begin && x < x_end;
            uint64_t idx = (uint64_t)x + (uint64_t)y * p.width;
            lanes[l] = Lane();
            if (active[l] && guide && p.old_chains && idx < p.old_chains_len) {
                const lam_markov_chain& c = p.old_chains[idx];
                lanes[l].tentative.light_source = vec3(c.light_source[0], c.light_source[1], c.light_source[2]);
                lanes[l].tentative.mean_cosine = c.mean_cosine;
                lanes[l].tentative.weight_sum = c.weight_sum;
                lanes[l].tentative.num_samples = c.num_samples;
                lanes[l].tentative.score = c.score;
            }
            own_seed[l] = rand_u32(x * y) + p.seed_offset + y;
            pixel_color[l] = pixel_normal[l] = pixel_albedo[l] = pixel_emission[l] = out_radiance[l] = vec3(0.0f);
            pixel_ty[l] = 0;
            sample[l] = Sample();
            sample_valid[l] = false;
            pdf[l] = 0.0f;
            R[l] = lam_reservoir{};
        }
        MC snapshot[SUBGROUP];
        for (uint32_t i = 0; i < p.samples; ++i) {
            for (uint32_t l = 0; l < SUBGROUP; ++l) snapshot[l] = active[l] ? lanes[l].tentative : MC();
            for (uint32_t l = 0; l < SUBGROUP; ++l)
                if (active[l]) fill_mc_screen_space_states(lanes[l], &own_seed[l], snapshot, active, x_base + l, y);
            for (uint32_t l = 0; l < SUBGROUP; ++l) {
                if (!active[l]) continue;
                SampleReturn rs = rt_sample(lanes[l], x_base + l, y, own_seed[l]);
                pixel_normal[l] = rs.normal;
                pixel_albedo[l] = rs.albedo;
                pixel_emission[l] = rs.emission;
                pixel_ty[l] = rs.ty;
                pixel_color[l] = pixel_color[l] + rs.color;
                out_radiance[l] = out_radiance[l] + rs.out_radiance;
                own_seed[l] = rand_u32(own_seed[l]);
                if (p.restir == LAM_RESTIR_PER_PIXEL) {
                    if (rs.valid) {
                        sample_valid[l] = true;
                        Sample s;
                        s.visible_point = rs.visible_point;
                        s.visible_normal = normalised_to_u32(rs.visible_normal);
                        s.sample_point = rs.point;
                        s.sample_normal = normalised_to_u32(pixel_normal[l]);
                        s.out_radiance = out_radiance[l] / u2f(p.samples);
                        s.ty = pixel_ty[l];
                        s.roughness = conv_rough(rs.roughness);
                        sample[l] = s;
                        pdf[l] += rs.pdf;
                    }
                } else if (p.restir == LAM_RESTIR_PER_SAMPLE) {
                    Sample s;
                    s.visible_point = rs.visible_point;
                    s.visible_normal = normalised_to_u32(rs.visible_normal);
                    s.sample_point = rs.point;
                    s.sample_normal = normalised_to_u32(rs.normal);
                    s.out_radiance = rs.out_radiance;
                    s.ty = rs.ty;
                    s.roughness = conv_rough(rs.roughness);
                    if (s.ty != SKY && rs.valid) {
                        float w = p_hat(s);
                        R[l] = update(s, w, R[l], own_seed[l]);
                        own_seed[l] = rand_u32(own_seed[l]);
                        uint32_t c = conf_of(R[l].packed_confidence_valid);
                        R[l].W = safe_div(R[l].w, u2f(c) * p_hat(sam_from_res(R[l])));
                    } else if (s.ty == SKY) {
                        R[l].ty = SKY;
                    }
                }
            }
            // subgroupShuffle(tentative, (sub_id + 1) % 32)
            MC shuffled[SUBGROUP];
            for (uint32_t l = 0; l < SUBGROUP; ++l) {
                uint32_t src = (l + 1u) % SUBGROUP;
                shuffled[l] = active[src] ? lanes[src].tentative : MC();
            }
            for (uint32_t l = 0; l < SUBGROUP; ++l) if (active[l]) lanes[l].tentative = shuffled[l];
        }
        for (uint32_t l = 0; l < SUBGROUP; ++l) {
            if (!active[l]) continue;
            pixels++;
            uint32_t x = x_base + l;
            uint64_t idx = (uint64_t)x + (uint64_t)y * p.width;
            pdf[l] /= u2f(p.samples);
            if (p.restir != LAM_RESTIR_DISABLED && p.info) {
                lam_info& inf = p.info[idx];
                vec3 cl = lanes[l].camera_loc;
                float a[9] = {cl.x, cl.y, cl.z, pixel_emission[l].x, pixel_emission[l].y, pixel_emission[l].z,
                              pixel_albedo[l].x, pixel_albedo[l].y, pixel_albedo[l].z};
                std::memcpy(inf.arr, a, sizeof(a));
            }
            if (guide && p.chains && idx < p.chains_len) {
                lam_markov_chain& c = p.chains[idx];
                const MC& t = lanes[l].tentative;
                c.light_source[0] = t.light_source.x;
                c.light_source[1] = t.light_source.y;
                c.light_source[2] = t.light_source.z;
                c.mean_cosine = t.mean_cosine;
                c.weight_sum = t.weight_sum;
                c.num_samples = t.num_samples;
                c.score = t.score;
                c._pad = 0;
            }
            vec3 col = max3(pixel_color[l] / u2f(p.samples), 0.0f);
            if (p.out_normal) st4(p.out_normal, idx, pixel_normal[l]);
            if (p.out_albedo) st4(p.out_albedo, idx, pixel_albedo[l]);
            if (p.out_color) st4(p.out_color, idx, col);
            if (p.restir == LAM_RESTIR_PER_PIXEL) {
                if (sample[l].ty != SKY && sample_valid[l]) {
                    float w = p_hat(sample[l]);
                    R[l] = update(sample[l], w, R[l], own_seed[l]);
                    own_seed[l] = rand_u32(own_seed[l]);
                    uint32_t c = conf_of(R[l].packed_confidence_valid);
                    R[l].W = safe_div(R[l].w, u2f(c) * p_hat(sam_from_res(R[l])));
                } else if (sample[l].ty == SKY) {
                    R[l].ty = SKY;
                }
            }
            if (p.reservoirs) p.reservoirs[idx] = R[l];
        }
    }
    static void st4(float* img, uint64_t idx, vec3 v) {
        img[4 * idx + 0] = v.x;
        img[4 * idx + 1] = v.y;
        img[4 * idx + 2] = v.z;
        img[4 * idx + 3] = 1.0f;
    }
};

}  // namespace

// Debug views, src/debug/{front_face,reflectance,tangent}.wesl: one primary ray per pixel.  The
// candidate test of these shaders keeps only triangles whose diffuse alpha is not near zero
// (no exception for transparent materials); the oracle's scene marks every BLAS opaque or not,
// and debug renders of non-opaque geometry use the same alpha rule as the path shaders here.
static int render_debug(const Scene& sc, const RenderParams& p, RenderCounters* counters) {
    PT pt(sc, p);
    for (uint32_t y = 0; y < p.height; ++y) {
        for (uint32_t x = 0; x < p.width; ++x) {
            Ray r = pt.create_ray(x, y);
            Hit h = sc.trace(r.origin, r.direction, p.tmin, p.tmax, false);
            vec3 c(0.0f);
            if (p.quality == LAM_DEBUG_TANGENT) {
                vec3 dir = h.hit ? normalize(h.ov0 - h.ov1) : vec3(0.0f);
                c = (correct_tangent(dir) + vec3(1.0f)) / 2.0f;
            } else if (h.hit && p.quality == LAM_DEBUG_FRONT_FACE) {
                float g = 1.0f / (h.t + 1.0f);
                c = h.front ? vec3(0.0f, g, 0.0f) : vec3(g, 0.0f, 0.0f);
            } else if (h.hit) {
                // reflectance.wesl:88 reads material_idx[geometry_index], i.e. instance 0's table
                const lam_material& m = pt.material_of(0, h.prim);
                vec2 ior = unpack2x16float(m.refractive_index);
                c = vec3(ior.x / 5.0f, ior.y / 5.0f, 0.0f);
            }
            uint64_t idx = (uint64_t)x + (uint64_t)y * p.width;
            if (p.out_color) PT::st4(p.out_color, idx, c);
            if (p.out_normal) PT::st4(p.out_normal, idx, vec3(0.0f));
            if (p.out_albedo) PT::st4(p.out_albedo, idx, vec3(0.0f));
        }
    }
    if (counters) {
        counters->segments = (uint64_t)p.width * p.height;
        counters->samples = counters->segments;
    }
    return LAM_OK;
}

int render(const Scene& scene, const RenderParams& p, RenderCounters* counters) {
    if (p.width == 0 || p.height == 0 || p.samples == 0) return LAM_ERR_INVALID_ARGUMENT;
    if (p.quality >= LAM_DEBUG_FRONT_FACE) return render_debug(scene, p, counters);
    uint32_t y0 = p.crop_w ? p.crop_y0 : 0u;
    uint32_t y1 = p.crop_w ? std::min(p.height, p.crop_y0 + p.crop_h) : p.height;
    uint32_t x0 = p.crop_w ? (p.crop_x0 / SUBGROUP) * SUBGROUP : 0u;
    uint32_t x1 = p.crop_w ? std::min(p.width, p.crop_x0 + p.crop_w) : p.width;
    std::vector<std::pair<uint32_t, uint32_t>> groups;
    for (uint32_t y = y0; y < y1; ++y)
        for (uint32_t xb = x0; xb < x1; xb += SUBGROUP) groups.push_back({y, xb});
    int threads = std::max(1, p.threads);
    std::vector<uint64_t> segs_t(threads, 0), pix_t(threads, 0);
    parallel_for((long long)groups.size(), threads, 4, [&](long long g, int t) {
        PT pt(scene, p);
        pt.rt_main_subgroup(groups[g].first, groups[g].second);
        segs_t[t] += pt.segments;
        pix_t[t] += pt.pixels;
    });
    uint64_t segs = 0, pixels = 0;
    for (int t = 0; t < threads; ++t) { segs += segs_t[t]; pixels += pix_t[t]; }
    if (counters) {
        counters->segments = segs;
        counters->samples = pixels * p.samples;
    }
    return LAM_OK;
}

// ---------------------------------------------------------------- temporal_resampling.wesl:37-65
int temporal_resampling(lam_reservoir* cur, const lam_reservoir* old, uint32_t width, uint32_t height,
                        uint32_t seed_offset) {
    for (uint32_t y = 0; y < height; ++y) {
        for (uint32_t x = 0; x < width; ++x) {
            uint64_t idx = (uint64_t)x + (uint64_t)y * width;
            uint32_t own_seed = rand_u32(x * y) + rand_u32(seed_offset + y);
            lam_reservoir Rs = cur[idx];
            lam_reservoir R = old ? old[idx] : lam_reservoir{};
            if (dot(u32_to_normalised(R.sample_normal), u32_to_normalised(Rs.sample_normal)) < 0.95f) R = lam_reservoir{};
            if (Rs.ty == SKY) continue;
            float w = p_hat(sam_from_res(R));
            bool picked;
            R = merge(Rs, R, w, own_seed, &picked);
            uint32_t c = conf_of(R.packed_confidence_valid);
            R.W = safe_div(R.w, u2f(c) * p_hat(sam_from_res(R)));
            cur[idx] = R;
        }
    }
    return LAM_OK;
}

// ---------------------------------------------------------------- spatial_resampling.wesl:35-194
static float jacobian_determinant(const Sample& q, const Sample& r) {
    vec3 q1_to_q2 = q.sample_point - q.visible_point;
    vec3 r1_to_q2 = r.sample_point - q.visible_point;
    vec3 vn = u32_to_normalised(q.visible_normal);
    float cos_theta_r = dot(normalize(r1_to_q2), vn);
    float cos_theta_q = dot(normalize(q1_to_q2), vn);
    return safe_div(cos_theta_r * len_sqrd(q1_to_q2), cos_theta_q * len_sqrd(r1_to_q2));
}

int spatial_resampling(const lam_reservoir* cur, const lam_info* info, uint32_t width, uint32_t height,
                       uint32_t is_samples, uint32_t is_space, uint32_t seed_offset, float* out_color) {
    if (is_samples > 128 || is_space < 2) return LAM_ERR_INVALID_ARGUMENT;
    std::vector<lam_reservoir> Q(is_samples + 1);
    for (uint32_t y = 0; y < height; ++y) {
        for (uint32_t x = 0; x < width; ++x) {
            uint64_t idx = (uint64_t)x + (uint64_t)y * width;
            uint32_t own_seed = rand_u32(x * y) + rand_u32(seed_offset) + y;
            lam_reservoir Rs = cur[idx];
            uint32_t Z = 0;
            vec3 Rs_normal = u32_to_normalised(Rs.sample_normal);
            Q[0] = Rs;
            if (Rs.ty == SKY) continue;
            uint32_t sample_is_samples = 0;
            for (uint32_t i = 0; i < is_samples; ++i) {
                uint32_t max_val = (is_space * is_space) - 1u;
                uint32_t min_space = is_space / 2u;
                uint32_t self_idx = min_space + (min_space * is_space);
                uint32_t rnd = rand_u32(own_seed) % max_val;
                if (rnd >= self_idx) rnd = rnd + 1u;
                uint32_t xn = rnd % is_space, yn = rnd / is_space;
                int32_t nbx = (int32_t)xn - (int32_t)min_space, nby = (int32_t)yn - (int32_t)min_space;
                own_seed = rand_u32(own_seed);
                int32_t ox = (int32_t)x + nbx, oy = (int32_t)y + nby;
                if (ox < 0 || oy < 0 || (nbx == 0 && nby == 0)) continue;
                if ((uint32_t)ox >= width || (uint32_t)oy >= height) continue;
                const lam_reservoir& Rn = cur[(uint64_t)ox + (uint64_t)oy * width];
                vec3 Rn_normal = u32_to_normalised(Rn.sample_normal);
                float similarity = dot(Rn_normal, Rs_normal);
                if (similarity < 0.9f || Rn.ty != Rs.ty || absf(Rs.roughness - Rn.roughness) > 0.1f) continue;
                float jac = jacobian_determinant(sam_from_res(Rn), sam_from_res(Rs));
                if (Rs.ty != DIFFUSE) continue;
                float p_hat_dashed_q = p_hat(sam_from_res(Rn)) * jac;
                bool picked;
                Rs = merge(Rs, Rn, p_hat_dashed_q, own_seed, &picked);
                own_seed = rand_u32(own_seed);
                if (picked) Rs_normal = u32_to_normalised(Rs.sample_normal);
                Q[sample_is_samples + 1u] = Rn;
                own_seed = rand_u32(own_seed);
                sample_is_samples++;
            }
            for (uint32_t j = 0; j < sample_is_samples + 1u; ++j)
                if (p_hat(sam_from_res(Q[j])) > 0.0f) Z = Z + conf_of(Q[j].packed_confidence_valid);
            float Z_times_p_hat = u2f(Z) * p_hat(sam_from_res(Rs));
            Rs.W = safe_div(Rs.w, Z_times_p_hat);
            const float* a = info[idx].arr;
            vec3 albedo(a[6], a[7], a[8]), emission(a[3], a[4], a[5]);
            vec3 pix = fma3(v3(Rs.out_radiance) * Rs.W, albedo, emission);
            out_color[4 * idx + 0] = pix.x;
            out_color[4 * idx + 1] = pix.y;
            out_color[4 * idx + 2] = pix.z;
            out_color[4 * idx + 3] = 1.0f;
        }
    }
    return LAM_OK;
}

// ---------------------------------------------------------------- end_of_frame.wesl:14-99
void process_gi_reservoirs(lam_reservoir* r, uint64_t n, uint32_t cap) {
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t c = conf_of(r[i].packed_confidence_valid);
        if (c > cap) {
            float mul = u2f(cap) / u2f(c);
            r[i].w *= mul;
            r[i].packed_confidence_valid = pack_conf(cap, valid_of(r[i].packed_confidence_valid));
        }
    }
}

void process_world_markov_chains(uint32_t* world, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t* e = world + i * W_STRIDE;
        if (e[W_TIMEOUT] == 0u) {
            e[W_SEC] = 0u;
            e[W_NUM] = 0u;
            e[W_LUM] = e[W_LUM + 1] = e[W_LUM + 2] = 0u;
            e[W_LOCK] = 0u;
            continue;
        }
        uint32_t old_num = e[W_NUM];
        if (old_num != 0u) {
            uint32_t prod = old_num * 8u;
            uint32_t nn = prod / 9u + ((prod % 9u) != 0u ? 1u : 0u);
            float mul = u2f(nn) / u2f(old_num);
            for (int k = 0; k < 3; ++k) e[W_LUM + k] = f2bits(bits2f(e[W_LUM + k]) * mul);
            e[W_NUM] = nn;
        }
        e[W_TIMEOUT] = e[W_TIMEOUT] - 1u;
    }
}

void average_frames(const float* const* frames, uint32_t n, uint32_t width, uint32_t height, float* out) {
    uint64_t P = (uint64_t)width * height;
    for (uint64_t i = 0; i < P; ++i) {
        float a[4] = {0, 0, 0, 0};
        for (uint32_t f = 0; f < n; ++f)
            for (int c = 0; c < 4; ++c) a[c] = a[c] + (frames[f][4 * i + c] / u2f(n));
        out[3 * i + 0] = a[0];
        out[3 * i + 1] = a[1];
        out[3 * i + 2] = a[2];
    }
}

}  // namespace oracle
