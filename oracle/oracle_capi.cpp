// oracle_capi.cpp - TEST INFRASTRUCTURE ONLY (the CPU oracle; see oracle_math.h).
// C entry points of the oracle, plus the host-side packing restatements:
//   Material::new and its packing   src/lib.rs:96-182 (f16/bf16 per half 2.6.0)
//   Camera::from_proj_view          src/camera.rs:15-24, 59-70 (4x4 inverse; FP64 cofactors here)
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <new>

#include "oracle_pt.h"

using namespace oracle;

extern "C" {

int oracle_scene_create(const lam_scene_desc* desc, void** out) {
    if (!out) return LAM_ERR_INVALID_ARGUMENT;
    Scene* s = new (std::nothrow) Scene();
    if (!s) return LAM_ERR_OUT_OF_MEMORY;
    int rc = s->load(desc);
    if (rc != LAM_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return LAM_OK;
}

void oracle_scene_destroy(void* scene) { delete (Scene*)scene; }

int oracle_trace(const void* scene, const lam_ray* rays, uint64_t n, uint32_t mode, lam_hit* hits, int32_t threads,
                 int32_t bruteforce) {
    if (!scene || (!rays && n) || (!hits && n)) return LAM_ERR_INVALID_ARGUMENT;
    const Scene& sc = *(const Scene*)scene;
    int th = threads > 0 ? threads : 1;
    parallel_for((long long)n, th, 256, [&](long long i, int) {
        const lam_ray& r = rays[i];
        vec3 o(r.origin[0], r.origin[1], r.origin[2]), d(r.direction[0], r.direction[1], r.direction[2]);
        Hit h = bruteforce ? sc.trace_bruteforce(o, d, r.tmin, r.tmax) : sc.trace(o, d, r.tmin, r.tmax, mode == LAM_TRACE_ANY);
        lam_hit& out = hits[i];
        if (h.hit) {
            out.t = h.t;
            out.u = h.u;
            out.v = h.v;
            out.primitive_index = h.prim;
            out.instance_index = h.inst;
            out.kind = h.front ? LAM_HIT_FRONT : LAM_HIT_BACK;
        } else {
            out.t = 0.0f;
            out.u = out.v = 0.0f;
            out.primitive_index = 0xFFFFFFFFu;
            out.instance_index = 0xFFFFFFFFu;
            out.kind = LAM_HIT_NONE;
        }
    });
    return LAM_OK;
}

int oracle_render(const void* scene, oracle_render_args* a) {
    if (!scene || !a || !a->camera) return LAM_ERR_INVALID_ARGUMENT;
    RenderParams p;
    p.width = a->width;
    p.height = a->height;
    p.samples = a->samples;
    p.quality = a->quality;
    p.restir = a->restir;
    p.max_depth = a->max_depth;
    p.guide = a->guide;
    p.seed_offset = a->seed_offset;
    p.tmin = a->tmin;
    p.tmax = a->tmax;
    p.camera = *a->camera;
    p.crop_x0 = a->crop_x0;
    p.crop_y0 = a->crop_y0;
    p.crop_w = a->crop_w;
    p.crop_h = a->crop_h;
    p.threads = a->threads;
    p.chains = a->chains;
    p.old_chains = a->old_chains;
    p.chains_len = a->chains_len;
    p.old_chains_len = a->old_chains_len;
    p.world = a->world;
    p.old_world = a->old_world;
    p.world_len = a->world_len;
    p.reservoirs = a->reservoirs;
    p.info = a->info;
    p.out_color = a->out_color;
    p.out_normal = a->out_normal;
    p.out_albedo = a->out_albedo;
    RenderCounters c;
    int rc = render(*(const Scene*)scene, p, &c);
    a->segments_out = c.segments;
    a->samples_out = c.samples;
    return rc;
}

int oracle_temporal_resampling(lam_reservoir* cur, const lam_reservoir* old, uint32_t w, uint32_t h, uint32_t s) {
    return temporal_resampling(cur, old, w, h, s);
}
int oracle_spatial_resampling(const lam_reservoir* cur, const lam_info* info, uint32_t w, uint32_t h, uint32_t n,
                              uint32_t space, uint32_t s, float* out) {
    return spatial_resampling(cur, info, w, h, n, space, s, out);
}
void oracle_process_gi_reservoirs(lam_reservoir* r, uint64_t n, uint32_t cap) { process_gi_reservoirs(r, n, cap); }
void oracle_process_world_markov_chains(uint32_t* w, uint64_t n) { process_world_markov_chains(w, n); }
void oracle_average_frames(const float* const* f, uint32_t n, uint32_t w, uint32_t h, float* out) {
    average_frames(f, n, w, h, out);
}

uint32_t oracle_rand_u32(uint32_t s) { return rand_u32(s); }
float oracle_rand_f32(uint32_t s) { return rand_f32(s); }
uint16_t oracle_f32_to_f16(float f) { return f32_to_f16(f); }
float oracle_f16_to_f32(uint16_t h) { return f16_to_f32(h); }
uint16_t oracle_f32_to_bf16(float f) { return f32_to_bf16(f); }
uint32_t oracle_normalised_to_u32(const float n[3]) { return normalised_to_u32(vec3(n[0], n[1], n[2])); }
void oracle_u32_to_normalised(uint32_t u, float out[3]) {
    vec3 v = u32_to_normalised(u);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

// Material::new, src/lib.rs:132-182
int oracle_material_new(const float uv1[2], const float uv2[2], const float uv3[2], const uint16_t recolour[2],
                        uint16_t diffuse, int32_t emission, int32_t attributes, float emissive_scale,
                        float diffuse_scale, const float* ior, uint32_t ty, lam_material* out) {
    auto pack2xf16 = [](const float f[2]) { return (uint32_t)f32_to_f16(f[0]) | ((uint32_t)f32_to_f16(f[1]) << 16); };
    auto opt = [](int32_t v, uint16_t* o) {
        if (v < 0) { *o = 0xFFFF; return true; }
        if (v >= 0xFFFF) return false;
        *o = (uint16_t)v;
        return true;
    };
    uint16_t e, a;
    if (!opt(emission, &e) || !opt(attributes, &a)) return LAM_ERR_INVALID_ARGUMENT;
    float vac[2] = {1.0f, 1.0f};
    const float* r = ior ? ior : vac;
    out->tex_pos_1 = pack2xf16(uv1);
    out->tex_pos_2 = pack2xf16(uv2);
    out->tex_pos_3 = pack2xf16(uv3);
    out->tex_pos_recolour = (uint32_t)recolour[0] | ((uint32_t)recolour[1] << 16);
    out->tex_idx_diffuse_emission = (uint32_t)diffuse | ((uint32_t)e << 16);
    out->tex_idx_attributes_ty = (uint32_t)a | ((uint32_t)(uint16_t)ty << 16);
    out->emission_scale = (uint32_t)f32_to_bf16(emissive_scale) | ((uint32_t)f32_to_bf16(diffuse_scale) << 16);
    out->refractive_index = pack2xf16(r);
    return LAM_OK;
}

static bool invert4(const float m[16], float out[16]) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    double inv[16];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    if (det == 0.0 || !std::isfinite(det)) return false;
    for (int i = 0; i < 16; ++i) out[i] = (float)(inv[i] / det);
    return true;
}

int oracle_camera_from_proj_view(const float proj[16], const float view[16], lam_camera* out) {
    if (!invert4(proj, out->projection_inverse)) return LAM_ERR_PROJECTION_UNINVERTIBLE;
    if (!invert4(view, out->view_inverse)) return LAM_ERR_VIEW_UNINVERTIBLE;
    return LAM_OK;
}

int oracle_invert_3x4(const float m[12], float out[12]) { return invert_3x4(m, out) ? 1 : 0; }

int oracle_wbw(const float o[3], const float d[3], const float v0[3], const float v1[3], const float v2[3],
               float* t_f32, float* t, float* u, float* v, int32_t* front) {
    vec3 O(o[0], o[1], o[2]), D(d[0], d[1], d[2]);
    vec3 A(v0[0], v0[1], v0[2]), B(v1[0], v1[1], v1[2]), C(v2[0], v2[1], v2[2]);
    WbwRay r = wbw_setup(D);
    float tf;
    if (!wbw_f32(r, O, A, B, C, &tf)) return 0;
    *t_f32 = tf;
    bool fr;
    wbw_f64(O, D, A, B, C, t, u, v, &fr);
    *front = fr ? 1 : 0;
    return 1;
}

}  // extern "C"
