// wavefront.cu - rt_main of the reference (src/path_tracing/general.wesl:506-975) as a wavefront:
//
//   generate   one thread per pixel: seed chain, camera ray per sample of the wave
//   extend     persistent warps: closest hit for every queued path (traverse.cuh)
//   shade      one bounce of rt_sample for every queued path; survivors are appended to the next queue
//   accumulate one thread per pixel: per-sample colours summed in sample order, reservoirs, outputs
//   shuffle    (Markov guiding) the per-sample subgroup shuffle of the tentative chains
//
// Path state lives in HBM as structure-of-arrays indexed by path id = sample_in_wave * pixels + pixel.
// A wave holds `spp_wave` samples of every pixel; samples of one pixel are independent except through
// the Markov chains and per-sample ReSTIR, which therefore run one sample per wave.
#include <algorithm>
#include <cstring>
#include <vector>

#include "guide.cuh"
#include "guide_net.cuh"
#include "materials.cuh"
#include "scene.h"
#include "tracer.h"
#include "traverse.cuh"
#include "wavefront.cuh"

namespace lam {


struct Isect {
    v3 color;
    float t;
    v3 emission;
    uint32_t ty;
    v3 normal;
    bool front_face;
    v3 tangent;
    float2 roughness, roughness_transparent;
    float ior_low, ior_high;
};

// ray_hit's post-query part (general.wesl:1080-1137) for a committed triangle.
// A committed procedural hit is a generated intersection (general.wesl:1068-1075, 1100-1102): the
// handler's t, normal and tangent (phit_a = normal, t; phit_b = tangent), barycentrics 0, back face.
LAM_DEV void make_isect(const DevScene& S, const DevInstance* insts, uint2 hit, float3 o, float3 d, Isect& r,
                        const float4* phit_a = nullptr, const float4* phit_b = nullptr, uint32_t path = 0u) {
    const float4* tp = S.tris + 3u * hit.x;
    const float4 a = ld_keep(tp);
    float t, bu, bv;
    bool front;
    v3 tg, n;
    if (phit_a && (insts[hit.y].flags & INST_PROCEDURAL)) {
        const float4 pa = phit_a[path], pb = phit_b[path];
        t = pa.w;
        bu = bv = 0.0f;
        front = false;
        n = mk(pa.x, pa.y, pa.z);
        tg = mk(pb.x, pb.y, pb.z);
    } else {
        float m[12];
        {
            const float4* ip = reinterpret_cast<const float4*>(insts + hit.y);
            const float4 a0 = ld_keep(ip), a1 = ld_keep(ip + 1), a2 = ld_keep(ip + 2);
            m[0] = a0.x; m[1] = a0.y; m[2] = a0.z; m[3] = a0.w; m[4] = a1.x; m[5] = a1.y;
            m[6] = a1.z; m[7] = a1.w; m[8] = a2.x; m[9] = a2.y; m[10] = a2.z; m[11] = a2.w;
        }
        float3 oo, od;
        object_ray(m, o, d, &oo, &od);
        const float4 b = ld_keep(tp + 1), c = ld_keep(tp + 2);
        wbw_f64(oo, od, a, b, c, &t, &bu, &bv, &front);
        v3 v0 = mk(a.x, a.y, a.z), v1 = mk(b.x, b.y, b.z), v2 = mk(c.x, c.y, c.z);
        tg = normalize(v0 - v1);
        {
            float ax = fabsf(tg.x), ay = fabsf(tg.y), az = fabsf(tg.z);
            bool xl = ax > ay && ax > az, yl = ay > ax && ay > az;
            bool rev = xl ? tg.x < 0.0f : (yl ? tg.y < 0.0f : tg.z < 0.0f);
            if (rev) tg = -tg;
        }
        n = normalize(cross(tg, v0 - v2));
    }
    r.t = t;
    r.front_face = front;
    const uint32_t prim = __float_as_uint(a.w);
    const lam_material mt = load_material(S, hit.y, prim);
    const uint32_t idx_d = mt.tex_idx_diffuse_emission & 0xFFFFu, idx_e = mt.tex_idx_diffuse_emission >> 16;
    const uint32_t idx_a = mt.tex_idx_attributes_ty & 0xFFFFu;
    r.ty = mt.tex_idx_attributes_ty >> 16;
    float2 ri = unpack2x16float(mt.refractive_index);
    r.ior_low = ri.x;
    r.ior_high = ri.y;
    v3 dw = mk(d.x, d.y, d.z);
    r.normal = dot(dw, n) > 0.0f ? -n : n;
    r.tangent = tg;
    float2 uv = hit_uv(mt, bu, bv);
    float4 dc = tex_sample(S, S.diffuse_first, S.diffuse_count, idx_d, uv.x, uv.y);
    float4 rc = recolour_load(S, mt.tex_pos_recolour & 0xFFFFu, mt.tex_pos_recolour >> 16);
    v3 diffuse = mk(dc.x, dc.y, dc.z) * mk(rc.x, rc.y, rc.z);
    r.color = diffuse;
    float es_x = __uint_as_float((mt.emission_scale & 0xFFFFu) << 16);
    float es_y = __uint_as_float((mt.emission_scale >> 16) << 16);
    r.emission = splat(0.0f);
    if (idx_e != 0xFFFFu) {
        float4 ec = tex_sample(S, S.emission_first, S.emission_count, idx_e, uv.x, uv.y);
        r.emission = mk(ec.x, ec.y, ec.z) * es_x;
    }
    r.emission = r.emission + diffuse * es_y;
    r.roughness = make_float2(0.0f, 0.0f);
    r.roughness_transparent = make_float2(0.0f, 0.0f);
    if (idx_a != 0xFFFFu) {
        float4 at = tex_sample(S, S.attr_first, S.attr_count, idx_a, uv.x, uv.y);
        r.roughness = make_float2(at.x, at.y);
        r.roughness_transparent = make_float2(at.z, at.w);
    }
}

// ---------------------------------------------------------------- BSDF helpers (general.wesl:1206-1289)
LAM_DEV v3 to_onb(v3 src, v3 up, v3 tangent) {
    v3 s = tangent, t = cross(up, s);
    v3 inv_s = cross(up, t), inv_up = cross(t, s), inv_t = cross(s, up);
    return fma3(splat(src.x), inv_s, fma3(splat(src.y), inv_up, inv_t * src.z));
}
LAM_DEV v3 from_onb(v3 src, v3 up, v3 tangent) {
    v3 s = tangent, t = cross(up, s);
    return fma3(splat(src.x), s, fma3(splat(src.y), up, t * src.z));
}
LAM_DEV v3 from_onb_no_tangent(v3 src, v3 up) {
    v3 other = near_zero(up.x) ? mk(1.0f, 0.0f, 0.0f) : mk(0.0f, 1.0f, 0.0f);
    return from_onb(src, up, normalize(cross(up, other)));
}
LAM_DEV v3 cosine_hemisphere(uint32_t seed, v3 n, v3 t) {
    float r1 = rand_f32(seed), r2 = rand_f32(seed + 1u);
    float phi = TAU_F * r1;
    v3 h = mk(cosf(phi) * sqrtf(r2), sqrtf(1.0f - r2), sinf(phi) * sqrtf(r2));
    return from_onb(h, n, t);
}
LAM_DEV v3 sample_vndf_ggx(uint32_t seed, v3 view, float2 rough) {
    float u1 = rand_f32(seed), u2 = rand_f32(seed + 1u);
    v3 in = mk(view.x * rough.x, view.y, view.z * rough.y);
    if (v3_near_zero(in)) in = mk(0.0f, -1.0f, 0.0f);
    v3 wi = normalize(in);
    float phi = TAU_F * u1;
    float y = fmaf(1.0f - u2, 1.0f + wi.y, -wi.y);
    float st = sqrtf(clampf(fmaf(y, -y, 1.0f), 0.0f, 1.0f));
    v3 wm = mk(st * cosf(phi), y, st * sinf(phi)) + wi;
    v3 out = mk(wm.x * rough.x, wm.y, wm.z * rough.y);
    if (v3_near_zero(out)) out = mk(0.0f, 1.0f, 0.0f);
    return normalize(out);
}
// Density (per solid angle) of the direction the reference's metallic bounce produces
// (general.wesl:718, 892-897).  get_normal hands sample_vndf_ggx V = to_onb(rd, n, t), and to_onb
// (shared.wesl:39-46) is not the inverse of from_onb: for an orthonormal frame it returns
// -from_onb(rd), so V is a fixed vector of the frame's coordinates, not rd seen from the surface.
// The sampler's point p is uniform on the cap {y >= -wi.y} of the unit sphere (wi = the stretched,
// normalised V); u = p + wi lies on the unit sphere through the origin; the microfacet normal is
// m = normalize(S u) with S = diag(ax, 1, ay), expressed through from_onb; the true incoming
// direction R (rd in from_onb's frame) is reflected about m and, when that points below the surface,
// mirrored about the normal.  Change of variables:
//   u -> direction:     4 (u . wi) / (2 pi (1 + wi.y))   on the cap's image
//   m = S u / |S u|:    dw_u / dw_m = 1 / (ax ay |S^-1 m|^3)
//   w = reflect(R, m):  dw_m / dw   = 1 / (4 |w . m|)
// and the mirror adds the density of the mirrored direction.
LAM_DEV float metal_raw_pdf(v3 R, v3 wi, float ax, float ay, v3 w) {
    v3 h = w - R;
    const float hl = len(h);
    if (!(hl > 0.0f)) return 0.0f;
    h = h * (1.0f / hl);
    if (h.y < 0.0f) h = -h;
    const v3 us = mk(h.x / ax, h.y, h.z / ay);
    const float ul = len(us);
    const v3 u = us * (1.0f / ul);
    const float uw = dot(u, wi);
    if (!(uw > 0.0f)) return 0.0f;
    const float py = 2.0f * uw * u.y - wi.y;  // the cap point p = 2 (u . wi) u - wi
    if (py < -wi.y) return 0.0f;
    const float dens_u = 4.0f * uw / (TAU_F * (1.0f + wi.y));
    const float dens_m = dens_u / (ax * ay * ul * ul * ul);
    const float wm = fabsf(dot(w, h));
    return wm > 0.0f ? dens_m / (4.0f * wm) : 0.0f;
}
LAM_DEV float metal_pdf(v3 rd, v3 n, v3 t, float ax, float ay, v3 w_world) {
    const v3 t3 = cross(n, t);  // from_onb's third axis
    const v3 W = mk(dot(w_world, t), dot(w_world, n), dot(w_world, t3));
    if (!(W.y > 0.0f)) return 0.0f;
    const v3 V = to_onb(rd, n, t);
    const v3 R = mk(dot(rd, t), dot(rd, n), dot(rd, t3));
    const v3 wi = normalize(mk(V.x * ax, V.y, V.z * ay));
    return metal_raw_pdf(R, wi, ax, ay, W) + metal_raw_pdf(R, wi, ax, ay, mk(W.x, -W.y, W.z));
}
// Metallic vertices the learned guide is mixed in at: a microfacet (Medium / High) reflection with no
// Fresnel choice (index ratio 1) and both roughnesses at least this
constexpr float METAL_GUIDE_MIN_ROUGHNESS = 0.1f;

LAM_DEV float reflectance(float c, float ri) {
    float r0 = (1.0f - ri) / (1.0f + ri);
    float r0s = r0 * r0;
    return fmaf(1.0f - r0s, powf(1.0f - c, 5.0f), r0s);
}
LAM_DEV v3 oren_nayar(v3 incoming, v3 reflected, float rough, v3 color) {
    float rr = rough * HALF_PI_F;
    float rr2 = rr * rr;
    v3 a = fma3(color * 0.17f, splat(rr2 / (rr2 + 0.13f)), splat(1.0f - (0.5f * (rr2 / (rr2 + 0.33f)))));
    float b = 0.45f * (rr2 / (rr2 + 0.09f));
    float s = fmaf(-reflected.y, incoming.y, dot(reflected, incoming));
    float t = 1.0f;
    if (s > 0.0f) {
        t = fmaxf(reflected.y, incoming.y);
        if (near_zero(t)) t = 0.001f;
    }
    return fma3(splat(b), splat(s / t), a);
}
LAM_DEV float g_lobe(float x, float u, float t1, float t2) {
    float tau = x < u ? t1 : t2;
    float dd = x - u;
    return expf(-((dd * dd) * (tau * tau)) * 0.5f);
}

// ---------------------------------------------------------------- wave buffers
// lobes of the Markov mixture kept for the learned-guide kernel: one per resampling candidate
constexpr uint32_t MIX_LOBES = NUM_RESAMPLES;

struct WaveBuffers {
    uint32_t width = 0, height = 0, npix = 0, spp_wave = 0;
    uint64_t paths = 0;
    bool full = false, guide = false;
    bool mem_capped = false;  // spp_wave was reduced to fit device memory
    float4 *ray_o = nullptr, *ray_d = nullptr, *ray_o2 = nullptr, *ray_d2 = nullptr;  // two queues' rays
    float4 *qthr0 = nullptr, *qthr1 = nullptr, *qacc0 = nullptr, *qacc1 = nullptr;  // two queues' path state
    uint4 *qmisc0 = nullptr, *qmisc1 = nullptr;
    uint2* hit = nullptr;
    uint32_t *queue0 = nullptr, *queue1 = nullptr;
    float4 *thr = nullptr, *acc = nullptr;
    float* brdf = nullptr;
    uint32_t *seed = nullptr, *flags = nullptr;
    // restir / guide state
    float4 *ort = nullptr, *orad = nullptr, *ppoint = nullptr, *pnormal = nullptr, *vpoint = nullptr,
           *vnormal = nullptr, *lnormal = nullptr, *ldir = nullptr;
    // per pixel
    float4 *pix_color = nullptr, *pix_orad = nullptr, *pix_emission = nullptr, *pix_albedo = nullptr;
    lam_markov_chain *tent_snap = nullptr, *tent_live = nullptr;
    // learned guiding: deferred diffuse vertices and the per-path training-record lists
    bool learned = false;
    uint32_t* dq = nullptr;
    float4 *def_n = nullptr, *def_t = nullptr, *def_c = nullptr, *def_o = nullptr, *def_d = nullptr, *def_a = nullptr;
    uint32_t* rec_head = nullptr;
    float4 *def_r = nullptr, *def_lobe = nullptr;  // the Markov sampler's or the metal's draw; Markov lobes
    float* def_lw = nullptr;
    uint32_t* def_kind = nullptr;                  // DEF_DIFFUSE / DEF_METAL
    float4 *phit_a = nullptr, *phit_b = nullptr;  // procedural hits (allocated on first use)
    uint8_t* shade_key = nullptr;                  // material-ordered shading (allocated on first use)
    uint32_t *shade_order = nullptr, *shade_bc = nullptr;
    uint32_t* ctr = nullptr;  // [0..1] queue counts, [2..3] work counters, [4] error flags,
                              // [8..11] segment counters, [12] diffuse-queue count, [13] records
    std::vector<void*> allocs;
    int sms = 148, grid_extend = 0, grid_shade = 0, grid_guide = 0, grid_sort = 0;
};

static void free_wave(WaveBuffers* w) {
    if (!w) return;
    for (void* p : w->allocs) cudaFree(p);
    delete w;
}

template <class T>
static int walloc(WaveBuffers* w, T** p, size_t count) {
    *p = nullptr;
    if (!count) return LAM_OK;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (wavefront state)");
    w->allocs.push_back(*p);
    return LAM_OK;
}

LAM_DEV void create_ray(const Args& A, uint32_t x, uint32_t y, v3* o, v3* d) {
    float hx = __uint2float_rn(A.width) / 2.0f, hy = __uint2float_rn(A.height) / 2.0f;
    float nx = (__uint2float_rn(x) / hx) - 1.0f, ny = (__uint2float_rn(y) / hy) - 1.0f;
    float v[4] = {nx, -ny, 1.0f, 1.0f};
    const float* P = A.cam.projection_inverse;
    float q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = P[i] * v[0] + P[4 + i] * v[1] + P[8 + i] * v[2] + P[12 + i] * v[3];
    float l = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = q[i] / l;
    const float* V = A.cam.view_inverse;
    *d = mk(V[0] * q[0] + V[4] * q[1] + V[8] * q[2] + V[12] * 0.0f, V[1] * q[0] + V[5] * q[1] + V[9] * q[2] + V[13] * 0.0f,
            V[2] * q[0] + V[6] * q[1] + V[10] * q[2] + V[14] * 0.0f);
    *o = A.camera_pos;
}

LAM_DEV uint32_t advance_fill_seed(uint32_t s) {
#pragma unroll 4
    for (int i = 0; i < 12; ++i) {
        s = rand_u32(s);
        s = rand_u32(s);
    }
    return s;
}

// ---------------------------------------------------------------- generate
__global__ void __launch_bounds__(WAVE_BLOCK) generate_kernel(Args A) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) *A.count_in = A.npix * A.wave_count;
    if (p >= A.npix) return;
    const uint32_t x = p % A.width, y = p / A.width;
    uint32_t st;
    if (A.wave_first == 0u) {
        st = rand_u32(x * y) + A.seed_offset + y;
        A.pix_color[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (A.pix_orad) A.pix_orad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (A.tent_live) {
            MC t = (A.old_chains && p < A.old_chains_len) ? mc_load(A.old_chains + p) : mc_zero();
            mc_store(A.tent_live + p, t);
            mc_store(A.tent_snap + p, t);
        }
        if (A.reservoirs && A.restir == LAM_RESTIR_PER_SAMPLE) A.reservoirs[p] = lam_reservoir{};
    } else {
        st = A.pixel_seed[p];
        if (A.tent_live) mc_store(A.tent_live + p, mc_load(A.tent_snap + p));
    }
    v3 o, d;
    create_ray(A, x, y, &o, &d);
    for (uint32_t j = 0; j < A.wave_count; ++j) {
        const uint32_t path = j * A.npix + p;
        const uint32_t fill_seed = st;
        st = advance_fill_seed(st);
        A.ray_o[path] = make_float4(o.x, o.y, o.z, 0.0f);
        A.ray_d[path] = make_float4(d.x, d.y, d.z, 0.0f);
        A.qthr[path] = make_float4(1.0f, 1.0f, 1.0f, -1.0f);
        A.qacc[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        A.qmisc[path] = make_uint4(0u, st, 0u, 0u);
        if (A.ort) {
            A.ort[path] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            A.orad[path] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            A.ppoint[path] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(TY_SKY));
            A.pnormal[path] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(fill_seed));
            A.vpoint[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            A.vnormal[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (A.lnormal) {
            A.lnormal[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            A.ldir[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (A.rec_head) A.rec_head[path] = NO_REC;
        A.q_in[path] = path;
        st = rand_u32(st);
    }
    A.pixel_seed[p] = st;
}

// ---------------------------------------------------------------- extend
template <bool ALPHA>
__global__ void __launch_bounds__(WAVE_BLOCK) extend_kernel(Args A) {
    __shared__ TraceSmem sm;
    const uint4* tl;
    const DevInstance* in;
    stage_tlas(A.S, sm, tl, in);
    const uint32_t n = *A.count_in;
    const uint32_t lane = threadIdx.x & 31u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(A.segments, (unsigned long long)n);      // this render
        atomicAdd(A.segments + 1, (unsigned long long)n);  // since the pipeline's buffers were created
    }
    uint32_t err = 0u;
    (void)lane;
    trace_persistent<false, ALPHA>(
        A.S, tl, in, n, A.work, err,
        [&](uint32_t i, float3& o, float3& d, float& t0, float& t1) {
            const float4 o4 = ld_stream(A.ray_o + i), d4 = ld_stream(A.ray_d + i);
            o = make_float3(o4.x, o4.y, o4.z);
            d = make_float3(d4.x, d4.y, d4.z);
            t0 = A.tmin;
            t1 = A.tmax;
        },
        [&](uint32_t i, const TraceResult& tr) { A.hit[i] = make_uint2(tr.tri, tr.inst); });
    if (err) atomicOr(A.err, err);
}

// ---------------------------------------------------------------- shade (one bounce of rt_sample)
template <int Q, bool GUIDE>
struct Shader {
    LAM_DEV static v3 get_normal(v3 rd, v3 n, v3 t, uint32_t seed, float2 rough) {
        if (Q == LAM_QUALITY_LOW) return n;
        return from_onb(sample_vndf_ggx(seed, to_onb(rd, n, t), rough), n, t);
    }
    LAM_DEV static v3 make_diffuse(v3 hit_color, v3 rd, v3 n, v3 t, float rough, v3 new_dir) {
        if (Q == LAM_QUALITY_LOW) return splat(1.0f);
        return oren_nayar(to_onb(rd, n, t), new_dir, rough, hit_color);
    }
    // returns (weights.xyz, ior); picked_idx < 0 means "not picked yet"
    LAM_DEV static float4 pick_ref_idx(float* picked_idx, float low, float high, uint32_t seed) {
        if (Q == LAM_QUALITY_LOW) return make_float4(1.0f, 1.0f, 1.0f, low);
        if (Q == LAM_QUALITY_MEDIUM) {
            if (*picked_idx < 0.0f) *picked_idx = rand_f32(seed);
            return make_float4(1.0f, 1.0f, 1.0f, mixf(low, high, *picked_idx));
        }
        if (*picked_idx < 0.0f) {
            float pi = rand_f32(seed);
            *picked_idx = pi;
            float lambda = mixf(760.0f, 340.0f, pi);
            float x = fmaf(1.056f, g_lobe(lambda, 599.8f, 0.0264f, 0.0323f),
                           fmaf(0.362f, g_lobe(lambda, 442.0f, 0.0624f, 0.0374f), -(0.065f * g_lobe(lambda, 501.1f, 0.049f, 0.0382f))));
            float y = fmaf(0.821f, g_lobe(lambda, 568.8f, 0.0213f, 0.0248f), 0.286f * g_lobe(lambda, 530.9f, 0.0613f, 0.0322f));
            float z = fmaf(1.217f, g_lobe(lambda, 437.0f, 0.0845f, 0.0278f), 0.681f * g_lobe(lambda, 459.0f, 0.0385f, 0.0725f));
            v3 rgb = mk(3.2406f, -0.9689f, 0.0557f) * x + mk(-1.5372f, 1.8758f, -0.204f) * y + mk(-0.4986f, 0.0415f, 1.057f) * z;
            return make_float4(saturate(rgb.x) * 3.910f, saturate(rgb.y) * 4.411f, saturate(rgb.z) * 5.511f, mixf(low, high, pi));
        }
        return make_float4(1.0f, 1.0f, 1.0f, mixf(low, high, *picked_idx));
    }
};

// 16 screen-space candidates of the sample (general.wesl:367-385), recomputed from the seed the
// sample started its fill with.
// The 21 resampling candidates of a Markov-guided bounce, in shared memory while the bounce is
// shaded: field major with one column per thread (conflict-free), the six words of a chain that
// resampling and the mixture read (light xyz, mean cosine, weight sum, sample count); 64.5 KB per
// 128-thread CTA.  As a per-thread array they lived in local memory (616 bytes of stack per thread,
// spilling out of L1 at 12 warps per SM); here the ReSTIR GI frame loop runs 3% faster.  Five words
// (kappa computed when a candidate is stored) with four CTAs per SM at 128 registers was slower:
// 23.7 against 19.9 ms per frame.
constexpr uint32_t CAND_WORDS = 6;
constexpr uint32_t CAND_SMEM = CAND_WORDS * NUM_RESAMPLES * WAVE_BLOCK * sizeof(float);
constexpr uint32_t GUIDE_SHADE_SMEM = CAND_SMEM;  // dynamic shared memory of the guided shade kernel
struct Cands {
    float* b;  // this thread's column
    LAM_DEV float* at(int k, int f) const { return b + (k * (int)CAND_WORDS + f) * WAVE_BLOCK; }
    LAM_DEV void put(int k, const MC& m) {
        *at(k, 0) = m.light.x;
        *at(k, 1) = m.light.y;
        *at(k, 2) = m.light.z;
        *at(k, 3) = m.mean_cosine;
        *at(k, 4) = m.weight_sum;
        *at(k, 5) = __uint_as_float(m.num_samples);
    }
    LAM_DEV MC get(int k) const {
        MC m;
        m.light = mk(*at(k, 0), *at(k, 1), *at(k, 2));
        m.mean_cosine = *at(k, 3);
        m.weight_sum = *at(k, 4);
        m.num_samples = __float_as_uint(*at(k, 5));
        m.score = 0.0f;
        return m;
    }
    LAM_DEV float weight(int k) const { return *at(k, 4); }
};

LAM_DEV void screen_candidates(const Args& A, uint32_t pixel, uint32_t fill_seed, Cands& cand) {
    const uint32_t x = pixel % A.width, y = pixel / A.width;
    const uint32_t gbase = x & ~31u;
    uint32_t s = fill_seed;
    const uint32_t sub = rand_u32(s) % 32u;
    MC sh = (gbase + sub < A.width) ? mc_load(A.tent_snap + (uint64_t)y * A.width + gbase + sub) : mc_zero();
    for (int i = 0; i < 4; ++i) cand.put(i, sh);
#pragma unroll 1
    for (int i = 4; i < 16; ++i) {
        uint32_t xr = rand_u32(s);
        s = xr;
        uint32_t yr = rand_u32(s);
        s = yr;
        int32_t dx = (int32_t)(xr % 91u) - 45, dy = (int32_t)(yr % 91u) - 45;
        uint32_t nx = (uint32_t)((int32_t)x + dx), ny = (uint32_t)((int32_t)y + dy);
        uint64_t idx = (uint32_t)(nx + ny * A.width);
        if (A.old_chains && A.old_chains_len) {
            idx = idx < A.old_chains_len ? idx : A.old_chains_len - 1;
            cand.put(i, mc_load(A.old_chains + idx));
        } else {
            cand.put(i, mc_zero());
        }
    }
}

// Learned guiding: colour-weighted luminance of the radiance a path carried back to each recorded
// vertex, (scol_final - scol_vertex) / throughput_vertex, written as the record's training weight.
LAM_DEV void finalize_records(const Args& A, uint32_t path, v3 scol) {
    uint32_t r = A.rec_head[path];
    for (int guard = 0; r != NO_REC && guard < 256; ++guard) {
        float* R = A.recs + (size_t)r * GUIDE_RECORD_STRIDE;
        const float c[3] = {scol.x - R[16], scol.y - R[17], scol.z - R[18]};
        const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
        float w = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (R[13 + k] > 0.0f && c[k] > 0.0f) w += lw[k] * (c[k] / R[13 + k]);
        R[12] = (w < 3.0e38f) ? w : 0.0f;
        r = __float_as_uint(R[19]);
    }
}

// ---------------------------------------------------------------- material-ordered shading
// A stable counting sort of the queue by shading class (sky, diffuse, metallic, transparent), so that
// the shade kernel runs one class at a time across the whole GPU: its warps take one branch, and
// every SM's caches hold one class's code, materials and textures.  (A sort within blocks, whose
// warps are as uniform, gave no gain: the grid-wide order is what pays.)  The three kernels split
// the queue into one contiguous chunk per block: count the classes of the chunk, scan the counts
// (class major, then block), and write each position to its slot in the order.  Within a class the
// queue order is kept, so the shade kernel's reads stay nearly sequential.  A procedural hit's
// leaf record holds its primitive in the same word as a triangle's.

// The chunk of queue positions [*beg, *end) of block b of nb (a multiple of the block size).
LAM_DEV void sort_chunk(uint32_t n, uint32_t b, uint32_t nb, uint32_t* beg, uint32_t* end) {
    const uint32_t per = (n + nb - 1u) / nb;
    const uint32_t c = (per + WAVE_BLOCK - 1u) / WAVE_BLOCK * WAVE_BLOCK;
    *beg = min(n, b * c);
    *end = min(n, *beg + c);
}

// BATCH: each path's scene is its request's (lam_batch_render).
template <bool BATCH>
__global__ void __launch_bounds__(WAVE_BLOCK) shade_keys_kernel(const __grid_constant__ Args A) {
    __shared__ uint32_t cnt[SHADE_CLASSES];
    if (threadIdx.x < SHADE_CLASSES) cnt[threadIdx.x] = 0u;
    __syncthreads();
    uint32_t beg, end;
    sort_chunk(*A.count_in, blockIdx.x, gridDim.x, &beg, &end);
    const uint32_t lane = threadIdx.x & 31u;
    // U tiles per step, each stage's loads issued for all of them before the next stage's: a class
    // is a chain of four dependent loads (hit; triangle word and instance; material index; material)
    constexpr uint32_t U = 4;
    for (uint32_t t = beg; t < end; t += U * WAVE_BLOCK) {
        bool v[U];
        uint2 h[U];
        const DevScene* S[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint32_t j = t + q * WAVE_BLOCK + threadIdx.x;
            v[q] = j < end;
            S[q] = &A.S;
            // plain loads: the shade kernel reads the hit (and a batched path's flags) again next
            if (BATCH && v[q]) S[q] = &A.reqs[A.segs[A.qmisc[j].z >> 16].req].S;
            h[q] = v[q] ? A.hit[j] : make_uint2(NO_HIT, 0u);
        }
        uint32_t prim[U], mcount[U], moff[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const bool hit = h[q].x != NO_HIT;
            prim[q] = hit ? __float_as_uint(ld_keep(S[q]->tris + 3u * h[q].x).w) : 0u;
            mcount[q] = hit ? S[q]->inst[h[q].y].mat_count : 0u;
            moff[q] = hit ? S[q]->inst[h[q].y].mat_offset : 0u;
        }
        uint32_t mi[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q)
            mi[q] = clamp_idx(mcount[q] ? __ldg(S[q]->mat_idx + moff[q] + clamp_idx(prim[q], mcount[q])) : 0u,
                              S[q]->material_count);
        uint32_t k[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint32_t j = t + q * WAVE_BLOCK + threadIdx.x;
            k[q] = SHADE_CLASSES;
            if (v[q]) {
                if (h[q].x == NO_HIT) {
                    k[q] = SHADE_SKY;
                } else {
                    // tex_idx_attributes_ty: the type in its upper half (as load_material reads it)
                    const uint32_t ty = __ldg(reinterpret_cast<const uint32_t*>(S[q]->materials + mi[q]) + 5) >> 16;
                    k[q] = ty == TY_METALLIC ? SHADE_METALLIC : (ty == TY_TRANSPARENT ? SHADE_TRANSPARENT : SHADE_DIFFUSE);
                }
                A.shade_key[j] = (uint8_t)k[q];
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < U; ++q)
#pragma unroll
            for (uint32_t c = 0; c < SHADE_CLASSES; ++c) {
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, k[q] == c);
                if (lane == 0u && m) atomicAdd(&cnt[c], (uint32_t)__popc(m));
            }
    }
    __syncthreads();
    if (threadIdx.x < SHADE_CLASSES) A.shade_bc[blockIdx.x * SHADE_CLASSES + threadIdx.x] = cnt[threadIdx.x];
}

// One block of SORT_BLOCKS_MAX threads: thread b turns block b's counts into its first slot per
// class (exclusive, class-major: all of class 0, then class 1, ...).
__global__ void __launch_bounds__(SORT_BLOCKS_MAX) shade_scan_kernel(const __grid_constant__ Args A, uint32_t nb) {
    __shared__ uint32_t warp_sum[SORT_BLOCKS_MAX / 32];
    __shared__ uint32_t class_base;
    const uint32_t b = threadIdx.x, lane = b & 31u, wid = b >> 5;
    if (b == 0u) class_base = 0u;
    for (uint32_t c = 0; c < SHADE_CLASSES; ++c) {
        const uint32_t v = b < nb ? A.shade_bc[b * SHADE_CLASSES + c] : 0u;
        uint32_t x = v;  // inclusive scan within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31u) warp_sum[wid] = x;
        __syncthreads();
        if (wid == 0u) {
            uint32_t s = warp_sum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
                if (lane >= (uint32_t)o) s += y;
            }
            warp_sum[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = (wid ? warp_sum[wid - 1u] : 0u) + x - v;
        if (b < nb) A.shade_bc[b * SHADE_CLASSES + c] = class_base + before;
        __syncthreads();
        if (b == 0u) class_base += warp_sum[SORT_BLOCKS_MAX / 32 - 1];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(WAVE_BLOCK) shade_scatter_kernel(const __grid_constant__ Args A) {
    // U tiles per step: their ranks come from one pass of ballots, so that a step takes three
    // barriers instead of three per tile
    constexpr uint32_t NW = WAVE_BLOCK / 32, U = 4;
    __shared__ uint32_t wcnt[U][NW][SHADE_CLASSES];
    __shared__ uint32_t next[SHADE_CLASSES];
    if (threadIdx.x < SHADE_CLASSES) next[threadIdx.x] = A.shade_bc[blockIdx.x * SHADE_CLASSES + threadIdx.x];
    __syncthreads();
    uint32_t beg, end;
    sort_chunk(*A.count_in, blockIdx.x, gridDim.x, &beg, &end);
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    for (uint32_t t = beg; t < end; t += U * WAVE_BLOCK) {
        uint32_t k[U], rank[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint32_t j = t + q * WAVE_BLOCK + threadIdx.x;
            k[q] = j < end ? (uint32_t)A.shade_key[j] : SHADE_CLASSES;
            rank[q] = 0u;
#pragma unroll
            for (uint32_t c = 0; c < SHADE_CLASSES; ++c) {
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, k[q] == c);
                if (k[q] == c) rank[q] = (uint32_t)__popc(m & below);
                if (lane == 0u) wcnt[q][wid][c] = (uint32_t)__popc(m);
            }
        }
        __syncthreads();
        // a position's slot: its class's next slot, then the earlier tiles' and earlier warps' lanes
        // of its class, then its rank within its warp (stable: tiles, warps and lanes in order)
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            if (k[q] < SHADE_CLASSES) {
                uint32_t slot = next[k[q]] + rank[q];
                for (uint32_t p = 0; p < q; ++p)
                    for (uint32_t w = 0; w < NW; ++w) slot += wcnt[p][w][k[q]];
                for (uint32_t w = 0; w < wid; ++w) slot += wcnt[q][w][k[q]];
                A.shade_order[slot] = t + q * WAVE_BLOCK + threadIdx.x;
            }
        }
        __syncthreads();
        if (threadIdx.x < SHADE_CLASSES) {
            uint32_t add = 0u;
#pragma unroll
            for (uint32_t q = 0; q < U; ++q)
#pragma unroll
                for (uint32_t w = 0; w < NW; ++w) add += wcnt[q][w][threadIdx.x];
            next[threadIdx.x] += add;
        }
        __syncthreads();
    }
}

template <int Q, bool GUIDE, bool LEARN, bool BATCH>
// Six CTAs per SM for the unguided forms: the kernel waits on chains of dependent gathers (queue ->
// hit -> triangle -> material -> texture), so resident warps matter more than the few registers
// that spill (measured: 79 ms against 87 ms per 16-spp step at 1080p).  The Markov-guided forms keep
// their registers (160; three CTAs per SM, which their shared-memory candidates also allow).
__global__ void __launch_bounds__(WAVE_BLOCK, (GUIDE ? 1 : 6)) shade_kernel(const __grid_constant__ Args A) {
    const uint32_t n = *A.count_in;
    const uint32_t lane = threadIdx.x & 31u;
    Grid G;
    G.world = A.world;
    G.old_world = A.old_world;
    G.len = A.world_len;
    G.mod_m = A.world_mod_m;
    G.camera_loc = A.camera_pos;
    const bool rec = A.ort != nullptr;
    // learned guiding without Markov chains: what the bounce decides for a deferred vertex (normal and
    // roughness, tangent and seed, albedo or the metal's reflection), held per thread until the append
    // at the end gives the vertex its slot in the guide kernel's queue, where it is then written
    constexpr bool STASH = LEARN && !GUIDE;
    __shared__ float4 def_stash[STASH ? 3 : 1][STASH ? WAVE_BLOCK : 1];
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;; base += gridDim.x * blockDim.x) {
        if (base >= n) break;
        const uint32_t j = base + lane;  // work item; i: the queue position it shades
        const uint32_t i = (A.shade_order && j < n) ? A.shade_order[j] : j;
        {
            // the next iteration's queue-ordered inputs have known addresses: start them towards L2
            const uint32_t jnext = j + gridDim.x * blockDim.x;
            if (jnext < n) {
                if (A.shade_order) {
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.shade_order + jnext));
                } else {
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.q_in + jnext));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.hit + jnext));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.ray_o + jnext));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.ray_d + jnext));
                }
            }
        }
        bool cont = false, deferred = false;
        uint32_t def_kind = DEF_DIFFUSE;  // with `deferred`: what kind of vertex the guide kernel gets
        uint32_t path = 0;
        v3 ro = splat(0.0f), rd = splat(0.0f);  // the outgoing ray once the bounce is shaded
        float seg_w = 0.0f;                     // a batched path's segment, carried in the ray's w
        float4 o_thr = make_float4(0.0f, 0.0f, 0.0f, 0.0f), o_acc = o_thr;  // the outgoing state
        uint4 o_misc = make_uint4(0u, 0u, 0u, 0u);
        if (i < n) {
            path = A.q_in[i];
            const uint4 misc = ld_stream(A.qmisc + i);
            uint32_t fl = misc.z;
            // per-render fields; a batched render takes them from the path's request
            const DevScene* Sp = &A.S;
            uint32_t pixel, sample_index, samples = A.samples;
            float4 *out_normal = A.out_normal, *out_albedo = A.out_albedo;
            if (BATCH) {
                const BatchSeg sg = A.segs[fl >> 16];
                const BatchReq& R = A.reqs[sg.req];
                Sp = &R.S;
                const uint32_t rel = path - sg.path_base;
                pixel = rel % R.npix;
                sample_index = sg.first + rel / R.npix;
                samples = R.samples;
                out_normal = R.out_normal;
                out_albedo = R.out_albedo;
            } else {
                pixel = path % A.npix;
                sample_index = A.wave_first + path / A.npix;
            }
            const DevScene& S = *Sp;
            const bool last_sample = sample_index + 1u == samples;
            const uint32_t depth = fl & 0xFFu;
            bool last_not_vmf = (fl >> 8) & 1u;
            const float4 o4 = ld_stream(A.ray_o + i), d4 = ld_stream(A.ray_d + i);
            ro = mk(o4.x, o4.y, o4.z);
            rd = mk(d4.x, d4.y, d4.z);
            seg_w = o4.w;
            float4 th = ld_stream(A.qthr + i);
            v3 color = mk(th.x, th.y, th.z);
            float picked = th.w;
            float4 ac = ld_stream(A.qacc + i);
            v3 scol = mk(ac.x, ac.y, ac.z);
            float cached_pdf = ac.w, cached_brdf = __uint_as_float(misc.x);
            uint32_t seed = misc.y;
            v3 orc = splat(1.0f), orad = splat(0.0f);
            float sum_mc = 0.0f;
            float4 pp = make_float4(0, 0, 0, 0), pn = make_float4(0, 0, 0, 0);
            if (rec) {
                float4 t0 = A.ort[path], t1 = A.orad[path];
                orc = mk(t0.x, t0.y, t0.z);
                sum_mc = t0.w;
                orad = mk(t1.x, t1.y, t1.z);
                pp = A.ppoint[path];
                pn = A.pnormal[path];
            }
            v3 last_normal = splat(0.0f), last_dir = splat(0.0f);
            if (GUIDE) {
                float4 a = A.lnormal[path], b = A.ldir[path];
                last_normal = mk(a.x, a.y, a.z);
                last_dir = mk(b.x, b.y, b.z);
            }
            MC tentative = GUIDE ? mc_load(A.tent_live + pixel) : mc_zero();
            const uint2 h = ld_stream(A.hit + i);  // hits are stored by queue position (extend shares this queue)
            bool terminated = false;
            const bool hit = h.x != NO_HIT;
            Isect is;
            v3 new_pos, bg = splat(0.0f);
            // what the chain updates take from either branch: radiance arriving at ro, its emitted
            // part, and whether the previous direction came from the cosine lobe
            v3 g_rad = splat(0.0f), g_out = splat(0.0f);
            bool g_nvmf = false;
            if (hit) {
                make_isect(S, S.inst, h, make_float3(ro.x, ro.y, ro.z), make_float3(rd.x, rd.y, rd.z), is, A.phit_a,
                           A.phit_b, path);
                new_pos = fma3(rd, splat(is.t), ro);
                if (depth != 0u) {
                    v3 est = GUIDE ? grid_radiance(G, new_pos, is.normal, rd) : splat(0.0f);
                    v3 rad_refl = strip_nan3(((is.color * est) * cached_brdf) / cached_pdf);
                    v3 rad_out = (is.emission * cached_brdf) / cached_pdf;
                    g_rad = rad_out + rad_refl;
                    g_out = rad_out;
                    g_nvmf = last_not_vmf;
                }
            } else {
                bg = sky_sample(S, rd);
                new_pos = fma3(rd, splat(A.tmax), ro);
                if (depth == 1u && rec) {
                    A.vpoint[path] = make_float4(new_pos.x, new_pos.y, new_pos.z, 0.0f);
                    A.vnormal[path] = make_float4(-rd.x, -rd.y, -rd.z, 0.0f);
                }
                if (depth == 0u && last_sample) {
                    if (out_normal) out_normal[pixel] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                    if (out_albedo) out_albedo[pixel] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                    if (A.pix_emission) {
                        A.pix_emission[pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        A.pix_albedo[pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    }
                }
                if (depth != 0u) {
                    orad = fma3(orc, bg, orad);
                    g_rad = (bg * cached_brdf) / cached_pdf;
                    g_out = g_rad;
                }
            }
            // one call site for the chain updates of hit and sky lanes (general.wesl:677-684 and
            // :928-935 run the same updates), so a warp with both kinds runs them once
            if (depth != 0u) {
                if (GUIDE) grid_add_radiance_warp(G, ro, last_normal, last_dir, g_rad);
                float weight = len(g_rad);
                if (weight > 0.0f) {
                    if (GUIDE) {
                        MC st = update_chain(ro, new_pos, weight, seed, false, grid_load(G, ro, last_normal, last_dir, false),
                                             1.0f, sum_mc);
                        grid_store_warp(G, ro, last_normal, last_dir, st);
                        tentative = update_chain(ro, new_pos, len(g_out), seed, g_nvmf, tentative,
                                                 depth == 1u ? 1.0f : 0.5f, sum_mc);
                    }
                    seed++;
                }
            }
            if (hit) {
                last_normal = is.normal;
                last_dir = rd;
                last_not_vmf = false;
                ro = new_pos;
                if (depth == 0u) {
                    if (rec) {
                        pp = make_float4(ro.x, ro.y, ro.z, __uint_as_float(is.ty));
                        pn = make_float4(is.normal.x, is.normal.y, is.normal.z, pn.w);
                    }
                    if (last_sample) {
                        if (out_normal) out_normal[pixel] = make_float4(is.normal.x, is.normal.y, is.normal.z, 1.0f);
                        if (out_albedo) out_albedo[pixel] = make_float4(is.color.x, is.color.y, is.color.z, 1.0f);
                        if (A.pix_emission) {
                            A.pix_emission[pixel] = make_float4(is.emission.x, is.emission.y, is.emission.z, 0.0f);
                            A.pix_albedo[pixel] = make_float4(is.color.x, is.color.y, is.color.z, 0.0f);
                        }
                    }
                } else if (depth == 1u && rec) {
                    A.vpoint[path] = make_float4(ro.x, ro.y, ro.z, 0.0f);
                    A.vnormal[path] = make_float4(is.normal.x, is.normal.y, is.normal.z, 0.0f);
                }
                scol = fma3(color, is.emission, scol);
                if (depth != 0u) orad = fma3(orc, is.emission, orad);
                v3 assign_normal = Shader<Q, GUIDE>::get_normal(rd, is.normal, is.tangent, seed, is.roughness);
                v3 normal = Shader<Q, GUIDE>::get_normal(rd, is.normal, is.tangent, seed, is.roughness_transparent);
                bool should_reflect = false;
                seed += 1u;
                float4 cri = Shader<Q, GUIDE>::pick_ref_idx(&picked, is.ior_low, is.ior_high, seed);
                float ri = cri.w;
                seed += 1u;
                if (!(!is.front_face && is.ty == TY_TRANSPARENT)) ri = 1.0f / ri;
                v3 cw = mk(cri.x, cri.y, cri.z);
                color = color * cw;
                orc = orc * cw;
                if (ri != 1.0f) {
                    float cos_theta = fminf(dot(-rd, normal), 1.0f);
                    float sin_theta = sqrtf(1.0f - (cos_theta * cos_theta));
                    bool cannot_refract = (ri * sin_theta) > 1.0f;
                    float pdf = reflectance(cos_theta, ri);
                    if (cannot_refract || (pdf > rand_f32(seed))) should_reflect = true;
                    seed += 1u;
                }
                if (!should_reflect || is.ty == TY_TRANSPARENT) {
                    color = color * is.color;
                    if (depth != 0u) orc = orc * is.color;
                }
                if (!should_reflect) {
                    normal = assign_normal;
                    seed += 1u;
                }
                // fill_mc_world_space_states + resample_mcmm (general.wesl:389-425)
                extern __shared__ float cand_smem[];  // GUIDE_SHADE_SMEM bytes in the guided kernels, else none
                Cands cand{cand_smem + threadIdx.x};
                MC s = mc_zero();
                if (GUIDE) {
                    screen_candidates(A, pixel, __float_as_uint(pn.w), cand);
                    // the four world-space candidates: their jittered positions first (the seed
                    // advances as in general.wesl:390-398), then their cells' reads together
                    {
                        v3 wpos[4];
                        bool wold[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            bool rc = rand_f32(seed) < 0.7f;
                            float jm = rc ? 0.75f : 1.0f;
                            float j0 = rand_f32_ptr(&seed);
                            float j1 = rand_f32_ptr(&seed);
                            v3 jit = (mk(j0, 0.0f, j1) * 0.15000000596046448f) * jm;
                            wpos[q] = ro + from_onb_no_tangent(jit, is.normal);
                            wold[q] = rc;
                            seed += 1u;
                        }
                        MC wc[4];
                        grid_load_n<4>(G, wpos, is.normal, rd, wold, wc);
#pragma unroll
                        for (int q = 0; q < 4; ++q) cand.put(16 + q, wc[q]);
                    }
                    cand.put(20, tentative);
                    sum_mc = 0.0f;
                    int sel = -1;
                    // the resampling loop stays rolled: the guided kernel is large, and unrolled its
                    // candidate loops needed 222 registers (2 CTAs per SM) and stalled on instruction fetch
#pragma unroll 1
                    for (int k = 0; k < NUM_RESAMPLES; ++k) {
                        seed = rand_u32(seed);
                        const float wk = cand.weight(k);
                        sum_mc += wk;
                        if (rand_f32(seed) * sum_mc < wk) sel = k;
                        seed = rand_u32(seed);
                    }
                    if (sel >= 0) s = cand.get(sel);
                } else {
                    for (int k = 16; k < 20; ++k) {
                        seed = rand_u32(rand_u32(seed)) + 1u;
                    }
#pragma unroll 7
                    for (int k = 0; k < NUM_RESAMPLES; ++k) seed = rand_u32(rand_u32(seed));
                }
                const bool reflecting = should_reflect || is.ty == TY_METALLIC;
                if (!reflecting) {
                    if (LEARN && !GUIDE && is.ty == TY_DIFFUSE && depth + 1u < A.max_depth) {
                        // the guide kernel draws the direction; it uses the seeds of the cosine branch
                        deferred = true;
                        def_kind = DEF_DIFFUSE;
                        def_stash[0][threadIdx.x] = make_float4(is.normal.x, is.normal.y, is.normal.z, is.roughness.x);
                        def_stash[1][threadIdx.x] = make_float4(is.tangent.x, is.tangent.y, is.tangent.z, __uint_as_float(seed));
                        def_stash[2][threadIdx.x] = make_float4(is.color.x, is.color.y, is.color.z, 0.0f);
                        seed += 3u;
                    } else if (is.ty == TY_DIFFUSE) {
                        v3 dir_cos = cosine_hemisphere(seed, is.normal, is.tangent);
                        float cos_pdf = fmaxf(dot(dir_cos, is.normal) / PI_F, 0.0f);
                        float theta = rand_f32(seed) * TAU_F;
                        seed += 1u;
                        float xi = rand_f32(seed);
                        seed += 1u;
                        float c0 = 1.0f, c1 = 0.0f;
                        v3 dir_markov = splat(0.0f);
                        if (GUIDE) {
                            v3 ld = light_dir(s, ro);
                            v3 mean = normalize(ld);
                            float kappa = get_kappa(s);
                            float W1 = logf(1.0f + (xi * exp_minus_one(-2.0f * kappa))) / kappa;
                            float W = 1.0f + W1;
                            float nV = sqrtf(-fmaf(W1, W1, 2.0f * W1));
                            v3 Xs = from_onb_no_tangent(mk(strip_nan(cosf(theta) * nV), W, strip_nan(sinf(theta) * nV)), mean);
                            dir_markov = normalize(Xs);
                            float u0 = 0.2f, u1 = 0.8f;
                            if (!(s.weight_sum > 0.0f) || near_zero(len(ld)) || near_zero(s.weight_sum) || near_zero(len(Xs))) {
                                u0 = 1.0f;
                                u1 = 0.0f;
                            }
                            float cs = u0 + u1;
                            c0 = u0 / cs;
                            c1 = u1 / cs;
                        }
                        float rnd = rand_f32(seed);
                        seed += 1u;
                        v3 dir;
                        if (rnd < c0) {
                            dir = dir_cos;
                            last_not_vmf = true;
                        } else {
                            dir = dir_markov;
                        }
                        float mix_pdf = 0.0f;
                        if (GUIDE && c1 != 0.0f && sum_mc > 0.0f) {
#pragma unroll 1
                            for (int k = 0; k < NUM_RESAMPLES; ++k) {
                                if (!(cand.weight(k) > 0.0f)) continue;
                                const MC ck = cand.get(k);
                                mix_pdf += vmf_pdf_fast(normalize(light_dir(ck, ro)), get_kappa(ck), dir) *
                                           (ck.weight_sum / sum_mc);
                            }
                        }
                        // general.wesl:840 weights by the cosine pdf of the cosine branch's draw even when
                        // dir is the vMF draw; LAM_GUIDE_PDF_AT_SAMPLE evaluates it at dir (unbiased)
                        const float cos_term = GUIDE && A.pdf_at_sample ? fmaxf(dot(dir, is.normal) / PI_F, 0.0f) : cos_pdf;
                        float avg_pdf = (c0 * cos_term) + (c1 == 0.0f ? 0.0f : c1 * fmaxf(mix_pdf, 0.0f));
                        if (GUIDE && LEARN && depth + 1u < A.max_depth) {
                            // learned + Markov: the guide kernel mixes this draw with the network's.  It
                            // needs the Markov mixture pdf at any direction, so the lobes go with the path;
                            // the pdf of this draw is recomputed from them (the same function the guide
                            // kernel evaluates), with the cosine term at the drawn direction
                            deferred = true;
                            A.def_kind[path] = DEF_DIFFUSE;
                            float pref = c0 * fmaxf(dot(dir, is.normal) / PI_F, 0.0f);
                            float4* lobe = A.def_lobe + (size_t)path * MIX_LOBES;
                            float* lw = A.def_lw + (size_t)path * MIX_LOBES;
#pragma unroll 1
                            for (int k = 0; k < NUM_RESAMPLES; ++k) {
                                const MC ck = cand.get(k);
                                const bool use = c1 != 0.0f && sum_mc > 0.0f && ck.weight_sum > 0.0f;
                                const v3 mean = use ? normalize(light_dir(ck, ro)) : splat(0.0f);
                                const float kappa = use ? get_kappa(ck) : 0.0f;
                                const float wk = use ? c1 * (ck.weight_sum / sum_mc) : 0.0f;
                                lobe[k] = make_float4(mean.x, mean.y, mean.z, kappa);
                                lw[k] = wk;
                                if (use) pref += wk * vmf_pdf_fast(mean, kappa, dir);
                            }
                            A.def_n[path] = make_float4(is.normal.x, is.normal.y, is.normal.z, is.roughness.x);
                            A.def_t[path] = make_float4(is.tangent.x, is.tangent.y, is.tangent.z, __uint_as_float(seed));
                            A.def_c[path] = make_float4(is.color.x, is.color.y, is.color.z, c0);
                            A.def_r[path] = make_float4(dir.x, dir.y, dir.z, pref);
                        } else {
                            v3 diffuse = Shader<Q, GUIDE>::make_diffuse(is.color, rd, is.normal, is.tangent, is.roughness.x, dir);
                            cached_pdf = avg_pdf;
                            cached_brdf = fmaxf(dot(dir, is.normal) / PI_F, 0.0f);
                            float nf = fabsf(cached_brdf) / fmaxf(avg_pdf, 0.001f);
                            color = (color * nf) * diffuse;
                            orc = (orc * nf) * diffuse;
                            rd = dir;
                        }
                    } else if (is.ty == TY_TRANSPARENT) {
                        cached_pdf = 1.0f;
                        cached_brdf = 1.0f;
                        rd = refract(rd, normal, ri);
                    }
                } else {
                    cached_pdf = 1.0f;
                    cached_brdf = 1.0f;
                    const v3 rd_in = rd;
                    rd = reflect(rd, normal);
                    if (dot(rd, is.normal) < 0.0f) rd = reflect(rd, is.normal);
                    if (LEARN && A.guide_metal && Q != LAM_QUALITY_LOW && is.ty == TY_METALLIC && ri == 1.0f &&
                        is.roughness.x >= METAL_GUIDE_MIN_ROUGHNESS && is.roughness.y >= METAL_GUIDE_MIN_ROUGHNESS &&
                        depth + 1u < A.max_depth) {
                        // the guide kernel mixes this reflection with the network's lobes (the path's
                        // throughput already holds the albedo, the whole weight of this bounce)
                        deferred = true;
                        def_kind = DEF_METAL;
                        const float4 dn = make_float4(is.normal.x, is.normal.y, is.normal.z, is.roughness.x);
                        const float4 dt = make_float4(is.tangent.x, is.tangent.y, is.tangent.z, __uint_as_float(seed));
                        const float4 dr = make_float4(rd.x, rd.y, rd.z, is.roughness.y);
                        if (STASH) {
                            def_stash[0][threadIdx.x] = dn;
                            def_stash[1][threadIdx.x] = dt;
                            def_stash[2][threadIdx.x] = dr;
                        } else {
                            A.def_kind[path] = DEF_METAL;
                            A.def_n[path] = dn;
                            A.def_t[path] = dt;
                            A.def_r[path] = dr;
                        }
                        rd = rd_in;  // the deferred path keeps its incoming direction
                    }
                }
                cont = depth + 1u < A.max_depth;
                terminated = !cont;
            } else {
                scol = fma3(color, bg, scol);
                terminated = true;
            }
            if (terminated && GUIDE) {
                // final training at the primary vertex (general.wesl:942-948)
                v3 spt = mk(pp.x, pp.y, pp.z), snm = mk(pn.x, pn.y, pn.z);
                float4 vp = A.vpoint[path];
                v3 start_dir;
                {
                    v3 o0;
                    create_ray(A, pixel % A.width, pixel / A.width, &o0, &start_dir);
                }
                MC wc = grid_load(G, spt, snm, start_dir, false);
                MC st = update_chain(spt, mk(vp.x, vp.y, vp.z), len(orad), seed, false, wc, 1.0f, sum_mc);
                grid_store_warp(G, spt, snm, start_dir, st);
                grid_add_radiance_warp(G, spt, snm, start_dir, orad);
            }
            if (LEARN && terminated && A.rec_head) finalize_records(A, path, scol);
            // write back
            const uint32_t nfl = (fl & 0xFFFF0000u) | (depth + 1u) | (last_not_vmf ? 0x100u : 0u);
            o_thr = make_float4(color.x, color.y, color.z, picked);
            o_acc = make_float4(scol.x, scol.y, scol.z, cached_pdf);
            o_misc = make_uint4(__float_as_uint(cached_brdf), seed, nfl, 0u);
            // a finished path leaves its radiance by path for the accumulate kernel; a deferred one its
            // live state at its slot in the guide kernel's queue, and a continuing one its state at its
            // slot in the next queue (both below)
            if (!cont) A.acc[path] = o_acc;
            if (rec) {
                A.ort[path] = make_float4(orc.x, orc.y, orc.z, sum_mc);
                A.orad[path] = make_float4(orad.x, orad.y, orad.z, 0.0f);
                A.ppoint[path] = pp;
                A.pnormal[path] = pn;
            }
            if (GUIDE) {
                A.lnormal[path] = make_float4(last_normal.x, last_normal.y, last_normal.z, 0.0f);
                A.ldir[path] = make_float4(last_dir.x, last_dir.y, last_dir.z, 0.0f);
                mc_store(A.tent_live + pixel, tentative);
            }
        }
        // warp-aggregated appends of the surviving paths: deferred ones to the guide kernel's queue, with
        // their live state at their slot there (the guide kernel reads it in queue order), the others
        // to the next queue
        if (LEARN) {
            const uint32_t dmask = __ballot_sync(0xFFFFFFFFu, deferred);
            if (dmask) {
                uint32_t slot = 0;
                if (lane == 0) slot = atomicAdd(A.dq_count, __popc(dmask));
                slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
                if (deferred) {
                    const uint32_t q = slot + __popc(dmask & ((1u << lane) - 1u));
                    A.dq[q] = path;
                    A.def_o[q] = make_float4(ro.x, ro.y, ro.z, 0.0f);
                    A.def_d[q] = make_float4(rd.x, rd.y, rd.z, 0.0f);
                    A.thr[q] = o_thr;
                    A.def_a[q] = o_acc;
                    A.brdf[q] = __uint_as_float(o_misc.x);
                    A.seed[q] = o_misc.y;
                    A.flags[q] = o_misc.z;
                    if (STASH) {
                        A.def_kind[q] = def_kind;
                        A.def_n[q] = def_stash[0][threadIdx.x];
                        A.def_t[q] = def_stash[1][threadIdx.x];
                        if (def_kind == DEF_METAL) A.def_r[q] = def_stash[2][threadIdx.x];
                        else A.def_c[q] = def_stash[2][threadIdx.x];
                    }
                }
            }
        }
        const bool next = cont && !deferred;
        const uint32_t mask = __ballot_sync(0xFFFFFFFFu, next);
        if (mask) {
            uint32_t slot = 0;
            if (lane == 0) slot = atomicAdd(A.count_out, __popc(mask));
            slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
            if (next) {
                const uint32_t s = slot + __popc(mask & ((1u << lane) - 1u));
                A.q_out[s] = path;
                A.ray_o_out[s] = make_float4(ro.x, ro.y, ro.z, seg_w);
                A.ray_d_out[s] = make_float4(rd.x, rd.y, rd.z, 0.0f);
                A.qthr_out[s] = o_thr;
                A.qacc_out[s] = o_acc;
                A.qmisc_out[s] = o_misc;
            }
        }
    }
}

// ---------------------------------------------------------------- learned guiding: deferred diffuse sampling
// One-sample MIS of the cosine lobe (probability 1 - f) and the network's vMF mixture (probability f):
// pdf(w) = (1 - f) cos/pi + f q(w).  With NET false (untrained network, f = 0) this is the plain cosine
// branch of the shade kernel, with the same seeds and the same arithmetic.
constexpr uint32_t GUIDE_SMEM = net::LAYERS * net::LAYER_BYTES + 2u * net::X_BYTES + 64u + 128u;
constexpr uint32_t GUIDE_TMEM_COLS = 128;  // accumulators of tiles A (columns 0..63) and B (64..127)

// The Markov sampler's mixture pdf at w from the lobes the shade kernel kept for the path:
// c0 cos/pi + sum_k w_k vMF_k(w), where w_k already includes the vMF branch's probability.
LAM_DEV float markov_mixture_pdf(const Args& A, uint32_t path, float c0, v3 n, v3 w) {
    float p = c0 * fmaxf(dot(w, n) / PI_F, 0.0f);
    const float4* lobe = A.def_lobe + (size_t)path * MIX_LOBES;
    const float* lw = A.def_lw + (size_t)path * MIX_LOBES;
#pragma unroll 1
    for (int k = 0; k < NUM_RESAMPLES; ++k) {
        const float wk = lw[k];
        if (wk != 0.0f) {
            const float4 l = lobe[k];
            p += wk * vmf_pdf_fast(mk(l.x, l.y, l.z), l.w, w);
        }
    }
    return p;
}

// MARKOV: the learned + Markov three-way mixture.  The shade kernel drew the Markov sampler's direction
// (cosine lobe or a candidate's vMF lobe, with the reference's seeds) and kept its lobes; here that draw
// is taken with probability 1 - f and the network's with probability f, and the sample is weighted by
// (1 - f) p_markov(w) + f q(w), p_markov being the Markov sampler's whole mixture pdf.
// Training record of a deferred vertex: the query, the chosen direction and the throughput and
// accumulated colour at the vertex (finalize_records turns them into the weight when the path ends).
// A Bernoulli subset of the vertices (probability rec_prob), so that the record buffer samples every
// pixel and depth of the wave instead of filling up with the first vertices shaded.
LAM_DEV void record_vertex(const Args& A, uint32_t path, uint32_t seed0, v3 ro, v3 n, v3 rd, v3 dir, v3 color_pre,
                           float4 ac) {
    if (A.recs && rand_f32(rand_u32(seed0 ^ 0x2C1B3C6Du)) < A.rec_prob) {
        const uint32_t r = atomicAdd(A.rec_count, 1u);
        if (r < A.rec_cap) {
            float* R = A.recs + (size_t)r * GUIDE_RECORD_STRIDE;
            const float v[GUIDE_RECORD_STRIDE] = {ro.x, ro.y, ro.z, n.x, n.y, n.z, -rd.x, -rd.y, -rd.z, dir.x,
                                                  dir.y, dir.z, 0.0f, color_pre.x, color_pre.y, color_pre.z,
                                                  ac.x, ac.y, ac.z, __uint_as_float(A.rec_head[path])};
#pragma unroll
            for (uint32_t k = 0; k < GUIDE_RECORD_STRIDE; ++k) R[k] = v[k];
            A.rec_head[path] = r;
        }
    }
}

// A deferred rough-metal vertex: the reference's reflection (drawn by the shade kernel) with
// probability 1 - f, the network's lobes with f, weighted by p_metal(w) / ((1 - f) p_metal(w) + f q(w))
// (the reference's weight of this bounce is 1 once the albedo is in the throughput, i.e. the BSDF
// times the cosine equals the albedo times p_metal).  Untrained (NET false) it is the reference's
// bounce, unchanged.
template <bool NET, bool MARKOV>
LAM_DEV void guide_finish_metal(const Args& A, uint32_t q, uint32_t path, const net::Lobes* L) {
    const uint32_t v = MARKOV ? path : q;  // where the shade kernel left the vertex's records
    const float4 d4 = A.def_d[q], dn = A.def_n[v], dt = A.def_t[v], dr = A.def_r[v];
    v3 dir = mk(dr.x, dr.y, dr.z);
    if (NET) {
        const float4 th = A.thr[q];
        const v3 rd = mk(d4.x, d4.y, d4.z), n = mk(dn.x, dn.y, dn.z), t = mk(dt.x, dt.y, dt.z);
        const uint32_t seed0 = __float_as_uint(dt.w);
        const float f = A.guide_frac;
        uint32_t h = rand_u32(seed0 ^ 0x68E31DA4u);
        if (rand_f32(h) < f) {
            h = rand_u32(h);
            const float u0 = rand_f32(h);
            h = rand_u32(h);
            const float u1 = rand_f32(h);
            h = rand_u32(h);
            const float u2 = rand_f32(h);
            dir = net::mixture_sample(*L, u0, u1, u2);
        }
        const float pm = metal_pdf(rd, n, t, dn.w, dr.w, dir);
        const float mix = (1.0f - f) * pm + f * net::mixture_pdf(*L, dir);
        const float wgt = mix > 0.0f ? pm / mix : 0.0f;
        A.thr[q] = make_float4(th.x * wgt, th.y * wgt, th.z * wgt, th.w);
        if (MARKOV) {
            const float4 oc = A.ort[path];
            A.ort[path] = make_float4(oc.x * wgt, oc.y * wgt, oc.z * wgt, oc.w);
        }
    }
    A.def_d[q] = make_float4(dir.x, dir.y, dir.z, 0.0f);
}

// The vertex at guide queue slot q of path `path`: its live state (origin, direction, throughput,
// sample colour, brdf, seed, flags) is stored by slot.  What the shade kernel decided at the vertex
// (kind, frame, albedo, the metal's reflection) is stored by slot too, except after the Markov-guided
// shade kernel (MARKOV), which keeps it and the Markov draw and lobes by path.  Training records are
// kept by path.
template <int Q, bool NET, bool MARKOV>
LAM_DEV void guide_finish(const Args& A, uint32_t q, uint32_t path, const net::Lobes* L, bool& out) {
    const uint32_t v = MARKOV ? path : q;
    if (A.def_kind[v] == DEF_METAL) {
        guide_finish_metal<NET, MARKOV>(A, q, path, L);
        out = true;
        return;
    }
    const float4 o4 = A.def_o[q], d4 = A.def_d[q], dn = A.def_n[v], dt = A.def_t[v], dc = A.def_c[v];
    const float4 th = A.thr[q], ac = A.def_a[q];
    const v3 ro = mk(o4.x, o4.y, o4.z), rd = mk(d4.x, d4.y, d4.z), n = mk(dn.x, dn.y, dn.z), t = mk(dt.x, dt.y, dt.z);
    const uint32_t seed0 = __float_as_uint(dt.w);
    v3 color = mk(th.x, th.y, th.z);
    v3 dir;
    float pdf;
    if (MARKOV) {
        const float4 dr = A.def_r[path];
        dir = mk(dr.x, dr.y, dr.z);
        pdf = dr.w;
        if (NET) {
            const float f = A.guide_frac;
            uint32_t h = rand_u32(seed0 ^ 0x68E31DA4u);
            const float u = rand_f32(h);
            if (u < f) {
                h = rand_u32(h);
                const float u0 = rand_f32(h);
                h = rand_u32(h);
                const float u1 = rand_f32(h);
                h = rand_u32(h);
                const float u2 = rand_f32(h);
                dir = net::mixture_sample(*L, u0, u1, u2);
                pdf = markov_mixture_pdf(A, path, dc.w, n, dir);
                A.flags[q] |= 0x100u;  // not drawn from a chain's vMF lobe (general.wesl:469-472)
            }
            pdf = (1.0f - f) * pdf + f * net::mixture_pdf(*L, dir);
        }
    } else {
        const v3 dir_cos = cosine_hemisphere(seed0, n, t);
        dir = dir_cos;
        pdf = fmaxf(dot(dir_cos, n) / PI_F, 0.0f);
    }
    if (NET && !MARKOV) {
        const float f = A.guide_frac;
        uint32_t h = rand_u32(seed0 ^ 0x68E31DA4u);
        const float u = rand_f32(h);
        if (u < f) {
            h = rand_u32(h);
            const float u0 = rand_f32(h);
            h = rand_u32(h);
            const float u1 = rand_f32(h);
            h = rand_u32(h);
            const float u2 = rand_f32(h);
            dir = net::mixture_sample(*L, u0, u1, u2);
        }
        pdf = (1.0f - f) * fmaxf(dot(dir, n) / PI_F, 0.0f) + f * net::mixture_pdf(*L, dir);
    }
    const v3 diffuse = Shader<Q, false>::make_diffuse(mk(dc.x, dc.y, dc.z), rd, n, t, dn.w, dir);
    const float cached_brdf = fmaxf(dot(dir, n) / PI_F, 0.0f);
    const float nf = fabsf(cached_brdf) / fmaxf(pdf, 0.001f);
    const v3 color_pre = color;
    color = (color * nf) * diffuse;
    if (MARKOV) {
        // the out-radiance colour the Markov chains train on takes the same factor (general.wesl:863)
        const float4 oc = A.ort[path];
        const v3 orc = (mk(oc.x, oc.y, oc.z) * nf) * diffuse;
        A.ort[path] = make_float4(orc.x, orc.y, orc.z, oc.w);
    }
    A.thr[q] = make_float4(color.x, color.y, color.z, th.w);
    A.brdf[q] = cached_brdf;
    A.def_a[q] = make_float4(ac.x, ac.y, ac.z, pdf);
    A.def_d[q] = make_float4(dir.x, dir.y, dir.z, 0.0f);
    record_vertex(A, path, seed0, ro, n, rd, dir, color_pre, ac);
    out = true;
}

template <int Q, bool NET, bool MARKOV>
__global__ void __launch_bounds__(WAVE_BLOCK) guide_sample_kernel(Args A) {
    const uint32_t n = *A.dq_count;
    const uint32_t lane = threadIdx.x & 31u;
    if (!NET) {
        for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += gridDim.x * blockDim.x) {
            const uint32_t i = base + lane;
            bool go = false;
            uint32_t path = 0;
            if (i < n) {
                path = A.dq[i];
                guide_finish<Q, false, MARKOV>(A, i, path, nullptr, go);
            }
            const uint32_t mask = __ballot_sync(0xFFFFFFFFu, go);
            uint32_t slot = 0;
            if (lane == 0 && mask) slot = atomicAdd(A.count_out, __popc(mask));
            slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
            if (go) {
                const uint32_t s = slot + __popc(mask & ((1u << lane) - 1u));
                A.q_out[s] = path;
                A.ray_o_out[s] = A.def_o[i];
                A.ray_d_out[s] = A.def_d[i];
                A.qthr_out[s] = A.thr[i];
                A.qacc_out[s] = A.def_a[i];
                A.qmisc_out[s] = make_uint4(__float_as_uint(A.brdf[i]), A.seed[i], A.flags[i], 0u);
            }
        }
        return;
    }
    // tensor-core path: two 128-row tiles (A, B) per pass, one row of each per thread, so that tile B's
    // MMAs run while tile A's epilogue does and both tiles' gathers are in flight together
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 127u) & ~uintptr_t(127));
    uint8_t* W = sm;
    uint8_t* XA = sm + net::LAYERS * net::LAYER_BYTES;
    uint8_t* XB = XA + net::X_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(XB + net::X_BYTES);
    uint32_t* slot_t = reinterpret_cast<uint32_t*>(bars + 2);
    {
        const uint4* src = reinterpret_cast<const uint4*>(A.guide_w);
        uint4* dst = reinterpret_cast<uint4*>(W);
        for (uint32_t i = threadIdx.x; i < net::LAYERS * net::LAYER_BYTES / 16u; i += blockDim.x) dst[i] = src[i];
    }
    if (threadIdx.x == 0) {
        net::mbar_init(bars);
        net::mbar_init(bars + 1);
    }
    if (threadIdx.x < 32) net::tmem_alloc(slot_t, GUIDE_TMEM_COLS);
    net::fence_before();
    __syncthreads();
    net::fence_after();
    const uint32_t tmem = *slot_t;
    const uint32_t bar_a = net::smem_u32(bars), bar_b = net::smem_u32(bars + 1);
    const uint32_t w_addr = net::smem_u32(W), xa = net::smem_u32(XA), xb = net::smem_u32(XB);
    const uint32_t t_row = tmem + ((threadIdx.x & ~31u) << 16);
    uint32_t phase = 0;
    bool failed = false;
    const uint32_t pairs = (n + 2u * net::TILE - 1) / (2u * net::TILE);
    for (uint32_t pair = blockIdx.x; pair < pairs; pair += gridDim.x) {
        const uint32_t ia = pair * 2u * net::TILE + threadIdx.x, ib = ia + net::TILE;
        const bool va = ia < n, vb = ib < n;
        const uint32_t pa = va ? A.dq[ia] : 0u, pb = vb ? A.dq[ib] : 0u;
        // origin and direction are stored by slot (rows ia and ib are read in order); the normal too,
        // except after the Markov-guided shade kernel, which keeps it by path
        auto query = [&](bool v, uint32_t slot, uint32_t path, uint8_t* X) {
            net::Query q{mk(0.0f, 0.0f, 0.0f), mk(0.0f, 1.0f, 0.0f), mk(0.0f, 1.0f, 0.0f)};
            if (v) {
                const uint32_t r = MARKOV ? path : slot;
                const float4 o4 = A.def_o[slot], d4 = A.def_d[slot], dn = A.def_n[r];
                q.pos = mk(o4.x, o4.y, o4.z);
                q.n = mk(dn.x, dn.y, dn.z);
                q.wo = mk(-d4.x, -d4.y, -d4.z);
                // the sampling epilogue reads these after the network: start them toward L2 now
                asm volatile("prefetch.global.L2 [%0];" ::"l"(A.def_t + r));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(A.def_c + r));
            }
            float f[net::WIDTH];
            net::encode_features(q, A.box, f);
            net::store_row(X, net::X_RG, threadIdx.x, f);
        };
        query(va, ia, pa, XA);
        query(vb, ib, pb, XB);
        bool ok = true;
        for (uint32_t l = 0; l < (uint32_t)net::LAYERS; ++l) {
            net::fence_async_smem();
            net::fence_before();
            if (__syncthreads_or(failed ? 1 : 0)) {
                failed = true;
                ok = false;
                break;
            }
            if (threadIdx.x == 0) {
                net::fence_after();
                net::issue_fwd(tmem, xa, w_addr + l * net::LAYER_BYTES);
                net::mma_commit(bar_a);
                net::issue_fwd(tmem + 64u, xb, w_addr + l * net::LAYER_BYTES);
                net::mma_commit(bar_b);
            }
            if (!net::mbar_wait(bar_a, phase)) failed = true;
            net::fence_after();
            if (l < 3u) net::epilogue_relu(t_row, XA, threadIdx.x);
            if (!net::mbar_wait(bar_b, phase)) failed = true;
            net::fence_after();
            if (l < 3u) net::epilogue_relu(t_row + 64u, XB, threadIdx.x);
            phase ^= 1u;
        }
        if (!ok) break;
        for (uint32_t h = 0; h < 2u; ++h) {
            const bool v = h == 0u ? va : vb;
            const uint32_t path = h == 0u ? pa : pb, q = h == 0u ? ia : ib;
            float raw[net::OUT];
            net::head_read(t_row + 64u * h, raw);
            bool go = false;
            if (v) {
                net::Lobes L;
                net::lobes_from_raw(raw, L);
                guide_finish<Q, true, MARKOV>(A, q, path, &L, go);
            }
            const uint32_t mask = __ballot_sync(0xFFFFFFFFu, go);
            uint32_t slot = 0;
            if (lane == 0 && mask) slot = atomicAdd(A.count_out, __popc(mask));
            slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
            if (go) {
                const uint32_t s = slot + __popc(mask & ((1u << lane) - 1u));
                A.q_out[s] = path;
                A.ray_o_out[s] = A.def_o[q];
                A.ray_d_out[s] = A.def_d[q];
                A.qthr_out[s] = A.thr[q];
                A.qacc_out[s] = A.def_a[q];
                A.qmisc_out[s] = make_uint4(__float_as_uint(A.brdf[q]), A.seed[q], A.flags[q], 0u);
            }
        }
    }
    if (failed) {
        // let MMAs still in flight finish before TMEM is freed
        net::mbar_wait(bar_a, phase ^ 1u, net::DRAIN_TRIES);
        net::mbar_wait(bar_b, phase ^ 1u, net::DRAIN_TRIES);
    }
    net::fence_before();
    failed = __syncthreads_or(failed ? 1 : 0) != 0;
    if (failed && threadIdx.x == 0) atomicOr(A.err, 1u << 8);
    if (threadIdx.x < 32) {
        net::fence_after();
        net::tmem_free(tmem, GUIDE_TMEM_COLS);
    }
}

// ---------------------------------------------------------------- per-pixel accumulate / outputs
LAM_DEV void reservoir_update(lam_reservoir& R, v3 vp, uint32_t vn, v3 sp, uint32_t sn, v3 orad, uint32_t ty,
                              float rough, float w_new, uint32_t seed) {
    R.w = R.w + w_new;
    uint32_t c = (R.packed_confidence_valid & 0x7FFFFFFFu) + 1u;
    R.packed_confidence_valid = (c & 0x7FFFFFFFu) | (R.packed_confidence_valid & 0x80000000u);
    if (rand_f32(seed) * R.w < w_new) {
        R.visible_point[0] = vp.x; R.visible_point[1] = vp.y; R.visible_point[2] = vp.z;
        R.visible_normal = vn;
        R.sample_point[0] = sp.x; R.sample_point[1] = sp.y; R.sample_point[2] = sp.z;
        R.sample_normal = sn;
        R.out_radiance[0] = orad.x; R.out_radiance[1] = orad.y; R.out_radiance[2] = orad.z;
        R.ty = ty;
        R.roughness = rough;
        R.packed_confidence_valid |= 0x80000000u;
    }
}
LAM_DEV float res_p_hat(const lam_reservoir& R) {
    return fmaxf(len(mk(R.out_radiance[0], R.out_radiance[1], R.out_radiance[2])), 0.00001f);
}

template <int Q>
__global__ void __launch_bounds__(WAVE_BLOCK) accumulate_kernel(Args A, uint32_t is_last_wave) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.npix) return;
    float4 pc = A.pix_color[p];
    v3 col = mk(pc.x, pc.y, pc.z);
    v3 orsum = splat(0.0f);
    if (A.pix_orad) {
        float4 t = A.pix_orad[p];
        orsum = mk(t.x, t.y, t.z);
    }
    for (uint32_t j = 0; j < A.wave_count; ++j) {
        const uint32_t path = j * A.npix + p;
        float4 a = A.acc[path];
        col = col + mk(a.x, a.y, a.z);
        if (A.pix_orad) {
            float4 o = A.orad[path];
            orsum = orsum + mk(o.x, o.y, o.z);
        }
        if (A.restir == LAM_RESTIR_PER_SAMPLE && A.reservoirs) {
            float4 pp = A.ppoint[path], pn = A.pnormal[path], vp = A.vpoint[path], vn = A.vnormal[path], o = A.orad[path];
            uint32_t ty = __float_as_uint(pp.w);
            lam_reservoir R = A.reservoirs[p];
            if (ty != TY_SKY) {
                v3 orr = mk(o.x, o.y, o.z);
                float w = fmaxf(len(orr), 0.00001f);
                uint32_t st = A.pixel_seed[p];
                reservoir_update(R, mk(vp.x, vp.y, vp.z), normalised_to_u32(mk(vn.x, vn.y, vn.z)), mk(pp.x, pp.y, pp.z),
                                 normalised_to_u32(mk(pn.x, pn.y, pn.z)), orr, ty, 0.0f, w, st);
                A.pixel_seed[p] = rand_u32(st);
                uint32_t c = R.packed_confidence_valid & 0x7FFFFFFFu;
                R.W = safe_div(R.w, __uint2float_rn(c) * res_p_hat(R));
            } else {
                R.ty = TY_SKY;
            }
            A.reservoirs[p] = R;
        }
    }
    A.pix_color[p] = make_float4(col.x, col.y, col.z, 0.0f);
    if (A.pix_orad) A.pix_orad[p] = make_float4(orsum.x, orsum.y, orsum.z, 0.0f);
    if (!is_last_wave) return;
    const float inv_n = __uint2float_rn(A.samples);
    if (A.out_color) {
        v3 c = col / inv_n;
        A.out_color[p] = make_float4(fmaxf(c.x, 0.0f), fmaxf(c.y, 0.0f), fmaxf(c.z, 0.0f), 1.0f);
    }
    const uint32_t last_path = (A.wave_count - 1u) * A.npix + p;
    if (A.restir != LAM_RESTIR_DISABLED && A.info) {
        float4 e = A.pix_emission[p], al = A.pix_albedo[p];
        lam_info inf;
        inf.arr[0] = A.camera_pos.x; inf.arr[1] = A.camera_pos.y; inf.arr[2] = A.camera_pos.z;
        inf.arr[3] = e.x; inf.arr[4] = e.y; inf.arr[5] = e.z;
        inf.arr[6] = al.x; inf.arr[7] = al.y; inf.arr[8] = al.z;
        A.info[p] = inf;
    }
    if (A.tent_snap && A.chains && p < A.chains_len) A.chains[p] = A.tent_snap[p];
    if (A.reservoirs) {
        if (A.restir == LAM_RESTIR_PER_PIXEL) {
            float4 pp = A.ppoint[last_path], pn = A.pnormal[last_path], vp = A.vpoint[last_path], vn = A.vnormal[last_path];
            uint32_t ty = __float_as_uint(pp.w);
            lam_reservoir R = lam_reservoir{};
            if (ty != TY_SKY) {
                v3 orr = orsum / inv_n;
                float w = fmaxf(len(orr), 0.00001f);
                uint32_t st = A.pixel_seed[p];
                reservoir_update(R, mk(vp.x, vp.y, vp.z), normalised_to_u32(mk(vn.x, vn.y, vn.z)), mk(pp.x, pp.y, pp.z),
                                 normalised_to_u32(mk(pn.x, pn.y, pn.z)), orr, ty, 0.0f, w, st);
                uint32_t c = R.packed_confidence_valid & 0x7FFFFFFFu;
                R.W = safe_div(R.w, __uint2float_rn(c) * res_p_hat(R));
            } else {
                R.ty = TY_SKY;
            }
            A.reservoirs[p] = R;
        } else if (A.restir == LAM_RESTIR_DISABLED) {
            A.reservoirs[p] = lam_reservoir{};
        }
    }
}

// subgroupShuffle(tentative, (lane + 1) % 32) after each sample (general.wesl:349-361, 582)
__global__ void shuffle_kernel(Args A) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.npix) return;
    const uint32_t x = p % A.width, y = p / A.width;
    const uint32_t src_x = (x & ~31u) + (((x & 31u) + 1u) & 31u);
    MC t = src_x < A.width ? mc_load(A.tent_live + (uint64_t)y * A.width + src_x) : mc_zero();
    mc_store(A.tent_snap + p, t);
}

// Device bytes of wave state per path: rays of two queues (64), live state of two queues (96), hit
// (8), two queue entries (8), state by path (44); ReSTIR / Markov / learned-guide extras.
constexpr uint64_t WAVE_BYTES_PER_PATH = 220, WAVE_BYTES_FULL = 96, WAVE_BYTES_GUIDE = 32, WAVE_BYTES_LEARNED = 108,
                   WAVE_BYTES_THREE_WAY = 20 * MIX_LOBES;

static int alloc_wave(WaveBuffers* w, uint32_t npix, bool full, bool guide, bool learned) {
    const size_t P = w->paths;
    int rc = 0;
    rc |= walloc(w, &w->ray_o, P);
    rc |= walloc(w, &w->ray_d, P);
    rc |= walloc(w, &w->ray_o2, P);
    rc |= walloc(w, &w->ray_d2, P);
    rc |= walloc(w, &w->qthr0, P);
    rc |= walloc(w, &w->qthr1, P);
    rc |= walloc(w, &w->qacc0, P);
    rc |= walloc(w, &w->qacc1, P);
    rc |= walloc(w, &w->qmisc0, P);
    rc |= walloc(w, &w->qmisc1, P);
    rc |= walloc(w, &w->hit, P);
    rc |= walloc(w, &w->queue0, P);
    rc |= walloc(w, &w->queue1, P);
    rc |= walloc(w, &w->thr, P);
    rc |= walloc(w, &w->acc, P);
    rc |= walloc(w, &w->brdf, P);
    rc |= walloc(w, &w->seed, P);
    rc |= walloc(w, &w->flags, P);
    rc |= walloc(w, &w->pix_color, npix);
    rc |= walloc(w, &w->ctr, 64);
    if (full) {
        rc |= walloc(w, &w->ort, P);
        rc |= walloc(w, &w->orad, P);
        rc |= walloc(w, &w->ppoint, P);
        rc |= walloc(w, &w->pnormal, P);
        rc |= walloc(w, &w->vpoint, P);
        rc |= walloc(w, &w->vnormal, P);
        rc |= walloc(w, &w->pix_orad, npix);
        rc |= walloc(w, &w->pix_emission, npix);
        rc |= walloc(w, &w->pix_albedo, npix);
    }
    if (guide) {
        rc |= walloc(w, &w->lnormal, P);
        rc |= walloc(w, &w->ldir, P);
        rc |= walloc(w, &w->tent_snap, npix);
        rc |= walloc(w, &w->tent_live, npix);
    }
    if (learned) {
        rc |= walloc(w, &w->dq, P);
        rc |= walloc(w, &w->def_n, P);
        rc |= walloc(w, &w->def_t, P);
        rc |= walloc(w, &w->def_c, P);
        rc |= walloc(w, &w->def_o, P);
        rc |= walloc(w, &w->def_d, P);
        rc |= walloc(w, &w->def_a, P);
        rc |= walloc(w, &w->rec_head, P);
        rc |= walloc(w, &w->def_r, P);
        rc |= walloc(w, &w->def_kind, P);
        if (guide) {
            rc |= walloc(w, &w->def_lobe, P * MIX_LOBES);
            rc |= walloc(w, &w->def_lw, P * MIX_LOBES);
        }
    }
    return rc;
}

static int ensure_wave(lam_pipeline* pl, uint32_t width, uint32_t height, bool full, bool guide, bool learned) {
    const uint32_t npix = width * height;
    uint32_t spp_wave = 1;
    if (!guide && pl->opts.restir_temporal != LAM_RESTIR_PER_SAMPLE) {
        // aim for ~32M paths in flight (about 7 GB of wave state at 1080p), at most the sample count:
        // the deep bounces of a small wave leave the persistent traversal tail-bound (1080p, 16 spp:
        // 1058 Mrays/s with 4-spp waves, 1089 with 8, 1104 with one 16-spp wave)
        uint64_t target = pl->wave_paths ? pl->wave_paths : (32ull << 20);
        spp_wave = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(pl->opts.samples, target / std::max(1u, npix)));
    }
    WaveBuffers* w = pl->wave;
    // a wave that was shrunk to fit device memory is kept while the request is larger
    if (w && w->width == width && w->height == height && w->full == full && w->guide == guide && w->learned == learned &&
        (w->spp_wave == spp_wave || (w->mem_capped && w->spp_wave < spp_wave)))
        return LAM_OK;
    free_wave(w);
    pl->wave = nullptr;
    // at most half of the free device memory; if an allocation still fails, halve the wave
    bool capped = false;
    size_t free_b = 0, total_b = 0;
    if (spp_wave > 1 && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const uint64_t per_path = WAVE_BYTES_PER_PATH + (full ? WAVE_BYTES_FULL : 0) + (guide ? WAVE_BYTES_GUIDE : 0) +
                                  (learned ? WAVE_BYTES_LEARNED : 0) + (guide && learned ? WAVE_BYTES_THREE_WAY : 0);
        const uint64_t fit = (uint64_t)(free_b / 2) / (per_path * std::max(1u, npix));
        if (fit < spp_wave) {
            spp_wave = (uint32_t)std::max<uint64_t>(1, fit);
            capped = true;
        }
    }
    for (;;) {
        w = new WaveBuffers();
        w->width = width;
        w->height = height;
        w->npix = npix;
        w->spp_wave = spp_wave;
        w->paths = (uint64_t)npix * spp_wave;
        w->full = full;
        w->guide = guide;
        w->learned = learned;
        if (alloc_wave(w, npix, full, guide, learned) == LAM_OK) break;
        free_wave(w);
        if (spp_wave == 1) return LAM_ERR_CUDA;  // the failed allocation set the error message
        (void)cudaGetLastError();                // an out-of-memory error is not sticky
        spp_wave = std::max(1u, spp_wave / 2u);
        capped = true;
    }
    w->mem_capped = capped;
    cudaMemset(w->ctr, 0, 64 * sizeof(uint32_t));
    pl->total_segments = 0;
    pl->prof_segments_base = 0;
    cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, pl->device);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, extend_kernel<false>, WAVE_BLOCK, 0);
    w->grid_extend = w->sms * std::max(1, occ);
    occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, shade_kernel<LAM_QUALITY_MEDIUM, false, false, false>, WAVE_BLOCK, 0);
    w->grid_shade = w->sms * std::max(1, occ);
    w->grid_sort = std::min(SORT_BLOCKS_MAX, w->sms * 6);
    if (guide) {
        const void* ks[] = {(const void*)shade_kernel<LAM_QUALITY_LOW, true, false, false>,
                            (const void*)shade_kernel<LAM_QUALITY_MEDIUM, true, false, false>,
                            (const void*)shade_kernel<LAM_QUALITY_HIGH, true, false, false>,
                            (const void*)shade_kernel<LAM_QUALITY_LOW, true, true, false>,
                            (const void*)shade_kernel<LAM_QUALITY_MEDIUM, true, true, false>,
                            (const void*)shade_kernel<LAM_QUALITY_HIGH, true, true, false>};
        for (const void* k : ks) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GUIDE_SHADE_SMEM);
            if (e != cudaSuccess) {
                free_wave(w);
                return cuda_error(e, "guided shade kernel attributes");
            }
        }
    }
    if (learned) {
        cudaError_t e = cudaSuccess;
        auto attrs = [&](const void* k) {
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, GUIDE_SMEM);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        };
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_LOW, true, false>);
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_MEDIUM, true, false>);
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_HIGH, true, false>);
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_LOW, true, true>);
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_MEDIUM, true, true>);
        attrs((const void*)guide_sample_kernel<LAM_QUALITY_HIGH, true, true>);
        // resident CTAs per SM from the kernel's registers and shared memory (the occupancy query
        // under-reports this kernel); at most 4 keep the 128-column TMEM allocations within 512 columns
        cudaFuncAttributes fa{};
        int regs_sm = 0, smem_sm = 0, smem_reserved = 0;
        const void* sized = guide ? (const void*)guide_sample_kernel<LAM_QUALITY_MEDIUM, true, true>
                                  : (const void*)guide_sample_kernel<LAM_QUALITY_MEDIUM, true, false>;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, sized);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, pl->device);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, pl->device);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, pl->device);
        if (e != cudaSuccess) {
            free_wave(w);
            return cuda_error(e, "guide kernel attributes");
        }
        const int regs_block = ((fa.numRegs + 7) / 8) * 8 * WAVE_BLOCK;
        const int by_regs = regs_block > 0 ? regs_sm / regs_block : 1;
        const int by_smem = smem_sm / (int)(GUIDE_SMEM + fa.sharedSizeBytes + smem_reserved);
        w->grid_guide = w->sms * std::min(4, std::max(1, std::min(by_regs, by_smem)));
    }
    pl->wave = w;
    return LAM_OK;
}

int ensure_handler(lam_pipeline* pl) {
    if (pl->handler) return LAM_OK;
    HandlerModule* m = new HandlerModule();
    int rc = load_handler_module(pl->handler_cubin, m);
    if (rc) {
        free_handler_module(m);
        return rc;
    }
    pl->handler = m;
    return LAM_OK;
}

template <int Q>
static void launch_guide(bool net, bool markov, int grid, cudaStream_t st, const Args& A) {
    if (markov) {
        if (net) guide_sample_kernel<Q, true, true><<<grid, WAVE_BLOCK, GUIDE_SMEM, st>>>(A);
        else guide_sample_kernel<Q, false, true><<<grid, WAVE_BLOCK, 0, st>>>(A);
    } else {
        if (net) guide_sample_kernel<Q, true, false><<<grid, WAVE_BLOCK, GUIDE_SMEM, st>>>(A);
        else guide_sample_kernel<Q, false, false><<<grid, WAVE_BLOCK, 0, st>>>(A);
    }
}

template <int Q>
static void launch_shade(bool guide, bool learned, dim3 g, dim3 b, cudaStream_t st, const Args& A) {
    if (guide && learned) shade_kernel<Q, true, true, false><<<g, b, GUIDE_SHADE_SMEM, st>>>(A);
    else if (guide) shade_kernel<Q, true, false, false><<<g, b, GUIDE_SHADE_SMEM, st>>>(A);
    else if (learned) shade_kernel<Q, false, true, false><<<g, b, 0, st>>>(A);
    else shade_kernel<Q, false, false, false><<<g, b, 0, st>>>(A);
}


// ---------------------------------------------------------------- batched renders: kernels
LAM_DEV uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Segment of pixel thread t (segments sorted by pix_thread_base).
LAM_DEV uint32_t find_seg(const BatchSeg* segs, uint32_t nsegs, uint32_t t) {
    uint32_t lo = 0, hi = nsegs - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (segs[mid].pix_thread_base <= t) lo = mid;
        else hi = mid - 1u;
    }
    return lo;
}

// create_ray (general.wesl:1158-1173) with a request's camera and image size.
LAM_DEV void create_ray_req(const BatchReq& R, uint32_t x, uint32_t y, v3* o, v3* d) {
    float hx = __uint2float_rn(R.width) / 2.0f, hy = __uint2float_rn(R.height) / 2.0f;
    float nx = (__uint2float_rn(x) / hx) - 1.0f, ny = (__uint2float_rn(y) / hy) - 1.0f;
    float v[4] = {nx, -ny, 1.0f, 1.0f};
    const float* P = R.cam.projection_inverse;
    float q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = P[i] * v[0] + P[4 + i] * v[1] + P[8 + i] * v[2] + P[12 + i] * v[3];
    float l = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = q[i] / l;
    const float* V = R.cam.view_inverse;
    *d = mk(V[0] * q[0] + V[4] * q[1] + V[8] * q[2] + V[12] * 0.0f, V[1] * q[0] + V[5] * q[1] + V[9] * q[2] + V[13] * 0.0f,
            V[2] * q[0] + V[6] * q[1] + V[10] * q[2] + V[14] * 0.0f);
    *o = R.camera_pos;
}

// Zeroes the per-request completion counters and stamps the batch start.
__global__ void batch_start_kernel(uint32_t* done, unsigned long long* times, uint32_t n) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) done[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) times[n] = global_timer_ns();
}

// One thread per (segment, pixel): the request's seed chain and camera ray for each of the
// segment's samples (as generate_kernel does for a single render).
__global__ void __launch_bounds__(WAVE_BLOCK) batch_generate_kernel(const __grid_constant__ Args A) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *A.count_in = A.npix;  // paths of this wave
    if (t >= A.pix_threads) return;
    const uint32_t k = find_seg(A.segs, A.nsegs, t);
    const BatchSeg sg = A.segs[k];
    const BatchReq& R = A.reqs[sg.req];
    const uint32_t p = t - sg.pix_thread_base;
    const uint32_t x = p % R.width, y = p / R.width;
    uint32_t st;
    if (sg.first == 0u) {
        st = rand_u32(x * y) + R.seed_offset + y;
        A.pix_color[R.pix_base + p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
        st = A.pixel_seed[R.pix_base + p];
    }
    v3 o, d;
    create_ray_req(R, x, y, &o, &d);
    for (uint32_t j = 0; j < sg.count; ++j) {
        const uint32_t path = sg.path_base + j * R.npix + p;
        st = advance_fill_seed(st);
        A.ray_o[path] = make_float4(o.x, o.y, o.z, __uint_as_float(k));
        A.ray_d[path] = make_float4(d.x, d.y, d.z, 0.0f);
        A.qthr[path] = make_float4(1.0f, 1.0f, 1.0f, -1.0f);
        A.qacc[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        A.qmisc[path] = make_uint4(0u, st, k << 16, 0u);
        A.q_in[path] = path;
        st = rand_u32(st);
    }
    A.pixel_seed[R.pix_base + p] = st;
}

template <bool ALPHA>
__global__ void __launch_bounds__(WAVE_BLOCK) extend_batch_kernel(const __grid_constant__ Args A) {
    const uint32_t n = *A.count_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(A.segments, (unsigned long long)n);
        atomicAdd(A.segments + 1, (unsigned long long)n);
    }
    uint32_t err = 0u;
    trace_persistent_multi<false, ALPHA>(
        n, A.work, err,
        [&](uint32_t i, float3& o, float3& d, float& t0, float& t1, const DevScene*& sp) {
            const float4 o4 = A.ray_o[i], d4 = A.ray_d[i];
            o = make_float3(o4.x, o4.y, o4.z);
            d = make_float3(d4.x, d4.y, d4.z);
            t0 = A.tmin;
            t1 = A.tmax;
            sp = &A.reqs[A.segs[__float_as_uint(o4.w)].req].S;  // the ray carries its segment
        },
        [&](uint32_t i, const TraceResult& tr) { A.hit[i] = make_uint2(tr.tri, tr.inst); });
    if (err) atomicOr(A.err, err);
}

// One thread per (segment, pixel): sums the segment's samples in sample order; after a request's
// last sample writes its mean colour and, for the last pixel to finish, its completion time.
__global__ void __launch_bounds__(WAVE_BLOCK) batch_accumulate_kernel(const __grid_constant__ Args A) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.pix_threads) return;
    const BatchSeg sg = A.segs[find_seg(A.segs, A.nsegs, t)];
    const BatchReq& R = A.reqs[sg.req];
    const uint32_t p = t - sg.pix_thread_base;
    const float4 pc = A.pix_color[R.pix_base + p];
    v3 col = mk(pc.x, pc.y, pc.z);
    for (uint32_t j = 0; j < sg.count; ++j) {
        const float4 a = A.acc[sg.path_base + j * R.npix + p];
        col = col + mk(a.x, a.y, a.z);
    }
    A.pix_color[R.pix_base + p] = make_float4(col.x, col.y, col.z, 0.0f);
    if (sg.first + sg.count != R.samples) return;
    if (R.out_color) {
        const v3 c = col / __uint2float_rn(R.samples);
        R.out_color[p] = make_float4(fmaxf(c.x, 0.0f), fmaxf(c.y, 0.0f), fmaxf(c.z, 0.0f), 1.0f);
    }
    __threadfence();
    if (atomicAdd(A.req_done + sg.req, 1u) + 1u == R.npix) A.req_time[sg.req] = global_timer_ns();
}
}  // namespace lam

using namespace lam;

extern "C" int lam_tracer_create_pipeline(const lam_tracer* t, const lam_pipeline_layout* layout,
                                          const lam_tracer_options* o, lam_pipeline** out) {
    if (!t || !layout || !o || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_tracer_create_pipeline: null argument");
    if (o->samples == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "samples must be nonzero (NonZeroU32)");
    if (o->max_depth == 0 || o->max_depth > 255) return set_error(LAM_ERR_INVALID_ARGUMENT, "max_depth must be in 1..255");
    if (o->restir_temporal > LAM_RESTIR_PER_PIXEL) return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown ReSTIR mode");
    {
        const uint32_t g = o->guide_mode, learned = g & ~(uint32_t)LAM_GUIDE_METAL;
        const bool ok = g == LAM_GUIDE_NONE || g == LAM_GUIDE_MARKOV || g == (LAM_GUIDE_MARKOV | LAM_GUIDE_PDF_AT_SAMPLE) ||
                        ((learned == LAM_GUIDE_LEARNED || learned == (LAM_GUIDE_LEARNED | LAM_GUIDE_MARKOV)));
        if (!ok) return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown guide mode");
    }
    if (t->quality > LAM_QUALITY_HIGH && (t->quality < LAM_DEBUG_FRONT_FACE || t->quality > LAM_DEBUG_TANGENT))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown shader");
    lam_pipeline* p = new lam_pipeline();
    p->quality = t->quality;
    p->opts = *o;
    p->layout = *layout;
    p->intersection_handler = t->intersection_handler;
    cudaGetDevice(&p->device);
    if (!p->intersection_handler.empty()) {
        std::string log;
        int rc = compile_handler_cubin(p->intersection_handler, &p->handler_cubin, &log);
        if (rc) {
            delete p;
            return set_error(rc, log);
        }
    }
    *out = p;
    return LAM_OK;
}

extern "C" int lam_pipeline_destroy(lam_pipeline* p) {
    if (!p) return LAM_OK;
    free_wave(p->wave);
    free_batch(p->batch);
    free_handler_module(p->handler);
    for (auto& t : p->timed) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.end);
    }
    for (cudaEvent_t e : p->event_pool) cudaEventDestroy(e);
    delete p;
    return LAM_OK;
}

extern "C" int lam_pipeline_set_wave_paths(lam_pipeline* p, uint64_t max_paths) {
    if (!p) return set_error(LAM_ERR_INVALID_ARGUMENT, "null pipeline");
    p->wave_paths = max_paths;
    return LAM_OK;
}

extern "C" int lam_pipeline_set_shade_order(lam_pipeline* p, uint32_t order) {
    if (!p) return set_error(LAM_ERR_INVALID_ARGUMENT, "null pipeline");
    if (order != LAM_SHADE_ORDER_AUTO && order != LAM_SHADE_ORDER_QUEUE && order != LAM_SHADE_ORDER_MATERIAL)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown shade order");
    p->shade_order = order;
    return LAM_OK;
}

extern "C" int lam_pipeline_set_guide(lam_pipeline* p, lam_guide* g) {
    if (!p) return set_error(LAM_ERR_INVALID_ARGUMENT, "null pipeline");
    p->guide = g;
    return LAM_OK;
}

extern "C" int lam_pipeline_set_profiling(lam_pipeline* p, int enabled) {
    if (!p) return set_error(LAM_ERR_INVALID_ARGUMENT, "null pipeline");
    p->profiling = enabled != 0;
    return LAM_OK;
}

extern "C" int lam_render_profile_get(lam_pipeline* p, lam_stage_times* out) {
    if (!p || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    for (auto& t : p->timed) {
        cudaError_t e = cudaEventSynchronize(t.end);
        if (e != cudaSuccess) return cuda_error(e, "lam_render_profile_get");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t.start, t.end);
        switch (t.stage) {
            case 0: p->prof.generate_ms += ms; break;
            case 1: p->prof.extend_ms += ms; p->prof.extend_launches++; break;
            case 2: p->prof.shade_ms += ms; p->prof.shade_launches++; break;
            case 4: p->prof.train_ms += ms; break;
            default: p->prof.accumulate_ms += ms; break;
        }
        p->event_pool.push_back(t.start);
        p->event_pool.push_back(t.end);
    }
    p->timed.clear();
    lam_render_stats s;
    p->stats_pending = true;
    int rc = lam_render_stats_get(p, &s);
    if (rc) return rc;
    *out = p->prof;
    out->ray_segments = p->total_segments - p->prof_segments_base;
    return LAM_OK;
}

extern "C" int lam_render_profile_reset(lam_pipeline* p) {
    if (!p) return set_error(LAM_ERR_INVALID_ARGUMENT, "null pipeline");
    lam_stage_times tmp;
    int rc = lam_render_profile_get(p, &tmp);
    if (rc) return rc;
    p->prof = lam_stage_times{};
    p->prof_segments_base = p->total_segments;
    return LAM_OK;
}

// Reads the device counters of the last render (synchronises the device).
extern "C" int lam_render_stats_get(const lam_pipeline* p, lam_render_stats* out) {
    if (!p || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    lam_pipeline* q = const_cast<lam_pipeline*>(p);
    if (q->stats_pending && q->stats_ctr) {
        uint32_t host[16];
        cudaError_t e = cudaMemcpy(host, q->stats_ctr, sizeof(host), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_error(e, "lam_render_stats_get");
        unsigned long long segs, total;
        std::memcpy(&segs, host + 8, sizeof(segs));
        std::memcpy(&total, host + 10, sizeof(total));
        q->stats.ray_segments = segs;
        q->total_segments = total;
        q->stats.error_flags = host[4];
        q->stats_pending = false;
    }
    *out = q->stats;
    return LAM_OK;
}

extern "C" int lam_render(lam_pipeline* pl, const lam_scene* s, lam_data_buffers* b, const lam_camera* cam,
                          const lam_frame_targets* tg, uint32_t seed_offset, void* stream) {
    if (!pl || !s || !b || !cam || !tg) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_render: null argument");
    if (tg->width == 0 || tg->height == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_render: empty target");
    if (tg->width != b->width || tg->height != b->height)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_render: targets and data buffers differ in size");
    if ((uint64_t)tg->width * tg->height > 0xFFFFFFFFull / 4)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_render: target too large");
    if (s->instance_count > pl->layout.blas_count || s->diffuse_count > pl->layout.diffuse_count ||
        s->emission_count > pl->layout.emission_count || s->attribute_count > pl->layout.attribute_count)
        return set_error(LAM_ERR_LAYOUT_MISMATCH, "scene bindings exceed the pipeline layout counts");
    if (pl->quality >= LAM_DEBUG_FRONT_FACE) return render_debug(pl, s, cam, tg, (cudaStream_t)stream);
    const bool guide = (pl->opts.guide_mode & LAM_GUIDE_MARKOV) != 0u;
    const bool learned = (pl->opts.guide_mode & LAM_GUIDE_LEARNED) != 0u;
    const uint32_t restir = pl->opts.restir_temporal;
    if (learned && !pl->guide) return set_error(LAM_ERR_INVALID_ARGUMENT, "LAM_GUIDE_LEARNED needs lam_pipeline_set_guide");
    if (learned && restir != LAM_RESTIR_DISABLED)
        return set_error(LAM_ERR_UNSUPPORTED, "learned guiding runs with ReSTIR disabled");
    const bool full = guide || restir != LAM_RESTIR_DISABLED;
    pl->stats_ctr = nullptr;  // the counters may move with the wave buffers
    pl->stats_pending = false;
    int rc = ensure_wave(pl, tg->width, tg->height, full, guide, learned);
    if (rc) return rc;
    WaveBuffers* w = pl->wave;
    cudaStream_t st = (cudaStream_t)stream;
    Args A;
    std::memset(&A, 0, sizeof(A));
    A.S = s->dev;
    A.cam = *cam;
    A.width = tg->width;
    A.height = tg->height;
    A.npix = w->npix;
    A.samples = pl->opts.samples;
    A.max_depth = pl->opts.max_depth;
    A.restir = restir;
    A.seed_offset = seed_offset;
    A.pdf_at_sample = (pl->opts.guide_mode & LAM_GUIDE_PDF_AT_SAMPLE) != 0u;
    A.guide_metal = (pl->opts.guide_mode & LAM_GUIDE_METAL) != 0u;
    A.tmin = pl->opts.tmin;
    A.tmax = pl->opts.tmax;
    A.ray_o = w->ray_o;
    A.ray_d = w->ray_d;
    A.hit = w->hit;
    A.err = w->ctr + 4;
    A.segments = reinterpret_cast<unsigned long long*>(w->ctr + 8);
    A.thr = w->thr;
    A.acc = w->acc;
    A.brdf = w->brdf;
    A.seed = w->seed;
    A.flags = w->flags;
    A.ort = w->ort;
    A.orad = w->orad;
    A.ppoint = w->ppoint;
    A.pnormal = w->pnormal;
    A.vpoint = w->vpoint;
    A.vnormal = w->vnormal;
    A.lnormal = w->lnormal;
    A.ldir = w->ldir;
    A.pix_color = w->pix_color;
    A.pix_orad = w->pix_orad;
    A.pix_emission = w->pix_emission;
    A.pix_albedo = w->pix_albedo;
    A.tent_snap = w->tent_snap;
    A.tent_live = w->tent_live;
    const bool screen = (b->types & LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE) != 0u;
    const bool world = (b->types & LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE) != 0u;
    A.old_chains = guide && screen ? (const lam_markov_chain*)b->old_chains : nullptr;
    A.old_chains_len = b->chain_len;
    A.chains = guide && screen ? (lam_markov_chain*)b->chains : nullptr;
    A.chains_len = b->chain_len;
    A.world = (uint32_t*)b->world;
    A.old_world = (const uint32_t*)b->old_world;
    A.world_len = b->world_len;
    A.world_mod_m = ~0ull / std::max<uint64_t>(1, b->world_len) + 1ull;  // grid_index's remainder multiplier
    A.reservoirs = (lam_reservoir*)b->reservoirs;
    if (b->reservoir_len < w->npix) A.reservoirs = nullptr;
    A.info = (lam_info*)b->info;
    A.pixel_seed = (uint32_t*)b->pixel_seed;
    A.out_color = (float4*)tg->color;
    A.out_normal = (float4*)tg->normal;
    A.out_albedo = (float4*)tg->albedo;
    A.camera_pos = v3{cam->view_inverse[12], cam->view_inverse[13], cam->view_inverse[14]};
    std::memcpy(A.box, s->bounds, sizeof(A.box));
    // procedural geometry with a handler: the run-time-linked extend kernel
    const bool proc = s->dev.has_procedural && !pl->handler_cubin.empty();
    if (proc) {
        if ((rc = ensure_handler(pl))) return rc;
        if (!w->phit_a && (walloc(w, &w->phit_a, w->paths) || walloc(w, &w->phit_b, w->paths)))
            return LAM_ERR_CUDA;
        A.phit_a = w->phit_a;
        A.phit_b = w->phit_b;
    }
    lam_guide* gd = learned ? pl->guide : nullptr;
    if (gd) {
        A.dq = w->dq;
        A.dq_count = w->ctr + 12;
        A.def_n = w->def_n;
        A.def_t = w->def_t;
        A.def_c = w->def_c;
        A.def_o = w->def_o;
        A.def_d = w->def_d;
        A.def_a = w->def_a;
        A.def_r = w->def_r;
        A.def_kind = w->def_kind;
        A.def_lobe = w->def_lobe;
        A.def_lw = w->def_lw;
        A.rec_cap = gd->opts.record_capacity;
        A.rec_count = w->ctr + 13;
        A.guide_w = gd->packed;
        std::memcpy(A.box, s->bounds, sizeof(A.box));
    }
    if (guide && !world) return set_error(LAM_ERR_INVALID_ARGUMENT, "Markov guiding needs MARKOV_CHAIN_WORLD_SPACE buffers");
    // automatic order: sorted except under Markov guiding, which measured faster in queue order
    const bool sorted = pl->shade_order == LAM_SHADE_ORDER_MATERIAL || (pl->shade_order == LAM_SHADE_ORDER_AUTO && !guide);
    if (sorted) {
        if (!w->shade_order && (walloc(w, &w->shade_key, w->paths) || walloc(w, &w->shade_order, w->paths) ||
                                walloc(w, &w->shade_bc, (size_t)SORT_BLOCKS_MAX * SHADE_CLASSES)))
            return LAM_ERR_CUDA;
        A.shade_key = w->shade_key;
        A.shade_order = w->shade_order;
        A.shade_bc = w->shade_bc;
    }
    const bool alpha = !s->dev.all_opaque;
    const dim3 blk(WAVE_BLOCK);
    const dim3 gpix((w->npix + WAVE_BLOCK - 1) / WAVE_BLOCK);
    uint32_t launches = 0;
    auto ev = [&]() {
        cudaEvent_t e;
        if (!pl->event_pool.empty()) {
            e = pl->event_pool.back();
            pl->event_pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    };
    // stage 0 generate, 1 extend, 2 shade, 3 accumulate/shuffle
    auto begin = [&](int stage) -> int {
        if (!pl->profiling) return -1;
        lam_pipeline::Timed t{stage, ev(), ev()};
        cudaEventRecord(t.start, st);
        pl->timed.push_back(t);
        return (int)pl->timed.size() - 1;
    };
    auto end = [&](int h) {
        if (h >= 0) cudaEventRecord(pl->timed[h].end, st);
    };
    cudaMemsetAsync(w->ctr, 0, 10 * sizeof(uint32_t), st);  // keeps the cumulative counter ctr[10..11]
    for (uint32_t first = 0; first < pl->opts.samples;) {
        // learned guiding: record training vertices while the guide has seen fewer than train_spp
        // samples per pixel; sample the network once it has taken a training step
        const bool training = gd && gd->records && gd->trained_spp < gd->opts.train_spp;
        uint32_t count = std::min(w->spp_wave, pl->opts.samples - first);
        // the guide takes steps_per_wave Adam steps after each training wave; training waves stay at
        // ~8M paths (4 spp at 1080p) whatever the wave size of the rest of the render
        if (training) count = std::min<uint32_t>(count, std::max<uint32_t>(1u, (uint32_t)((8ull << 20) / w->npix)));
        A.wave_first = first;
        A.wave_count = count;
        uint32_t* qa = w->queue0;
        uint32_t* qb = w->queue1;
        uint32_t* ca = w->ctr + 0;
        uint32_t* cb = w->ctr + 1;
        float4 *rao = w->ray_o, *rad = w->ray_d, *rbo = w->ray_o2, *rbd = w->ray_d2;  // rays of qa, qb
        float4 *tha = w->qthr0, *thb = w->qthr1, *aca = w->qacc0, *acb = w->qacc1;   // path state of qa, qb
        uint4 *mia = w->qmisc0, *mib = w->qmisc1;
        A.q_in = qa;
        A.count_in = ca;
        A.ray_o = rao;
        A.ray_d = rad;
        A.qthr = tha;
        A.qacc = aca;
        A.qmisc = mia;
        const bool use_net = gd && gd->steps > 0;
        A.recs = training ? gd->records : nullptr;
        if (training) {
            // expected diffuse vertices of the wave: at most one per path and bounce
            const double expected = (double)w->npix * A.wave_count * std::max(1u, pl->opts.max_depth - 1u);
            A.rec_prob = (float)std::min(1.0, 1.25 * gd->opts.record_capacity / std::max(1.0, expected));
        }
        A.rec_head = training ? w->rec_head : nullptr;
        A.guide_frac = use_net ? gd->opts.guide_fraction : 0.0f;
        if (training) cudaMemsetAsync(w->ctr + 13, 0, sizeof(uint32_t), st);
        int h = begin(0);
        generate_kernel<<<gpix, blk, 0, st>>>(A);
        end(h);
        ++launches;
        for (uint32_t depth = 0; depth < pl->opts.max_depth; ++depth) {
            A.q_in = qa;
            A.q_out = qb;
            A.count_in = ca;
            A.count_out = cb;
            A.ray_o = rao;
            A.ray_d = rad;
            A.ray_o_out = rbo;
            A.ray_d_out = rbd;
            A.qthr = tha;
            A.qacc = aca;
            A.qmisc = mia;
            A.qthr_out = thb;
            A.qacc_out = acb;
            A.qmisc_out = mib;
            A.work = w->ctr + 2;
            cudaMemsetAsync(w->ctr + 2, 0, sizeof(uint32_t), st);
            cudaMemsetAsync(cb, 0, sizeof(uint32_t), st);
            h = begin(1);
            if (proc) {
                void* kargs[] = {&A};
                cudaLaunchKernel((const void*)pl->handler->extend, dim3(w->grid_extend), blk, kargs, 0, st);
            } else if (alpha) {
                extend_kernel<true><<<w->grid_extend, blk, 0, st>>>(A);
            } else {
                extend_kernel<false><<<w->grid_extend, blk, 0, st>>>(A);
            }
            end(h);
            h = begin(2);
            if (gd) cudaMemsetAsync(w->ctr + 12, 0, sizeof(uint32_t), st);
            if (sorted) {
                shade_keys_kernel<false><<<w->grid_sort, blk, 0, st>>>(A);
                shade_scan_kernel<<<1, SORT_BLOCKS_MAX, 0, st>>>(A, (uint32_t)w->grid_sort);
                shade_scatter_kernel<<<w->grid_sort, blk, 0, st>>>(A);
                launches += 3;
            }
            switch (pl->quality) {
                case LAM_QUALITY_LOW: launch_shade<LAM_QUALITY_LOW>(guide, learned, w->grid_shade, blk, st, A); break;
                case LAM_QUALITY_HIGH: launch_shade<LAM_QUALITY_HIGH>(guide, learned, w->grid_shade, blk, st, A); break;
                default: launch_shade<LAM_QUALITY_MEDIUM>(guide, learned, w->grid_shade, blk, st, A); break;
            }
            launches += 2;
            if (gd) {
                const int gg = use_net ? w->grid_guide : w->grid_shade;
                switch (pl->quality) {
                    case LAM_QUALITY_LOW: launch_guide<LAM_QUALITY_LOW>(use_net, guide, gg, st, A); break;
                    case LAM_QUALITY_HIGH: launch_guide<LAM_QUALITY_HIGH>(use_net, guide, gg, st, A); break;
                    default: launch_guide<LAM_QUALITY_MEDIUM>(use_net, guide, gg, st, A); break;
                }
                ++launches;
            }
            end(h);
            std::swap(qa, qb);
            std::swap(ca, cb);
            std::swap(rao, rbo);
            std::swap(rad, rbd);
            std::swap(tha, thb);
            std::swap(aca, acb);
            std::swap(mia, mib);
        }
        h = begin(3);
        if (guide) {
            shuffle_kernel<<<gpix, blk, 0, st>>>(A);
            ++launches;
        }
        const uint32_t last = first + A.wave_count >= pl->opts.samples ? 1u : 0u;
        accumulate_kernel<0><<<gpix, blk, 0, st>>>(A, last);
        end(h);
        ++launches;
        if (training) {
            h = begin(4);
            for (uint32_t k = 0; k < gd->opts.steps_per_wave; ++k) {
                rc = guide_grad_and_update(gd, gd->records, GUIDE_RECORD_STRIDE, gd->opts.record_capacity, w->ctr + 13,
                                           gd->opts.batch, false, 1.0f / (float)gd->opts.batch, s->bounds, 1u, nullptr,
                                           nullptr, st);
                if (rc) return rc;
                launches += 2;
            }
            end(h);
            gd->trained_spp += A.wave_count;
        }
        first += count;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "lam_render launch");
    pl->stats.samples = (uint64_t)w->npix * pl->opts.samples;
    pl->stats_ctr = w->ctr;
    pl->stats.kernel_launches = launches;
    pl->stats_pending = true;
    return LAM_OK;
}

// ---------------------------------------------------------------- batched renders: host side
namespace lam {

struct BatchState {
    WaveBuffers* wave = nullptr;  // path state for `capacity` paths
    uint32_t capacity = 0;
    BatchReq* reqs = nullptr;
    BatchSeg* segs = nullptr;
    uint32_t* done = nullptr;
    unsigned long long* times = nullptr;
    float4* pix_color = nullptr;
    uint32_t* pixel_seed = nullptr;
    size_t reqs_cap = 0, segs_cap = 0, done_cap = 0, times_cap = 0, pix_cap = 0, seed_cap = 0;
    uint64_t generation = 0;  // bumped whenever a buffer moves (invalidates a captured graph)
    uint32_t last_n = 0;
    cudaStream_t stream = nullptr;  // capture stream (the legacy default stream cannot be captured)
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<char> graph_key;
};

void free_batch(BatchState* b) {
    if (!b) return;
    free_wave(b->wave);
    cudaFree(b->reqs);
    cudaFree(b->segs);
    cudaFree(b->done);
    cudaFree(b->times);
    cudaFree(b->pix_color);
    cudaFree(b->pixel_seed);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->ev_in) cudaEventDestroy(b->ev_in);
    if (b->ev_out) cudaEventDestroy(b->ev_out);
    delete b;
}

struct BatchPlan {
    std::vector<BatchSeg> segs;
    std::vector<uint32_t> wave_begin, wave_nsegs, wave_paths, wave_threads;
    std::vector<uint32_t> pix_base;
    size_t pixels = 0;
};

// Shortest requests first (pixels x samples); each wave takes whole sample planes of requests until
// `capacity` paths.
static BatchPlan plan_batch(const lam_batch_request* r, uint32_t n, uint32_t capacity) {
    BatchPlan P;
    P.pix_base.resize(n);
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) {
        order[i] = i;
        P.pix_base[i] = (uint32_t)P.pixels;
        P.pixels += (size_t)r[i].targets.width * r[i].targets.height;
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return (uint64_t)r[a].targets.width * r[a].targets.height * r[a].samples <
               (uint64_t)r[b].targets.width * r[b].targets.height * r[b].samples;
    });
    uint32_t used = 0, threads = 0, begin = 0;
    auto close = [&]() {
        if (P.segs.size() == begin) return;
        P.wave_begin.push_back(begin);
        P.wave_nsegs.push_back((uint32_t)P.segs.size() - begin);
        P.wave_paths.push_back(used);
        P.wave_threads.push_back(threads);
        begin = (uint32_t)P.segs.size();
        used = threads = 0;
    };
    for (uint32_t q : order) {
        const uint32_t npix = r[q].targets.width * r[q].targets.height;
        uint32_t first = 0;
        while (first < r[q].samples) {
            uint32_t fit = (capacity - used) / npix;
            if (fit == 0 || P.segs.size() - begin >= 255) {
                close();
                fit = capacity / npix;
            }
            fit = std::min(fit, r[q].samples - first);
            BatchSeg sg;
            sg.req = q;
            sg.first = first;
            sg.count = fit;
            sg.path_base = used;
            sg.pix_thread_base = threads;
            P.segs.push_back(sg);
            used += fit * npix;
            threads += npix;
            first += fit;
        }
    }
    close();
    return P;
}

template <class T>
static int dgrow(BatchState* b, T** p, size_t* cap, size_t need) {
    if (*cap >= need && *p) return LAM_OK;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    b->generation++;
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(1, need) * sizeof(T));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (batch)");
    *cap = need;
    return LAM_OK;
}

static int batch_wave_buffers(BatchState* b, uint32_t capacity) {
    if (b->wave && b->capacity >= capacity) return LAM_OK;
    b->generation++;
    free_wave(b->wave);
    b->wave = nullptr;
    WaveBuffers* w = new WaveBuffers();
    w->paths = capacity;
    int rc = 0;
    rc |= walloc(w, &w->ray_o, capacity);
    rc |= walloc(w, &w->ray_d, capacity);
    rc |= walloc(w, &w->ray_o2, capacity);
    rc |= walloc(w, &w->ray_d2, capacity);
    rc |= walloc(w, &w->qthr0, capacity);
    rc |= walloc(w, &w->qthr1, capacity);
    rc |= walloc(w, &w->qacc0, capacity);
    rc |= walloc(w, &w->qacc1, capacity);
    rc |= walloc(w, &w->qmisc0, capacity);
    rc |= walloc(w, &w->qmisc1, capacity);
    rc |= walloc(w, &w->hit, capacity);
    rc |= walloc(w, &w->queue0, capacity);
    rc |= walloc(w, &w->queue1, capacity);
    rc |= walloc(w, &w->thr, capacity);
    rc |= walloc(w, &w->acc, capacity);
    rc |= walloc(w, &w->brdf, capacity);
    rc |= walloc(w, &w->seed, capacity);
    rc |= walloc(w, &w->flags, capacity);
    rc |= walloc(w, &w->ctr, 64);
    if (rc) {
        free_wave(w);
        return LAM_ERR_CUDA;
    }
    cudaMemset(w->ctr, 0, 64 * sizeof(uint32_t));
    b->wave = w;
    b->capacity = capacity;
    return LAM_OK;
}

static void batch_key(const lam_batch_request* r, uint32_t n, const lam_batch_tuning& t, uint64_t generation,
                      bool sorted, std::vector<char>& key) {
    const size_t base = sizeof(uint32_t) + n * sizeof(lam_batch_request) + sizeof(t) + sizeof(generation);
    key.resize(base + 1);
    char* k = key.data();
    std::memcpy(k, &n, sizeof(n));
    std::memcpy(k + sizeof(n), r, n * sizeof(lam_batch_request));
    std::memcpy(k + sizeof(n) + n * sizeof(lam_batch_request), &t, sizeof(t));
    std::memcpy(k + sizeof(n) + n * sizeof(lam_batch_request) + sizeof(t), &generation, sizeof(generation));
    k[base] = sorted ? 1 : 0;
}

}  // namespace lam

extern "C" int lam_batch_render(lam_pipeline* pl, const lam_batch_request* reqs, uint32_t n,
                                const lam_batch_tuning* tuning_in, void* stream) {
    if (!pl || (n && !reqs)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_batch_render: null argument");
    if (n == 0) return LAM_OK;
    if (pl->quality >= LAM_DEBUG_FRONT_FACE) return set_error(LAM_ERR_UNSUPPORTED, "batched renders use the path-tracing shaders");
    if (pl->opts.guide_mode != LAM_GUIDE_NONE || pl->opts.restir_temporal != LAM_RESTIR_DISABLED)
        return set_error(LAM_ERR_UNSUPPORTED, "batched renders are plain path tracing (no guiding, ReSTIR disabled)");
    uint32_t max_pix = 0;
    bool all_opaque = true;
    for (uint32_t i = 0; i < n; ++i) {
        const lam_batch_request& r = reqs[i];
        if (!r.scene || r.samples == 0 || r.targets.width == 0 || r.targets.height == 0)
            return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_batch_render: request without scene, samples or size");
        if ((uint64_t)r.targets.width * r.targets.height > (1u << 26))
            return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_batch_render: request image too large");
        const lam_scene* sc = r.scene;
        if (sc->instance_count > pl->layout.blas_count || sc->diffuse_count > pl->layout.diffuse_count ||
            sc->emission_count > pl->layout.emission_count || sc->attribute_count > pl->layout.attribute_count)
            return set_error(LAM_ERR_LAYOUT_MISMATCH, "a request's scene exceeds the pipeline layout counts");
        if (sc->dev.has_procedural && !pl->handler_cubin.empty())
            return set_error(LAM_ERR_UNSUPPORTED, "batched renders do not run intersection handlers");
        max_pix = std::max(max_pix, r.targets.width * r.targets.height);
        all_opaque = all_opaque && sc->dev.all_opaque;
    }
    lam_batch_tuning t{};
    if (tuning_in) t = *tuning_in;
    if (!t.wave_paths) t.wave_paths = 8u << 20;
    t.wave_paths = std::max(t.wave_paths, max_pix);
    if (!pl->batch) pl->batch = new BatchState();
    BatchState* b = pl->batch;
    pl->stats_ctr = nullptr;  // the counters may move with the batch buffers
    pl->stats_pending = false;
    int rc = batch_wave_buffers(b, t.wave_paths);
    if (rc) return rc;
    WaveBuffers* w = b->wave;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int occ_e = 0, occ_s = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e, extend_batch_kernel<false>, WAVE_BLOCK, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, shade_kernel<LAM_QUALITY_MEDIUM, false, false, true>, WAVE_BLOCK, 0);
    const int grid_e = sms * (int)(t.extend_blocks_per_sm ? std::min<uint32_t>(t.extend_blocks_per_sm, std::max(1, occ_e))
                                                          : (uint32_t)std::max(1, occ_e));
    const int grid_s = sms * (int)(t.shade_blocks_per_sm ? t.shade_blocks_per_sm : (uint32_t)std::max(1, occ_s));
    const BatchPlan P = plan_batch(reqs, n, t.wave_paths);
    // material-ordered shading (no Markov guiding here, so the automatic order sorts)
    const bool sorted = pl->shade_order != LAM_SHADE_ORDER_QUEUE;
    const int grid_sort = std::min(SORT_BLOCKS_MAX, sms * 6);
    if (sorted && !w->shade_order) {
        b->generation++;  // a captured graph does not know the new buffers
        if (walloc(w, &w->shade_key, b->capacity) || walloc(w, &w->shade_order, b->capacity) ||
            walloc(w, &w->shade_bc, (size_t)SORT_BLOCKS_MAX * SHADE_CLASSES))
            return LAM_ERR_CUDA;
    }
    // device tables (uploaded before any capture)
    if (dgrow(b, &b->reqs, &b->reqs_cap, n) || dgrow(b, &b->segs, &b->segs_cap, P.segs.size()) ||
        dgrow(b, &b->done, &b->done_cap, n) || dgrow(b, &b->times, &b->times_cap, n + 1) ||
        dgrow(b, &b->pix_color, &b->pix_cap, P.pixels) || dgrow(b, &b->pixel_seed, &b->seed_cap, P.pixels))
        return LAM_ERR_CUDA;
    std::vector<BatchReq> hr(n);
    for (uint32_t i = 0; i < n; ++i) {
        const lam_batch_request& r = reqs[i];
        BatchReq& q = hr[i];
        q.S = r.scene->dev;
        q.cam = r.camera;
        q.camera_pos = v3{r.camera.view_inverse[12], r.camera.view_inverse[13], r.camera.view_inverse[14]};
        q.width = r.targets.width;
        q.height = r.targets.height;
        q.npix = q.width * q.height;
        q.samples = r.samples;
        q.seed_offset = r.seed_offset;
        q.pix_base = P.pix_base[i];
        q.out_color = (float4*)r.targets.color;
        q.out_normal = (float4*)r.targets.normal;
        q.out_albedo = (float4*)r.targets.albedo;
    }
    cudaError_t e = cudaMemcpy(b->reqs, hr.data(), n * sizeof(BatchReq), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->segs, P.segs.data(), P.segs.size() * sizeof(BatchSeg), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "lam_batch_render tables");
    b->last_n = n;
    if (!b->stream) {
        if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_error(e, "batch stream");
    }
    cudaStream_t caller = (cudaStream_t)stream;
    cudaStream_t st = b->stream;
    cudaEventRecord(b->ev_in, caller);
    cudaStreamWaitEvent(st, b->ev_in, 0);

    Args A;
    std::memset(&A, 0, sizeof(A));
    A.max_depth = pl->opts.max_depth;
    A.restir = LAM_RESTIR_DISABLED;
    A.tmin = pl->opts.tmin;
    A.tmax = pl->opts.tmax;
    A.ray_o = w->ray_o;
    A.ray_d = w->ray_d;
    A.hit = w->hit;
    A.err = w->ctr + 4;
    A.segments = reinterpret_cast<unsigned long long*>(w->ctr + 8);
    A.thr = w->thr;
    A.acc = w->acc;
    A.brdf = w->brdf;
    A.seed = w->seed;
    A.flags = w->flags;
    A.pix_color = b->pix_color;
    A.pixel_seed = b->pixel_seed;
    A.reqs = b->reqs;
    A.req_done = b->done;
    A.req_time = b->times;
    if (sorted) {
        A.shade_key = w->shade_key;
        A.shade_order = w->shade_order;
        A.shade_bc = w->shade_bc;
    }
    const dim3 blk(WAVE_BLOCK);
    uint32_t launches = 0;
    auto record = [&]() {
        cudaMemsetAsync(w->ctr, 0, 10 * sizeof(uint32_t), st);
        batch_start_kernel<<<1, 256, 0, st>>>(b->done, b->times, n);
        for (size_t wv = 0; wv < P.wave_begin.size(); ++wv) {
            A.segs = b->segs + P.wave_begin[wv];
            A.nsegs = P.wave_nsegs[wv];
            A.pix_threads = P.wave_threads[wv];
            A.npix = P.wave_paths[wv];
            uint32_t* qa = w->queue0;
            uint32_t* qb = w->queue1;
            uint32_t* ca = w->ctr + 0;
            uint32_t* cb = w->ctr + 1;
            float4 *rao = w->ray_o, *rad = w->ray_d, *rbo = w->ray_o2, *rbd = w->ray_d2;  // rays of qa, qb
            float4 *tha = w->qthr0, *thb = w->qthr1, *aca = w->qacc0, *acb = w->qacc1;   // path state of qa, qb
            uint4 *mia = w->qmisc0, *mib = w->qmisc1;
            A.q_in = qa;
            A.count_in = ca;
            A.ray_o = rao;
            A.ray_d = rad;
            A.qthr = tha;
            A.qacc = aca;
            A.qmisc = mia;
            const dim3 gp((A.pix_threads + WAVE_BLOCK - 1) / WAVE_BLOCK);
            batch_generate_kernel<<<gp, blk, 0, st>>>(A);
            for (uint32_t depth = 0; depth < pl->opts.max_depth; ++depth) {
                A.q_in = qa;
                A.q_out = qb;
                A.count_in = ca;
                A.count_out = cb;
                A.ray_o = rao;
                A.ray_d = rad;
                A.ray_o_out = rbo;
                A.ray_d_out = rbd;
                A.qthr = tha;
                A.qacc = aca;
                A.qmisc = mia;
                A.qthr_out = thb;
                A.qacc_out = acb;
                A.qmisc_out = mib;
                A.work = w->ctr + 2;
                cudaMemsetAsync(w->ctr + 2, 0, sizeof(uint32_t), st);
                cudaMemsetAsync(cb, 0, sizeof(uint32_t), st);
                if (all_opaque) extend_batch_kernel<false><<<grid_e, blk, 0, st>>>(A);
                else extend_batch_kernel<true><<<grid_e, blk, 0, st>>>(A);
                if (sorted) {
                    shade_keys_kernel<true><<<grid_sort, blk, 0, st>>>(A);
                    shade_scan_kernel<<<1, SORT_BLOCKS_MAX, 0, st>>>(A, (uint32_t)grid_sort);
                    shade_scatter_kernel<<<grid_sort, blk, 0, st>>>(A);
                    launches += 3;
                }
                switch (pl->quality) {
                    case LAM_QUALITY_LOW: shade_kernel<LAM_QUALITY_LOW, false, false, true><<<grid_s, blk, 0, st>>>(A); break;
                    case LAM_QUALITY_HIGH: shade_kernel<LAM_QUALITY_HIGH, false, false, true><<<grid_s, blk, 0, st>>>(A); break;
                    default: shade_kernel<LAM_QUALITY_MEDIUM, false, false, true><<<grid_s, blk, 0, st>>>(A); break;
                }
                launches += 2;
                std::swap(qa, qb);
                std::swap(ca, cb);
                std::swap(rao, rbo);
                std::swap(rad, rbd);
                std::swap(tha, thb);
                std::swap(aca, acb);
                std::swap(mia, mib);
            }
            batch_accumulate_kernel<<<gp, blk, 0, st>>>(A);
            launches += 2;
        }
    };
    if (t.use_graph) {
        std::vector<char> key;
        batch_key(reqs, n, t, b->generation, sorted, key);
        if (!b->graph || key != b->graph_key) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_error(e, "lam_batch_render capture");
            record();
            e = cudaStreamEndCapture(st, &g);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_error(e, "lam_batch_render graph");
            b->graph_key = key;
        }
        e = cudaGraphLaunch(b->graph, st);
        if (e != cudaSuccess) return cuda_error(e, "lam_batch_render graph launch");
    } else {
        record();
    }
    cudaEventRecord(b->ev_out, st);
    cudaStreamWaitEvent(caller, b->ev_out, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "lam_batch_render launch");
    pl->stats.samples = 0;
    for (uint32_t i = 0; i < n; ++i) pl->stats.samples += (uint64_t)reqs[i].targets.width * reqs[i].targets.height * reqs[i].samples;
    pl->stats.kernel_launches = launches;
    pl->stats_ctr = w->ctr;
    pl->stats_pending = true;
    return LAM_OK;
}

extern "C" int lam_batch_latencies(lam_pipeline* pl, uint32_t n, double* ms) {
    if (!pl || !ms) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    BatchState* b = pl->batch;
    if (!b || b->last_n != n) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_batch_latencies: n differs from the last batch");
    std::vector<unsigned long long> h(n + 1);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), b->times, (n + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "lam_batch_latencies");
    for (uint32_t i = 0; i < n; ++i) ms[i] = (double)(long long)(h[i] - h[n]) * 1e-6;
    return LAM_OK;
}

extern "C" int lam_batch_autotune(lam_pipeline* pl, const lam_batch_request* reqs, uint32_t n, uint32_t spp_divisor,
                                  lam_batch_tuning* out, void* stream) {
    if (!pl || !out || (n && !reqs)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_batch_autotune: null argument");
    std::vector<lam_batch_request> r(reqs, reqs + n);
    const uint32_t div = std::max(1u, spp_divisor);
    for (auto& q : r) q.samples = std::max(1u, q.samples / div);
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // each candidate runs as it will be used (CUDA graph on): one call to capture the graph and touch
    // the buffers, then the best of three timed replays
    auto timeit = [&](const lam_batch_tuning& t, float* ms) -> int {
        int rc = lam_batch_render(pl, r.data(), n, &t, stream);
        if (rc) return rc;
        *ms = 3.0e38f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, st);
            rc = lam_batch_render(pl, r.data(), n, &t, stream);
            if (rc) return rc;
            cudaEventRecord(e1, st);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) return cuda_error(e, "lam_batch_autotune");
            float m = 0.0f;
            cudaEventElapsedTime(&m, e0, e1);
            *ms = std::min(*ms, m);
        }
        return LAM_OK;
    };
    lam_batch_tuning best{};
    best.use_graph = 1;
    float best_ms = 3.0e38f;
    int rc = LAM_OK;
    // coordinate 1: queue size
    for (uint32_t wp : {2u << 20, 4u << 20, 8u << 20, 16u << 20, 32u << 20}) {
        lam_batch_tuning t = best;
        t.wave_paths = wp;
        float ms = 0;
        if ((rc = timeit(t, &ms))) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    // coordinate 2: shade CTAs per SM; coordinate 3: extend CTAs per SM
    for (int c = 0; c < 2 && rc == LAM_OK; ++c) {
        lam_batch_tuning base = best;
        for (uint32_t v : {1u, 2u, 3u, 4u, 6u}) {
            lam_batch_tuning t = base;
            if (c == 0) t.shade_blocks_per_sm = v;
            else t.extend_blocks_per_sm = v;
            float ms = 0;
            if ((rc = timeit(t, &ms))) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    best.use_graph = 1;
    *out = best;
    return LAM_OK;
}

extern "C" int lam_pipeline_trace_rays(lam_pipeline* pl, const lam_scene* s, const lam_ray* rays, uint32_t n,
                                       uint32_t mode, lam_hit* hits, void* stream) {
    if (!pl || !s || (n && (!rays || !hits))) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_pipeline_trace_rays: null argument");
    if (!s->dev.has_procedural || pl->handler_cubin.empty()) return lam_trace_rays(s, rays, n, mode, hits, stream);
    if (mode != LAM_TRACE_CLOSEST && mode != LAM_TRACE_ANY)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_pipeline_trace_rays: unknown mode");
    if (n == 0) return LAM_OK;
    if (int rc = check_trace_call(s, n, "lam_pipeline_trace_rays")) return rc;
    int rc = ensure_handler(pl);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* scratch = nullptr;  // [0] work counter, [1] error flags
    cudaError_t e = cudaMallocAsync((void**)&scratch, 8, st);
    if (e != cudaSuccess) return cuda_error(e, "lam_pipeline_trace_rays scratch");
    cudaMemsetAsync(scratch, 0, 8, st);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    DevScene S = s->dev;
    uint32_t* counter = scratch;
    uint32_t* err = scratch + 1;
    void* kargs[] = {&S, &rays, &n, &hits, &counter, &err};
    cudaKernel_t k = mode == LAM_TRACE_ANY ? pl->handler->trace_any : pl->handler->trace_closest;
    e = cudaLaunchKernel((const void*)k, dim3(sms * 8), dim3(TRACE_BLOCK), kargs, 0, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(scratch, st);
        return cuda_error(e, "procedural trace launch");
    }
    uint32_t err_flags = 0;
    cudaMemcpyAsync(&err_flags, err, 4, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(scratch, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "lam_pipeline_trace_rays");
    if (err_flags & ERR_STACK_OVERFLOW) return set_error(LAM_ERR_STACK_OVERFLOW, "traversal stack overflow");
    return LAM_OK;
}
