// debug.cu - the reference's debugging shaders (src/debug/mod.rs:1-56) as one kernel over the
// same traversal: one thread per pixel, one primary ray (pixel corner, no jitter).
//   FrontFace   (debug/front_face.wesl:44-102):  green = 1 / (t + 1) on a front face, red on a back face
//   Reflectance (debug/reflectance.wesl:40-95):  (ior_low / 5, ior_high / 5, 0) of the hit material
//   Tangent     (debug/tangent.wesl:50-118):     (corrected normalize(v0 - v1) + 1) / 2 in object space
// The candidate test of these shaders accepts a non-opaque triangle only when its diffuse alpha is
// not near zero (no exception for transparent materials).  normal and albedo outputs are zero.
#include "materials.cuh"
#include "scene.h"
#include "tracer.h"
#include "traverse.cuh"

namespace lam {

struct DebugArgs {
    DevScene S;
    lam_camera cam;
    uint32_t width, height, mode;
    float tmin, tmax;
    float4 *color, *normal, *albedo;
};

template <bool ALPHA>
__global__ void __launch_bounds__(128) debug_kernel(DebugArgs A) {
    __shared__ TraceSmem sm;
    const uint4* tl;
    const DevInstance* in;
    stage_tlas(A.S, sm, tl, in);
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.width * A.height) return;
    const uint32_t x = p % A.width, y = p / A.width;
    // create_ray (debug/*.wesl, identical to general.wesl:1158-1173)
    float hx = __uint2float_rn(A.width) / 2.0f, hy = __uint2float_rn(A.height) / 2.0f;
    float v[4] = {(__uint2float_rn(x) / hx) - 1.0f, -((__uint2float_rn(y) / hy) - 1.0f), 1.0f, 1.0f};
    const float* P = A.cam.projection_inverse;
    float q[4];
    for (int i = 0; i < 4; ++i) q[i] = P[i] * v[0] + P[4 + i] * v[1] + P[8 + i] * v[2] + P[12 + i] * v[3];
    float l = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int i = 0; i < 4; ++i) q[i] = q[i] / l;
    const float* V = A.cam.view_inverse;
    float3 d = make_float3(V[0] * q[0] + V[4] * q[1] + V[8] * q[2] + V[12] * 0.0f,
                           V[1] * q[0] + V[5] * q[1] + V[9] * q[2] + V[13] * 0.0f,
                           V[2] * q[0] + V[6] * q[1] + V[10] * q[2] + V[14] * 0.0f);
    float3 o = make_float3(V[12], V[13], V[14]);
    Traverser<false, ALPHA> T;
    uint2 stack[TRAVERSAL_STACK];
    uint32_t err = 0;
    T.transparent_passes = false;
    T.init(A.S, o, d, A.tmin, A.tmax);
    while (T.step(A.S, tl, in, stack, err)) {
    }
    float3 c = make_float3(0.0f, 0.0f, 0.0f);
    const TraceResult& r = T.res;
    if (A.mode == LAM_DEBUG_TANGENT) {
        float3 dir = make_float3(0.0f, 0.0f, 0.0f);
        if (r.tri != NO_HIT) {
            const float4* tp = A.S.tris + 3u * r.tri;
            float4 a = __ldg(tp), b = __ldg(tp + 1);
            v3 t = normalize(mk(a.x - b.x, a.y - b.y, a.z - b.z));
            dir = make_float3(t.x, t.y, t.z);
        }
        float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
        bool xl = ax > ay && ax > az, yl = ay > ax && ay > az;
        bool rev = xl ? dir.x < 0.0f : (yl ? dir.y < 0.0f : dir.z < 0.0f);
        if (rev) dir = make_float3(-dir.x, -dir.y, -dir.z);
        c = make_float3((dir.x + 1.0f) / 2.0f, (dir.y + 1.0f) / 2.0f, (dir.z + 1.0f) / 2.0f);
    } else if (r.tri != NO_HIT) {
        float m[12];
        for (int k = 0; k < 12; ++k) m[k] = in[r.inst].inv[k];
        float3 oo, od;
        object_ray(m, o, d, &oo, &od);
        const float4* tp = A.S.tris + 3u * r.tri;
        float t, bu, bv;
        bool front;
        wbw_f64(oo, od, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), &t, &bu, &bv, &front);
        if (A.mode == LAM_DEBUG_FRONT_FACE) {
            float g = 1.0f / (t + 1.0f);
            c = front ? make_float3(0.0f, g, 0.0f) : make_float3(g, 0.0f, 0.0f);
        } else {
            // reflectance.wesl:88 indexes the material tables by geometry_index (always 0 here), not
            // by the instance index
            lam_material mt = load_material(A.S, 0u, r.prim);
            float2 ior = unpack2x16float(mt.refractive_index);
            c = make_float3(ior.x / 5.0f, ior.y / 5.0f, 0.0f);
        }
    }
    if (A.color) A.color[p] = make_float4(c.x, c.y, c.z, 1.0f);
    if (A.normal) A.normal[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    if (A.albedo) A.albedo[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    (void)err;
}

int render_debug(lam_pipeline* pl, const lam_scene* s, const lam_camera* cam, const lam_frame_targets* tg,
                 cudaStream_t st) {
    DebugArgs A;
    A.S = s->dev;
    A.cam = *cam;
    A.width = tg->width;
    A.height = tg->height;
    A.mode = pl->quality;
    A.tmin = pl->opts.tmin;
    A.tmax = pl->opts.tmax;
    A.color = (float4*)tg->color;
    A.normal = (float4*)tg->normal;
    A.albedo = (float4*)tg->albedo;
    const uint32_t n = tg->width * tg->height;
    dim3 grid((n + 127) / 128), block(128);
    if (s->dev.all_opaque) debug_kernel<false><<<grid, block, 0, st>>>(A);
    else debug_kernel<true><<<grid, block, 0, st>>>(A);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "debug render launch");
    pl->stats.samples = n;
    pl->stats.kernel_launches = 1;
    pl->stats_pending = false;
    pl->stats.ray_segments = n;
    return LAM_OK;
}

}  // namespace lam
