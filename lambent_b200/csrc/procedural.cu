// procedural.cu - traversal kernels for scenes with procedural (AABB) geometry.  Built as LTO
// intermediate code with the intersection handler left external (lam_user_intersect), embedded in
// the library, and linked with the user's handler source at run time (handler_jit.cpp): the
// reference compiles its handler into the ray-query shader the same way (src/lib.rs:291-295,
// general.wesl:1068-1075).
#define LAM_HAVE_HANDLER 1
#include "materials.cuh"
#include "traverse.cuh"
#include "wavefront.cuh"

using namespace lam;

// The wavefront extend step (extend_kernel) with the handler: also records the handler's normal,
// tangent and t for procedural hits, which the shade kernel reads.
extern "C" __global__ void __launch_bounds__(WAVE_BLOCK) lam_proc_extend(const __grid_constant__ Args A) {
    __shared__ TraceSmem sm;
    const uint4* tl;
    const DevInstance* in;
    stage_tlas(A.S, sm, tl, in);
    const uint32_t n = *A.count_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(A.segments, (unsigned long long)n);
        atomicAdd(A.segments + 1, (unsigned long long)n);
    }
    uint32_t err = 0u;
    trace_persistent<false, true>(
        A.S, tl, in, n, A.work, err,
        [&](uint32_t i, float3& o, float3& d, float& t0, float& t1) {
            const float4 o4 = A.ray_o[i], d4 = A.ray_d[i];
            o = make_float3(o4.x, o4.y, o4.z);
            d = make_float3(d4.x, d4.y, d4.z);
            t0 = A.tmin;
            t1 = A.tmax;
        },
        [&](uint32_t i, const TraceResult& tr) {
            A.hit[i] = make_uint2(tr.tri, tr.inst);
            if (tr.tri != NO_HIT && (in[tr.inst].flags & INST_PROCEDURAL)) {
                const uint32_t path = A.q_in[i];
                A.phit_a[path] = make_float4(tr.pn.x, tr.pn.y, tr.pn.z, tr.t);
                A.phit_b[path] = make_float4(tr.ptg.x, tr.ptg.y, tr.ptg.z, 0.0f);
            }
        });
    if (err) atomicOr(A.err, err);
}

// lam_trace_rays with the handler (closest or any hit).
template <bool ANY>
LAM_DEV void proc_trace(const DevScene& S, const lam_ray* __restrict__ rays, uint32_t n, lam_hit* __restrict__ hits,
                        uint32_t* __restrict__ counter, uint32_t* __restrict__ err_out) {
    __shared__ TraceSmem sm;
    const uint4* tl;
    const DevInstance* in;
    stage_tlas(S, sm, tl, in);
    uint32_t err = 0u;
    auto load = [&](uint32_t i, float3& o, float3& d, float& t0, float& t1) {
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + i));
        const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
        o = make_float3(r0.x, r0.y, r0.z);
        d = make_float3(r1.x, r1.y, r1.z);
        t0 = r0.w;
        t1 = r1.w;
    };
    auto store = [&](uint32_t i, const TraceResult& tr) {
        lam_hit h;
        if (tr.tri == NO_HIT) {
            h.t = 0.0f; h.u = 0.0f; h.v = 0.0f;
            h.primitive_index = NO_HIT;
            h.instance_index = NO_HIT;
            h.kind = LAM_HIT_NONE;
        } else if (in[tr.inst].flags & INST_PROCEDURAL) {
            h.t = tr.t; h.u = 0.0f; h.v = 0.0f;
            h.primitive_index = tr.prim;
            h.instance_index = tr.inst;
            h.kind = LAM_HIT_BACK;
        } else {
            const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + i));
            const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
            const float3 o = make_float3(r0.x, r0.y, r0.z), d = make_float3(r1.x, r1.y, r1.z);
            float m[12];
            for (int q = 0; q < 12; ++q) m[q] = in[tr.inst].inv[q];
            float3 oo, od;
            object_ray(m, o, d, &oo, &od);
            const float4* tp = S.tris + 3u * tr.tri;
            bool front;
            wbw_f64(oo, od, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), &h.t, &h.u, &h.v, &front);
            h.primitive_index = tr.prim;
            h.instance_index = tr.inst;
            h.kind = front ? LAM_HIT_FRONT : LAM_HIT_BACK;
        }
        hits[i] = h;
    };
    trace_persistent<ANY, true>(S, tl, in, n, counter, err, load, store);
    if (err) atomicOr(err_out, err);
}

extern "C" __global__ void __launch_bounds__(TRACE_BLOCK)
lam_proc_trace_closest(DevScene S, const lam_ray* rays, uint32_t n, lam_hit* hits, uint32_t* counter, uint32_t* err) {
    proc_trace<false>(S, rays, n, hits, counter, err);
}
extern "C" __global__ void __launch_bounds__(TRACE_BLOCK)
lam_proc_trace_any(DevScene S, const lam_ray* rays, uint32_t n, lam_hit* hits, uint32_t* counter, uint32_t* err) {
    proc_trace<true>(S, rays, n, hits, counter, err);
}
