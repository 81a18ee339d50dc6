// traverse.cuh - two-level compressed-BVH8 traversal with the watertight triangle test.
//
// Replaces the driver ray query used by ray_hit (src/path_tracing/general.wesl:1053-1078):
// RayDesc(flags 0, cull mask 0xFF, T_MIN, T_MAX, origin, direction), committed closest hit.
// Contract (identical to the CPU oracle's):
//   * hit iff tmin < t < tmax; no face culling; opaque geometry commits without a callback;
//     non-opaque geometry runs the reference's alpha test (general.wesl:1059-1067);
//   * per triangle: Woop-Benthin-Wald watertight test in f32 with this exact operation order
//     (explicit __f*_rn intrinsics, never contracted) and an FP64 recomputation of the three
//     edge functions when any is exactly zero;
//   * ties in t go to the lowest (instance, primitive) pair;
//   * instances are entered with the f32 object-space ray o' = M^-1 o, d' = M^-1 d (fixed fma order).
// The box test evaluates each slab plane as one FMA against the node's quantization grid; the
// far distance is scaled by (1 + 2^-20) and child boxes carry one grid step of outward padding,
// which together cover the f32 rounding of the slab distances.
#pragma once
#include "device_math.cuh"
#include "scene.h"

namespace lam {

constexpr int TRAVERSAL_STACK = 32;
constexpr uint32_t NO_HIT = 0xFFFFFFFFu;
enum : uint32_t { ERR_STACK_OVERFLOW = 1u };

struct TravRay {
    float3 o, d, inv;
    uint32_t oct;
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

LAM_DEV float sel3(int k, float x, float y, float z) { return k == 0 ? x : (k == 1 ? y : z); }

LAM_DEV float safe_rcp(float x) {
    float y = fabsf(x) < 1e-30f ? copysignf(1e-30f, x) : x;
    // approximate reciprocal (<= 1 ulp): the slab distances only need to be conservative, which the
    // 2^-20 far-distance margin and the one-step box padding guarantee
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
}

LAM_DEV void setup_ray(TravRay& r, float3 o, float3 d) {
    r.o = o;
    r.d = d;
    r.inv = make_float3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    r.oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = sel3(kz, d.x, d.y, d.z);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    // shear constants from one IEEE reciprocal (the oracle uses the same three operations); any
    // constants serve, as long as every triangle a ray meets is tested with the same ones
    r.Sz = __fdiv_rn(1.0f, dz);
    r.Sx = __fmul_rn(sel3(kx, d.x, d.y, d.z), r.Sz);
    r.Sy = __fmul_rn(sel3(ky, d.x, d.y, d.z), r.Sz);
}

// setup_ray without the reciprocal and products of the shear constants (restores a ray whose Sx, Sy, Sz
// are known).
LAM_DEV void setup_ray_keep_shear(TravRay& r, float3 o, float3 d) {
    r.o = o;
    r.d = d;
    r.inv = make_float3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    r.oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = sel3(kz, d.x, d.y, d.z);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
}

LAM_DEV void object_ray(const float* m, float3 o, float3 d, float3* oo, float3* od) {
    oo->x = __fmaf_rn(m[0], o.x, __fmaf_rn(m[1], o.y, __fmaf_rn(m[2], o.z, m[3])));
    oo->y = __fmaf_rn(m[4], o.x, __fmaf_rn(m[5], o.y, __fmaf_rn(m[6], o.z, m[7])));
    oo->z = __fmaf_rn(m[8], o.x, __fmaf_rn(m[9], o.y, __fmaf_rn(m[10], o.z, m[11])));
    od->x = __fmaf_rn(m[0], d.x, __fmaf_rn(m[1], d.y, __fmul_rn(m[2], d.z)));
    od->y = __fmaf_rn(m[4], d.x, __fmaf_rn(m[5], d.y, __fmul_rn(m[6], d.z)));
    od->z = __fmaf_rn(m[8], d.x, __fmaf_rn(m[9], d.y, __fmul_rn(m[10], d.z)));
}

// Watertight test (f32).  Returns true with the IEEE quotient t = T / det when the ray crosses
// the triangle and t could beat `limit` (callers apply the exact tmin / limit / tie rules).
LAM_DEV bool wbw_f32(const TravRay& r, float4 a, float4 b, float4 c, float limit, float* t_out) {
    float Ax0 = __fsub_rn(a.x, r.o.x), Ay0 = __fsub_rn(a.y, r.o.y), Az0 = __fsub_rn(a.z, r.o.z);
    float Bx0 = __fsub_rn(b.x, r.o.x), By0 = __fsub_rn(b.y, r.o.y), Bz0 = __fsub_rn(b.z, r.o.z);
    float Cx0 = __fsub_rn(c.x, r.o.x), Cy0 = __fsub_rn(c.y, r.o.y), Cz0 = __fsub_rn(c.z, r.o.z);
    float Akx = sel3(r.kx, Ax0, Ay0, Az0), Aky = sel3(r.ky, Ax0, Ay0, Az0), Akz = sel3(r.kz, Ax0, Ay0, Az0);
    float Bkx = sel3(r.kx, Bx0, By0, Bz0), Bky = sel3(r.ky, Bx0, By0, Bz0), Bkz = sel3(r.kz, Bx0, By0, Bz0);
    float Ckx = sel3(r.kx, Cx0, Cy0, Cz0), Cky = sel3(r.ky, Cx0, Cy0, Cz0), Ckz = sel3(r.kz, Cx0, Cy0, Cz0);
    float Ax = __fmaf_rn(-r.Sx, Akz, Akx), Ay = __fmaf_rn(-r.Sy, Akz, Aky);
    float Bx = __fmaf_rn(-r.Sx, Bkz, Bkx), By = __fmaf_rn(-r.Sy, Bkz, Bky);
    float Cx = __fmaf_rn(-r.Sx, Ckz, Ckx), Cy = __fmaf_rn(-r.Sy, Ckz, Cky);
    float U = __fmaf_rn(Cx, By, -__fmul_rn(Cy, Bx));
    float V = __fmaf_rn(Ax, Cy, -__fmul_rn(Ay, Cx));
    float W = __fmaf_rn(Bx, Ay, -__fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
    float T = __fmaf_rn(U, Az, __fmaf_rn(V, Bz, __fmul_rn(W, Cz)));
    // conservative early out: |T / det| certainly above the current limit
    if (fabsf(T) > __fmul_rn(fabsf(det), limit) * 1.00000095367431640625f) return false;
    *t_out = __fdiv_rn(T, det);
    return true;
}

// FP64 re-evaluation of the committed hit (same formulas as the oracle, never contracted).
LAM_DEV void wbw_f64(float3 of, float3 df, float4 p0, float4 p1, float4 p2, float* t, float* u, float* v,
                     bool* front) {
    TravRay sel;
    // only the axis selection of setup_ray is needed
    {
        float ax = fabsf(df.x), ay = fabsf(df.y), az = fabsf(df.z);
        int kz = 0;
        float m = ax;
        if (ay > m) { kz = 1; m = ay; }
        if (az > m) kz = 2;
        int kx = kz + 1 == 3 ? 0 : kz + 1;
        int ky = kx + 1 == 3 ? 0 : kx + 1;
        if (sel3(kz, df.x, df.y, df.z) < 0.0f) { int tt = kx; kx = ky; ky = tt; }
        sel.kx = kx; sel.ky = ky; sel.kz = kz;
    }
    double o[3] = {of.x, of.y, of.z}, d[3] = {df.x, df.y, df.z};
    double P0[3] = {p0.x, p0.y, p0.z}, P1[3] = {p1.x, p1.y, p1.z}, P2[3] = {p2.x, p2.y, p2.z};
    double a[3], b[3], c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = __dsub_rn(P0[k], o[k]);
        b[k] = __dsub_rn(P1[k], o[k]);
        c[k] = __dsub_rn(P2[k], o[k]);
    }
    const int kx = sel.kx, ky = sel.ky, kz = sel.kz;
    double dkx = kx == 0 ? d[0] : (kx == 1 ? d[1] : d[2]);
    double dky = ky == 0 ? d[0] : (ky == 1 ? d[1] : d[2]);
    double dkz = kz == 0 ? d[0] : (kz == 1 ? d[1] : d[2]);
    auto pick = [&](const double* q, int k) { return k == 0 ? q[0] : (k == 1 ? q[1] : q[2]); };
    double Sx = __ddiv_rn(dkx, dkz), Sy = __ddiv_rn(dky, dkz), Sz = __ddiv_rn(1.0, dkz);
    double Ax = __dsub_rn(pick(a, kx), __dmul_rn(Sx, pick(a, kz))), Ay = __dsub_rn(pick(a, ky), __dmul_rn(Sy, pick(a, kz)));
    double Bx = __dsub_rn(pick(b, kx), __dmul_rn(Sx, pick(b, kz))), By = __dsub_rn(pick(b, ky), __dmul_rn(Sy, pick(b, kz)));
    double Cx = __dsub_rn(pick(c, kx), __dmul_rn(Sx, pick(c, kz))), Cy = __dsub_rn(pick(c, ky), __dmul_rn(Sy, pick(c, kz)));
    double U = __dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx));
    double V = __dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx));
    double W = __dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax));
    double det = __dadd_rn(__dadd_rn(U, V), W);
    double Az = __dmul_rn(Sz, pick(a, kz)), Bz = __dmul_rn(Sz, pick(b, kz)), Cz = __dmul_rn(Sz, pick(c, kz));
    double T = __dadd_rn(__dadd_rn(__dmul_rn(U, Az), __dmul_rn(V, Bz)), __dmul_rn(W, Cz));
    *t = __double2float_rn(__ddiv_rn(T, det));
    *u = __double2float_rn(__ddiv_rn(V, det));
    *v = __double2float_rn(__ddiv_rn(W, det));
    double e1[3] = {__dsub_rn(P1[0], P0[0]), __dsub_rn(P1[1], P0[1]), __dsub_rn(P1[2], P0[2])};
    double e2[3] = {__dsub_rn(P2[0], P0[0]), __dsub_rn(P2[1], P0[1]), __dsub_rn(P2[2], P0[2])};
    double n0 = __dsub_rn(__dmul_rn(e1[1], e2[2]), __dmul_rn(e1[2], e2[1]));
    double n1 = __dsub_rn(__dmul_rn(e1[2], e2[0]), __dmul_rn(e1[0], e2[2]));
    double n2 = __dsub_rn(__dmul_rn(e1[0], e2[1]), __dmul_rn(e1[1], e2[0]));
    double nd = __dadd_rn(__dadd_rn(__dmul_rn(n0, d[0]), __dmul_rn(n1, d[1])), __dmul_rn(n2, d[2]));
    *front = nd < 0.0;
}

// Byte k of w as the float 1 + byte * 2^-15 (the byte in mantissa bits 8..15 of 1.0f): one byte
// permute turns a quantized child coordinate into an exact float.
LAM_DEV float qone(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x3F800000u, 0x7604u + (k << 4)));
}

// Intersects the 8 children of one node.  Outputs the node group (child_base, internal hits in
// bits 24..31 in octant order | imask) and the leaf group (leaf_base, item hits in bits 0..23).
LAM_DEV void intersect_node(const uint4* __restrict__ np, const TravRay& r, float tmin, float tmax, uint2& ng,
                            uint2& tg) {
    const uint4 n0 = ld_keep(np), n1 = ld_keep(np + 1), n2 = ld_keep(np + 2), n3 = ld_keep(np + 3), n4 = ld_keep(np + 4);
    const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    const uint32_t imask = n0.w >> 24;
    const float sx = __uint_as_float((n0.w & 0xFFu) << 23);
    const float sy = __uint_as_float(((n0.w >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((n0.w >> 16) & 0xFFu) << 23);
    const float adx = __fmul_rn(sx, r.inv.x), ady = __fmul_rn(sy, r.inv.y), adz = __fmul_rn(sz, r.inv.z);
    const float aox = __fmul_rn(__fsub_rn(px, r.o.x), r.inv.x);
    const float aoy = __fmul_rn(__fsub_rn(py, r.o.y), r.inv.y);
    const float aoz = __fmul_rn(__fsub_rn(pz, r.o.z), r.inv.z);
    // near plane = lo plane when the inverse direction is positive
    const bool fx = r.inv.x < 0.0f, fy = r.inv.y < 0.0f, fz = r.inv.z < 0.0f;
    const uint32_t nx0 = fx ? n3.z : n2.x, nx1 = fx ? n3.w : n2.y, fx0 = fx ? n2.x : n3.z, fx1 = fx ? n2.y : n3.w;
    const uint32_t ny0 = fy ? n4.x : n2.z, ny1 = fy ? n4.y : n2.w, fy0 = fy ? n2.z : n4.x, fy1 = fy ? n2.w : n4.y;
    const uint32_t nz0 = fz ? n4.z : n3.x, nz1 = fz ? n4.w : n3.y, fz0 = fz ? n3.x : n4.z, fz1 = fz ? n3.y : n4.w;
    // Hit-mask contribution of each slot, four slots per word: bits (bits 5..7 of meta, unary) at
    // position `at` (bits 0..4; internal children sit at 24 + slot, which is XORed with the octant).
    // A byte is internal when its position is 24..31 (bits 3 and 4 set); bit 0 of each byte of
    // inner_* flags it, so inner_* * oct holds the octant in exactly the internal bytes.
    const uint32_t ma = n1.z, mb = n1.w;
    const uint32_t inner_a = ((ma & (ma << 1)) >> 4) & 0x01010101u, inner_b = ((mb & (mb << 1)) >> 4) & 0x01010101u;
    const uint32_t at_a = (ma ^ (inner_a * r.oct)) & 0x1F1F1F1Fu, at_b = (mb ^ (inner_b * r.oct)) & 0x1F1F1F1Fu;
    const uint32_t bits_a = (ma >> 5) & 0x07070707u, bits_b = (mb >> 5) & 0x07070707u;
    uint32_t hits = 0u;
    // t = q * adx + aox with q read as 1 + q * 2^-15: t = (1 + q * 2^-15) * (2^15 adx) + (aox - 2^15 adx).
    // Rounding B adds at most 2^-9 of a grid step (plus 2^-24 |aox|) to each plane distance, far inside
    // the builder's one-step outward padding and the 2^-20 far-plane margin.  This saves the
    // subtraction of an integer-to-float conversion per plane.  Should 2^15 adx overflow, the plane
    // distance is NaN, which fmaxf / fminf ignore: the test only becomes more permissive.
    const float Ax = 32768.0f * adx, Ay = 32768.0f * ady, Az = 32768.0f * adz;
    const float Bx = __fmaf_rn(-32768.0f, adx, aox), By = __fmaf_rn(-32768.0f, ady, aoy),
                Bz = __fmaf_rn(-32768.0f, adz, aoz);
#pragma unroll
    for (uint32_t i = 0; i < 8; ++i) {
        const uint32_t k = i & 3u;
        const float tnx = __fmaf_rn(qone(i < 4 ? nx0 : nx1, k), Ax, Bx);
        const float tny = __fmaf_rn(qone(i < 4 ? ny0 : ny1, k), Ay, By);
        const float tnz = __fmaf_rn(qone(i < 4 ? nz0 : nz1, k), Az, Bz);
        const float tfx = __fmaf_rn(qone(i < 4 ? fx0 : fx1, k), Ax, Bx);
        const float tfy = __fmaf_rn(qone(i < 4 ? fy0 : fy1, k), Ay, By);
        const float tfz = __fmaf_rn(qone(i < 4 ? fz0 : fz1, k), Az, Bz);
        const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
        const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
        if (tn <= tf * 1.00000095367431640625f)
            hits |= __byte_perm(i < 4 ? bits_a : bits_b, 0u, 0x4440u + k) << __byte_perm(i < 4 ? at_a : at_b, 0u, 0x4440u + k);
    }
    ng = make_uint2(n1.x, (hits & 0xFF000000u) | imask);
    tg = make_uint2(n1.y, hits & 0x00FFFFFFu);
}

struct TraceResult {
    uint32_t tri;   // global triangle slot, NO_HIT if none
    uint32_t inst;
    uint32_t prim;
    float t;        // f32 watertight distance
#ifdef LAM_HAVE_HANDLER
    float3 pn, ptg; // normal and tangent of a committed procedural hit (from the handler)
#endif
};

}  // namespace lam
#ifdef LAM_HAVE_HANDLER
// The intersection handler, linked in at run time (lam_tracer_set_intersection_handler).
extern "C" __device__ lam_aabb_intersection lam_user_intersect(const lam_ray_intersection& i);
#endif
namespace lam {

// Conservative ray / box test in the ray's own space (procedural candidates reach the handler only
// when the ray crosses their box inside (tmin, limit), as the driver's AABB candidates do).
LAM_DEV bool ray_box(const TravRay& r, float4 lo, float4 hi, float tmin, float limit) {
    const float tx0 = (lo.x - r.o.x) * r.inv.x, tx1 = (hi.x - r.o.x) * r.inv.x;
    const float ty0 = (lo.y - r.o.y) * r.inv.y, ty1 = (hi.y - r.o.y) * r.inv.y;
    const float tz0 = (lo.z - r.o.z) * r.inv.z, tz1 = (hi.z - r.o.z) * r.inv.z;
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), limit));
    return tn <= tf * 1.00000095367431640625f;
}

// Position of the r-th (from 0) set bit of m; r < popc(m).  Four population counts of halving
// windows (cheaper here than __fns).
LAM_DEV uint32_t nth_set_bit(uint32_t m, uint32_t r) {
    uint32_t pos = 0u, c = __popc(m & 0xFFFFu);
    if (r >= c) { r -= c; m >>= 16; pos += 16u; }
    c = __popc(m & 0xFFu);
    if (r >= c) { r -= c; m >>= 8; pos += 8u; }
    c = __popc(m & 0xFu);
    if (r >= c) { r -= c; m >>= 4; pos += 4u; }
    c = __popc(m & 0x3u);
    if (r >= c) { r -= c; m >>= 2; pos += 2u; }
    return pos + ((r >= (m & 1u)) ? 1u : 0u);
}

enum : int { STEP_MORE = 0, STEP_DONE = 1, STEP_COOP = 2 };

// Per-warp shared memory of the cooperative triangle phase (one slot per lane).
struct CoopScratch {
    float ox[32], oy[32], oz[32], sx[32], sy[32], sz[32], tmin[32], lim[32];
    uint32_t perm[32], excl[32], mask[32], base[32], item[32];
    unsigned long long key[32];
    const float4* tris[32];  // the owner's triangle array (lanes of one warp may trace different scenes)
};

// Alpha-test callback for non-opaque geometry: candidate accepted unless the diffuse texel's
// alpha is near zero, transparent materials always accepted (general.wesl:1059-1067).
LAM_DEV bool alpha_accept(const DevScene& S, uint32_t inst, uint32_t prim, float bu, float bv, bool transparent_passes);

// Resumable traversal: init() then step() until it returns false.  One step intersects one node
// and tests the leaf items it exposes, so a warp can refill lanes whose rays have finished
// (after Aila and Laine, "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009).
template <bool ANY, bool ALPHA>
struct Traverser {
    TravRay R;
    float3 wo, wd;
    float wSx, wSy, wSz;  // the world ray's shear constants, restored when an instance is left
    float tmin, best_t;
    uint2 ng, tg;
    int sp, blas_base;
    uint32_t cur_inst, cur_flags;
    TraceResult res;
    bool transparent_passes = true;  // transparent materials pass the alpha test (path shaders)

    LAM_DEV void init(const DevScene& S, float3 o, float3 d, float t0, float t1) {
        wo = o;
        wd = d;
        tmin = t0;
        best_t = t1;
        res.tri = NO_HIT;
        res.inst = NO_HIT;
        res.prim = NO_HIT;
        res.t = t1;
        sp = 0;
        blas_base = -1;
        cur_inst = 0u;
        cur_flags = 0u;
        setup_ray(R, o, d);
        wSx = R.Sx;
        wSy = R.Sy;
        wSz = R.Sz;
        ng = S.tlas_node_count ? make_uint2(0u, (1u << (24u + R.oct)) | 1u) : make_uint2(0u, 0u);
        tg = make_uint2(0u, 0u);
    }

    LAM_DEV void push(uint2* stack, uint2 g, uint32_t& err) {
        if (sp < TRAVERSAL_STACK) stack[sp++] = g;
        else err |= ERR_STACK_OVERFLOW;
    }

    // One traversal step: one node, then the leaf items it exposes.  Returns STEP_MORE, STEP_DONE
    // (res is final), or, with COOP, STEP_COOP when the exposed items are triangles of an opaque
    // instance: they are left in tg for the warp's shared triangle phase (coop_triangles), after
    // which finish_coop() completes the step.  `stack` holds TRAVERSAL_STACK entries owned by this
    // lane (kept outside the struct so that the struct itself stays in registers).
    template <bool COOP>
    LAM_DEV int step_impl(const DevScene& S, const uint4* __restrict__ tlas_nodes, const DevInstance* __restrict__ insts,
                          uint2* stack, uint32_t& err) {
        if (ng.y > 0x00FFFFFFu) {
            const uint32_t k = __ffs(ng.y >> 24) - 1u;
            ng.y &= ~(1u << (24u + k));
            const uint32_t slot = k ^ R.oct;
            const uint32_t child = ng.x + __popc(ng.y & ((1u << slot) - 1u) & 0xFFu);
            if (ng.y > 0x00FFFFFFu) push(stack, ng, err);
            // one call site for TLAS and BLAS nodes: lanes of a warp on either level share one test
            // (two call sites run the 8-wide test twice whenever a warp straddles the levels)
            intersect_node((blas_base < 0 ? tlas_nodes : S.blas_nodes) + 5u * child, R, tmin, best_t, ng, tg);
        } else {
            tg = ng;
            ng = make_uint2(0u, 0u);
        }
        if (COOP && blas_base >= 0 && tg.y != 0u && (cur_flags & (INST_OPAQUE | INST_PROCEDURAL)) == INST_OPAQUE)
            return STEP_COOP;
        while (tg.y != 0u) {
            const uint32_t k = __ffs(tg.y) - 1u;
            tg.y &= tg.y - 1u;
            const uint32_t item = tg.x + k;
            if (blas_base < 0) {
                const uint32_t id = __ldg(S.tlas_items + item);
                const DevInstance& I = insts[id];
                const uint32_t flags = I.flags;
                const uint32_t root = I.blas_root;
                if (!(flags & INST_VISIBLE) || root == NO_HIT) continue;
                if (tg.y != 0u) push(stack, tg, err);
                if (ng.y > 0x00FFFFFFu) push(stack, ng, err);
                blas_base = sp;
                cur_inst = id;
                cur_flags = flags;
                float m[12];
#pragma unroll
                for (int q = 0; q < 12; ++q) m[q] = I.inv[q];
                float3 oo, od;
                object_ray(m, wo, wd, &oo, &od);
                setup_ray(R, oo, od);
                ng = make_uint2(root, (1u << (24u + R.oct)) | 1u);
                tg = make_uint2(0u, 0u);
                return STEP_MORE;
            }
            const float4* tp = S.tris + 3u * item;
            if (cur_flags & INST_PROCEDURAL) {
#ifdef LAM_HAVE_HANDLER
                const float4 lo = __ldg(tp), hi = __ldg(tp + 1);
                if (!ray_box(R, lo, hi, tmin, best_t)) continue;
                const uint32_t prim = __float_as_uint(lo.w);
                lam_ray_intersection ri;
                ri.kind = LAM_INTERSECTION_AABB;
                ri.t = best_t;
                const float* fw = S.inst_fwd + 16u * cur_inst;
                ri.instance_custom_data = __float_as_uint(fw[12]);
                ri.instance_index = cur_inst;
                ri.sbt_record_offset = 0u;
                ri.geometry_index = 0u;
                ri.primitive_index = prim;
                ri.barycentrics[0] = 0.0f;
                ri.barycentrics[1] = 0.0f;
                ri.front_face = 0u;
#pragma unroll
                for (int q = 0; q < 12; ++q) {
                    ri.object_to_world[q] = fw[q];
                    ri.world_to_object[q] = insts[cur_inst].inv[q];
                }
                ri.world_origin[0] = wo.x; ri.world_origin[1] = wo.y; ri.world_origin[2] = wo.z;
                ri.world_direction[0] = wd.x; ri.world_direction[1] = wd.y; ri.world_direction[2] = wd.z;
                ri.object_origin[0] = R.o.x; ri.object_origin[1] = R.o.y; ri.object_origin[2] = R.o.z;
                ri.object_direction[0] = R.d.x; ri.object_direction[1] = R.d.y; ri.object_direction[2] = R.d.z;
                ri.tmin = tmin;
                ri.aabb_min[0] = lo.x; ri.aabb_min[1] = lo.y; ri.aabb_min[2] = lo.z;
                ri.aabb_max[0] = hi.x; ri.aabb_max[1] = hi.y; ri.aabb_max[2] = hi.z;
                const lam_aabb_intersection ai = lam_user_intersect(ri);
                const float t = ai.t;
                const bool better = ai.hit && t > tmin &&
                                    (t < best_t || (t == best_t && res.tri != NO_HIT &&
                                                    (cur_inst < res.inst || (cur_inst == res.inst && prim < res.prim))));
                if (!better) continue;
                best_t = t;
                res.tri = item;
                res.inst = cur_inst;
                res.prim = prim;
                res.pn = make_float3(ai.normal[0], ai.normal[1], ai.normal[2]);
                res.ptg = make_float3(ai.tangent[0], ai.tangent[1], ai.tangent[2]);
                if (ANY) {
                    res.t = best_t;
                    return STEP_DONE;
                }
#endif
                continue;
            }
            const float4 a = ld_keep(tp), b = ld_keep(tp + 1), c = ld_keep(tp + 2);
            float t;
            if (!wbw_f32(R, a, b, c, best_t, &t)) continue;
            const uint32_t prim = __float_as_uint(a.w);
            bool better = t > tmin && (t < best_t || (t == best_t && res.tri != NO_HIT &&
                                                      (cur_inst < res.inst || (cur_inst == res.inst && prim < res.prim))));
            if (!better) continue;
            if (ALPHA && !(cur_flags & INST_OPAQUE)) {
                float rt, ru, rv;
                bool fr;
                wbw_f64(R.o, R.d, a, b, c, &rt, &ru, &rv, &fr);
                if (!alpha_accept(S, cur_inst, prim, ru, rv, transparent_passes)) continue;
            }
            best_t = t;
            res.tri = item;
            res.inst = cur_inst;
            res.prim = prim;
            if (ANY) {
                res.t = best_t;
                return STEP_DONE;
            }
        }
        return tail(stack) ? STEP_MORE : STEP_DONE;
    }

    // Returns false once the traversal has finished (res is final).
    LAM_DEV bool step(const DevScene& S, const uint4* __restrict__ tlas_nodes, const DevInstance* __restrict__ insts,
                      uint2* stack, uint32_t& err) {
        return step_impl<false>(S, tlas_nodes, insts, stack, err) == STEP_MORE;
    }

    // End of a step: leave a finished instance, pop the next group; false when the ray is done.
    LAM_DEV bool tail(uint2* stack) {
        if (ng.y <= 0x00FFFFFFu) {
            if (blas_base >= 0 && sp == blas_base) {
                blas_base = -1;
                setup_ray_keep_shear(R, wo, wd);
                R.Sx = wSx;
                R.Sy = wSy;
                R.Sz = wSz;
            }
            if (sp == 0) {
                res.t = best_t;
                return false;
            }
            ng = stack[--sp];
        }
        return true;
    }

    // Completes a STEP_COOP step once the warp has tested this lane's triangles.
    LAM_DEV bool finish_coop(uint2* stack, bool hit_now) {
        if (ANY && hit_now) {
            res.t = best_t;
            return false;
        }
        return tail(stack);
    }

    // The warp's shared triangle phase: every lane of the warp takes part.  The pending triangles
    // (tg) of the lanes with `want` are dealt out over all 32 lanes; each tester runs the watertight
    // test against its owner's ray and folds (t, primitive) into the owner's slot with a 64-bit
    // shared-memory atomic minimum.  The owner then commits the minimum under the same rules as the
    // serial loop (closest, ties to the lowest (instance, primitive)), so results are bit-identical.
    // Returns whether this lane committed a new hit.
    LAM_DEV bool coop_triangles(bool want, const DevScene& S, CoopScratch& ws) {
        return coop_triangles_from(want, S.tris, ws);
    }
    LAM_DEV bool coop_triangles_from(bool want, const float4* my_tris, CoopScratch& ws) {
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t mask = want ? tg.y : 0u;
        const uint32_t cnt = __popc(mask);
        uint32_t incl = cnt;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        ws.excl[lane] = incl - cnt;
        ws.mask[lane] = mask;
        ws.base[lane] = tg.x;
        ws.ox[lane] = R.o.x;
        ws.oy[lane] = R.o.y;
        ws.oz[lane] = R.o.z;
        ws.sx[lane] = R.Sx;
        ws.sy[lane] = R.Sy;
        ws.sz[lane] = R.Sz;
        ws.perm[lane] = (uint32_t)R.kx | ((uint32_t)R.ky << 2) | ((uint32_t)R.kz << 4);
        ws.tmin[lane] = tmin;
        ws.lim[lane] = best_t;
        ws.key[lane] = ~0ull;
        ws.tris[lane] = my_tris;
        __syncwarp();
        for (uint32_t c0 = 0; c0 < total; c0 += 32u) {
            const uint32_t j = c0 + lane;
            bool has = false;
            unsigned long long key = 0ull;
            uint32_t owner = 0u, item = 0u;
            if (j < total) {
                // owner of test j: the last lane whose exclusive count is <= j
                uint32_t lo = 0u, hi = 31u;
#pragma unroll
                for (int it = 0; it < 5; ++it) {
                    const uint32_t mid = (lo + hi + 1u) >> 1;
                    if (ws.excl[mid] <= j) lo = mid;
                    else hi = mid - 1u;
                }
                owner = lo;
                const uint32_t bit = nth_set_bit(ws.mask[owner], j - ws.excl[owner]);
                item = ws.base[owner] + bit;
                TravRay r;
                r.o = make_float3(ws.ox[owner], ws.oy[owner], ws.oz[owner]);
                r.Sx = ws.sx[owner];
                r.Sy = ws.sy[owner];
                r.Sz = ws.sz[owner];
                const uint32_t pm = ws.perm[owner];
                r.kx = (int)(pm & 3u);
                r.ky = (int)((pm >> 2) & 3u);
                r.kz = (int)((pm >> 4) & 3u);
                const float4* tp = ws.tris[owner] + 3u * item;
                const float4 a = ld_keep(tp), b = ld_keep(tp + 1), c = ld_keep(tp + 2);
                float t;
                if (wbw_f32(r, a, b, c, ws.lim[owner], &t) && t > ws.tmin[owner]) {
                    const uint32_t u = __float_as_uint(t);
                    const uint32_t ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);  // float order as unsigned
                    key = ((unsigned long long)ord << 32) | __float_as_uint(a.w);
                    atomicMin(&ws.key[owner], key);
                    has = true;
                }
            }
            __syncwarp();
            if (has && key == ws.key[owner]) ws.item[owner] = item;  // (t, primitive) names one triangle
            __syncwarp();
        }
        bool hit_now = false;
        if (want) {
            const unsigned long long key = ws.key[lane];
            if (key != ~0ull) {
                const uint32_t ord = (uint32_t)(key >> 32);
                const float t = __uint_as_float((ord & 0x80000000u) ? (ord & 0x7FFFFFFFu) : ~ord);
                const uint32_t prim = (uint32_t)key;
                const bool better = t < best_t || (t == best_t && res.tri != NO_HIT &&
                                                   (cur_inst < res.inst || (cur_inst == res.inst && prim < res.prim)));
                if (better) {
                    best_t = t;
                    res.tri = ws.item[lane];
                    res.inst = cur_inst;
                    res.prim = prim;
                    hit_now = true;
                }
            }
            tg.y = 0u;
        }
        __syncwarp();
        return hit_now;
    }
};

// Lanes below this many active rays trigger a refill of the idle lanes from the work queue.
#ifndef LAM_REFILL_THRESHOLD
#define LAM_REFILL_THRESHOLD 28
#endif
constexpr int REFILL_THRESHOLD = LAM_REFILL_THRESHOLD;

// Persistent warp loop over work items [0, n) claimed with a global counter.  `load(i, o, d, t0, t1)`
// fetches item i; `store(i, res)` consumes a finished traversal.  Every lane of the warp must call it,
// in blocks of 128 threads.  Triangle tests of opaque instances are dealt out over the whole warp
// (Traverser::coop_triangles): with one ray per lane, a step exposes 0 to 24 triangles per lane, and
// a per-lane loop would run as long as the busiest lane.
template <bool ANY, bool ALPHA, class Load, class Store>
LAM_DEV void trace_persistent(const DevScene& S, const uint4* __restrict__ tl, const DevInstance* __restrict__ in,
                              uint32_t n, uint32_t* __restrict__ work, uint32_t& err, Load load, Store store) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    __shared__ CoopScratch coop_ws[4];  // one per warp of a 128-thread block
    CoopScratch& ws = coop_ws[(threadIdx.x >> 5) & 3u];
    Traverser<ANY, ALPHA> T;
    uint2 stack[TRAVERSAL_STACK];
    bool active = false, exhausted = false;
    uint32_t item = 0;
    for (;;) {
        const uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
        if (!exhausted && __popc(act) < REFILL_THRESHOLD) {
            const uint32_t need = ~act;
            const uint32_t leader = __ffs(need) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(work, (uint32_t)__popc(need));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (!active) {
                const uint32_t i = base + __popc(need & lt_mask);
                if (i < n) {
                    float3 o, d;
                    float t0, t1;
                    load(i, o, d, t0, t1);
                    T.init(S, o, d, t0, t1);
                    item = i;
                    active = true;
                }
            }
            if (base + (uint32_t)__popc(need) >= n) exhausted = true;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;
        int code = STEP_MORE;
        if (active) code = T.template step_impl<true>(S, tl, in, stack, err);
        const bool want = active && code == STEP_COOP;
        if (__any_sync(0xFFFFFFFFu, want)) {  // warp-uniform: triangle tests dealt out over all lanes
            const bool hit_now = T.coop_triangles(want, S, ws);
            if (want) code = T.finish_coop(stack, hit_now) ? STEP_MORE : STEP_DONE;
        }
        if (active && code == STEP_DONE) {
            store(item, T.res);
            active = false;
        }
    }
}

// As trace_persistent, for work items that belong to different scenes: `load(i, o, d, t0, t1, sp)`
// also returns the item's scene, whose TLAS and instances are read from global memory.
template <bool ANY, bool ALPHA, class Load, class Store>
LAM_DEV void trace_persistent_multi(uint32_t n, uint32_t* __restrict__ work, uint32_t& err, Load load, Store store) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    __shared__ CoopScratch coop_ws[4];  // one per warp of a 128-thread block
    CoopScratch& ws = coop_ws[(threadIdx.x >> 5) & 3u];
    Traverser<ANY, ALPHA> T;
    uint2 stack[TRAVERSAL_STACK];
    const DevScene* sp = nullptr;
    bool active = false, exhausted = false;
    uint32_t item = 0;
    for (;;) {
        const uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
        if (!exhausted && __popc(act) < REFILL_THRESHOLD) {
            const uint32_t need = ~act;
            const uint32_t leader = __ffs(need) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(work, (uint32_t)__popc(need));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (!active) {
                const uint32_t i = base + __popc(need & lt_mask);
                if (i < n) {
                    float3 o, d;
                    float t0, t1;
                    load(i, o, d, t0, t1, sp);
                    T.init(*sp, o, d, t0, t1);
                    item = i;
                    active = true;
                }
            }
            if (base + (uint32_t)__popc(need) >= n) exhausted = true;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;
        int code = STEP_MORE;
        if (active) code = T.template step_impl<true>(*sp, sp->tlas_nodes, sp->inst, stack, err);
        const bool want = active && code == STEP_COOP;
        if (__any_sync(0xFFFFFFFFu, want)) {
            const bool hit_now = T.coop_triangles_from(want, want ? sp->tris : nullptr, ws);
            if (want) code = T.finish_coop(stack, hit_now) ? STEP_MORE : STEP_DONE;
        }
        if (active && code == STEP_DONE) {
            store(item, T.res);
            active = false;
        }
    }
}

constexpr int TRACE_BLOCK = 128;
constexpr uint32_t SMEM_INSTANCES = 128;

struct TraceSmem {
    DevInstance inst[SMEM_INSTANCES];
};

// Copies the instance records into shared memory when they fit (every instance entry reads one);
// returns the pointers the traversal should use.  The TLAS nodes stay in global memory, where
// they are L1-resident: one node-test call site then loads TLAS and BLAS nodes alike through the
// read-only path (staging them in shared memory made those loads generic: 1104 against 1118
// Mrays/s).
LAM_DEV void stage_tlas(const DevScene& S, TraceSmem& sm, const uint4*& tl, const DevInstance*& in) {
    tl = S.tlas_nodes;
    in = S.inst;
    if (S.instance_count <= SMEM_INSTANCES) {
        const uint4* src = reinterpret_cast<const uint4*>(S.inst);
        uint4* dst = reinterpret_cast<uint4*>(sm.inst);
        for (uint32_t i = threadIdx.x; i < S.instance_count * 4u; i += blockDim.x) dst[i] = src[i];
        in = sm.inst;
    }
    __syncthreads();
}

}  // namespace lam
