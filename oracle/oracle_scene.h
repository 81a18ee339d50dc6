// oracle_scene.h - TEST INFRASTRUCTURE ONLY (the CPU oracle; see oracle_math.h).
//
// CPU restatement of the ray-query contract that the reference gets from its GPU driver
// (rayQueryInitialize / rayQueryProceed / rayQueryGetCommittedIntersection,
// src/path_tracing/general.wesl:1053-1078; BLAS/TLAS build, examples/cornell_box/src/main.rs:464-563):
//   * closest hit with tmin < t < tmax, no face culling, opaque geometry auto-commits;
//   * the per-triangle test is the watertight test of Woop, Benthin and Wald (JCGT 2013),
//     evaluated in IEEE f32 with fixed operation order and an FP64 fallback for zero edge
//     functions; ties in t are broken by the lowest (instance, primitive) index;
//   * the committed t and barycentrics are re-evaluated in FP64 for the winning triangle and
//     rounded to f32;
//   * instances are traversed in object space with the ray transformed by the f32 inverse of
//     the 3x4 instance matrix (inverse computed in FP64, rounded to f32).
// The acceleration structure here is a plain binary SAH BVH with conservative FP64 box tests;
// it shares nothing with the product's BVH8.
#pragma once
#include <cstdint>
#include <vector>
#include "oracle_math.h"
#include "../include/lambent.h"

namespace oracle {

struct Tex {
    std::vector<uint8_t> rgba;
    uint32_t w = 0, h = 0;
};

struct BNode {
    double lo[3], hi[3];
    int32_t left = -1, right = -1;  // children (internal)
    int32_t first = 0, count = 0;   // leaf range into the item index list (count > 0)
};

struct Bvh {
    std::vector<BNode> nodes;
    std::vector<uint32_t> items;
    void build(const std::vector<double>& boxes /* 6 per item */, uint32_t n);
};

struct Blas {
    std::vector<float> v;          // 3 floats per vertex
    std::vector<uint32_t> idx;     // 3 per triangle (expanded for non-indexed input)
    uint32_t tri_count = 0;
    bool opaque = true;
    Bvh bvh;
};

struct Instance {
    float xf[12];                  // object -> world, 3x4 row-major
    float inv[12];                 // world -> object (f32 rounding of the FP64 inverse)
    uint32_t blas = 0, mask = 0xFF, custom = 0;
    std::vector<uint32_t> mat;     // per-primitive material index
};

struct Hit {
    bool hit = false;
    float t = 0, u = 0, v = 0;     // FP64-refined, rounded to f32
    uint32_t prim = 0, inst = 0;
    bool front = false;
    vec3 ov0, ov1, ov2;            // object-space vertices of the committed triangle
};

struct Scene {
    std::vector<Blas> blas;
    std::vector<Instance> inst;
    Bvh tlas;
    std::vector<lam_material> materials;
    std::vector<Tex> diffuse, emission, attributes;
    Tex recolour;
    std::vector<uint8_t> sky;      // 6 * sky_size^2 * 4
    uint32_t sky_size = 0;

    int load(const lam_scene_desc* d);
    // closest (any_hit = false) or any hit.  Rays with tmin < t < tmax.
    Hit trace(vec3 o, vec3 d, float tmin, float tmax, bool any_hit) const;
    Hit trace_bruteforce(vec3 o, vec3 d, float tmin, float tmax) const;

    // texture helpers (nearest filter, clamp-to-edge: wgpu SamplerDescriptor::default())
    void sample(const std::vector<Tex>& arr, uint32_t layer, float u, float v, float out[4]) const;
    void load_recolour(uint32_t x, uint32_t y, float out[4]) const;
    vec3 background(vec3 dir) const;
    bool alpha_accept(uint32_t inst, uint32_t prim, float bu, float bv) const;
};

// Instance-matrix inverse (FP64 adjugate / determinant, rounded to f32).  Returns false if singular.
bool invert_3x4(const float m[12], float out[12]);
// World ray -> object ray with the f32 inverse (fixed fma order).
void object_ray(const float inv[12], vec3 o, vec3 d, vec3* oo, vec3* od);

// Watertight f32 test; returns true and t (f32 T/det) on hit.
struct WbwRay { int kx, ky, kz; float Sx, Sy, Sz; };
WbwRay wbw_setup(vec3 d);
bool wbw_f32(const WbwRay& r, vec3 o, vec3 v0, vec3 v1, vec3 v2, float* t_out);
// FP64 re-evaluation of t, u, v (weights of v1, v2) and facing.
void wbw_f64(vec3 o, vec3 d, vec3 v0, vec3 v1, vec3 v2, float* t, float* u, float* v, bool* front);

}  // namespace oracle
