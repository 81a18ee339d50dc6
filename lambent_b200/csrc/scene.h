// scene.h - device-resident scene (group 0 + group 2 bindings of the reference) and the
// internal handle types behind the C-ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/lambent.h"

namespace lam {

// Per-instance record, 64 bytes (4 x float4).
struct DevInstance {
    float inv[12];        // world -> object, 3x4 row-major (f32 rounding of the FP64 inverse)
    uint32_t blas_root;   // global node index of the BLAS root, 0xFFFFFFFF for an empty BLAS
    uint32_t mat_offset;  // first entry of this instance's material-index table in mat_idx
    uint32_t mat_count;
    uint32_t flags;       // INST_OPAQUE | INST_VISIBLE
};
static_assert(sizeof(DevInstance) == 64, "instance record is 64 bytes");
enum : uint32_t { INST_OPAQUE = 1u, INST_VISIBLE = 2u, INST_PROCEDURAL = 4u };

struct DevTexLayer {
    uint32_t offset;      // first texel (RGBA8 as u32) in the texel pool
    uint32_t w, h;
    uint32_t pad;
};

struct DevScene {
    const uint4* blas_nodes;      // 5 uint4 per node, all BLASes concatenated
    const uint4* tlas_nodes;
    const float4* tris;           // 3 float4 per triangle slot: (v0, prim bits), (v1, 0), (v2, 0)
    const uint32_t* tlas_items;   // instance ids in TLAS leaf order
    const DevInstance* inst;
    const uint32_t* mat_idx;
    const lam_material* materials;
    const uint32_t* texels;
    const DevTexLayer* layers;    // diffuse | emission | attributes | recolour
    const uint32_t* sky;          // 6 * sky_size^2 texels, or null
    uint32_t material_count;
    uint32_t diffuse_first, diffuse_count;
    uint32_t emission_first, emission_count;
    uint32_t attr_first, attr_count;
    uint32_t recolour_layer;
    uint32_t sky_size;
    uint32_t tlas_node_count;
    uint32_t instance_count;
    uint32_t all_opaque;
    uint32_t has_procedural;      // some instance holds AABB geometry
    const float* inst_fwd;        // per instance: object-to-world 3x4, custom index, 3 zeros (procedural scenes)
};

}  // namespace lam

struct lam_scene {
    lam::DevScene dev{};
    std::vector<void*> allocations;
    lam_scene_stats stats{};
    float bounds[6] = {0, 0, 0, 0, 0, 0};  // union of the instance world boxes: lo xyz, hi xyz
    uint32_t blas_count = 0, instance_count = 0, material_count = 0;
    uint32_t diffuse_count = 0, emission_count = 0, attribute_count = 0;
    int device = 0;
};

namespace lam {
// thread-local error reporting shared by all translation units
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
// Checks shared by the ray-query entry points: n within LAM_TRACE_MAX_RAYS (the 32-bit work counter
// overshoots n by at most one claim per warp of the grid and must not wrap) and the current device
// being the scene's (the kernels dereference the scene's device pointers).
int check_trace_call(const lam_scene* s, uint32_t n, const char* who);
}  // namespace lam
