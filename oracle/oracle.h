/* oracle.h - TEST INFRASTRUCTURE ONLY.  C API of the CPU oracle library (liblambent_oracle.so),
 * loaded with ctypes by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker of the CUDA product.  Nothing in the product links or includes it. */
#ifndef LAMBENT_ORACLE_H
#define LAMBENT_ORACLE_H
#include <stdint.h>
#include "../include/lambent.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_render_args {
    uint32_t width, height, samples, quality, restir, max_depth, guide, seed_offset;
    float tmin, tmax;
    const lam_camera* camera;
    uint32_t crop_x0, crop_y0, crop_w, crop_h;   /* crop_w == 0: whole image */
    int32_t threads;
    lam_markov_chain* chains;
    const lam_markov_chain* old_chains;
    uint64_t chains_len, old_chains_len;
    uint32_t* world;                              /* 14 u32 per entry */
    const uint32_t* old_world;
    uint64_t world_len;
    lam_reservoir* reservoirs;
    lam_info* info;
    float* out_color;
    float* out_normal;
    float* out_albedo;
    uint64_t segments_out;                        /* written: ray segments traced */
    uint64_t samples_out;                         /* written: pixels * spp */
} oracle_render_args;

int oracle_scene_create(const lam_scene_desc* desc, void** out);
void oracle_scene_destroy(void* scene);
/* mode: LAM_TRACE_CLOSEST / LAM_TRACE_ANY; bruteforce != 0 tests every triangle */
int oracle_trace(const void* scene, const lam_ray* rays, uint64_t n, uint32_t mode, lam_hit* hits,
                 int32_t threads, int32_t bruteforce);
int oracle_render(const void* scene, oracle_render_args* args);
int oracle_temporal_resampling(lam_reservoir* cur, const lam_reservoir* old, uint32_t width, uint32_t height,
                               uint32_t seed_offset);
int oracle_spatial_resampling(const lam_reservoir* cur, const lam_info* info, uint32_t width, uint32_t height,
                              uint32_t is_samples, uint32_t is_space, uint32_t seed_offset, float* out_color);
void oracle_process_gi_reservoirs(lam_reservoir* r, uint64_t n, uint32_t confidence_cap);
void oracle_process_world_markov_chains(uint32_t* world, uint64_t n);
void oracle_average_frames(const float* const* frames, uint32_t n, uint32_t width, uint32_t height, float* out_rgb);

/* known-answer helpers */
uint32_t oracle_rand_u32(uint32_t s);
float oracle_rand_f32(uint32_t s);
uint16_t oracle_f32_to_f16(float f);
float oracle_f16_to_f32(uint16_t h);
uint16_t oracle_f32_to_bf16(float f);
uint32_t oracle_normalised_to_u32(const float n[3]);
void oracle_u32_to_normalised(uint32_t u, float out[3]);
int oracle_material_new(const float uv1[2], const float uv2[2], const float uv3[2], const uint16_t recolour[2],
                        uint16_t diffuse, int32_t emission, int32_t attributes, float emissive_scale,
                        float diffuse_scale, const float* ior, uint32_t ty, lam_material* out);
int oracle_camera_from_proj_view(const float proj[16], const float view[16], lam_camera* out);
int oracle_invert_3x4(const float m[12], float out[12]);
/* single watertight test: returns 1 on hit; t_f32 from the f32 test, t/u/v/front from FP64 */
int oracle_wbw(const float o[3], const float d[3], const float v0[3], const float v1[3], const float v2[3],
               float* t_f32, float* t, float* u, float* v, int32_t* front);

#ifdef __cplusplus
}
#endif
#endif
