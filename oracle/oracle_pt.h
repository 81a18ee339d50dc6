// oracle_pt.h - TEST INFRASTRUCTURE ONLY (the CPU oracle; see oracle_math.h).
// Restatement of the reference path tracer and its follow-up passes on the CPU.
#pragma once
#include <cstdint>
#include "oracle_scene.h"

namespace oracle {

struct RenderParams {
    uint32_t width = 0, height = 0;
    uint32_t samples = 4;
    uint32_t quality = LAM_QUALITY_MEDIUM;
    uint32_t restir = LAM_RESTIR_PER_PIXEL;
    uint32_t max_depth = 5;
    uint32_t guide = LAM_GUIDE_NONE;
    uint32_t seed_offset = 0;
    float tmin = 1e-4f, tmax = 1000.0f;
    lam_camera camera{};
    // Pixel window [x0, x0 + w) x [y0, y0 + h) of the full image to render (a crop keeps the
    // full-image ray generation and seeds).  w == 0 renders the whole image.
    uint32_t crop_x0 = 0, crop_y0 = 0, crop_w = 0, crop_h = 0;
    int threads = 1;
    // temporal buffers (any may be null when the corresponding feature is off)
    lam_markov_chain* chains = nullptr;
    const lam_markov_chain* old_chains = nullptr;
    uint64_t chains_len = 0, old_chains_len = 0;
    uint32_t* world = nullptr;            // 14 u32 per entry
    const uint32_t* old_world = nullptr;
    uint64_t world_len = 0;
    lam_reservoir* reservoirs = nullptr;
    lam_info* info = nullptr;
    // outputs (rgba32f, width*height*4; may be null)
    float* out_color = nullptr;
    float* out_normal = nullptr;
    float* out_albedo = nullptr;
};

struct RenderCounters {
    uint64_t segments = 0;
    uint64_t samples = 0;
};

int render(const Scene& scene, const RenderParams& p, RenderCounters* counters);

int temporal_resampling(lam_reservoir* cur, const lam_reservoir* old, uint32_t width, uint32_t height,
                        uint32_t seed_offset);
int spatial_resampling(const lam_reservoir* cur, const lam_info* info, uint32_t width, uint32_t height,
                       uint32_t is_samples, uint32_t is_space, uint32_t seed_offset, float* out_color);
void process_gi_reservoirs(lam_reservoir* r, uint64_t n, uint32_t confidence_cap);
void process_world_markov_chains(uint32_t* world, uint64_t n);
void average_frames(const float* const* frames, uint32_t n, uint32_t width, uint32_t height, float* out_rgb);

}  // namespace oracle
