// tracer.h - internal objects behind lam_pipeline_layout / lam_tracer / lam_pipeline /
// lam_data_buffers.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/lambent.h"

struct lam_pipeline_layout {
    uint32_t blas_count = 1, diffuse_count = 1, emission_count = 1, attribute_count = 1;
};

struct lam_tracer {
    uint32_t quality = LAM_QUALITY_MEDIUM;
    std::string intersection_handler;  // empty = default (always miss)
};

// DataBuffers (src/data_buffer/mod.rs:103-114): temporal buffers current/old per kind.
struct lam_data_buffers {
    uint32_t width = 1, height = 1;
    uint32_t world_size = 1;
    uint32_t types = 0;
    void* reservoirs = nullptr;      // lam_reservoir[max(1, W*H if SPATIAL)]
    void* old_reservoirs = nullptr;
    void* info = nullptr;            // lam_info[W*H]
    void* chains = nullptr;          // lam_markov_chain[max(1, W*H if SCREEN)]
    void* old_chains = nullptr;
    void* world = nullptr;           // lam_world_markov_chain[max(1, world_size if WORLD)]
    void* old_world = nullptr;
    void* pixel_seed = nullptr;      // u32[W*H] seed chain between waves of one render
    size_t reservoir_len = 1, chain_len = 1, world_len = 1, pixels = 1;
};

namespace lam {

struct WaveBuffers;  // defined in wavefront.cu

}  // namespace lam

struct lam_pipeline {
    uint32_t quality = LAM_QUALITY_MEDIUM;
    lam_tracer_options opts{};
    lam_pipeline_layout layout{};
    std::string intersection_handler;
    lam::WaveBuffers* wave = nullptr;  // scratch reused across renders
    lam_render_stats stats{};
    bool stats_pending = false;
    int device = 0;
    // stage profiling: (stage, start, end) event triples recorded by lam_render
    bool profiling = false;
    struct Timed {
        int stage;
        cudaEvent_t start, end;
    };
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> event_pool;
    lam_stage_times prof{};
    uint64_t prof_segments_base = 0;
    uint64_t total_segments = 0;
};

namespace lam {
int set_intersection_handler(lam_tracer* t, const char* src);
// Debug views (FrontFace / Reflectance / Tangent), debug.cu.
int render_debug(lam_pipeline* pl, const lam_scene* s, const lam_camera* cam, const lam_frame_targets* tg,
                 cudaStream_t st);
}
