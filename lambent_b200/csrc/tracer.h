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
// A pipeline's intersection handler, linked into the procedural traversal kernels (handler_jit.cpp).
struct HandlerModule {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t extend = nullptr, trace_closest = nullptr, trace_any = nullptr;
};
int compile_handler_cubin(const std::string& source, std::vector<char>* cubin, std::string* log);
int load_handler_module(const std::vector<char>& cubin, HandlerModule* m);
void free_handler_module(HandlerModule* m);
struct BatchState;   // defined in wavefront.cu
void free_batch(BatchState* b);

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
    lam_guide* guide = nullptr;  // learned guide (not owned)
    uint64_t wave_paths = 0;     // bound on the paths of one wave (0: about 32M)
    uint32_t shade_order = LAM_SHADE_ORDER_AUTO;
    std::vector<char> handler_cubin;   // intersection handler linked with the procedural kernels
    lam::HandlerModule* handler = nullptr;  // loaded on first use
    lam::BatchState* batch = nullptr;  // lam_batch_render state
    uint32_t* stats_ctr = nullptr;     // device counters of the last render (single or batched)
};

// Learned guiding network state (guide_net.cu).
struct lam_guide {
    lam_guide_options opts{};
    int device = 0, sms = 148;
    uint32_t parts = 1;                 // gradient partial slots (one per SM)
    float *master = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    uint16_t* packed = nullptr;         // BF16 weights in the MMA tile layout
    float *partial = nullptr, *partial_loss = nullptr;
    uint32_t* err = nullptr;
    float* records = nullptr;           // render-side training records, record_capacity entries
    uint64_t steps = 0;
    uint32_t trained_spp = 0;
    uint32_t wait_tries = 1u << 20;     // lam_guide_set_wait_limit
    bool kernels_ready = false;
    std::vector<void*> allocs;
};

namespace lam {
// Render-side training record: pos, normal, wo, wi, weight (the public lam_guide_record), then the
// path throughput and accumulated colour at the vertex, and the previous record of the same path.
constexpr uint32_t GUIDE_RECORD_STRIDE = 20;
int guide_grad_and_update(lam_guide* g, const float* recs, uint32_t stride, uint32_t n, const uint32_t* n_dev,
                          uint32_t batch, bool sequential, float scale, const float box[6], uint32_t mode, float* grad,
                          float* loss, cudaStream_t st);
int guide_check_error(const lam_guide* g);

int set_intersection_handler(lam_tracer* t, const char* src);
// Debug views (FrontFace / Reflectance / Tangent), debug.cu.
int render_debug(lam_pipeline* pl, const lam_scene* s, const lam_camera* cam, const lam_frame_targets* tg,
                 cudaStream_t st);
}
