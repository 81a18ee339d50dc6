// wavefront.cuh - kernel arguments of the wavefront renderer (wavefront.cu) shared with the
// run-time-linked procedural traversal kernels (procedural.cu).
#pragma once
#include "device_math.cuh"
#include "scene.h"
#include "guide.cuh"

namespace lam {

constexpr int WAVE_BLOCK = 128;
enum : uint32_t { DEF_DIFFUSE = 0u, DEF_METAL = 1u };  // kinds of vertices deferred to the learned guide
constexpr uint32_t NO_REC = 0xFFFFFFFFu;
// classes of material-ordered shading: what a bounce runs differs between sky lanes, diffuse,
// metallic and transparent vertices
enum : uint32_t { SHADE_SKY = 0u, SHADE_DIFFUSE = 1u, SHADE_METALLIC = 2u, SHADE_TRANSPARENT = 3u, SHADE_CLASSES = 4u };
constexpr int SORT_BLOCKS_MAX = 1024;  // blocks of the class-count and scatter kernels (one scan block)

// ---------------------------------------------------------------- batched renders
// A request of lam_batch_render: its scene, camera, image and samples.
struct BatchReq {
    DevScene S;
    lam_camera cam;
    v3 camera_pos;
    uint32_t width, height, npix, samples, seed_offset;
    uint32_t pix_base;  // first entry of this request's pixels in the batch's per-pixel pools
    float4 *out_color, *out_normal, *out_albedo;
};
// A segment of a wave: `count` consecutive samples (from `first`) of every pixel of one request,
// as paths path_base + s * npix + pixel.
struct BatchSeg {
    uint32_t req, first, count, path_base;
    uint32_t pix_thread_base;  // first generate/accumulate thread of the segment within its wave
};

// ---------------------------------------------------------------- kernel arguments
struct Args {
    DevScene S;
    lam_camera cam;
    uint32_t width, height, npix, samples, max_depth, restir, seed_offset;
    float tmin, tmax;
    uint32_t wave_first, wave_count;
    uint32_t pdf_at_sample;  // LAM_GUIDE_PDF_AT_SAMPLE: Markov mixture pdf with its cosine term at the chosen direction
    uint32_t guide_metal;    // LAM_GUIDE_METAL: the learned guide is mixed in at rough metallic vertices too
    // wave buffers
    float4 *ray_o, *ray_d;          // rays by position in q_in (the generate kernel's queue is the identity)
    float4 *ray_o_out, *ray_d_out;  // rays by position in q_out, written where a path is appended
    // a live path's core state by position in q_in / q_out: throughput (xyz) and picked IOR (w); radiance
    // sum (xyz) and cached pdf (w); (cached brdf bits, seed, flags, 0).  thr / brdf / seed / flags below
    // hold the same fields of a deferred vertex by its guide-queue slot, and acc the radiance of a
    // finished path by path.
    float4 *qthr, *qacc;
    uint4* qmisc;
    float4 *qthr_out, *qacc_out;
    uint4* qmisc_out;
    uint2* hit;  // (triangle slot, instance) of the closest hit, by position in the current queue
    // material-ordered shading (lam_pipeline_set_shade_order): the class of each queued hit, the queue
    // positions in class order (null: the shade kernel takes them in queue order), and per-block class
    // counts, which the scan turns into the blocks' first output slots
    uint8_t* shade_key;
    uint32_t *shade_order, *shade_bc;
    uint32_t *q_in, *q_out;
    uint32_t *count_in, *count_out, *work;
    uint32_t* err;
    unsigned long long* segments;
    float4 *thr, *acc;
    float* brdf;
    uint32_t *seed, *flags;
    float4 *ort, *orad, *ppoint, *pnormal, *vpoint, *vnormal, *lnormal, *ldir;
    float4 *pix_color, *pix_orad, *pix_emission, *pix_albedo;
    lam_markov_chain *tent_snap, *tent_live;
    // data buffers
    const lam_markov_chain* old_chains;
    lam_markov_chain* chains;
    uint64_t chains_len, old_chains_len;
    uint32_t* world;
    const uint32_t* old_world;
    uint64_t world_len;
    uint64_t world_mod_m;    // ~0 / world_len + 1: multiplier of the fast remainder that indexes the grid
    lam_reservoir* reservoirs;
    lam_info* info;
    uint32_t* pixel_seed;
    // outputs
    float4 *out_color, *out_normal, *out_albedo;
    v3 camera_pos;
    // learned guiding: the guide kernel's queue dq (path ids); a deferred vertex's normal and
    // roughness, tangent and seed, albedo (by slot in dq, by path after the Markov-guided shade
    // kernel); its origin, incoming then outgoing direction, and sample colour and cached pdf by slot
    // in dq (thr, brdf, seed and flags above hold the rest)
    uint32_t *dq, *dq_count;
    float4 *def_n, *def_t, *def_c;
    float4 *def_o, *def_d, *def_a;
    // learned + Markov guiding (three-way mixture): the Markov sampler's direction and pdf, and its
    // candidate lobes (mean, kappa) with their mixture weights (times the vMF branch's probability)
    float4* def_r;           // also a rough-metal vertex's reflection (xyz) and roughness y (w)
    uint32_t* def_kind;      // what a deferred vertex is: DEF_DIFFUSE or DEF_METAL
    float4* def_lobe;        // MIX_LOBES per path
    float* def_lw;           // MIX_LOBES per path; 0: no lobe
    float* recs;             // training records (GUIDE_RECORD_STRIDE floats), null when not training
    uint32_t rec_cap;
    float rec_prob;          // probability that a deferred vertex is recorded
    uint32_t *rec_count, *rec_head;
    const uint16_t* guide_w; // packed BF16 weights
    float guide_frac;
    float box[6];
    // procedural hits (run-time-linked intersection handler): per path (normal, t), (tangent, 0)
    float4 *phit_a, *phit_b;
    // batched renders
    const BatchReq* reqs;
    const BatchSeg* segs;    // this wave's segments
    uint32_t nsegs, pix_threads;
    uint32_t* req_done;      // per request: pixels finished
    unsigned long long* req_time;  // per request: global timer at completion; [n] = batch start
};

}  // namespace lam
