/*
 * lambent.h - C-ABI of the B200-native Lambent path-tracing hot path.
 *
 * Every entry point returns an int status (LAM_OK == 0, negative on error) and never
 * throws or aborts across the ABI.  lam_last_error_message() returns a thread-local
 * description of the last failure on the calling thread.  Handles are opaque; each is
 * thread-compatible (one thread at a time per handle).  Device pointers are plain CUDA
 * global-memory pointers; `stream` arguments are cudaStream_t values passed as void*
 * (NULL = the legacy default stream).
 *
 * Each declaration cites the reference (Vecvec/Lambent) interface it replaces as
 * path:line inside that project.
 */
#ifndef LAMBENT_B200_H
#define LAMBENT_B200_H

#include <stddef.h>
#include <stdint.h>
#include "lambent_handler.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum {
    LAM_OK = 0,
    LAM_ERR_INVALID_ARGUMENT = -1,        /* bad size, NULL handle, u16::MAX texture index */
    LAM_ERR_OUT_OF_MEMORY = -2,
    LAM_ERR_CUDA = -3,                    /* a CUDA runtime call failed */
    LAM_ERR_NOT_BUILT = -4,
    LAM_ERR_PROJECTION_UNINVERTIBLE = -5, /* CameraError::ProjectionUninvertable, src/camera.rs:53-57 */
    LAM_ERR_VIEW_UNINVERTIBLE = -6,       /* CameraError::ViewUninvertable */
    LAM_ERR_TEXTURE = -7,                 /* TextureError, src/textures.rs:93-97 */
    LAM_ERR_COMPILE = -8,                 /* intersection-handler compile error (src/lib.rs:424 panics) */
    LAM_ERR_LAYOUT_MISMATCH = -9,         /* bound resources exceed the pipeline layout counts */
    LAM_ERR_UNSUPPORTED = -10,
    LAM_ERR_DEVICE_TIMEOUT = -11,         /* a bounded device-side wait gave up */
    LAM_ERR_STACK_OVERFLOW = -12,         /* traversal stack overflow recorded by a kernel */
    LAM_ERR_CALLBACK = -13                /* a caller-supplied callback returned nonzero */
};

/* ---------------------------------------------------------------- enums */
/* MaterialType, src/lib.rs:194-203; SKY, src/importance_sampling/shared.wesl:7-10 */
enum { LAM_DIFFUSE = 0, LAM_METALLIC = 1, LAM_TRANSPARENT = 2, LAM_SKY = 0xFF };

/* path_tracing::{Low, Medium, High}, src/path_tracing/mod.rs:66-147;
 * debug::{FrontFace, Reflectance, Tangent}, src/debug/mod.rs:1-56 */
enum {
    LAM_QUALITY_LOW = 0,
    LAM_QUALITY_MEDIUM = 1,
    LAM_QUALITY_HIGH = 2,
    LAM_DEBUG_FRONT_FACE = 16,
    LAM_DEBUG_REFLECTANCE = 17,
    LAM_DEBUG_TANGENT = 18
};

/* RestirTemporalMode, src/path_tracing/mod.rs:31-41 (PerPixel is the default) */
enum { LAM_RESTIR_DISABLED = 0, LAM_RESTIR_PER_SAMPLE = 1, LAM_RESTIR_PER_PIXEL = 2 };

/* Directional sampler used at diffuse vertices.
 * LAM_GUIDE_NONE    - BSDF (cosine) sampling only: the branch the reference takes when no
 *                     Markov chain is valid (src/path_tracing/general.wesl:812-815).
 * LAM_GUIDE_MARKOV  - the reference's vMF Markov-chain mixture (general.wesl:764-866).
 * LAM_GUIDE_LEARNED - cosine BSDF sampler combined with the learned lobe mixture by
 *                     one-sample MIS (no counterpart in the reference; see lam_guide).
 * LAM_GUIDE_METAL   - modifier bit for the learned modes: the learned lobes are also mixed in at
 *                     rough metallic vertices (Medium / High, index ratio 1, both roughnesses >= 0.1)
 *                     with the reference's reflection, weighted by their mixture pdf (unbiased).
 * LAM_GUIDE_LEARNED | LAM_GUIDE_MARKOV - a three-way one-sample-MIS mixture: with probability 1 - f
 *                     the Markov sampler's draw (cosine lobe or a chain's vMF lobe, as LAM_GUIDE_MARKOV
 *                     draws it), with probability f the network's; the sample is weighted by
 *                     (1 - f) p_markov(w) + f q(w), p_markov being the Markov mixture's pdf with its
 *                     cosine term at w (unbiased).  ReSTIR must be disabled.
 * LAM_GUIDE_PDF_AT_SAMPLE - modifier bit for LAM_GUIDE_MARKOV, no counterpart in the reference.
 *                     The reference weights a guided sample by 0.2 * cos(w_c)/pi + 0.8 * vMF(w),
 *                     where w_c is the cosine branch's own draw (general.wesl:793, 840), also when
 *                     the vMF branch chose w; the estimate is then biased (about +4% on the Cornell
 *                     box).  With this bit the cosine term is evaluated at w, which makes the
 *                     mixture pdf the density w was drawn from and the estimator unbiased.  Without
 *                     it LAM_GUIDE_MARKOV renders what the reference renders. */
enum { LAM_GUIDE_NONE = 0, LAM_GUIDE_MARKOV = 1, LAM_GUIDE_LEARNED = 2, LAM_GUIDE_PDF_AT_SAMPLE = 4, LAM_GUIDE_METAL = 8 };

/* BufferType bitflags, src/data_buffer/mod.rs:18-27 */
enum {
    LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE = 1u << 0,
    LAM_BUFFER_SPATIAL_RESAMPLING = 1u << 1,
    LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE = 1u << 2,
    LAM_BUFFER_ALL = 7u
};

/* wgpu::BufferUsages bits used by Descriptor::buffer_descriptor (src/lib.rs:64-69) */
enum { LAM_USAGE_COPY_DST = 0x8, LAM_USAGE_UNIFORM = 0x40, LAM_USAGE_STORAGE = 0x80 };

/* AccelerationStructureGeometryFlags::OPAQUE (examples/cornell_box/src/main.rs:469) */
enum { LAM_GEOMETRY_OPAQUE = 1u };

/* lam_trace_rays modes */
enum { LAM_TRACE_CLOSEST = 0, LAM_TRACE_ANY = 1 };

/* lam_hit.kind */
enum { LAM_HIT_NONE = 0, LAM_HIT_FRONT = 1, LAM_HIT_BACK = 2 };

/* ---------------------------------------------------------------- plain data (bit-exact with the reference) */

/* Material, src/lib.rs:83-94 / src/bindings.wesl:48-57 - 8 x u32 = 32 bytes */
typedef struct lam_material {
    uint32_t tex_pos_1;                /* 2 x f16 UV of vertex 0 */
    uint32_t tex_pos_2;                /* 2 x f16 UV of vertex 1 */
    uint32_t tex_pos_3;                /* 2 x f16 UV of vertex 2 */
    uint32_t tex_pos_recolour;         /* 2 x u16 texel of the recolour texture */
    uint32_t tex_idx_diffuse_emission; /* u16 diffuse layer | u16 emission layer << 16 (0xFFFF = none) */
    uint32_t tex_idx_attributes_ty;    /* u16 attribute layer (0xFFFF = none) | u16 type << 16 */
    uint32_t emission_scale;           /* bf16 emissive-texture scale | bf16 diffuse scale << 16 */
    uint32_t refractive_index;         /* 2 x f16: low (760 nm) | high (340 nm) << 16 */
} lam_material;

/* Camera, src/camera.rs:6-11 - two column-major 4x4 f32 matrices = 128 bytes */
typedef struct lam_camera {
    float projection_inverse[16];
    float view_inverse[16];
} lam_camera;

/* MarcovChainState, src/bindings.wesl:3-9 (storage layout, 32 bytes) */
typedef struct lam_markov_chain {
    float light_source[3];
    float mean_cosine;
    float weight_sum;
    uint32_t num_samples;
    float score;
    uint32_t _pad;
} lam_markov_chain;

/* WorldMarcovChainState, src/bindings.wesl:33-40 (56 bytes) */
typedef struct lam_world_markov_chain {
    uint32_t secondary_hash;
    uint32_t num_samples;
    uint32_t luminance[3];     /* f32 bit patterns */
    uint32_t lock;
    uint32_t chain_light_source[3];
    uint32_t chain_mean_cosine;
    uint32_t chain_weight_sum;
    uint32_t chain_num_samples;
    uint32_t chain_score;
    uint32_t timeout;
} lam_world_markov_chain;

/* Reservoir, src/bindings.wesl:158-169 (64 bytes) */
typedef struct lam_reservoir {
    float visible_point[3];
    uint32_t visible_normal;   /* octahedral snorm16x2 */
    float sample_point[3];
    uint32_t sample_normal;
    float out_radiance[3];
    uint32_t ty;
    float roughness;
    float w;
    uint32_t packed_confidence_valid; /* 31-bit M | valid << 31 */
    float W;
} lam_reservoir;

/* CompressedInfo, src/bindings.wesl:63-65 (36 bytes): cam_loc, emission, albedo */
typedef struct lam_info {
    float arr[9];
} lam_info;

/* Buffer descriptor returned by the Descriptor impls (src/lib.rs:184-192, src/camera.rs:43-51) */
typedef struct lam_buffer_descriptor {
    const void* contents;
    size_t size;
    uint32_t usage;
} lam_buffer_descriptor;

/* ---------------------------------------------------------------- scene input */

/* One bottom-level geometry (BlasTriangleGeometry, examples/cornell_box/src/main.rs:464-470, 547-560). */
typedef struct lam_blas_desc {
    const float* vertices;    /* host pointer, vertex_count * vertex_stride floats */
    uint32_t vertex_count;
    uint32_t vertex_stride;   /* floats per vertex: 3 or 4 (the reference uses [f32;4]) */
    const uint32_t* indices;  /* NULL: non-indexed, triangle i = vertices 3i..3i+2 */
    uint32_t index_count;     /* multiple of 3 (or 3 * triangle count when non-indexed) */
    uint32_t flags;           /* LAM_GEOMETRY_OPAQUE: skip the alpha test (general.wesl:1059-1067) */
    /* Procedural geometry instead of triangles (AABB geometry of a BLAS): aabb_count boxes of
     * 6 floats (min xyz, max xyz).  Candidates go to the pipeline's intersection handler; without
     * one they miss, as the reference's default handler does. */
    const float* aabbs;
    uint32_t aabb_count;
} lam_blas_desc;

/* The no-vertex-return input format (Vertices / Indices, src/lib.rs:439-454, bindings.wesl:83-113,
 * get_vertices general.wesl): a Vertices blob is geometry_stride (u32) and 12 zero bytes followed by
 * [f32; 4] vertices; an Indices array of length 1 means "no indices" (the vertex index is used
 * directly).  Triangle p of geometry g reads the index slots geometry_stride * g + 3p + {0, 1, 2}.
 * Fills *out with a BLAS whose vertices point into the blob (it must outlive *out) and whose index
 * list (owned by *out; release it with lam_blas_desc_free) lists the triangles geometry by geometry,
 * numbered consecutively.  Out-of-range slots or vertex indices: LAM_ERR_INVALID_ARGUMENT. */
int lam_blas_from_vertices(const void* vertices_blob, size_t blob_bytes, const uint32_t* indices,
                           size_t index_count, uint32_t geometry_count, const uint32_t* triangles_per_geometry,
                           uint32_t flags, lam_blas_desc* out);
int lam_blas_desc_free(lam_blas_desc* desc);
/* The reference looks materials up by the primitive index within its geometry
 * (material_idx[instance].materials[primitive_index], general.wesl:1059); writes the table indexed
 * by the consecutive numbering of lam_blas_from_vertices (out: sum of triangles_per_geometry
 * entries).  An index past the end of `table` reads its last entry, as a clamped GPU load does. */
int lam_material_table_for_geometries(const uint32_t* table, uint32_t table_len, uint32_t geometry_count,
                                      const uint32_t* triangles_per_geometry, uint32_t* out);

/* One top-level instance (TlasInstance::new, main.rs:493-498) plus its material table
 * (binding 0/1 material_idx[instance].materials[primitive], bindings.wesl:59-70). */
typedef struct lam_instance_desc {
    float transform[12];              /* 3x4 row-major object-to-world */
    uint32_t blas;
    uint32_t custom_index;
    uint32_t mask;                    /* instance visible when (mask & 0xFF) != 0 */
    const uint32_t* material_indices; /* one u32 per primitive of the BLAS */
    uint32_t material_index_count;
} lam_instance_desc;

/* One RGBA8 texture layer (Rgba8Unorm 2D texture, src/textures.rs:41-90). */
typedef struct lam_texture_layer {
    const uint8_t* rgba8;
    uint32_t width;
    uint32_t height;
} lam_texture_layer;

typedef struct lam_scene_desc {
    const lam_blas_desc* blas;
    uint32_t blas_count;
    const lam_instance_desc* instances;
    uint32_t instance_count;
    const lam_material* materials;
    uint32_t material_count;
    const lam_texture_layer* diffuse;     /* bind group 2 binding 1 */
    uint32_t diffuse_count;
    const lam_texture_layer* emission;    /* binding 2 */
    uint32_t emission_count;
    const lam_texture_layer* attributes;  /* binding 3 */
    uint32_t attribute_count;
    const lam_texture_layer* recolour;    /* binding 4; NULL = 1x1 white (textures.rs:192-219) */
    const uint8_t* sky_faces;             /* 6 * sky_size^2 RGBA8 cube faces +X,-X,+Y,-Y,+Z,-Z; NULL = black */
    uint32_t sky_size;
} lam_scene_desc;

typedef struct lam_scene_stats {
    uint64_t triangle_count;
    uint64_t blas_node_count;
    uint64_t tlas_node_count;
    uint64_t device_bytes;
    double build_seconds;
} lam_scene_stats;

/* ---------------------------------------------------------------- tracing options */

/* RayTracingOptions / PathTracerOpts, src/low_level.rs:77-113, src/path_tracing/mod.rs:7-34 */
typedef struct lam_tracer_options {
    uint32_t samples;          /* SAMPLES override (default 4, low_level.rs:101) */
    float tmin;                /* T_MIN (default 1e-4) */
    float tmax;                /* T_MAX (default 1000) */
    uint32_t restir_temporal;  /* LAM_RESTIR_* (default PER_PIXEL) */
    uint32_t max_depth;        /* path vertices; the reference hard-codes BOUNCES = 5 (general.wesl:50) */
    uint32_t guide_mode;       /* LAM_GUIDE_* */
} lam_tracer_options;

/* Output images, bind group 1 bindings 1-3 (rgba32float storage textures, low_level.rs:413-442).
 * Device pointers to width*height*4 floats, row-major; any may be NULL. */
typedef struct lam_frame_targets {
    float* color;
    float* normal;
    float* albedo;
    uint32_t width;
    uint32_t height;
} lam_frame_targets;

/* One ray for lam_trace_rays: origin, tmin, direction, tmax (32 bytes). */
typedef struct lam_ray {
    float origin[3];
    float tmin;
    float direction[3];
    float tmax;
} lam_ray;

/* Committed intersection returned by lam_trace_rays (RayIntersection fields read at
 * general.wesl:1078-1093): barycentrics u,v weight vertices 1 and 2. */
typedef struct lam_hit {
    float t;
    float u;
    float v;
    uint32_t primitive_index;
    uint32_t instance_index;
    uint32_t kind;             /* LAM_HIT_* */
} lam_hit;

/* Render statistics of the last lam_render on a pipeline. */
typedef struct lam_render_stats {
    uint64_t ray_segments;     /* primary + extension rays traced */
    uint64_t samples;          /* pixels * spp */
    uint32_t kernel_launches;
    uint32_t error_flags;      /* bit 0: traversal stack overflow */
} lam_render_stats;

/* Per-stage device time of the renders since the last reset (CUDA events on the render stream). */
typedef struct lam_stage_times {
    double generate_ms;
    double extend_ms;
    double shade_ms;           /* shade + learned-guide sampling */
    double accumulate_ms;      /* accumulate + chain shuffle */
    uint64_t extend_launches;
    uint64_t shade_launches;
    uint64_t ray_segments;     /* segments traced by the timed renders */
    double train_ms;           /* learned-guide training steps */
} lam_stage_times;

/* Opaque handles */
typedef struct lam_pipeline_layout lam_pipeline_layout;
typedef struct lam_tracer lam_tracer;
typedef struct lam_pipeline lam_pipeline;
typedef struct lam_scene lam_scene;
typedef struct lam_data_buffers lam_data_buffers;
typedef struct lam_texture_loader lam_texture_loader;

/* Raw texture cuboids returned by lam_texture_loader_raw (README.md:39-43). */
typedef struct lam_raw_textures {
    uint8_t* cuboid[3];        /* diffuse, lit (emission), attributes: layers * height * width * 4 bytes */
    uint32_t width[3];
    uint32_t height[3];
    uint32_t layers[3];
    int32_t* layer_of_entry[3];/* per load() call: the layer in cuboid k, or -1 when not included */
    uint32_t entry_count;
} lam_raw_textures;

/* ---------------------------------------------------------------- library */
uint32_t lam_version(void);
const char* lam_last_error_message(void);

/* dispatch_size, src/lib.rs:207-219: workgroups of 64x1 over width x height. */
int lam_dispatch_size(uint32_t width, uint32_t height, uint32_t out_workgroups[2]);

/* ---------------------------------------------------------------- Material */
/* Material::new, src/lib.rs:132-163.  tex_idx_emission / tex_idx_attributes: -1 = None
 * (u16::MAX, lib.rs:165-170; passing 0xFFFF itself is LAM_ERR_INVALID_ARGUMENT where the
 * reference asserts).  EmissionScale::from_f32 (lib.rs:110-115).  refractive_index_range:
 * [low, high] or NULL for VACUUM 1..1 (lib.rs:148). */
int lam_material_new(const float tex_pos_1[2], const float tex_pos_2[2], const float tex_pos_3[2],
                     const uint16_t tex_pos_recolour[2], uint16_t tex_idx_diffuse,
                     int32_t tex_idx_emission, int32_t tex_idx_attributes,
                     float emissive_texture_scale, float diffuse_texture_scale,
                     const float* refractive_index_range, uint32_t material_type,
                     lam_material* out);

/* <[Material] as Descriptor>::buffer_descriptor, src/lib.rs:184-192 ("descriptor" in README.md:22-24) */
int lam_material_descriptor(const lam_material* materials, uint32_t count, uint32_t further_usages,
                            lam_buffer_descriptor* out);

/* refractive_indices::refractive_index_between, src/lib.rs:35-37 */
int lam_refractive_index_between(const float in_front[2], const float behind[2], float out[2]);

/* ---------------------------------------------------------------- Camera */
/* Camera::from_proj_view, src/camera.rs:15-24 ("Camera::new" in README.md:50-51).
 * proj/view: column-major 4x4. */
int lam_camera_new(const float proj[16], const float view[16], lam_camera* out);
int lam_camera_from_proj_view(const float proj[16], const float view[16], lam_camera* out);
/* Camera::update_from_proj_view, src/camera.rs:27-40 (either may be NULL) */
int lam_camera_update_from_proj_view(lam_camera* camera, const float* proj, const float* view);
/* impl Descriptor for Camera, src/camera.rs:43-51 (UNIFORM usage) */
int lam_camera_descriptor(const lam_camera* camera, uint32_t further_usages, lam_buffer_descriptor* out);

/* ---------------------------------------------------------------- TextureLoader */
/* TextureLoader::new / default, src/textures.rs:12-23 */
int lam_texture_loader_new(lam_texture_loader** out);
/* TextureLoader::load, src/textures.rs:25-28 and the 3-file form of README.md:34-37:
 * PNG files (8-bit gray/gray-alpha/RGB/RGBA/palette, non-interlaced); lit/attributes may be NULL. */
int lam_texture_loader_load(lam_texture_loader* loader, const char* diffuse_path,
                            const char* lit_path, const char* attributes_path);
/* TextureLoader::load_from_bytes, src/textures.rs:30-38 (PNG bytes; lit/attributes may be NULL). */
int lam_texture_loader_load_from_bytes(lam_texture_loader* loader,
                                       const uint8_t* diffuse, size_t diffuse_len,
                                       const uint8_t* lit, size_t lit_len,
                                       const uint8_t* attributes, size_t attributes_len);
/* Already-decoded RGBA8 pixels (what image::RgbaImage holds); lit/attributes may be NULL. */
int lam_texture_loader_load_rgba8(lam_texture_loader* loader, uint32_t width, uint32_t height,
                                  const uint8_t* diffuse, const uint8_t* lit, const uint8_t* attributes);
/* TextureLoader::raw (README.md:39-43): consumes the loader (the handle is freed even on error). */
int lam_texture_loader_raw(lam_texture_loader* loader, lam_raw_textures* out);
int lam_raw_textures_free(lam_raw_textures* raw);
int lam_texture_loader_free(lam_texture_loader* loader);

/* ---------------------------------------------------------------- pipeline layout / tracer */
/* low_level::pipeline_layout, src/low_level.rs:237-343 (counts are NonZeroU32). */
int lam_pipeline_layout_create(uint32_t blas_count, uint32_t diffuse_count, uint32_t emission_count,
                               uint32_t attribute_count, lam_pipeline_layout** out);
int lam_pipeline_layout_destroy(lam_pipeline_layout* layout);

/* RayTracer::<S>::new, src/lib.rs:268-279 (quality = LAM_QUALITY_* or LAM_DEBUG_*) */
int lam_tracer_create(uint32_t quality, lam_tracer** out);
/* RayTracer::set_intersection_handler, src/lib.rs:291-295 / IntersectionHandler,
 * src/low_level.rs:115-147.  cuda_source (CUDA C++) defines
 *   __device__ lam_aabb_intersection intersect(const lam_ray_intersection& i);
 * with the types of lambent_handler.h (included for it).  It is called for every candidate of
 * procedural (AABB) geometry and must return in finite time.  Pipelines created from the tracer
 * afterwards compile it with NVRTC and link it into their traversal kernels (nvJitLink);
 * a source that does not compile fails lam_tracer_create_pipeline with LAM_ERR_COMPILE and the
 * compiler's log.  NULL restores the default handler (always a miss,
 * src/default_intersection_handler.wesl). */
int lam_tracer_set_intersection_handler(lam_tracer* tracer, const char* cuda_source);
int lam_tracer_destroy(lam_tracer* tracer);
/* RayTracingOptions::default / PathTracerOpts::default (low_level.rs:101-113) */
int lam_tracer_options_default(lam_tracer_options* out);
/* RayTracer::create_pipeline, src/lib.rs:297-318 */
int lam_tracer_create_pipeline(const lam_tracer* tracer, const lam_pipeline_layout* layout,
                               const lam_tracer_options* options, lam_pipeline** out);
int lam_pipeline_destroy(lam_pipeline* pipeline);

/* ---------------------------------------------------------------- scene (BLAS/TLAS build) */
/* create_blas / create_tlas / build_acceleration_structures (main.rs:464-563) plus the
 * group-0 materials and group-2 textures: uploads everything and builds the BVH8. */
int lam_scene_create(const lam_scene_desc* desc, void* stream, lam_scene** out);
int lam_scene_update_materials(lam_scene* scene, const lam_material* materials, uint32_t count,
                               void* stream);
int lam_scene_stats_get(const lam_scene* scene, lam_scene_stats* out);
int lam_scene_destroy(lam_scene* scene);

/* Ray-query closest hit / any hit (rayQueryInitialize..GetCommittedIntersection,
 * general.wesl:1053-1078) for n rays held in device memory.  n <= LAM_TRACE_MAX_RAYS, and the
 * current device must be the scene's (LAM_ERR_INVALID_ARGUMENT otherwise).  The call waits for
 * its stream before it returns. */
#define LAM_TRACE_MAX_RAYS 0x7FFFFFFFu
int lam_trace_rays(const lam_scene* scene, const lam_ray* rays, uint32_t n, uint32_t mode,
                   lam_hit* hits, void* stream);

/* lam_trace_rays with the pipeline's intersection handler for procedural geometry (the reference
 * runs its ray queries inside the pipeline that holds the handler).  Procedural hits report the
 * handler's t, u = v = 0 and LAM_HIT_BACK (the reference's generated intersections carry no
 * barycentrics or facing).  Without a handler, or for scenes without procedural geometry, this is
 * lam_trace_rays. */
int lam_pipeline_trace_rays(lam_pipeline* pipeline, const lam_scene* scene, const lam_ray* rays, uint32_t n,
                            uint32_t mode, lam_hit* hits, void* stream);

/* Allocation-free form of lam_trace_rays; it has no counterpart in the reference.  For callers
 * that cannot allocate device memory while they run (a render loop inside a fixed frame budget,
 * where cudaMalloc/cudaFree can synchronise the device, or a host that reserves all of its GPU
 * memory up front): the query's scratch (a work counter and error flags) lives in a 256-byte
 * static device array that every GPU loading this library keeps until the process exits.
 * n must not exceed LAM_TRACE_STATIC_MAX_RAYS (larger n: LAM_ERR_INVALID_ARGUMENT).  All calls
 * share that array: calls that overlap on the GPU race and must be serialised.  The first call on
 * a device looks up the array's device address (in the CUDA runtime's primary context) and keeps
 * it for the life of the process; make that first call before any stream capture, and do not use
 * this entry point across cudaDeviceReset, which leaves the kept address stale.  Each call reads
 * the error flags back and waits for its stream before it returns.  The current device must be the
 * scene's.  Results are identical to lam_trace_rays. */
#define LAM_TRACE_STATIC_MAX_RAYS 0x7FFFFFFFu
int lam_trace_rays_static(const lam_scene* scene, const lam_ray* rays, uint32_t n, uint32_t mode,
                          lam_hit* hits, void* stream);

/* ---------------------------------------------------------------- DataBuffers */
/* DataBuffers::new, src/data_buffer/mod.rs:150-252 */
int lam_data_buffers_new(uint32_t width, uint32_t height, uint32_t world_space_buffer_size,
                         uint32_t buffer_types, lam_data_buffers** out);
/* DataBuffers::resize, src/data_buffer/mod.rs:259-267 */
int lam_data_buffers_resize(lam_data_buffers* buffers, uint32_t width, uint32_t height);
/* DataBuffers::advance_frame, src/data_buffer/mod.rs:272-349 (AdvanceOptions.confidence_cap) */
int lam_data_buffers_advance_frame(lam_data_buffers* buffers, uint32_t buffers_to_advance,
                                   uint32_t confidence_cap, void* stream);
/* Device pointers of the temporal buffers (which: 0 reservoirs, 1 old reservoirs, 2 info,
 * 3 chains, 4 old chains, 5 world chains, 6 old world chains, 7 per-pixel seed state). */
int lam_data_buffers_get(const lam_data_buffers* buffers, uint32_t which, void** device_ptr,
                         size_t* bytes);
int lam_data_buffers_destroy(lam_data_buffers* buffers);

/* ---------------------------------------------------------------- rendering */
/* One dispatch of rt_main (general.wesl:506-610) as a wavefront launch sequence. */
int lam_render(lam_pipeline* pipeline, const lam_scene* scene, lam_data_buffers* buffers,
               const lam_camera* camera, const lam_frame_targets* targets, uint32_t seed_offset,
               void* stream);
int lam_render_stats_get(const lam_pipeline* pipeline, lam_render_stats* out);
/* Stage timing (no counterpart in the reference, which has none): when enabled, lam_render records
 * CUDA events around its launches; lam_render_profile_get synchronises and sums them. */
int lam_pipeline_set_profiling(lam_pipeline* pipeline, int enabled);
int lam_render_profile_get(lam_pipeline* pipeline, lam_stage_times* out);
/* Wave size (no counterpart in the reference, whose rt_main holds one pixel's samples in a thread):
 * lam_render runs a frame's samples in waves of at most max(pixels, max_paths) paths; each path in
 * flight keeps about 220 bytes of device state.  0 restores the default of about 32M paths (one
 * 16-spp wave at 1080p, about 7 GB).  Markov guiding and per-sample ReSTIR always run one sample per
 * wave.  The image does not depend on the wave size; smaller waves trade speed for memory.  Takes
 * effect at the next lam_render.  lam_render itself caps a new wave at half the free device memory
 * and halves it while an allocation fails; a wave shrunk that way is kept for later, larger
 * requests. */
int lam_pipeline_set_wave_paths(lam_pipeline* pipeline, uint64_t max_paths);
/* Shading order (no counterpart in the reference, whose rt_main shades one pixel's path per
 * thread).  LAM_SHADE_ORDER_QUEUE shades the queued hits in the order extend found them;
 * LAM_SHADE_ORDER_MATERIAL first sorts them (stable) by what the bounce runs: sky, diffuse,
 * metallic, transparent, so that a warp's lanes take the same branch.  LAM_SHADE_ORDER_AUTO, the
 * default, sorts every render except Markov-guided ones, which run slower in class order.  A plain
 * render's image does not depend on the order;
 * under guiding, the world-grid and training updates land in another order, as they already may
 * between two runs.  The sort keeps 5 bytes per path of device state.  Takes effect at the next
 * lam_render or lam_batch_render. */
#define LAM_SHADE_ORDER_AUTO 0u
#define LAM_SHADE_ORDER_QUEUE 1u
#define LAM_SHADE_ORDER_MATERIAL 2u
int lam_pipeline_set_shade_order(lam_pipeline* pipeline, uint32_t order);
int lam_render_profile_reset(lam_pipeline* pipeline);

/* TemporalResampling main, src/importance_sampling/temporal_resampling.wesl:37-65 */
int lam_temporal_resampling(lam_data_buffers* buffers, uint32_t width, uint32_t height,
                            uint32_t seed_offset, void* stream);
/* SpatialResampling main, src/importance_sampling/spatial_resampling.wesl:52-194
 * (overrides IS_SAMPLES, IS_SPACE; writes targets->color). */
int lam_spatial_resampling(lam_data_buffers* buffers, const lam_frame_targets* targets,
                           uint32_t is_samples, uint32_t is_space, uint32_t seed_offset,
                           void* stream);

/* ---------------------------------------------------------------- batched renders
 * lam_batch_render: many independent render requests (own scene, camera, resolution and sample
 * count) as one wavefront.  Paths of every request share the same persistent launches, so small
 * requests fill the GPU together.  No reference counterpart: the reference dispatches one rt_main
 * per request.  Plain path tracing only (no ReSTIR, no guiding); each request writes the mean
 * colour of its samples to targets.color, and normal/albedo of its last sample when given.
 * Requests run shortest first (pixels x samples) and finish at different times inside the batch:
 * lam_batch_latencies reports, per request, the time from the batch start to its completion. */
typedef struct lam_batch_request {
    const lam_scene* scene;
    lam_camera camera;
    lam_frame_targets targets;
    uint32_t samples;
    uint32_t seed_offset;
} lam_batch_request;
/* Queue and launch sizes of a batch (0 = default).  use_graph: capture the launch sequence in a
 * CUDA graph on the first call and replay it while the requests (pointers, sizes, samples) and the
 * tuning stay the same. */
typedef struct lam_batch_tuning {
    uint32_t wave_paths;       /* paths per wave (queue size), >= the largest request's pixels */
    uint32_t extend_blocks_per_sm;
    uint32_t shade_blocks_per_sm;
    uint32_t use_graph;
} lam_batch_tuning;
int lam_batch_render(lam_pipeline* pipeline, const lam_batch_request* requests, uint32_t n,
                     const lam_batch_tuning* tuning, void* stream);
/* Milliseconds from the start of the last batch to each request's completion (synchronises). */
int lam_batch_latencies(lam_pipeline* pipeline, uint32_t n, double* ms);
/* Autotuner: times the batch (samples divided by `spp_divisor`, at least 1) under candidate wave
 * sizes and launch sizes, coordinate by coordinate, each as a CUDA-graph replay (best of three after
 * a capturing call), and writes the fastest to *out. */
int lam_batch_autotune(lam_pipeline* pipeline, const lam_batch_request* requests, uint32_t n,
                       uint32_t spp_divisor, lam_batch_tuning* out, void* stream);

/* ---------------------------------------------------------------- learned path guiding
 * No counterpart in the reference (its guiding is the Markov-chain cache, general.wesl:764-866).
 * A 4-layer MLP (64 wide, BF16 weights, FP32 accumulation on the tensor cores) maps a diffuse
 * vertex (position, normal, outgoing direction) to an 8-lobe vMF mixture over incident directions.
 * With guide_mode LAM_GUIDE_LEARNED and a guide attached to the pipeline, lam_render samples
 * that mixture with probability guide_fraction and the cosine BSDF lobe otherwise, and weights
 * the sample by the mixture pdf (one-sample MIS, balance heuristic): the estimate stays unbiased.
 * While fewer than train_spp samples per pixel have been rendered with the guide, every render
 * records its diffuse vertices (and the radiance their paths carried back) and takes
 * steps_per_wave Adam steps on them after each wave of samples.  Until the first training step
 * the guided render is the plain one, sample for sample.
 *
 * Parameters (lam_guide_get_params / set_params) are 4 x 64 x 64 f32, W[layer][out][in]:
 * layer input column 63 is the constant 1 (so W[l][o][63] is the bias), hidden unit 63 is that
 * constant (rows W[0..2][63][*] are unused), and head rows 40..63 are unused.  Head outputs:
 * 0-7 mixture logits, 8-15 log concentration (clamped to [-3, 6]), 16-23 / 24-31 / 32-39 the
 * x / y / z components of the (normalised) lobe means. */
#define LAM_GUIDE_PARAMS 16384u
#define LAM_GUIDE_OUTPUTS 40u
typedef struct lam_guide lam_guide;
typedef struct lam_guide_options {
    uint32_t train_spp;        /* samples per pixel that train the network (default 32) */
    uint32_t steps_per_wave;   /* Adam steps after each wave of training samples (default 32) */
    uint32_t batch;            /* training records per step, a multiple of 128 (default 16384) */
    uint32_t record_capacity;  /* training records kept per wave (default 2^21) */
    float learning_rate;       /* Adam step size (default 2e-3) */
    float guide_fraction;      /* probability of sampling the learned mixture (default 0.5) */
    uint32_t seed;             /* weight initialisation and minibatch selection */
} lam_guide_options;
/* A query: position, shading normal, outgoing direction (toward the previous vertex). */
typedef struct lam_guide_query {
    float pos[3], normal[3], wo[3];
} lam_guide_query;
/* A training record: a query, the sampled incident direction wi and the weight of -log q(wi):
 * the luminance of (BSDF * cos * incident radiance / pdf) the path carried back. */
typedef struct lam_guide_record {
    float pos[3], normal[3], wo[3], wi[3];
    float weight;
} lam_guide_record;

int lam_guide_options_default(lam_guide_options* out);
int lam_guide_create(const lam_guide_options* options, lam_guide** out);
int lam_guide_destroy(lam_guide* guide);
/* Host copies of the f32 master parameters.  set_params also resets the Adam state and the
 * count of trained samples. */
int lam_guide_get_params(const lam_guide* guide, float* params);
int lam_guide_set_params(lam_guide* guide, const float* params);
/* Raw head outputs (n x 40 f32, device) for n device queries; box = scene bounds lo xyz, hi xyz
 * (lam_scene_bounds) used to normalise positions. */
int lam_guide_eval(const lam_guide* guide, const lam_guide_query* queries, uint32_t n, const float box[6],
                   float* outputs, void* stream);
/* Loss  (1/n) sum -weight log q(wi)  and its gradient with respect to the parameters (f32, device,
 * LAM_GUIDE_PARAMS entries, zero for unused ones) over n device records. */
int lam_guide_loss_grad(lam_guide* guide, const lam_guide_record* records, uint32_t n, const float box[6],
                        float* grad, float* loss, void* stream);
/* steps Adam steps on minibatches of options.batch records drawn from the n device records. */
int lam_guide_train(lam_guide* guide, const lam_guide_record* records, uint32_t n, uint32_t steps,
                    const float box[6], void* stream);
/* Number of Adam steps taken and samples per pixel trained so far.  Also reports, once, a
 * tensor-core completion wait of the guide's kernels that gave up: LAM_ERR_DEVICE_TIMEOUT. */
int lam_guide_progress(const lam_guide* guide, uint64_t* steps, uint32_t* trained_spp);
/* Bounded device waits: the polls of an mbarrier that the guide's tensor-core kernels
 * (lam_guide_eval, lam_guide_loss_grad, lam_guide_train) make before a wait gives up (default 2^20).
 * A CTA whose wait gives up lets its MMAs in flight finish, frees its tensor memory, records the
 * timeout and returns; its outputs are then undefined.  0 makes every wait give up at once, which
 * exercises that path without a stalled device. */
int lam_guide_set_wait_limit(lam_guide* guide, uint32_t tries);
/* Attaches the guide used by lam_render when guide_mode is LAM_GUIDE_LEARNED (NULL detaches). */
int lam_pipeline_set_guide(lam_pipeline* pipeline, lam_guide* guide);
/* World-space bounds of the scene's geometry: lo xyz, hi xyz. */
int lam_scene_bounds(const lam_scene* scene, float box[6]);

/* average, examples/cornell_box/src/average_to_buf.wgsl:11-21: out_rgb[3*p+c] = mean over
 * the n rgba32f device images frames[0..n) (host array of device pointers). */
int lam_average_frames(const float* const* frames, uint32_t n, uint32_t width, uint32_t height,
                       float* out_rgb, void* stream);

/* ---------------------------------------------------------------- denoiser hand-off
 * OidnState::new / denoise, examples/cornell_box/src/main.rs:797-963: the averaged frame (RGB f32,
 * width * height * 3 floats, the layout lam_average_frames writes) goes to host memory, a host-side
 * filter (OIDN's RayTracing filter in the reference) works on it in place, and the result returns to
 * the device buffer.  A lam_denoiser owns the pinned host staging of one frame size.
 * lam_denoise_fn gets the colour (filtered in place) and, when lam_denoiser_run was given them, the
 * first-hit normal and albedo images repacked to RGB f32 (else NULL); it returns 0, or nonzero for an
 * error (lam_denoiser_run then returns LAM_ERR_CALLBACK and leaves the device frame unchanged).
 * lam_denoiser_run synchronises `stream` twice: before the filter runs and after the upload. */
typedef struct lam_denoiser lam_denoiser;
typedef int (*lam_denoise_fn)(void* user, float* rgb, const float* normal, const float* albedo,
                              uint32_t width, uint32_t height);
int lam_denoiser_create(uint32_t width, uint32_t height, lam_denoiser** out);
/* rgb: device, width * height * 3 f32, filtered in place; normal / albedo: device rgba32f images of the
 * same size (lam_frame_targets.normal / .albedo) or NULL. */
int lam_denoiser_run(lam_denoiser* denoiser, float* rgb, const float* normal, const float* albedo,
                     lam_denoise_fn filter, void* user, void* stream);
int lam_denoiser_destroy(lam_denoiser* denoiser);

#ifdef __cplusplus
}
#endif

#endif /* LAMBENT_B200_H */
