// @generated by gen_bindings.py from include/lambent.h - do not edit by hand.
#![allow(non_camel_case_types, non_upper_case_globals, clippy::all)]
#![no_std]

pub use core::ffi::{c_char, c_int, c_uint, c_void};

pub const LAM_OK: c_int = 0;
pub const LAM_ERR_INVALID_ARGUMENT: c_int = -1;
pub const LAM_ERR_OUT_OF_MEMORY: c_int = -2;
pub const LAM_ERR_CUDA: c_int = -3;
pub const LAM_ERR_NOT_BUILT: c_int = -4;
pub const LAM_ERR_PROJECTION_UNINVERTIBLE: c_int = -5;
pub const LAM_ERR_VIEW_UNINVERTIBLE: c_int = -6;
pub const LAM_ERR_TEXTURE: c_int = -7;
pub const LAM_ERR_COMPILE: c_int = -8;
pub const LAM_ERR_LAYOUT_MISMATCH: c_int = -9;
pub const LAM_ERR_UNSUPPORTED: c_int = -10;
pub const LAM_ERR_DEVICE_TIMEOUT: c_int = -11;
pub const LAM_ERR_STACK_OVERFLOW: c_int = -12;
pub const LAM_ERR_CALLBACK: c_int = -13;
pub const LAM_DIFFUSE: c_int = 0;
pub const LAM_METALLIC: c_int = 1;
pub const LAM_TRANSPARENT: c_int = 2;
pub const LAM_SKY: c_int = 0xFF;
pub const LAM_QUALITY_LOW: c_int = 0;
pub const LAM_QUALITY_MEDIUM: c_int = 1;
pub const LAM_QUALITY_HIGH: c_int = 2;
pub const LAM_DEBUG_FRONT_FACE: c_int = 16;
pub const LAM_DEBUG_REFLECTANCE: c_int = 17;
pub const LAM_DEBUG_TANGENT: c_int = 18;
pub const LAM_RESTIR_DISABLED: c_int = 0;
pub const LAM_RESTIR_PER_SAMPLE: c_int = 1;
pub const LAM_RESTIR_PER_PIXEL: c_int = 2;
pub const LAM_GUIDE_NONE: c_int = 0;
pub const LAM_GUIDE_MARKOV: c_int = 1;
pub const LAM_GUIDE_LEARNED: c_int = 2;
pub const LAM_GUIDE_PDF_AT_SAMPLE: c_int = 4;
pub const LAM_GUIDE_METAL: c_int = 8;
pub const LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE: c_int = 1 << 0;
pub const LAM_BUFFER_SPATIAL_RESAMPLING: c_int = 1 << 1;
pub const LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE: c_int = 1 << 2;
pub const LAM_BUFFER_ALL: c_int = 7;
pub const LAM_USAGE_COPY_DST: c_int = 0x8;
pub const LAM_USAGE_UNIFORM: c_int = 0x40;
pub const LAM_USAGE_STORAGE: c_int = 0x80;
pub const LAM_GEOMETRY_OPAQUE: c_int = 1;
pub const LAM_TRACE_CLOSEST: c_int = 0;
pub const LAM_TRACE_ANY: c_int = 1;
pub const LAM_HIT_NONE: c_int = 0;
pub const LAM_HIT_FRONT: c_int = 1;
pub const LAM_HIT_BACK: c_int = 2;
pub const LAM_TRACE_MAX_RAYS: u32 = 0x7FFFFFFF;
pub const LAM_TRACE_STATIC_MAX_RAYS: u32 = 0x7FFFFFFF;
pub const LAM_SHADE_ORDER_AUTO: u32 = 0;
pub const LAM_SHADE_ORDER_QUEUE: u32 = 1;
pub const LAM_SHADE_ORDER_MATERIAL: u32 = 2;
pub const LAM_GUIDE_PARAMS: u32 = 16384;
pub const LAM_GUIDE_OUTPUTS: u32 = 40;

#[repr(C)]
pub struct lam_pipeline_layout {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_tracer {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_pipeline {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_scene {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_data_buffers {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_texture_loader {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_guide {
    _private: [u8; 0],
}
#[repr(C)]
pub struct lam_denoiser {
    _private: [u8; 0],
}

pub type lam_denoise_fn = Option<unsafe extern "C" fn(user: *mut c_void, rgb: *mut f32, normal: *const f32, albedo: *const f32, width: u32, height: u32) -> c_int>;

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_material {
    pub tex_pos_1: u32,
    pub tex_pos_2: u32,
    pub tex_pos_3: u32,
    pub tex_pos_recolour: u32,
    pub tex_idx_diffuse_emission: u32,
    pub tex_idx_attributes_ty: u32,
    pub emission_scale: u32,
    pub refractive_index: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_camera {
    pub projection_inverse: [f32; 16],
    pub view_inverse: [f32; 16],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_markov_chain {
    pub light_source: [f32; 3],
    pub mean_cosine: f32,
    pub weight_sum: f32,
    pub num_samples: u32,
    pub score: f32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_world_markov_chain {
    pub secondary_hash: u32,
    pub num_samples: u32,
    pub luminance: [u32; 3],
    pub lock: u32,
    pub chain_light_source: [u32; 3],
    pub chain_mean_cosine: u32,
    pub chain_weight_sum: u32,
    pub chain_num_samples: u32,
    pub chain_score: u32,
    pub timeout: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_reservoir {
    pub visible_point: [f32; 3],
    pub visible_normal: u32,
    pub sample_point: [f32; 3],
    pub sample_normal: u32,
    pub out_radiance: [f32; 3],
    pub ty: u32,
    pub roughness: f32,
    pub w: f32,
    pub packed_confidence_valid: u32,
    pub W: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_info {
    pub arr: [f32; 9],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_buffer_descriptor {
    pub contents: *const c_void,
    pub size: usize,
    pub usage: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_blas_desc {
    pub vertices: *const f32,
    pub vertex_count: u32,
    pub vertex_stride: u32,
    pub indices: *const u32,
    pub index_count: u32,
    pub flags: u32,
    pub aabbs: *const f32,
    pub aabb_count: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_instance_desc {
    pub transform: [f32; 12],
    pub blas: u32,
    pub custom_index: u32,
    pub mask: u32,
    pub material_indices: *const u32,
    pub material_index_count: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_texture_layer {
    pub rgba8: *const u8,
    pub width: u32,
    pub height: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_scene_desc {
    pub blas: *const lam_blas_desc,
    pub blas_count: u32,
    pub instances: *const lam_instance_desc,
    pub instance_count: u32,
    pub materials: *const lam_material,
    pub material_count: u32,
    pub diffuse: *const lam_texture_layer,
    pub diffuse_count: u32,
    pub emission: *const lam_texture_layer,
    pub emission_count: u32,
    pub attributes: *const lam_texture_layer,
    pub attribute_count: u32,
    pub recolour: *const lam_texture_layer,
    pub sky_faces: *const u8,
    pub sky_size: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_scene_stats {
    pub triangle_count: u64,
    pub blas_node_count: u64,
    pub tlas_node_count: u64,
    pub device_bytes: u64,
    pub build_seconds: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_tracer_options {
    pub samples: u32,
    pub tmin: f32,
    pub tmax: f32,
    pub restir_temporal: u32,
    pub max_depth: u32,
    pub guide_mode: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_frame_targets {
    pub color: *mut f32,
    pub normal: *mut f32,
    pub albedo: *mut f32,
    pub width: u32,
    pub height: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_ray {
    pub origin: [f32; 3],
    pub tmin: f32,
    pub direction: [f32; 3],
    pub tmax: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_hit {
    pub t: f32,
    pub u: f32,
    pub v: f32,
    pub primitive_index: u32,
    pub instance_index: u32,
    pub kind: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_render_stats {
    pub ray_segments: u64,
    pub samples: u64,
    pub kernel_launches: u32,
    pub error_flags: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_stage_times {
    pub generate_ms: f64,
    pub extend_ms: f64,
    pub shade_ms: f64,
    pub accumulate_ms: f64,
    pub extend_launches: u64,
    pub shade_launches: u64,
    pub ray_segments: u64,
    pub train_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_raw_textures {
    pub cuboid: [*mut u8; 3],
    pub width: [u32; 3],
    pub height: [u32; 3],
    pub layers: [u32; 3],
    pub layer_of_entry: [*mut i32; 3],
    pub entry_count: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_batch_request {
    pub scene: *const lam_scene,
    pub camera: lam_camera,
    pub targets: lam_frame_targets,
    pub samples: u32,
    pub seed_offset: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_batch_tuning {
    pub wave_paths: u32,
    pub extend_blocks_per_sm: u32,
    pub shade_blocks_per_sm: u32,
    pub use_graph: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_guide_options {
    pub train_spp: u32,
    pub steps_per_wave: u32,
    pub batch: u32,
    pub record_capacity: u32,
    pub learning_rate: f32,
    pub guide_fraction: f32,
    pub seed: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_guide_query {
    pub pos: [f32; 3],
    pub normal: [f32; 3],
    pub wo: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lam_guide_record {
    pub pos: [f32; 3],
    pub normal: [f32; 3],
    pub wo: [f32; 3],
    pub wi: [f32; 3],
    pub weight: f32,
}

extern "C" {
    pub fn lam_blas_from_vertices(vertices_blob: *const c_void, blob_bytes: usize, indices: *const u32, index_count: usize, geometry_count: u32, triangles_per_geometry: *const u32, flags: u32, out: *mut lam_blas_desc) -> c_int;
    pub fn lam_blas_desc_free(desc: *mut lam_blas_desc) -> c_int;
    pub fn lam_material_table_for_geometries(table: *const u32, table_len: u32, geometry_count: u32, triangles_per_geometry: *const u32, out: *mut u32) -> c_int;
    pub fn lam_version() -> u32;
    pub fn lam_last_error_message() -> *const c_char;
    pub fn lam_dispatch_size(width: u32, height: u32, out_workgroups: *mut u32) -> c_int;
    pub fn lam_material_new(tex_pos_1: *const f32, tex_pos_2: *const f32, tex_pos_3: *const f32, tex_pos_recolour: *const u16, tex_idx_diffuse: u16, tex_idx_emission: i32, tex_idx_attributes: i32, emissive_texture_scale: f32, diffuse_texture_scale: f32, refractive_index_range: *const f32, material_type: u32, out: *mut lam_material) -> c_int;
    pub fn lam_material_descriptor(materials: *const lam_material, count: u32, further_usages: u32, out: *mut lam_buffer_descriptor) -> c_int;
    pub fn lam_refractive_index_between(in_front: *const f32, behind: *const f32, out: *mut f32) -> c_int;
    pub fn lam_camera_new(proj: *const f32, view: *const f32, out: *mut lam_camera) -> c_int;
    pub fn lam_camera_from_proj_view(proj: *const f32, view: *const f32, out: *mut lam_camera) -> c_int;
    pub fn lam_camera_update_from_proj_view(camera: *mut lam_camera, proj: *const f32, view: *const f32) -> c_int;
    pub fn lam_camera_descriptor(camera: *const lam_camera, further_usages: u32, out: *mut lam_buffer_descriptor) -> c_int;
    pub fn lam_texture_loader_new(out: *mut *mut lam_texture_loader) -> c_int;
    pub fn lam_texture_loader_load(loader: *mut lam_texture_loader, diffuse_path: *const c_char, lit_path: *const c_char, attributes_path: *const c_char) -> c_int;
    pub fn lam_texture_loader_load_from_bytes(loader: *mut lam_texture_loader, diffuse: *const u8, diffuse_len: usize, lit: *const u8, lit_len: usize, attributes: *const u8, attributes_len: usize) -> c_int;
    pub fn lam_texture_loader_load_rgba8(loader: *mut lam_texture_loader, width: u32, height: u32, diffuse: *const u8, lit: *const u8, attributes: *const u8) -> c_int;
    pub fn lam_texture_loader_raw(loader: *mut lam_texture_loader, out: *mut lam_raw_textures) -> c_int;
    pub fn lam_raw_textures_free(raw: *mut lam_raw_textures) -> c_int;
    pub fn lam_texture_loader_free(loader: *mut lam_texture_loader) -> c_int;
    pub fn lam_pipeline_layout_create(blas_count: u32, diffuse_count: u32, emission_count: u32, attribute_count: u32, out: *mut *mut lam_pipeline_layout) -> c_int;
    pub fn lam_pipeline_layout_destroy(layout: *mut lam_pipeline_layout) -> c_int;
    pub fn lam_tracer_create(quality: u32, out: *mut *mut lam_tracer) -> c_int;
    pub fn lam_tracer_set_intersection_handler(tracer: *mut lam_tracer, cuda_source: *const c_char) -> c_int;
    pub fn lam_tracer_destroy(tracer: *mut lam_tracer) -> c_int;
    pub fn lam_tracer_options_default(out: *mut lam_tracer_options) -> c_int;
    pub fn lam_tracer_create_pipeline(tracer: *const lam_tracer, layout: *const lam_pipeline_layout, options: *const lam_tracer_options, out: *mut *mut lam_pipeline) -> c_int;
    pub fn lam_pipeline_destroy(pipeline: *mut lam_pipeline) -> c_int;
    pub fn lam_scene_create(desc: *const lam_scene_desc, stream: *mut c_void, out: *mut *mut lam_scene) -> c_int;
    pub fn lam_scene_update_materials(scene: *mut lam_scene, materials: *const lam_material, count: u32, stream: *mut c_void) -> c_int;
    pub fn lam_scene_stats_get(scene: *const lam_scene, out: *mut lam_scene_stats) -> c_int;
    pub fn lam_scene_destroy(scene: *mut lam_scene) -> c_int;
    pub fn lam_trace_rays(scene: *const lam_scene, rays: *const lam_ray, n: u32, mode: u32, hits: *mut lam_hit, stream: *mut c_void) -> c_int;
    pub fn lam_pipeline_trace_rays(pipeline: *mut lam_pipeline, scene: *const lam_scene, rays: *const lam_ray, n: u32, mode: u32, hits: *mut lam_hit, stream: *mut c_void) -> c_int;
    pub fn lam_trace_rays_static(scene: *const lam_scene, rays: *const lam_ray, n: u32, mode: u32, hits: *mut lam_hit, stream: *mut c_void) -> c_int;
    pub fn lam_data_buffers_new(width: u32, height: u32, world_space_buffer_size: u32, buffer_types: u32, out: *mut *mut lam_data_buffers) -> c_int;
    pub fn lam_data_buffers_resize(buffers: *mut lam_data_buffers, width: u32, height: u32) -> c_int;
    pub fn lam_data_buffers_advance_frame(buffers: *mut lam_data_buffers, buffers_to_advance: u32, confidence_cap: u32, stream: *mut c_void) -> c_int;
    pub fn lam_data_buffers_get(buffers: *const lam_data_buffers, which: u32, device_ptr: *mut *mut c_void, bytes: *mut usize) -> c_int;
    pub fn lam_data_buffers_destroy(buffers: *mut lam_data_buffers) -> c_int;
    pub fn lam_render(pipeline: *mut lam_pipeline, scene: *const lam_scene, buffers: *mut lam_data_buffers, camera: *const lam_camera, targets: *const lam_frame_targets, seed_offset: u32, stream: *mut c_void) -> c_int;
    pub fn lam_render_stats_get(pipeline: *const lam_pipeline, out: *mut lam_render_stats) -> c_int;
    pub fn lam_pipeline_set_profiling(pipeline: *mut lam_pipeline, enabled: c_int) -> c_int;
    pub fn lam_render_profile_get(pipeline: *mut lam_pipeline, out: *mut lam_stage_times) -> c_int;
    pub fn lam_pipeline_set_wave_paths(pipeline: *mut lam_pipeline, max_paths: u64) -> c_int;
    pub fn lam_pipeline_set_shade_order(pipeline: *mut lam_pipeline, order: u32) -> c_int;
    pub fn lam_render_profile_reset(pipeline: *mut lam_pipeline) -> c_int;
    pub fn lam_temporal_resampling(buffers: *mut lam_data_buffers, width: u32, height: u32, seed_offset: u32, stream: *mut c_void) -> c_int;
    pub fn lam_spatial_resampling(buffers: *mut lam_data_buffers, targets: *const lam_frame_targets, is_samples: u32, is_space: u32, seed_offset: u32, stream: *mut c_void) -> c_int;
    pub fn lam_batch_render(pipeline: *mut lam_pipeline, requests: *const lam_batch_request, n: u32, tuning: *const lam_batch_tuning, stream: *mut c_void) -> c_int;
    pub fn lam_batch_latencies(pipeline: *mut lam_pipeline, n: u32, ms: *mut f64) -> c_int;
    pub fn lam_batch_autotune(pipeline: *mut lam_pipeline, requests: *const lam_batch_request, n: u32, spp_divisor: u32, out: *mut lam_batch_tuning, stream: *mut c_void) -> c_int;
    pub fn lam_guide_options_default(out: *mut lam_guide_options) -> c_int;
    pub fn lam_guide_create(options: *const lam_guide_options, out: *mut *mut lam_guide) -> c_int;
    pub fn lam_guide_destroy(guide: *mut lam_guide) -> c_int;
    pub fn lam_guide_get_params(guide: *const lam_guide, params: *mut f32) -> c_int;
    pub fn lam_guide_set_params(guide: *mut lam_guide, params: *const f32) -> c_int;
    pub fn lam_guide_eval(guide: *const lam_guide, queries: *const lam_guide_query, n: u32, box: *const f32, outputs: *mut f32, stream: *mut c_void) -> c_int;
    pub fn lam_guide_loss_grad(guide: *mut lam_guide, records: *const lam_guide_record, n: u32, box: *const f32, grad: *mut f32, loss: *mut f32, stream: *mut c_void) -> c_int;
    pub fn lam_guide_train(guide: *mut lam_guide, records: *const lam_guide_record, n: u32, steps: u32, box: *const f32, stream: *mut c_void) -> c_int;
    pub fn lam_guide_progress(guide: *const lam_guide, steps: *mut u64, trained_spp: *mut u32) -> c_int;
    pub fn lam_guide_set_wait_limit(guide: *mut lam_guide, tries: u32) -> c_int;
    pub fn lam_pipeline_set_guide(pipeline: *mut lam_pipeline, guide: *mut lam_guide) -> c_int;
    pub fn lam_scene_bounds(scene: *const lam_scene, box: *mut f32) -> c_int;
    pub fn lam_average_frames(frames: *const *const f32, n: u32, width: u32, height: u32, out_rgb: *mut f32, stream: *mut c_void) -> c_int;
    pub fn lam_denoiser_create(width: u32, height: u32, out: *mut *mut lam_denoiser) -> c_int;
    pub fn lam_denoiser_run(denoiser: *mut lam_denoiser, rgb: *mut f32, normal: *const f32, albedo: *const f32, filter: lam_denoise_fn, user: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn lam_denoiser_destroy(denoiser: *mut lam_denoiser) -> c_int;
}
