//! Safe Rust API over liblambent_b200 (the B200 / sm_100a C-ABI of the Lambent path-tracing hot path),
//! with the names and argument meaning of the Lambent crate:
//!
//!   Material::new / EmissionScale / MaterialType       src/lib.rs:83-203
//!   Camera::from_proj_view / update_from_proj_view     src/camera.rs:6-70
//!   TextureLoader::{new, load, load_from_bytes, raw}   src/textures.rs:12-91, README.md:29-45
//!   RayTracer::<S>::{new, set_intersection_handler,
//!                     create_pipeline}                  src/lib.rs:260-329
//!   path_tracing::{Low, Medium, High, PathTracerOpts,
//!                  RestirTemporalMode}                  src/path_tracing/mod.rs:7-147
//!   DataBuffers::{new, resize, advance_frame}          src/data_buffer/mod.rs:150-349
//!   dispatch_size                                      src/lib.rs:207-219
//!
//! Where the reference hands back wgpu objects, these types own the device-side state behind the
//! C-ABI handles and free it on drop.  Device pointers (frame targets, rays) are plain CUDA global
//! memory addresses; `stream` arguments are cudaStream_t values (null: the legacy default stream).
use core::marker::PhantomData;
use core::num::NonZeroU32;
use core::ops::Range;
use std::ffi::{CStr, CString};
use std::fmt;
use std::ptr;

pub use lambent_b200_sys as sys;

/// A failed C-ABI call: its status code (`sys::LAM_ERR_*`) and the library's message.
#[derive(Debug, Clone)]
pub struct Error {
    pub code: i32,
    pub message: String,
}

impl fmt::Display for Error {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "lambent_b200 error {}: {}", self.code, self.message)
    }
}

impl std::error::Error for Error {}

fn check(rc: i32) -> Result<(), Error> {
    if rc == sys::LAM_OK {
        return Ok(());
    }
    let msg = unsafe {
        let p = sys::lam_last_error_message();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    };
    Err(Error { code: rc, message: msg })
}

// ---------------------------------------------------------------- materials (src/lib.rs)

/// MaterialType, src/lib.rs:194-203.
#[repr(u8)]
#[derive(Clone, Copy, Debug)]
pub enum MaterialType {
    Diffuse = 0,
    Metallic = 1,
    Transparent = 2,
}

/// EmissionScale, src/lib.rs:96-121 (the library rounds both scales to bf16).
#[derive(Copy, Clone, Debug, Default)]
pub struct EmissionScale {
    pub emissive_texture_scale: f32,
    pub diffuse_texture_scale: f32,
}

impl EmissionScale {
    pub fn from_emission_scale(scale: f32) -> Self {
        Self { emissive_texture_scale: scale, diffuse_texture_scale: 0.0 }
    }
    pub fn from_f32(emissive_texture_scale: f32, diffuse_texture_scale: f32) -> Self {
        Self { emissive_texture_scale, diffuse_texture_scale }
    }
}

/// The 32-byte material record, bit-identical to the reference's Material.
#[repr(transparent)]
#[derive(Copy, Clone, Debug)]
pub struct Material(pub sys::lam_material);

impl Material {
    /// Material::new, src/lib.rs:132-163.  Panics when an optional index is u16::MAX, as the
    /// reference's map_optional_idx asserts.
    #[allow(clippy::too_many_arguments)]
    pub fn new(
        tex_pos_1: [f32; 2],
        tex_pos_2: [f32; 2],
        tex_pos_3: [f32; 2],
        tex_pos_recolour: [u16; 2],
        tex_idx_diffuse: u16,
        tex_idx_emission: Option<u16>,
        tex_idx_attributes: Option<u16>,
        emission_scale: EmissionScale,
        refractive_index: Option<Range<f32>>,
        ty: MaterialType,
    ) -> Self {
        let opt = |o: Option<u16>| -> i32 {
            match o {
                None => -1,
                Some(u) => {
                    assert_ne!(u16::MAX, u);
                    u as i32
                }
            }
        };
        let ior = refractive_index.map(|r| [r.start, r.end]);
        let mut out = sys::lam_material {
            tex_pos_1: 0,
            tex_pos_2: 0,
            tex_pos_3: 0,
            tex_pos_recolour: 0,
            tex_idx_diffuse_emission: 0,
            tex_idx_attributes_ty: 0,
            emission_scale: 0,
            refractive_index: 0,
        };
        let rc = unsafe {
            sys::lam_material_new(
                tex_pos_1.as_ptr(),
                tex_pos_2.as_ptr(),
                tex_pos_3.as_ptr(),
                tex_pos_recolour.as_ptr(),
                tex_idx_diffuse,
                opt(tex_idx_emission),
                opt(tex_idx_attributes),
                emission_scale.emissive_texture_scale,
                emission_scale.diffuse_texture_scale,
                ior.as_ref().map_or(ptr::null(), |a| a.as_ptr()),
                ty as u32,
                &mut out,
            )
        };
        check(rc).expect("lam_material_new");
        Material(out)
    }
}

// ---------------------------------------------------------------- camera (src/camera.rs)

/// CameraError, src/camera.rs:53-57.
#[derive(Debug)]
pub enum CameraError {
    ProjectionUninvertable([[f32; 4]; 4]),
    ViewUninvertable([[f32; 4]; 4]),
}

/// The 128-byte camera record: inverse projection and view, column-major.
#[repr(transparent)]
#[derive(Copy, Clone, Debug)]
pub struct Camera(pub sys::lam_camera);

fn flat(m: &[[f32; 4]; 4]) -> [f32; 16] {
    let mut o = [0.0f32; 16];
    for c in 0..4 {
        o[4 * c..4 * c + 4].copy_from_slice(&m[c]);
    }
    o
}

impl Camera {
    /// Camera::from_proj_view (README: Camera::new): normal (not inverted) matrices, columns first.
    pub fn from_proj_view(proj: [[f32; 4]; 4], view: [[f32; 4]; 4]) -> Result<Camera, CameraError> {
        let mut c = sys::lam_camera { projection_inverse: [0.0; 16], view_inverse: [0.0; 16] };
        let rc = unsafe { sys::lam_camera_from_proj_view(flat(&proj).as_ptr(), flat(&view).as_ptr(), &mut c) };
        match rc {
            sys::LAM_OK => Ok(Camera(c)),
            sys::LAM_ERR_PROJECTION_UNINVERTIBLE => Err(CameraError::ProjectionUninvertable(proj)),
            _ => Err(CameraError::ViewUninvertable(view)),
        }
    }

    pub fn new(proj: [[f32; 4]; 4], view: [[f32; 4]; 4]) -> Result<Camera, CameraError> {
        Self::from_proj_view(proj, view)
    }

    /// Camera::update_from_proj_view: either matrix may be None.
    pub fn update_from_proj_view(
        &mut self,
        proj: Option<[[f32; 4]; 4]>,
        view: Option<[[f32; 4]; 4]>,
    ) -> Result<(), CameraError> {
        let p = proj.map(|m| flat(&m));
        let v = view.map(|m| flat(&m));
        let rc = unsafe {
            sys::lam_camera_update_from_proj_view(
                &mut self.0,
                p.as_ref().map_or(ptr::null(), |a| a.as_ptr()),
                v.as_ref().map_or(ptr::null(), |a| a.as_ptr()),
            )
        };
        match rc {
            sys::LAM_OK => Ok(()),
            sys::LAM_ERR_PROJECTION_UNINVERTIBLE => Err(CameraError::ProjectionUninvertable(proj.unwrap())),
            _ => Err(CameraError::ViewUninvertable(view.unwrap())),
        }
    }
}

// ---------------------------------------------------------------- textures (src/textures.rs, README raw)

/// TextureLoader: decoded RGBA8 images, one entry per load().
pub struct TextureLoader {
    h: *mut sys::lam_texture_loader,
}

/// The three texture cuboids of TextureLoader::raw (README.md:39-43): layers x height x width x RGBA8.
pub struct RawTextures {
    pub diffuse: (Vec<u8>, u32, u32, u32),
    pub lit: (Vec<u8>, u32, u32, u32),
    pub attributes: (Vec<u8>, u32, u32, u32),
}

impl TextureLoader {
    pub fn new() -> Result<Self, Error> {
        let mut h = ptr::null_mut();
        check(unsafe { sys::lam_texture_loader_new(&mut h) })?;
        Ok(Self { h })
    }

    /// TextureLoader::load; the lit (emission) and attribute images are optional.
    pub fn load(&mut self, diffuse: &str, lit: Option<&str>, attributes: Option<&str>) -> Result<(), Error> {
        let c = |s: &str| CString::new(s).expect("path with a NUL byte");
        let (d, l, a) = (c(diffuse), lit.map(c), attributes.map(c));
        check(unsafe {
            sys::lam_texture_loader_load(
                self.h,
                d.as_ptr(),
                l.as_ref().map_or(ptr::null(), |x| x.as_ptr()),
                a.as_ref().map_or(ptr::null(), |x| x.as_ptr()),
            )
        })
    }

    /// TextureLoader::load_from_bytes (PNG bytes).
    pub fn load_from_bytes(&mut self, diffuse: &[u8], lit: Option<&[u8]>, attributes: Option<&[u8]>) -> Result<(), Error> {
        let p = |b: Option<&[u8]>| b.map_or((ptr::null(), 0usize), |x| (x.as_ptr(), x.len()));
        let (lp, ll) = p(lit);
        let (ap, al) = p(attributes);
        check(unsafe {
            sys::lam_texture_loader_load_from_bytes(self.h, diffuse.as_ptr(), diffuse.len(), lp, ll, ap, al)
        })
    }

    /// README `raw`: consumes the loader and returns the three cuboids.
    pub fn raw(mut self) -> Result<RawTextures, Error> {
        let mut r: sys::lam_raw_textures = unsafe { core::mem::zeroed() };
        let h = core::mem::replace(&mut self.h, ptr::null_mut());
        check(unsafe { sys::lam_texture_loader_raw(h, &mut r) })?;
        let take = |k: usize| {
            let n = r.layers[k] as usize * r.height[k] as usize * r.width[k] as usize * 4;
            let v = if n == 0 { Vec::new() } else { unsafe { std::slice::from_raw_parts(r.cuboid[k], n).to_vec() } };
            (v, r.width[k], r.height[k], r.layers[k])
        };
        let out = RawTextures { diffuse: take(0), lit: take(1), attributes: take(2) };
        unsafe { sys::lam_raw_textures_free(&mut r) };
        Ok(out)
    }
}

impl Drop for TextureLoader {
    fn drop(&mut self) {
        if !self.h.is_null() {
            unsafe { sys::lam_texture_loader_free(self.h) };
        }
    }
}

// ---------------------------------------------------------------- shaders and options

/// RayTracingShader: the quality levels of path_tracing and the views of debug.
pub trait RayTracingShader {
    const QUALITY: u32;
}

pub mod path_tracing {
    use super::*;

    pub struct Low;
    pub struct Medium;
    pub struct High;
    impl RayTracingShader for Low {
        const QUALITY: u32 = sys::LAM_QUALITY_LOW as u32;
    }
    impl RayTracingShader for Medium {
        const QUALITY: u32 = sys::LAM_QUALITY_MEDIUM as u32;
    }
    impl RayTracingShader for High {
        const QUALITY: u32 = sys::LAM_QUALITY_HIGH as u32;
    }

    /// RestirTemporalMode, src/path_tracing/mod.rs:31-41.
    #[derive(Default, Debug, Clone, Copy)]
    pub enum RestirTemporalMode {
        Disabled,
        PerSample,
        #[default]
        PerPixel,
    }

    /// PathTracerOpts, src/path_tracing/mod.rs:7-23, plus the path length (the reference's fixed
    /// BOUNCES = 5) and the directional sampler at diffuse vertices (sys::LAM_GUIDE_*).
    pub struct PathTracerOpts {
        pub samples: NonZeroU32,
        pub tmin: f32,
        pub tmax: f32,
        pub restir_temporal: RestirTemporalMode,
        pub max_depth: u32,
        pub guide_mode: u32,
    }

    impl Default for PathTracerOpts {
        fn default() -> Self {
            Self {
                samples: NonZeroU32::new(4).unwrap(),
                tmin: 0.0001,
                tmax: 1000.0,
                restir_temporal: RestirTemporalMode::default(),
                max_depth: 5,
                guide_mode: sys::LAM_GUIDE_NONE as u32,
            }
        }
    }

    impl PathTracerOpts {
        pub(crate) fn raw(&self) -> sys::lam_tracer_options {
            sys::lam_tracer_options {
                samples: self.samples.get(),
                tmin: self.tmin,
                tmax: self.tmax,
                restir_temporal: match self.restir_temporal {
                    RestirTemporalMode::Disabled => sys::LAM_RESTIR_DISABLED as u32,
                    RestirTemporalMode::PerSample => sys::LAM_RESTIR_PER_SAMPLE as u32,
                    RestirTemporalMode::PerPixel => sys::LAM_RESTIR_PER_PIXEL as u32,
                },
                max_depth: self.max_depth,
                guide_mode: self.guide_mode,
            }
        }
    }
}

pub mod debug {
    use super::*;

    pub struct FrontFace;
    pub struct Reflectance;
    pub struct Tangent;
    impl RayTracingShader for FrontFace {
        const QUALITY: u32 = sys::LAM_DEBUG_FRONT_FACE as u32;
    }
    impl RayTracingShader for Reflectance {
        const QUALITY: u32 = sys::LAM_DEBUG_REFLECTANCE as u32;
    }
    impl RayTracingShader for Tangent {
        const QUALITY: u32 = sys::LAM_DEBUG_TANGENT as u32;
    }
}

/// dispatch_size, src/lib.rs:207-219: workgroups of 64 x 1.
pub fn dispatch_size(width: u32, height: u32) -> (u32, u32) {
    let mut wg = [0u32; 2];
    unsafe { sys::lam_dispatch_size(width, height, wg.as_mut_ptr()) };
    (wg[0], wg[1])
}

// ---------------------------------------------------------------- tracer and pipeline (src/lib.rs)

/// RayTracer::<S>, src/lib.rs:260-329.  The CUDA device current on the calling thread runs it.
pub struct RayTracer<S: RayTracingShader> {
    h: *mut sys::lam_tracer,
    shader: PhantomData<S>,
}

impl<S: RayTracingShader> RayTracer<S> {
    pub fn new() -> Result<Self, Error> {
        let mut h = ptr::null_mut();
        check(unsafe { sys::lam_tracer_create(S::QUALITY, &mut h) })?;
        Ok(Self { h, shader: PhantomData })
    }

    /// set_intersection_handler: CUDA C++ source defining
    /// `__device__ lam_aabb_intersection intersect(const lam_ray_intersection&)`; None restores the
    /// default handler (every procedural candidate misses).
    pub fn set_intersection_handler(&mut self, cuda_source: Option<&str>) -> Result<(), Error> {
        let src = cuda_source.map(|s| CString::new(s).expect("handler source with a NUL byte"));
        check(unsafe {
            sys::lam_tracer_set_intersection_handler(self.h, src.as_ref().map_or(ptr::null(), |c| c.as_ptr()))
        })
    }

    /// create_pipeline, src/lib.rs:297-318: the counts of pipeline_layout (low_level.rs:237-343) and
    /// the options; the handler is compiled and linked here.
    pub fn create_pipeline(
        &self,
        blas_count: NonZeroU32,
        diffuse_count: NonZeroU32,
        emission_count: NonZeroU32,
        attribute_count: NonZeroU32,
        options: &path_tracing::PathTracerOpts,
    ) -> Result<Pipeline, Error> {
        let mut layout = ptr::null_mut();
        check(unsafe {
            sys::lam_pipeline_layout_create(
                blas_count.get(),
                diffuse_count.get(),
                emission_count.get(),
                attribute_count.get(),
                &mut layout,
            )
        })?;
        let opts = options.raw();
        let mut h = ptr::null_mut();
        let rc = unsafe { sys::lam_tracer_create_pipeline(self.h, layout, &opts, &mut h) };
        unsafe { sys::lam_pipeline_layout_destroy(layout) };
        check(rc)?;
        Ok(Pipeline { h })
    }
}

impl<S: RayTracingShader> Drop for RayTracer<S> {
    fn drop(&mut self) {
        unsafe { sys::lam_tracer_destroy(self.h) };
    }
}

/// A compiled path tracer (the reference's ComputePipeline).
pub struct Pipeline {
    h: *mut sys::lam_pipeline,
}

/// Output images (rgba32float, width * height * 4 floats, row-major device memory); any may be null.
pub struct FrameTargets {
    pub color: *mut f32,
    pub normal: *mut f32,
    pub albedo: *mut f32,
    pub width: u32,
    pub height: u32,
}

impl Pipeline {
    /// One dispatch of rt_main (general.wesl:506-610) with the seed offset of the immediate.
    pub fn render(
        &mut self,
        scene: &Scene,
        buffers: &mut DataBuffers,
        camera: &Camera,
        targets: &FrameTargets,
        seed_offset: u32,
        stream: *mut core::ffi::c_void,
    ) -> Result<(), Error> {
        let t = sys::lam_frame_targets {
            color: targets.color,
            normal: targets.normal,
            albedo: targets.albedo,
            width: targets.width,
            height: targets.height,
        };
        check(unsafe { sys::lam_render(self.h, scene.h, buffers.h, &camera.0, &t, seed_offset, stream) })
    }

    pub fn stats(&self) -> Result<sys::lam_render_stats, Error> {
        let mut s: sys::lam_render_stats = unsafe { core::mem::zeroed() };
        check(unsafe { sys::lam_render_stats_get(self.h, &mut s) })?;
        Ok(s)
    }

    /// Bounds the paths of one wave (about 220 bytes of device state each); 0 restores the default of
    /// about 32M paths.  The image does not depend on it.  No counterpart in the reference.
    pub fn set_wave_paths(&mut self, max_paths: u64) -> Result<(), Error> {
        check(unsafe { sys::lam_pipeline_set_wave_paths(self.h, max_paths) })
    }

    /// The order in which each bounce's hits are shaded.  No counterpart in the reference.
    pub fn set_shade_order(&mut self, order: ShadeOrder) -> Result<(), Error> {
        check(unsafe { sys::lam_pipeline_set_shade_order(self.h, order as u32) })
    }
}

/// Shading order of a pipeline's bounces: `Material` sorts each bounce's hits by shading class (sky,
/// diffuse, metallic, transparent) before shading, `Queue` shades them in traversal order, and
/// `Auto`, the default, sorts except under Markov guiding.  A plain render's image is the same in
/// every order.
#[repr(u32)]
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum ShadeOrder {
    Auto = sys::LAM_SHADE_ORDER_AUTO,
    Queue = sys::LAM_SHADE_ORDER_QUEUE,
    Material = sys::LAM_SHADE_ORDER_MATERIAL,
}

impl Drop for Pipeline {
    fn drop(&mut self) {
        unsafe { sys::lam_pipeline_destroy(self.h) };
    }
}

// ---------------------------------------------------------------- scene (BLAS / TLAS build)

/// A scene built on the device from a lam_scene_desc: BLASes, instances with their material tables,
/// materials, texture layers and the sky (create_blas / create_tlas / build_acceleration_structures
/// of examples/cornell_box/src/main.rs:464-563).
pub struct Scene {
    h: *mut sys::lam_scene,
}

impl Scene {
    /// Builds the scene.  Every pointer in `desc` is read during the call only.
    ///
    /// # Safety
    /// `desc` and the arrays it points to must be valid for the counts it gives.
    pub unsafe fn new(desc: &sys::lam_scene_desc, stream: *mut core::ffi::c_void) -> Result<Self, Error> {
        let mut h = ptr::null_mut();
        check(sys::lam_scene_create(desc, stream, &mut h))?;
        Ok(Self { h })
    }

    pub fn update_materials(&mut self, materials: &[Material], stream: *mut core::ffi::c_void) -> Result<(), Error> {
        check(unsafe {
            sys::lam_scene_update_materials(
                self.h,
                materials.as_ptr() as *const sys::lam_material,
                materials.len() as u32,
                stream,
            )
        })
    }
}

impl Drop for Scene {
    fn drop(&mut self) {
        unsafe { sys::lam_scene_destroy(self.h) };
    }
}

// ---------------------------------------------------------------- DataBuffers (src/data_buffer/mod.rs)

/// BufferType bitflags, src/data_buffer/mod.rs:18-27.
pub mod buffer_type {
    use super::sys;
    pub const MARKOV_CHAIN_SCREEN_SPACE: u32 = sys::LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE as u32;
    pub const SPATIAL_RESAMPLING: u32 = sys::LAM_BUFFER_SPATIAL_RESAMPLING as u32;
    pub const MARKOV_CHAIN_WORLD_SPACE: u32 = sys::LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE as u32;
    pub const ALL: u32 = sys::LAM_BUFFER_ALL as u32;
}

/// AdvanceOptions, src/data_buffer/mod.rs:436-472.
#[derive(Clone, Copy, Debug)]
pub struct AdvanceOptions {
    pub confidence_cap: u32,
}

impl AdvanceOptions {
    pub const RESPONSIVE: Self = Self { confidence_cap: 2 };
    pub const SEMI_INTERACTIVE: Self = Self { confidence_cap: 30 };
    pub const SLOW: Self = Self { confidence_cap: 100 };
}

pub struct DataBuffers {
    h: *mut sys::lam_data_buffers,
}

impl DataBuffers {
    /// DataBuffers::new, src/data_buffer/mod.rs:150-252.
    pub fn new(width: u32, height: u32, world_space_buffer_size: u32, buffers: u32) -> Result<Self, Error> {
        let mut h = ptr::null_mut();
        check(unsafe { sys::lam_data_buffers_new(width, height, world_space_buffer_size, buffers, &mut h) })?;
        Ok(Self { h })
    }

    pub fn resize(&mut self, width: u32, height: u32) -> Result<(), Error> {
        check(unsafe { sys::lam_data_buffers_resize(self.h, width, height) })
    }

    pub fn advance_frame(
        &mut self,
        buffers_to_advance: u32,
        options: AdvanceOptions,
        stream: *mut core::ffi::c_void,
    ) -> Result<(), Error> {
        check(unsafe { sys::lam_data_buffers_advance_frame(self.h, buffers_to_advance, options.confidence_cap, stream) })
    }
}

impl Drop for DataBuffers {
    fn drop(&mut self) {
        unsafe { sys::lam_data_buffers_destroy(self.h) };
    }
}
