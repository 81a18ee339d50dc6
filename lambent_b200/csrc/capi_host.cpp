// capi_host.cpp - host-only entry points of the C-ABI: errors, Material, Camera, TextureLoader,
// pipeline layout and tracer objects.  Reference interfaces are cited per function in
// include/lambent.h.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <mutex>
#include <unordered_set>
#include <string>
#include <vector>

#include "scene.h"
#include "tracer.h"

namespace lam {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return LAM_ERR_CUDA;
}

bool decode_png(const uint8_t* data, size_t n, std::vector<uint8_t>* rgba, uint32_t* w, uint32_t* h,
                std::string* why);

// ---- half 2.6.0 conversions (round to nearest even) used by Material::new (src/lib.rs:99-119, 172-176)
static uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

static uint16_t to_f16(float f) {
    uint32_t x = fbits(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    int32_t exp = (int32_t)((x >> 23) & 0xFFu);
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFF) return (uint16_t)(sign | 0x7C00u | (man ? 0x200u | (man >> 13) : 0u));
    int32_t he = exp - 112;  // rebias 127 -> 15
    if (he >= 31) return (uint16_t)(sign | 0x7C00u);
    if (he <= 0) {
        if (he < -10) return (uint16_t)sign;
        uint32_t full = man | 0x800000u;
        uint32_t shift = (uint32_t)(14 - he);
        uint32_t q = full >> shift;
        uint32_t rem = full & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (q & 1u))) ++q;
        return (uint16_t)(sign | q);
    }
    uint32_t out = sign | ((uint32_t)he << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (out & 1u))) ++out;
    return (uint16_t)out;
}

static uint16_t to_bf16(float f) {
    uint32_t x = fbits(f);
    if ((x & 0x7FFFFFFFu) > 0x7F800000u) return (uint16_t)((x >> 16) | 0x40u);
    uint32_t lsb = (x >> 16) & 1u;
    uint32_t rounding = 0x7FFFu + lsb;
    return (uint16_t)((x + rounding) >> 16);
}

static uint32_t pack2xf16(const float v[2]) { return (uint32_t)to_f16(v[0]) | ((uint32_t)to_f16(v[1]) << 16); }

// FP64 cofactor inverse of a column-major 4x4, rounded to f32.  False if singular.
static bool invert4(const float* m, float* out) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    // Gauss-Jordan with partial pivoting on [A | I]
    double aug[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            aug[r][c] = a[c * 4 + r];
            aug[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(aug[r][col]) > std::fabs(aug[piv][col])) piv = r;
        if (!(std::fabs(aug[piv][col]) > 0.0) || !std::isfinite(aug[piv][col])) return false;
        if (piv != col)
            for (int c = 0; c < 8; ++c) std::swap(aug[piv][c], aug[col][c]);
        double inv = 1.0 / aug[col][col];
        for (int c = 0; c < 8; ++c) aug[col][c] *= inv;
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            double f = aug[r][col];
            if (f != 0.0)
                for (int c = 0; c < 8; ++c) aug[r][c] -= f * aug[col][c];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double v = aug[r][4 + c];
            if (!std::isfinite(v)) return false;
            out[c * 4 + r] = (float)v;
        }
    return true;
}

}  // namespace lam

using namespace lam;

struct lam_texture_loader {
    struct Entry {
        std::vector<uint8_t> img[3];  // diffuse, lit, attributes (empty when not given)
        uint32_t w[3] = {0, 0, 0}, h[3] = {0, 0, 0};
    };
    std::vector<Entry> entries;
};

extern "C" {

uint32_t lam_version(void) { return 0x00010000u; }

const char* lam_last_error_message(void) { return g_last_error.c_str(); }

int lam_dispatch_size(uint32_t width, uint32_t height, uint32_t out[2]) {
    if (!out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_dispatch_size: null output");
    out[0] = (width + 63u) / 64u;
    out[1] = height;
    return LAM_OK;
}

int lam_material_new(const float uv1[2], const float uv2[2], const float uv3[2], const uint16_t recolour[2],
                     uint16_t tex_idx_diffuse, int32_t tex_idx_emission, int32_t tex_idx_attributes,
                     float emissive_texture_scale, float diffuse_texture_scale, const float* ior,
                     uint32_t material_type, lam_material* out) {
    if (!uv1 || !uv2 || !uv3 || !recolour || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_material_new: null argument");
    auto opt = [](int32_t v, uint16_t* o) {
        if (v < 0) { *o = 0xFFFFu; return true; }
        if (v >= 0xFFFF) return false;  // u16::MAX is reserved for "none" (lib.rs:165-170)
        *o = (uint16_t)v;
        return true;
    };
    uint16_t e, a;
    if (!opt(tex_idx_emission, &e) || !opt(tex_idx_attributes, &a))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "texture index u16::MAX is reserved for None");
    if (material_type > 0xFFFFu) return set_error(LAM_ERR_INVALID_ARGUMENT, "material type does not fit u16");
    const float vacuum[2] = {1.0f, 1.0f};
    const float* r = ior ? ior : vacuum;
    out->tex_pos_1 = pack2xf16(uv1);
    out->tex_pos_2 = pack2xf16(uv2);
    out->tex_pos_3 = pack2xf16(uv3);
    out->tex_pos_recolour = (uint32_t)recolour[0] | ((uint32_t)recolour[1] << 16);
    out->tex_idx_diffuse_emission = (uint32_t)tex_idx_diffuse | ((uint32_t)e << 16);
    out->tex_idx_attributes_ty = (uint32_t)a | (material_type << 16);
    out->emission_scale = (uint32_t)to_bf16(emissive_texture_scale) | ((uint32_t)to_bf16(diffuse_texture_scale) << 16);
    out->refractive_index = pack2xf16(r);
    return LAM_OK;
}

int lam_material_descriptor(const lam_material* m, uint32_t count, uint32_t further, lam_buffer_descriptor* out) {
    if ((!m && count) || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_material_descriptor: null argument");
    out->contents = m;
    out->size = (size_t)count * sizeof(lam_material);
    out->usage = LAM_USAGE_STORAGE | further;
    return LAM_OK;
}

int lam_refractive_index_between(const float in_front[2], const float behind[2], float out[2]) {
    if (!in_front || !behind || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    out[0] = behind[0] / in_front[0];
    out[1] = behind[1] / in_front[1];
    return LAM_OK;
}

int lam_camera_from_proj_view(const float proj[16], const float view[16], lam_camera* out) {
    if (!proj || !view || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_camera: null argument");
    lam_camera c;
    if (!invert4(proj, c.projection_inverse)) return set_error(LAM_ERR_PROJECTION_UNINVERTIBLE, "projection matrix is not invertible");
    if (!invert4(view, c.view_inverse)) return set_error(LAM_ERR_VIEW_UNINVERTIBLE, "view matrix is not invertible");
    *out = c;
    return LAM_OK;
}

int lam_camera_new(const float proj[16], const float view[16], lam_camera* out) {
    return lam_camera_from_proj_view(proj, view, out);
}

int lam_camera_update_from_proj_view(lam_camera* c, const float* proj, const float* view) {
    if (!c) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_camera_update_from_proj_view: null camera");
    float tmp[16];
    if (proj) {
        if (!invert4(proj, tmp)) return set_error(LAM_ERR_PROJECTION_UNINVERTIBLE, "projection matrix is not invertible");
        std::memcpy(c->projection_inverse, tmp, sizeof(tmp));
    }
    if (view) {
        if (!invert4(view, tmp)) return set_error(LAM_ERR_VIEW_UNINVERTIBLE, "view matrix is not invertible");
        std::memcpy(c->view_inverse, tmp, sizeof(tmp));
    }
    return LAM_OK;
}

int lam_camera_descriptor(const lam_camera* c, uint32_t further, lam_buffer_descriptor* out) {
    if (!c || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_camera_descriptor: null argument");
    out->contents = c;
    out->size = sizeof(lam_camera);
    out->usage = LAM_USAGE_UNIFORM | further;
    return LAM_OK;
}

// ---------------------------------------------------------------- TextureLoader
int lam_texture_loader_new(lam_texture_loader** out) {
    if (!out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null output");
    *out = new lam_texture_loader();
    return LAM_OK;
}

int lam_texture_loader_free(lam_texture_loader* l) {
    delete l;
    return LAM_OK;
}

static int decode_into(const uint8_t* bytes, size_t n, std::vector<uint8_t>* img, uint32_t* w, uint32_t* h) {
    std::string why;
    if (!decode_png(bytes, n, img, w, h, &why)) return set_error(LAM_ERR_TEXTURE, "texture decode failed: " + why);
    return LAM_OK;
}

int lam_texture_loader_load_from_bytes(lam_texture_loader* l, const uint8_t* diffuse, size_t dn, const uint8_t* lit,
                                       size_t ln, const uint8_t* attr, size_t an) {
    if (!l || !diffuse) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_texture_loader_load_from_bytes: null argument");
    lam_texture_loader::Entry e;
    int rc = decode_into(diffuse, dn, &e.img[0], &e.w[0], &e.h[0]);
    if (rc) return rc;
    if (lit && (rc = decode_into(lit, ln, &e.img[1], &e.w[1], &e.h[1]))) return rc;
    if (attr && (rc = decode_into(attr, an, &e.img[2], &e.w[2], &e.h[2]))) return rc;
    l->entries.push_back(std::move(e));
    return LAM_OK;
}

static int read_file(const char* path, std::vector<uint8_t>* out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return set_error(LAM_ERR_TEXTURE, std::string("cannot open texture file ") + path);
    out->assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return LAM_OK;
}

int lam_texture_loader_load(lam_texture_loader* l, const char* diffuse, const char* lit, const char* attr) {
    if (!l || !diffuse) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_texture_loader_load: null argument");
    std::vector<uint8_t> d, li, a;
    int rc = read_file(diffuse, &d);
    if (rc) return rc;
    if (lit && (rc = read_file(lit, &li))) return rc;
    if (attr && (rc = read_file(attr, &a))) return rc;
    return lam_texture_loader_load_from_bytes(l, d.data(), d.size(), lit ? li.data() : nullptr, li.size(),
                                              attr ? a.data() : nullptr, a.size());
}

int lam_texture_loader_load_rgba8(lam_texture_loader* l, uint32_t w, uint32_t h, const uint8_t* diffuse,
                                  const uint8_t* lit, const uint8_t* attr) {
    if (!l || !diffuse) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_texture_loader_load_rgba8: null argument");
    if (w == 0 || h == 0) return set_error(LAM_ERR_TEXTURE, "zero-sized image");
    lam_texture_loader::Entry e;
    const uint8_t* src[3] = {diffuse, lit, attr};
    for (int k = 0; k < 3; ++k) {
        if (!src[k]) continue;
        e.img[k].assign(src[k], src[k] + 4 * (size_t)w * h);
        e.w[k] = w;
        e.h[k] = h;
    }
    l->entries.push_back(std::move(e));
    return LAM_OK;
}

// Each cuboid is max(width) x max(height) x (number of entries that supplied that kind); smaller
// images are placed at the origin of their layer, the rest of the layer is zero.
int lam_texture_loader_raw(lam_texture_loader* l, lam_raw_textures* out) {
    if (!l || !out) {
        delete l;
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_texture_loader_raw: null argument");
    }
    std::memset(out, 0, sizeof(*out));
    out->entry_count = (uint32_t)l->entries.size();
    for (int k = 0; k < 3; ++k) {
        uint32_t W = 0, H = 0, layers = 0;
        for (auto& e : l->entries)
            if (!e.img[k].empty()) { W = std::max(W, e.w[k]); H = std::max(H, e.h[k]); ++layers; }
        out->width[k] = W;
        out->height[k] = H;
        out->layers[k] = layers;
        out->layer_of_entry[k] = (int32_t*)std::calloc(std::max<size_t>(1, l->entries.size()), sizeof(int32_t));
        size_t bytes = (size_t)W * H * 4 * layers;
        out->cuboid[k] = (uint8_t*)std::calloc(std::max<size_t>(1, bytes), 1);
        if (!out->layer_of_entry[k] || !out->cuboid[k]) {
            lam_raw_textures_free(out);
            delete l;
            return set_error(LAM_ERR_OUT_OF_MEMORY, "lam_texture_loader_raw: allocation failed");
        }
        uint32_t layer = 0;
        for (size_t i = 0; i < l->entries.size(); ++i) {
            auto& e = l->entries[i];
            if (e.img[k].empty()) { out->layer_of_entry[k][i] = -1; continue; }
            out->layer_of_entry[k][i] = (int32_t)layer;
            uint8_t* dst = out->cuboid[k] + (size_t)layer * W * H * 4;
            for (uint32_t y = 0; y < e.h[k]; ++y)
                std::memcpy(dst + (size_t)y * W * 4, e.img[k].data() + (size_t)y * e.w[k] * 4, (size_t)e.w[k] * 4);
            ++layer;
        }
    }
    delete l;
    return LAM_OK;
}

int lam_raw_textures_free(lam_raw_textures* raw) {
    if (!raw) return LAM_OK;
    for (int k = 0; k < 3; ++k) {
        std::free(raw->cuboid[k]);
        std::free(raw->layer_of_entry[k]);
        raw->cuboid[k] = nullptr;
        raw->layer_of_entry[k] = nullptr;
    }
    return LAM_OK;
}

// ---------------------------------------------------------------- pipeline layout / tracer
int lam_pipeline_layout_create(uint32_t blas, uint32_t diffuse, uint32_t emission, uint32_t attribute,
                               lam_pipeline_layout** out) {
    if (!out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null output");
    if (!blas || !diffuse || !emission || !attribute)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "pipeline layout counts must be nonzero (NonZeroU32)");
    lam_pipeline_layout* l = new lam_pipeline_layout();
    l->blas_count = blas;
    l->diffuse_count = diffuse;
    l->emission_count = emission;
    l->attribute_count = attribute;
    *out = l;
    return LAM_OK;
}

int lam_pipeline_layout_destroy(lam_pipeline_layout* l) {
    delete l;
    return LAM_OK;
}

int lam_tracer_create(uint32_t quality, lam_tracer** out) {
    if (!out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null output");
    if (quality > LAM_QUALITY_HIGH && (quality < LAM_DEBUG_FRONT_FACE || quality > LAM_DEBUG_TANGENT))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown shader quality");
    lam_tracer* t = new lam_tracer();
    t->quality = quality;
    *out = t;
    return LAM_OK;
}

int lam_tracer_destroy(lam_tracer* t) {
    delete t;
    return LAM_OK;
}

int lam_tracer_options_default(lam_tracer_options* o) {
    if (!o) return set_error(LAM_ERR_INVALID_ARGUMENT, "null output");
    o->samples = 4;
    o->tmin = 0.0001f;
    o->tmax = 1000.0f;
    o->restir_temporal = LAM_RESTIR_PER_PIXEL;
    o->max_depth = 5;
    o->guide_mode = LAM_GUIDE_NONE;
    return LAM_OK;
}

// ---------------------------------------------------------------- no-vertex-return input format
static std::mutex g_desc_mutex;
static std::unordered_set<const uint32_t*> g_desc_indices;  // index lists owned by adapter descs

int lam_blas_from_vertices(const void* blob, size_t blob_bytes, const uint32_t* indices, size_t index_count,
                           uint32_t geometry_count, const uint32_t* tris_per_geometry, uint32_t flags,
                           lam_blas_desc* out) {
    if (!blob || !out || (geometry_count && !tris_per_geometry))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_blas_from_vertices: null argument");
    if (blob_bytes < 16 || (blob_bytes - 16) % 16 != 0)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "Vertices blob: 16-byte header then [f32; 4] vertices");
    uint32_t stride;
    std::memcpy(&stride, blob, 4);
    const uint64_t vcount = (blob_bytes - 16) / 16;
    if (vcount > 0xFFFFFFFFull) return set_error(LAM_ERR_INVALID_ARGUMENT, "too many vertices");
    // arrayLength(&indices) == 1 selects the vertex index itself (get_vertices, general.wesl)
    const bool direct = !indices || index_count <= 1;
    uint64_t tris = 0;
    for (uint32_t g = 0; g < geometry_count; ++g) tris += tris_per_geometry[g];
    if (tris * 3 > 0xFFFFFFFFull) return set_error(LAM_ERR_INVALID_ARGUMENT, "too many triangles");
    std::vector<uint32_t> list;
    list.reserve((size_t)tris * 3);
    for (uint32_t g = 0; g < geometry_count; ++g)
        for (uint32_t p = 0; p < tris_per_geometry[g]; ++p)
            for (uint32_t j = 0; j < 3; ++j) {
                const uint64_t slot = (uint64_t)stride * g + 3ull * p + j;
                uint64_t v = slot;
                if (!direct) {
                    if (slot >= index_count) return set_error(LAM_ERR_INVALID_ARGUMENT, "index slot past the Indices array");
                    v = indices[slot];
                }
                if (v >= vcount) return set_error(LAM_ERR_INVALID_ARGUMENT, "vertex index past the Vertices blob");
                list.push_back((uint32_t)v);
            }
    uint32_t* owned = new uint32_t[std::max<size_t>(1, list.size())];
    if (!list.empty()) std::memcpy(owned, list.data(), list.size() * sizeof(uint32_t));
    {
        std::lock_guard<std::mutex> lk(g_desc_mutex);
        g_desc_indices.insert(owned);
    }
    out->vertices = reinterpret_cast<const float*>(static_cast<const char*>(blob) + 16);
    out->vertex_count = (uint32_t)vcount;
    out->vertex_stride = 4;
    out->indices = owned;
    out->index_count = (uint32_t)list.size();
    out->flags = flags;
    return LAM_OK;
}

int lam_blas_desc_free(lam_blas_desc* d) {
    if (!d || !d->indices) return LAM_OK;
    std::lock_guard<std::mutex> lk(g_desc_mutex);
    auto it = g_desc_indices.find(d->indices);
    if (it == g_desc_indices.end())
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_blas_desc_free: not made by lam_blas_from_vertices");
    g_desc_indices.erase(it);
    delete[] d->indices;
    d->indices = nullptr;
    d->index_count = 0;
    return LAM_OK;
}

int lam_material_table_for_geometries(const uint32_t* table, uint32_t table_len, uint32_t geometry_count,
                                      const uint32_t* tris_per_geometry, uint32_t* out) {
    if (!out || (geometry_count && !tris_per_geometry) || (table_len && !table))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_material_table_for_geometries: null argument");
    if (table_len == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "empty material table");
    size_t k = 0;
    for (uint32_t g = 0; g < geometry_count; ++g)
        for (uint32_t p = 0; p < tris_per_geometry[g]; ++p) out[k++] = table[p < table_len ? p : table_len - 1];
    return LAM_OK;
}

int lam_tracer_set_intersection_handler(lam_tracer* t, const char* src) {
    if (!t) return set_error(LAM_ERR_INVALID_ARGUMENT, "null tracer");
    return lam::set_intersection_handler(t, src);
}

}  // extern "C"
