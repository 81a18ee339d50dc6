// scene.cu - scene upload (BLAS/TLAS build, materials, textures) and the raw ray-query kernel.
//
// Replaces create_blas / create_tlas / build_acceleration_structures
// (examples/cornell_box/src/main.rs:464-563) and the group-0 / group-2 bindings
// (src/low_level.rs:237-397, src/textures.rs:41-243).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "bvh8.h"
#include "materials.cuh"
#include "scene.h"
#include "traverse.cuh"

namespace lam {

// Instance matrix inverse: FP64 adjugate / determinant rounded to f32 (the same procedure as
// the oracle, so the object-space rays agree bit for bit).
static bool invert_3x4(const float m[12], float out[12]) {
    double a = m[0], b = m[1], c = m[2];
    double d = m[4], e = m[5], f = m[6];
    double g = m[8], h = m[9], i = m[10];
    double A = e * i - f * h;
    double B = f * g - d * i;
    double C = d * h - e * g;
    double det = (a * A + b * B) + c * C;
    if (det == 0.0 || !std::isfinite(det)) return false;
    double r[9] = {A / det, (c * h - b * i) / det, (b * f - c * e) / det,
                   B / det, (a * i - c * g) / det, (c * d - a * f) / det,
                   C / det, (b * g - a * h) / det, (a * e - b * d) / det};
    double tx = m[3], ty = m[7], tz = m[11];
    for (int row = 0; row < 3; ++row) {
        out[row * 4 + 0] = (float)r[row * 3 + 0];
        out[row * 4 + 1] = (float)r[row * 3 + 1];
        out[row * 4 + 2] = (float)r[row * 3 + 2];
        out[row * 4 + 3] = (float)(-((r[row * 3 + 0] * tx + r[row * 3 + 1] * ty) + r[row * 3 + 2] * tz));
    }
    return true;
}

template <class T>
static int upload(lam_scene* s, const T* host, size_t count, const T** dev, cudaStream_t st) {
    *dev = nullptr;
    if (count == 0) return LAM_OK;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (scene)");
    s->allocations.push_back(p);
    e = cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync (scene)");
    *dev = (const T*)p;
    s->stats.device_bytes += count * sizeof(T);
    return LAM_OK;
}

static void free_scene(lam_scene* s) {
    for (void* p : s->allocations) cudaFree(p);
    s->allocations.clear();
}

}  // namespace lam

using namespace lam;

extern "C" int lam_scene_create(const lam_scene_desc* d, void* stream, lam_scene** out) {
    if (!d || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_create: null argument");
    *out = nullptr;
    if ((d->blas_count && !d->blas) || (d->instance_count && !d->instances) ||
        (d->material_count && !d->materials))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_create: null array with nonzero count");
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t st = (cudaStream_t)stream;

    // ---- validate and gather triangles per BLAS
    const uint32_t nb = d->blas_count;
    std::vector<uint32_t> tri_count(nb);
    std::vector<char> procedural(nb, 0);
    for (uint32_t b = 0; b < nb; ++b) {
        const lam_blas_desc& bd = d->blas[b];
        if (bd.aabb_count) {
            if (!bd.aabbs) return set_error(LAM_ERR_INVALID_ARGUMENT, "null aabbs");
            if (bd.index_count) return set_error(LAM_ERR_INVALID_ARGUMENT, "a BLAS holds triangles or AABBs, not both");
            for (uint32_t i = 0; i < bd.aabb_count; ++i)
                for (int k = 0; k < 3; ++k)
                    if (!(bd.aabbs[6 * (size_t)i + k] <= bd.aabbs[6 * (size_t)i + 3 + k]))
                        return set_error(LAM_ERR_INVALID_ARGUMENT, "AABB with min > max or NaN");
            procedural[b] = 1;
            tri_count[b] = bd.aabb_count;
            continue;
        }
        if (bd.vertex_stride != 3 && bd.vertex_stride != 4)
            return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_blas_desc.vertex_stride must be 3 or 4");
        if (bd.index_count % 3 != 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "index_count must be a multiple of 3");
        if (bd.vertex_count && !bd.vertices) return set_error(LAM_ERR_INVALID_ARGUMENT, "null vertices");
        if (bd.indices) {
            for (uint32_t i = 0; i < bd.index_count; ++i)
                if (bd.indices[i] >= bd.vertex_count)
                    return set_error(LAM_ERR_INVALID_ARGUMENT, "triangle index out of range");
        } else if (bd.index_count > bd.vertex_count) {
            return set_error(LAM_ERR_INVALID_ARGUMENT, "non-indexed BLAS needs index_count <= vertex_count");
        }
        tri_count[b] = bd.index_count / 3;
    }
    // ---- BLAS builds (one thread per BLAS, largest first)
    std::vector<Bvh8> bvh(nb);
    std::vector<std::vector<float4>> tri_data(nb);
    {
        std::vector<uint32_t> order(nb);
        for (uint32_t i = 0; i < nb; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return tri_count[a] > tri_count[b]; });
        std::atomic<uint32_t> next(0);
        auto work = [&]() {
            for (;;) {
                uint32_t q = next.fetch_add(1);
                if (q >= nb) break;
                uint32_t b = order[q];
                const lam_blas_desc& bd = d->blas[b];
                uint32_t n = tri_count[b];
                auto vtx = [&](uint32_t t, int c) {
                    uint32_t vi = bd.indices ? bd.indices[3 * t + c] : 3 * t + c;
                    return bd.vertices + (size_t)vi * bd.vertex_stride;
                };
                std::vector<float> boxes(6 * (size_t)n);
                if (procedural[b]) {
                    // AABB primitives: leaf slots hold (min, prim bits), (max, 0), (0)
                    std::memcpy(boxes.data(), bd.aabbs, boxes.size() * sizeof(float));
                    build_bvh8(boxes.data(), n, 3, &bvh[b]);
                    std::vector<float4>& td = tri_data[b];
                    td.resize(3 * (size_t)bvh[b].leaf_items.size());
                    for (size_t j = 0; j < bvh[b].leaf_items.size(); ++j) {
                        uint32_t t = bvh[b].leaf_items[j];
                        const float* a = bd.aabbs + 6 * (size_t)t;
                        float primbits;
                        std::memcpy(&primbits, &t, 4);
                        td[3 * j + 0] = make_float4(a[0], a[1], a[2], primbits);
                        td[3 * j + 1] = make_float4(a[3], a[4], a[5], 0.0f);
                        td[3 * j + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    }
                    continue;
                }
                for (uint32_t t = 0; t < n; ++t) {
                    for (int k = 0; k < 3; ++k) {
                        float lo = vtx(t, 0)[k], hi = lo;
                        for (int c = 1; c < 3; ++c) { lo = std::min(lo, vtx(t, c)[k]); hi = std::max(hi, vtx(t, c)[k]); }
                        boxes[6 * t + k] = lo;
                        boxes[6 * t + 3 + k] = hi;
                    }
                }
                build_bvh8(boxes.data(), n, 3, &bvh[b]);
                std::vector<float4>& td = tri_data[b];
                td.resize(3 * (size_t)bvh[b].leaf_items.size());
                for (size_t j = 0; j < bvh[b].leaf_items.size(); ++j) {
                    uint32_t t = bvh[b].leaf_items[j];
                    const float* p0 = vtx(t, 0);
                    const float* p1 = vtx(t, 1);
                    const float* p2 = vtx(t, 2);
                    float primbits;
                    std::memcpy(&primbits, &t, 4);
                    td[3 * j + 0] = make_float4(p0[0], p0[1], p0[2], primbits);
                    td[3 * j + 1] = make_float4(p1[0], p1[1], p1[2], 0.0f);
                    td[3 * j + 2] = make_float4(p2[0], p2[1], p2[2], 0.0f);
                }
            }
        };
        unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned i = 0; i < std::min<unsigned>(hw, std::max(1u, nb)); ++i) pool.emplace_back(work);
        for (auto& th : pool) th.join();
    }
    // ---- concatenate BLAS nodes / triangles with global offsets
    std::vector<uint32_t> node_off(nb), tri_off(nb);
    size_t total_nodes = 0, total_tris = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        node_off[b] = (uint32_t)total_nodes;
        tri_off[b] = (uint32_t)total_tris;
        total_nodes += bvh[b].nodes.size();
        total_tris += bvh[b].leaf_items.size();
    }
    if (total_nodes > 0x7FFFFFFFull || total_tris > 0x7FFFFFFFull)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "scene too large");
    std::vector<Bvh8Node> blas_nodes(total_nodes);
    std::vector<float4> tris(3 * total_tris);
    for (uint32_t b = 0; b < nb; ++b) {
        for (size_t i = 0; i < bvh[b].nodes.size(); ++i) {
            Bvh8Node nd = bvh[b].nodes[i];
            nd.child_base += node_off[b];
            nd.leaf_base += tri_off[b];
            blas_nodes[node_off[b] + i] = nd;
        }
        std::copy(tri_data[b].begin(), tri_data[b].end(), tris.begin() + 3 * (size_t)tri_off[b]);
    }
    // ---- instances and TLAS
    const uint32_t ni = d->instance_count;
    std::vector<DevInstance> inst(ni);
    std::vector<uint32_t> mat_idx;
    std::vector<float> iboxes(6 * (size_t)ni);
    // per instance: object-to-world 3x4, custom index bits, 3 zeros (read by intersection handlers)
    std::vector<float> fwd(16 * (size_t)ni);
    bool all_opaque = true, any_procedural = false;
    for (uint32_t i = 0; i < ni; ++i) {
        const lam_instance_desc& id = d->instances[i];
        if (id.blas >= nb) return set_error(LAM_ERR_INVALID_ARGUMENT, "instance references a missing BLAS");
        DevInstance& I = inst[i];
        if (!invert_3x4(id.transform, I.inv)) return set_error(LAM_ERR_INVALID_ARGUMENT, "singular instance transform");
        I.blas_root = bvh[id.blas].nodes.empty() ? NO_HIT : node_off[id.blas];
        I.mat_offset = (uint32_t)mat_idx.size();
        I.mat_count = id.material_indices ? id.material_index_count : 0u;
        if (I.mat_count) mat_idx.insert(mat_idx.end(), id.material_indices, id.material_indices + I.mat_count);
        bool opaque = (d->blas[id.blas].flags & LAM_GEOMETRY_OPAQUE) != 0u;
        all_opaque = all_opaque && opaque;
        I.flags = (opaque ? INST_OPAQUE : 0u) | ((id.mask & 0xFFu) ? INST_VISIBLE : 0u) |
                  (procedural[id.blas] ? INST_PROCEDURAL : 0u);
        any_procedural = any_procedural || procedural[id.blas];
        std::copy(id.transform, id.transform + 12, fwd.begin() + 16 * (size_t)i);
        std::memcpy(&fwd[16 * (size_t)i + 12], &id.custom_index, 4);
        // exact world box of the instance's transformed vertices (FP64), padded outward; a box of the
        // rotated object-space bounds would be up to 3^1.5 times larger and admit many rays that
        // cannot hit the instance
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        const lam_blas_desc& bd = d->blas[id.blas];
        const uint32_t nidx = procedural[id.blas] ? bd.aabb_count * 8u : tri_count[id.blas] * 3u;
        for (uint32_t k = 0; k < nidx; ++k) {
            float corner[3];
            const float* pv;
            if (procedural[id.blas]) {  // the 8 corners of every box
                const float* a = bd.aabbs + 6 * (size_t)(k >> 3);
                for (int c = 0; c < 3; ++c) corner[c] = a[((k >> c) & 1u) ? 3 + c : c];
                pv = corner;
            } else {
                const uint32_t vi = bd.indices ? bd.indices[k] : k;
                pv = bd.vertices + (size_t)vi * bd.vertex_stride;
            }
            for (int r = 0; r < 3; ++r) {
                const float* q = id.transform + 4 * r;
                double w = (double)q[0] * pv[0] + (double)q[1] * pv[1] + (double)q[2] * pv[2] + (double)q[3];
                lo[r] = std::min(lo[r], w);
                hi[r] = std::max(hi[r], w);
            }
        }
        if (nidx == 0)
            for (int r = 0; r < 3; ++r) lo[r] = hi[r] = (double)id.transform[4 * r + 3];
        double mag = 0.0;
        for (int k = 0; k < 3; ++k) mag = std::max({mag, std::fabs(lo[k]), std::fabs(hi[k]), hi[k] - lo[k]});
        double pad = mag * 1e-5 + 1e-30;
        for (int k = 0; k < 3; ++k) {
            iboxes[6 * i + k] = std::nextafter((float)(lo[k] - pad), -INFINITY);
            iboxes[6 * i + 3 + k] = std::nextafter((float)(hi[k] + pad), INFINITY);
        }
    }
    Bvh8 tlas;
    build_bvh8(iboxes.data(), ni, 1, &tlas);
    // ---- textures: one RGBA8 texel pool, layers diffuse | emission | attributes | recolour
    std::vector<DevTexLayer> layers;
    std::vector<uint32_t> texels;
    auto add_layers = [&](const lam_texture_layer* src, uint32_t n) -> int {
        if (n && !src) return set_error(LAM_ERR_INVALID_ARGUMENT, "null texture array");
        for (uint32_t i = 0; i < n; ++i) {
            const lam_texture_layer& L = src[i];
            if ((size_t)L.width * L.height && !L.rgba8) return set_error(LAM_ERR_TEXTURE, "null texture pixels");
            DevTexLayer dl;
            dl.offset = (uint32_t)texels.size();
            dl.w = L.width;
            dl.h = L.height;
            dl.pad = 0;
            size_t cnt = (size_t)L.width * L.height;
            size_t old = texels.size();
            texels.resize(old + cnt);
            if (cnt) std::memcpy(texels.data() + old, L.rgba8, cnt * 4);
            layers.push_back(dl);
        }
        return LAM_OK;
    };
    int rc;
    if ((rc = add_layers(d->diffuse, d->diffuse_count)) != LAM_OK) return rc;
    if ((rc = add_layers(d->emission, d->emission_count)) != LAM_OK) return rc;
    if ((rc = add_layers(d->attributes, d->attribute_count)) != LAM_OK) return rc;
    {
        static const uint8_t white[4] = {255, 255, 255, 255};
        lam_texture_layer w1{white, 1, 1};
        if ((rc = add_layers(d->recolour ? d->recolour : &w1, 1)) != LAM_OK) return rc;
    }
    if (texels.size() > 0xFFFFFFFFull) return set_error(LAM_ERR_INVALID_ARGUMENT, "texture pool too large");

    lam_scene* s = new lam_scene();
    cudaGetDevice(&s->device);
    DevScene& D = s->dev;
    auto fail = [&](int code) {
        free_scene(s);
        delete s;
        return code;
    };
    if ((rc = upload(s, reinterpret_cast<const uint4*>(blas_nodes.data()), blas_nodes.size() * 5, &D.blas_nodes, st))) return fail(rc);
    if ((rc = upload(s, reinterpret_cast<const uint4*>(tlas.nodes.data()), tlas.nodes.size() * 5, &D.tlas_nodes, st))) return fail(rc);
    if ((rc = upload(s, tris.data(), tris.size(), &D.tris, st))) return fail(rc);
    if ((rc = upload(s, tlas.leaf_items.data(), tlas.leaf_items.size(), &D.tlas_items, st))) return fail(rc);
    if ((rc = upload(s, inst.data(), inst.size(), &D.inst, st))) return fail(rc);
    if ((rc = upload(s, mat_idx.data(), mat_idx.size(), &D.mat_idx, st))) return fail(rc);
    if ((rc = upload(s, d->materials, d->material_count, &D.materials, st))) return fail(rc);
    if ((rc = upload(s, texels.data(), texels.size(), &D.texels, st))) return fail(rc);
    if ((rc = upload(s, layers.data(), layers.size(), &D.layers, st))) return fail(rc);
    if (any_procedural && (rc = upload(s, fwd.data(), fwd.size(), &D.inst_fwd, st))) return fail(rc);
    if (d->sky_faces && d->sky_size) {
        size_t n = 6 * (size_t)d->sky_size * d->sky_size;
        std::vector<uint32_t> sky(n);
        std::memcpy(sky.data(), d->sky_faces, n * 4);
        if ((rc = upload(s, sky.data(), n, &D.sky, st))) return fail(rc);
        D.sky_size = d->sky_size;
    }
    D.material_count = d->material_count;
    D.diffuse_first = 0;
    D.diffuse_count = d->diffuse_count;
    D.emission_first = d->diffuse_count;
    D.emission_count = d->emission_count;
    D.attr_first = d->diffuse_count + d->emission_count;
    D.attr_count = d->attribute_count;
    D.recolour_layer = D.attr_first + d->attribute_count;
    D.tlas_node_count = (uint32_t)tlas.nodes.size();
    D.instance_count = ni;
    D.all_opaque = all_opaque ? 1u : 0u;
    D.has_procedural = any_procedural ? 1u : 0u;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(cuda_error(e, "scene upload"));
    s->blas_count = nb;
    s->instance_count = ni;
    s->material_count = d->material_count;
    s->diffuse_count = d->diffuse_count;
    s->emission_count = d->emission_count;
    s->attribute_count = d->attribute_count;
    s->stats.triangle_count = total_tris;
    s->stats.blas_node_count = total_nodes;
    s->stats.tlas_node_count = tlas.nodes.size();
    s->stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int k = 0; k < 3; ++k) {
        s->bounds[k] = ni ? INFINITY : 0.0f;
        s->bounds[3 + k] = ni ? -INFINITY : 0.0f;
    }
    for (uint32_t i = 0; i < ni; ++i)
        for (int k = 0; k < 3; ++k) {
            s->bounds[k] = std::min(s->bounds[k], iboxes[6 * i + k]);
            s->bounds[3 + k] = std::max(s->bounds[3 + k], iboxes[6 * i + 3 + k]);
        }
    *out = s;
    return LAM_OK;
}

extern "C" int lam_scene_update_materials(lam_scene* s, const lam_material* m, uint32_t count, void* stream) {
    if (!s || (!m && count)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_update_materials: null argument");
    if (count != s->material_count)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_update_materials: count differs from the scene's");
    if (!count) return LAM_OK;
    cudaError_t e = cudaMemcpyAsync((void*)s->dev.materials, m, count * sizeof(lam_material), cudaMemcpyHostToDevice,
                                    (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_error(e, "lam_scene_update_materials");
    e = cudaStreamSynchronize((cudaStream_t)stream);
    return e == cudaSuccess ? LAM_OK : cuda_error(e, "lam_scene_update_materials");
}

extern "C" int lam_scene_stats_get(const lam_scene* s, lam_scene_stats* out) {
    if (!s || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_stats_get: null argument");
    *out = s->stats;
    return LAM_OK;
}

extern "C" int lam_scene_bounds(const lam_scene* s, float box[6]) {
    if (!s || !box) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_scene_bounds: null argument");
    std::memcpy(box, s->bounds, sizeof(s->bounds));
    return LAM_OK;
}

extern "C" int lam_scene_destroy(lam_scene* s) {
    if (!s) return LAM_OK;
    free_scene(s);
    delete s;
    return LAM_OK;
}

// ---------------------------------------------------------------- raw ray query kernel

namespace lam {

template <bool ANY, bool ALPHA>
__global__ void __launch_bounds__(TRACE_BLOCK) trace_rays_kernel(DevScene S, const lam_ray* __restrict__ rays,
                                                                 uint32_t n, lam_hit* __restrict__ hits,
                                                                 uint32_t* __restrict__ counter,
                                                                 uint32_t* __restrict__ err_out) {
    __shared__ TraceSmem sm;
    const uint4* tl;
    const DevInstance* in;
    stage_tlas(S, sm, tl, in);
    uint32_t err = 0u;
    auto load = [&](uint32_t i, float3& o, float3& d, float& t0, float& t1) {
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + i));
        const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
        o = make_float3(r0.x, r0.y, r0.z);
        d = make_float3(r1.x, r1.y, r1.z);
        t0 = r0.w;
        t1 = r1.w;
    };
    auto store = [&](uint32_t i, const TraceResult& tr) {
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(rays + i));
        const float4 r1 = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
        const float3 o = make_float3(r0.x, r0.y, r0.z), d = make_float3(r1.x, r1.y, r1.z);
        lam_hit h;
        if (tr.tri == NO_HIT) {
            h.t = 0.0f; h.u = 0.0f; h.v = 0.0f;
            h.primitive_index = NO_HIT;
            h.instance_index = NO_HIT;
            h.kind = LAM_HIT_NONE;
        } else {
            float m[12];
            for (int q = 0; q < 12; ++q) m[q] = in[tr.inst].inv[q];
            float3 oo, od;
            object_ray(m, o, d, &oo, &od);
            const float4* tp = S.tris + 3u * tr.tri;
            bool front;
            wbw_f64(oo, od, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), &h.t, &h.u, &h.v, &front);
            h.primitive_index = tr.prim;
            h.instance_index = tr.inst;
            h.kind = front ? LAM_HIT_FRONT : LAM_HIT_BACK;
        }
        hits[i] = h;
    };
    trace_persistent<ANY, ALPHA>(S, tl, in, n, counter, err, load, store);
    if (err) atomicOr(err_out, err);
}

int check_trace_call(const lam_scene* s, uint32_t n, const char* who) {
    if (n > LAM_TRACE_MAX_RAYS)
        return set_error(LAM_ERR_INVALID_ARGUMENT, std::string(who) + ": n exceeds LAM_TRACE_MAX_RAYS (2^31 - 1)");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_error(e, who);
    if (device != s->device)
        return set_error(LAM_ERR_INVALID_ARGUMENT, std::string(who) + ": the current device is not the scene's");
    return LAM_OK;
}

}  // namespace lam

extern "C" int lam_trace_rays(const lam_scene* s, const lam_ray* rays, uint32_t n, uint32_t mode, lam_hit* hits,
                              void* stream) {
    if (!s || (n && (!rays || !hits))) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_trace_rays: null argument");
    if (mode != LAM_TRACE_CLOSEST && mode != LAM_TRACE_ANY)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_trace_rays: unknown mode");
    if (n == 0) return LAM_OK;
    if (int rc = check_trace_call(s, n, "lam_trace_rays")) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* scratch = nullptr;  // [0] work counter, [1] error flags
    cudaError_t e = cudaMallocAsync((void**)&scratch, 8, st);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays scratch");
    cudaMemsetAsync(scratch, 0, 8, st);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    int per_sm = 8;
    dim3 grid(sms * per_sm), block(TRACE_BLOCK);
    const bool alpha = !s->dev.all_opaque;
    if (mode == LAM_TRACE_ANY) {
        if (alpha) trace_rays_kernel<true, true><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
        else trace_rays_kernel<true, false><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
    } else {
        if (alpha) trace_rays_kernel<false, true><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
        else trace_rays_kernel<false, false><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFreeAsync(scratch, st);
        return cuda_error(e, "trace_rays_kernel launch");
    }
    uint32_t err_flags = 0;
    cudaMemcpyAsync(&err_flags, scratch + 1, 4, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(scratch, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays");
    if (err_flags & ERR_STACK_OVERFLOW) return set_error(LAM_ERR_STACK_OVERFLOW, "traversal stack overflow");
    return LAM_OK;
}

// ---------------------------------------------------------------- allocation-free ray query
//
// lam_trace_rays_static: the same closest-hit / any-hit query as lam_trace_rays for callers that
// must not allocate device memory while they run (for example a render loop inside a fixed frame
// budget, where cudaMalloc / cudaFree can synchronise the device and stall the frame, or a host
// that reserves all of its GPU memory up front and forbids allocations afterwards).  Its only
// scratch - the work counter that hands rays to warps and the error flags - lives in the
// file-scope array below, which every GPU that loads this library holds until the process exits.
//
// Limits and sharing:
//   * n <= LAM_TRACE_STATIC_MAX_RAYS (2^31 - 1): the 32-bit work counter may overshoot n by one
//     claim per warp of the grid and must not wrap;
//   * every call uses the same array: calls that overlap on the GPU (different streams, or
//     several host threads) race on the counter and give wrong results; serialise them;
//   * the array keeps the last call's contents; each call clears the two words it uses first;
//   * the first call on a device resolves the array's device address with cudaGetSymbolAddress
//     (once per device, in the CUDA runtime's primary context of that device) and keeps it for the
//     life of the process; make that first call before any stream capture.  After cudaDeviceReset
//     the kept address is stale, so the entry point must not be used across a device reset;
//   * every call reads the error flags back and synchronises its stream before it returns.
namespace lam {

constexpr uint32_t STATIC_TRACE_WORDS = 64;  // 256 bytes; words 0 (work counter) and 1 (error flags) used
static __device__ __align__(256) uint32_t g_static_trace_scratch[STATIC_TRACE_WORDS];

constexpr int STATIC_TRACE_MAX_DEVICES = 64;
static std::atomic<uint32_t*> g_static_trace_ptr[STATIC_TRACE_MAX_DEVICES];

// Device address of g_static_trace_scratch on `device` (the current device); resolved once.
static int static_trace_scratch(int device, uint32_t** out) {
    if (device < 0 || device >= STATIC_TRACE_MAX_DEVICES)
        return set_error(LAM_ERR_UNSUPPORTED, "lam_trace_rays_static: device index beyond 63");
    uint32_t* p = g_static_trace_ptr[device].load(std::memory_order_acquire);
    if (!p) {
        void* addr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&addr, g_static_trace_scratch);
        if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static: cudaGetSymbolAddress");
        p = static_cast<uint32_t*>(addr);
        g_static_trace_ptr[device].store(p, std::memory_order_release);
    }
    *out = p;
    return LAM_OK;
}

}  // namespace lam

extern "C" int lam_trace_rays_static(const lam_scene* s, const lam_ray* rays, uint32_t n, uint32_t mode,
                                     lam_hit* hits, void* stream) {
    if (!s || (n && (!rays || !hits))) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_trace_rays_static: null argument");
    if (mode != LAM_TRACE_CLOSEST && mode != LAM_TRACE_ANY)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_trace_rays_static: unknown mode");
    if (n > LAM_TRACE_STATIC_MAX_RAYS)
        return set_error(LAM_ERR_INVALID_ARGUMENT,
                         "lam_trace_rays_static: n exceeds LAM_TRACE_STATIC_MAX_RAYS (2^31 - 1 rays per call)");
    if (n == 0) return LAM_OK;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static: cudaGetDevice");
    if (device != s->device)
        return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_trace_rays_static: the current device is not the scene's");
    uint32_t* scratch = nullptr;
    int rc = static_trace_scratch(device, &scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    e = cudaMemsetAsync(scratch, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static: clearing the scratch words");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    dim3 grid(sms * 8), block(TRACE_BLOCK);
    const bool alpha = !s->dev.all_opaque;
    if (mode == LAM_TRACE_ANY) {
        if (alpha) trace_rays_kernel<true, true><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
        else trace_rays_kernel<true, false><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
    } else {
        if (alpha) trace_rays_kernel<false, true><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
        else trace_rays_kernel<false, false><<<grid, block, 0, st>>>(s->dev, rays, n, hits, scratch, scratch + 1);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static: launch");
    uint32_t err_flags = 0;
    e = cudaMemcpyAsync(&err_flags, scratch + 1, sizeof(err_flags), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static: reading the error flags");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "lam_trace_rays_static");
    if (err_flags & ERR_STACK_OVERFLOW) return set_error(LAM_ERR_STACK_OVERFLOW, "traversal stack overflow");
    return LAM_OK;
}
