// oracle_scene.cpp - TEST INFRASTRUCTURE ONLY (the CPU oracle; see oracle_scene.h).
#include "oracle_scene.h"

#include <algorithm>
#include <cfloat>
#include <cstring>

namespace oracle {

// ---------------------------------------------------------------- instance transforms
bool invert_3x4(const float m[12], float out[12]) {
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

void object_ray(const float m[12], vec3 o, vec3 d, vec3* oo, vec3* od) {
    float r[3], s[3];
    for (int row = 0; row < 3; ++row) {
        const float* q = m + row * 4;
        r[row] = std::fma(q[0], o.x, std::fma(q[1], o.y, std::fma(q[2], o.z, q[3])));
        s[row] = std::fma(q[0], d.x, std::fma(q[1], d.y, q[2] * d.z));
    }
    *oo = vec3(r[0], r[1], r[2]);
    *od = vec3(s[0], s[1], s[2]);
}

// ---------------------------------------------------------------- watertight test (Woop, Benthin, Wald 2013)
WbwRay wbw_setup(vec3 d) {
    float a[3] = {absf(d.x), absf(d.y), absf(d.z)};
    int kz = 0;
    float m = a[0];
    if (a[1] > m) { kz = 1; m = a[1]; }
    if (a[2] > m) { kz = 2; }
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < 0.0f) std::swap(kx, ky);
    WbwRay r;
    r.kx = kx; r.ky = ky; r.kz = kz;
    // one IEEE reciprocal, then two products (lambent_b200/csrc/traverse.cuh setup_ray does the same)
    r.Sz = 1.0f / d[kz];
    r.Sx = d[kx] * r.Sz;
    r.Sy = d[ky] * r.Sz;
    return r;
}

bool wbw_f32(const WbwRay& r, vec3 o, vec3 v0, vec3 v1, vec3 v2, float* t_out) {
    vec3 A = v0 - o, B = v1 - o, C = v2 - o;
    float Ax = std::fma(-r.Sx, A[r.kz], A[r.kx]);
    float Ay = std::fma(-r.Sy, A[r.kz], A[r.ky]);
    float Bx = std::fma(-r.Sx, B[r.kz], B[r.kx]);
    float By = std::fma(-r.Sy, B[r.kz], B[r.ky]);
    float Cx = std::fma(-r.Sx, C[r.kz], C[r.kx]);
    float Cy = std::fma(-r.Sy, C[r.kz], C[r.ky]);
    float U = std::fma(Cx, By, -(Cy * Bx));
    float V = std::fma(Ax, Cy, -(Ay * Cx));
    float W = std::fma(Bx, Ay, -(By * Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = (U + V) + W;
    if (det == 0.0f) return false;
    float Az = r.Sz * A[r.kz];
    float Bz = r.Sz * B[r.kz];
    float Cz = r.Sz * C[r.kz];
    float T = std::fma(U, Az, std::fma(V, Bz, W * Cz));
    *t_out = T / det;
    return true;
}

void wbw_f64(vec3 of, vec3 df, vec3 v0f, vec3 v1f, vec3 v2f, float* t, float* u, float* v, bool* front) {
    WbwRay sel = wbw_setup(df);
    int kx = sel.kx, ky = sel.ky, kz = sel.kz;
    double o[3] = {of.x, of.y, of.z}, d[3] = {df.x, df.y, df.z};
    double p0[3] = {v0f.x, v0f.y, v0f.z}, p1[3] = {v1f.x, v1f.y, v1f.z}, p2[3] = {v2f.x, v2f.y, v2f.z};
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) { a[k] = p0[k] - o[k]; b[k] = p1[k] - o[k]; c[k] = p2[k] - o[k]; }
    double Sx = d[kx] / d[kz], Sy = d[ky] / d[kz], Sz = 1.0 / d[kz];
    double Ax = a[kx] - Sx * a[kz], Ay = a[ky] - Sy * a[kz];
    double Bx = b[kx] - Sx * b[kz], By = b[ky] - Sy * b[kz];
    double Cx = c[kx] - Sx * c[kz], Cy = c[ky] - Sy * c[kz];
    double U = Cx * By - Cy * Bx;
    double V = Ax * Cy - Ay * Cx;
    double W = Bx * Ay - By * Ax;
    double det = (U + V) + W;
    double Az = Sz * a[kz], Bz = Sz * b[kz], Cz = Sz * c[kz];
    double T = (U * Az + V * Bz) + W * Cz;
    *t = (float)(T / det);
    *u = (float)(V / det);
    *v = (float)(W / det);
    double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double nd = (n[0] * d[0] + n[1] * d[1]) + n[2] * d[2];
    *front = nd < 0.0;
}

// ---------------------------------------------------------------- BVH2 (binned SAH)
namespace {
struct Box {
    double lo[3], hi[3];
    void reset() { for (int k = 0; k < 3; ++k) { lo[k] = DBL_MAX; hi[k] = -DBL_MAX; } }
    void grow(const double* l, const double* h) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], l[k]); hi[k] = std::max(hi[k], h[k]); }
    }
    double area() const {
        double e[3];
        for (int k = 0; k < 3; ++k) e[k] = std::max(0.0, hi[k] - lo[k]);
        return 2.0 * (e[0] * e[1] + e[1] * e[2] + e[0] * e[2]);
    }
};
}  // namespace

void Bvh::build(const std::vector<double>& boxes, uint32_t n) {
    nodes.clear();
    items.resize(n);
    for (uint32_t i = 0; i < n; ++i) items[i] = i;
    if (n == 0) return;
    std::vector<double> cen(3 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5 * (boxes[6 * i + k] + boxes[6 * i + 3 + k]);
    struct Task { int32_t node; int32_t first, count; };
    std::vector<Task> stack;
    nodes.push_back(BNode());
    stack.push_back({0, 0, (int32_t)n});
    const int BINS = 16;
    while (!stack.empty()) {
        Task tk = stack.back();
        stack.pop_back();
        Box nb, cb;
        nb.reset(); cb.reset();
        for (int32_t i = tk.first; i < tk.first + tk.count; ++i) {
            uint32_t it = items[i];
            nb.grow(&boxes[6 * it], &boxes[6 * it + 3]);
            cb.grow(&cen[3 * it], &cen[3 * it]);
        }
        // Conservative padding: the f32 watertight hit point may sit ~1e-7 relative outside the box.
        double mag = 0.0;
        for (int k = 0; k < 3; ++k) mag = std::max({mag, std::fabs(nb.lo[k]), std::fabs(nb.hi[k]), nb.hi[k] - nb.lo[k]});
        double pad = mag * 1e-5 + 1e-30;
        BNode& node = nodes[tk.node];
        for (int k = 0; k < 3; ++k) { node.lo[k] = nb.lo[k] - pad; node.hi[k] = nb.hi[k] + pad; }
        if (tk.count <= 2) { node.first = tk.first; node.count = tk.count; continue; }
        int axis = 0;
        double ext = cb.hi[0] - cb.lo[0];
        for (int k = 1; k < 3; ++k) if (cb.hi[k] - cb.lo[k] > ext) { ext = cb.hi[k] - cb.lo[k]; axis = k; }
        int32_t mid = -1;
        if (ext > 0.0) {
            Box bb[BINS];
            int cnt[BINS] = {0};
            for (auto& b : bb) b.reset();
            double scale = BINS / ext;
            auto bin_of = [&](uint32_t it) {
                int b = (int)((cen[3 * it + axis] - cb.lo[axis]) * scale);
                return std::min(std::max(b, 0), BINS - 1);
            };
            for (int32_t i = tk.first; i < tk.first + tk.count; ++i) {
                uint32_t it = items[i];
                int b = bin_of(it);
                cnt[b]++;
                bb[b].grow(&boxes[6 * it], &boxes[6 * it + 3]);
            }
            double best = DBL_MAX;
            int best_split = -1;
            for (int s = 1; s < BINS; ++s) {
                Box l, r;
                l.reset(); r.reset();
                int nl = 0, nr = 0;
                for (int b = 0; b < s; ++b) if (cnt[b]) { l.grow(bb[b].lo, bb[b].hi); nl += cnt[b]; }
                for (int b = s; b < BINS; ++b) if (cnt[b]) { r.grow(bb[b].lo, bb[b].hi); nr += cnt[b]; }
                if (!nl || !nr) continue;
                double c = l.area() * nl + r.area() * nr;
                if (c < best) { best = c; best_split = s; }
            }
            if (best_split > 0) {
                auto it = std::partition(items.begin() + tk.first, items.begin() + tk.first + tk.count,
                                         [&](uint32_t x) { return bin_of(x) < best_split; });
                mid = (int32_t)(it - items.begin());
            }
        }
        if (mid <= tk.first || mid >= tk.first + tk.count) mid = tk.first + tk.count / 2;
        int32_t l = (int32_t)nodes.size();
        nodes.push_back(BNode());
        nodes.push_back(BNode());
        nodes[tk.node].left = l;
        nodes[tk.node].right = l + 1;
        stack.push_back({l, tk.first, mid - tk.first});
        stack.push_back({l + 1, mid, tk.first + tk.count - mid});
    }
}

static bool box_hit(const BNode& nd, const double o[3], const double d[3], double tmin, double tmax) {
    double t0 = tmin, t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.0) {
            if (o[k] < nd.lo[k] || o[k] > nd.hi[k]) return false;
            continue;
        }
        double inv = 1.0 / d[k];
        double a = (nd.lo[k] - o[k]) * inv, b = (nd.hi[k] - o[k]) * inv;
        if (a > b) std::swap(a, b);
        t0 = std::max(t0, a);
        t1 = std::min(t1, b);
        if (t0 > t1) return false;
    }
    return true;
}

// ---------------------------------------------------------------- scene load
int Scene::load(const lam_scene_desc* d) {
    if (!d) return LAM_ERR_INVALID_ARGUMENT;
    blas.resize(d->blas_count);
    for (uint32_t b = 0; b < d->blas_count; ++b) {
        const lam_blas_desc& bd = d->blas[b];
        if (bd.vertex_stride != 3 && bd.vertex_stride != 4) return LAM_ERR_INVALID_ARGUMENT;
        Blas& bl = blas[b];
        bl.v.resize(3 * (size_t)bd.vertex_count);
        for (uint32_t i = 0; i < bd.vertex_count; ++i)
            for (int k = 0; k < 3; ++k) bl.v[3 * i + k] = bd.vertices[(size_t)i * bd.vertex_stride + k];
        if (bd.indices) {
            bl.idx.assign(bd.indices, bd.indices + bd.index_count);
        } else {
            bl.idx.resize(bd.index_count);
            for (uint32_t i = 0; i < bd.index_count; ++i) bl.idx[i] = i;
        }
        bl.tri_count = (uint32_t)(bl.idx.size() / 3);
        for (uint32_t i : bl.idx) if (i >= bd.vertex_count) return LAM_ERR_INVALID_ARGUMENT;
        bl.opaque = (bd.flags & LAM_GEOMETRY_OPAQUE) != 0;
        std::vector<double> boxes(6 * (size_t)bl.tri_count);
        for (uint32_t t = 0; t < bl.tri_count; ++t) {
            for (int k = 0; k < 3; ++k) {
                double lo = DBL_MAX, hi = -DBL_MAX;
                for (int c = 0; c < 3; ++c) {
                    double x = bl.v[3 * bl.idx[3 * t + c] + k];
                    lo = std::min(lo, x);
                    hi = std::max(hi, x);
                }
                boxes[6 * t + k] = lo;
                boxes[6 * t + 3 + k] = hi;
            }
        }
        bl.bvh.build(boxes, bl.tri_count);
    }
    inst.resize(d->instance_count);
    std::vector<double> iboxes(6 * (size_t)d->instance_count);
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const lam_instance_desc& id = d->instances[i];
        if (id.blas >= d->blas_count) return LAM_ERR_INVALID_ARGUMENT;
        Instance& in = inst[i];
        std::memcpy(in.xf, id.transform, sizeof(in.xf));
        if (!invert_3x4(in.xf, in.inv)) return LAM_ERR_INVALID_ARGUMENT;
        in.blas = id.blas;
        in.mask = id.mask;
        in.custom = id.custom_index;
        if (id.material_indices) in.mat.assign(id.material_indices, id.material_indices + id.material_index_count);
        const Blas& bl = blas[id.blas];
        double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        if (!bl.bvh.nodes.empty()) {
            const BNode& r = bl.bvh.nodes[0];
            for (int c = 0; c < 8; ++c) {
                double p[3] = {(c & 1) ? r.hi[0] : r.lo[0], (c & 2) ? r.hi[1] : r.lo[1], (c & 4) ? r.hi[2] : r.lo[2]};
                for (int row = 0; row < 3; ++row) {
                    const float* q = in.xf + 4 * row;
                    double w = (double)q[0] * p[0] + (double)q[1] * p[1] + (double)q[2] * p[2] + (double)q[3];
                    lo[row] = std::min(lo[row], w);
                    hi[row] = std::max(hi[row], w);
                }
            }
        }
        for (int k = 0; k < 3; ++k) { iboxes[6 * i + k] = lo[k]; iboxes[6 * i + 3 + k] = hi[k]; }
    }
    tlas.build(iboxes, d->instance_count);
    materials.assign(d->materials, d->materials + d->material_count);
    auto copy_layers = [](const lam_texture_layer* src, uint32_t n, std::vector<Tex>& dst) {
        dst.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            dst[i].w = src[i].width;
            dst[i].h = src[i].height;
            dst[i].rgba.assign(src[i].rgba8, src[i].rgba8 + 4 * (size_t)src[i].width * src[i].height);
        }
    };
    copy_layers(d->diffuse, d->diffuse_count, diffuse);
    copy_layers(d->emission, d->emission_count, emission);
    copy_layers(d->attributes, d->attribute_count, attributes);
    if (d->recolour) {
        std::vector<Tex> r;
        copy_layers(d->recolour, 1, r);
        recolour = r[0];
    } else {
        recolour.w = recolour.h = 1;
        recolour.rgba = {255, 255, 255, 255};
    }
    sky_size = d->sky_faces ? d->sky_size : 0;
    if (sky_size) sky.assign(d->sky_faces, d->sky_faces + 6 * 4 * (size_t)sky_size * sky_size);
    return LAM_OK;
}

// ---------------------------------------------------------------- textures
void Scene::sample(const std::vector<Tex>& arr, uint32_t layer, float u, float v, float out[4]) const {
    if (layer >= arr.size() || arr[layer].w == 0 || arr[layer].h == 0) {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
        return;
    }
    const Tex& t = arr[layer];
    int32_t x = f2i(std::floor(u * (float)t.w));
    int32_t y = f2i(std::floor(v * (float)t.h));
    x = std::min(std::max(x, 0), (int32_t)t.w - 1);
    y = std::min(std::max(y, 0), (int32_t)t.h - 1);
    const uint8_t* p = &t.rgba[4 * ((size_t)y * t.w + x)];
    for (int c = 0; c < 4; ++c) out[c] = (float)p[c] / 255.0f;
}

void Scene::load_recolour(uint32_t x, uint32_t y, float out[4]) const {
    x = std::min(x, recolour.w - 1);
    y = std::min(y, recolour.h - 1);
    const uint8_t* p = &recolour.rgba[4 * ((size_t)y * recolour.w + x)];
    for (int c = 0; c < 4; ++c) out[c] = (float)p[c] / 255.0f;
}

// Cube-map face selection and (s, t) of the Vulkan cube-map table; nearest texel.
vec3 Scene::background(vec3 d) const {
    if (!sky_size) return vec3(0.0f);
    float ax = absf(d.x), ay = absf(d.y), az = absf(d.z);
    int face;
    float sc, tc, ma;
    if (ax >= ay && ax >= az) {
        ma = ax;
        if (d.x >= 0.0f) { face = 0; sc = -d.z; tc = -d.y; } else { face = 1; sc = d.z; tc = -d.y; }
    } else if (ay >= az) {
        ma = ay;
        if (d.y >= 0.0f) { face = 2; sc = d.x; tc = d.z; } else { face = 3; sc = d.x; tc = -d.z; }
    } else {
        ma = az;
        if (d.z >= 0.0f) { face = 4; sc = d.x; tc = -d.y; } else { face = 5; sc = -d.x; tc = -d.y; }
    }
    if (!(ma > 0.0f)) return vec3(0.0f);
    float s = 0.5f * (sc / ma + 1.0f), t = 0.5f * (tc / ma + 1.0f);
    int32_t x = f2i(std::floor(s * (float)sky_size));
    int32_t y = f2i(std::floor(t * (float)sky_size));
    x = std::min(std::max(x, 0), (int32_t)sky_size - 1);
    y = std::min(std::max(y, 0), (int32_t)sky_size - 1);
    const uint8_t* p = &sky[4 * (((size_t)face * sky_size + y) * sky_size + x)];
    return vec3(p[0] / 255.0f, p[1] / 255.0f, p[2] / 255.0f);
}

static uint32_t clamp_index(uint32_t i, size_t n) { return n == 0 ? 0 : (uint32_t)std::min<size_t>(i, n - 1); }

bool Scene::alpha_accept(uint32_t ii, uint32_t prim, float bu, float bv) const {
    const Instance& in = inst[ii];
    if (in.mat.empty() || materials.empty()) return true;
    const lam_material& m = materials[clamp_index(in.mat[clamp_index(prim, in.mat.size())], materials.size())];
    float bz = (1.0f - bu) - bv;
    vec2 t1 = unpack2x16float(m.tex_pos_1), t2 = unpack2x16float(m.tex_pos_2), t3 = unpack2x16float(m.tex_pos_3);
    float u = std::fma(t1.x, bz, std::fma(t2.x, bu, t3.x * bv));
    float v = std::fma(t1.y, bz, std::fma(t2.y, bu, t3.y * bv));
    uint32_t idx_d, idx_e, idx_a, ty;
    unpack_2xu16(m.tex_idx_diffuse_emission, &idx_d, &idx_e);
    unpack_2xu16(m.tex_idx_attributes_ty, &idx_a, &ty);
    float px[4];
    sample(diffuse, idx_d, u, v, px);
    return !near_zero(px[3]) || ty == TRANSPARENT;
}

// ---------------------------------------------------------------- traversal
Hit Scene::trace(vec3 o, vec3 d, float tmin, float tmax, bool any_hit) const {
    Hit best;
    float best_t = tmax;
    vec3 best_oo, best_od;
    if (tlas.nodes.empty()) return best;
    double wo[3] = {o.x, o.y, o.z}, wd[3] = {d.x, d.y, d.z};
    int32_t tstack[128];
    int tsp = 0;
    tstack[tsp++] = 0;
    while (tsp) {
        const BNode& tn = tlas.nodes[tstack[--tsp]];
        if (!box_hit(tn, wo, wd, tmin, best_t)) continue;
        if (tn.count == 0) {
            tstack[tsp++] = tn.left;
            tstack[tsp++] = tn.right;
            continue;
        }
        for (int32_t k = tn.first; k < tn.first + tn.count; ++k) {
            uint32_t ii = tlas.items[k];
            const Instance& in = inst[ii];
            if ((in.mask & 0xFFu) == 0u) continue;
            const Blas& bl = blas[in.blas];
            if (bl.bvh.nodes.empty()) continue;
            vec3 oo, od;
            object_ray(in.inv, o, d, &oo, &od);
            WbwRay wr = wbw_setup(od);
            double bo[3] = {oo.x, oo.y, oo.z}, bd[3] = {od.x, od.y, od.z};
            int32_t stack[128];
            int sp = 0;
            stack[sp++] = 0;
            while (sp) {
                const BNode& n = bl.bvh.nodes[stack[--sp]];
                if (!box_hit(n, bo, bd, tmin, best_t)) continue;
                if (n.count == 0) {
                    stack[sp++] = n.left;
                    stack[sp++] = n.right;
                    continue;
                }
                for (int32_t j = n.first; j < n.first + n.count; ++j) {
                    uint32_t prim = bl.bvh.items[j];
                    const float* p0 = &bl.v[3 * bl.idx[3 * prim]];
                    const float* p1 = &bl.v[3 * bl.idx[3 * prim + 1]];
                    const float* p2 = &bl.v[3 * bl.idx[3 * prim + 2]];
                    vec3 v0(p0[0], p0[1], p0[2]), v1(p1[0], p1[1], p1[2]), v2(p2[0], p2[1], p2[2]);
                    float t;
                    if (!wbw_f32(wr, oo, v0, v1, v2, &t)) continue;
                    if (!(t > tmin)) continue;
                    bool better = t < best_t ||
                                  (t == best_t && best.hit && (ii < best.inst || (ii == best.inst && prim < best.prim)));
                    if (!better) continue;
                    if (!bl.opaque) {
                        float rt, ru, rv;
                        bool fr;
                        wbw_f64(oo, od, v0, v1, v2, &rt, &ru, &rv, &fr);
                        if (!alpha_accept(ii, prim, ru, rv)) continue;
                    }
                    best.hit = true;
                    best.inst = ii;
                    best.prim = prim;
                    best_t = t;
                    best_oo = oo;
                    best_od = od;
                    best.ov0 = v0; best.ov1 = v1; best.ov2 = v2;
                    if (any_hit) { tsp = 0; sp = 0; break; }
                }
            }
            if (any_hit && best.hit) break;
        }
    }
    if (best.hit) wbw_f64(best_oo, best_od, best.ov0, best.ov1, best.ov2, &best.t, &best.u, &best.v, &best.front);
    return best;
}

Hit Scene::trace_bruteforce(vec3 o, vec3 d, float tmin, float tmax) const {
    Hit best;
    float best_t = tmax;
    vec3 best_oo, best_od;
    for (uint32_t ii = 0; ii < inst.size(); ++ii) {
        const Instance& in = inst[ii];
        if ((in.mask & 0xFFu) == 0u) continue;
        const Blas& bl = blas[in.blas];
        vec3 oo, od;
        object_ray(in.inv, o, d, &oo, &od);
        WbwRay wr = wbw_setup(od);
        for (uint32_t prim = 0; prim < bl.tri_count; ++prim) {
            const float* p0 = &bl.v[3 * bl.idx[3 * prim]];
            const float* p1 = &bl.v[3 * bl.idx[3 * prim + 1]];
            const float* p2 = &bl.v[3 * bl.idx[3 * prim + 2]];
            vec3 v0(p0[0], p0[1], p0[2]), v1(p1[0], p1[1], p1[2]), v2(p2[0], p2[1], p2[2]);
            float t;
            if (!wbw_f32(wr, oo, v0, v1, v2, &t)) continue;
            if (!(t > tmin) || !(t < best_t)) continue;
            if (!bl.opaque) {
                float rt, ru, rv;
                bool fr;
                wbw_f64(oo, od, v0, v1, v2, &rt, &ru, &rv, &fr);
                if (!alpha_accept(ii, prim, ru, rv)) continue;
            }
            best.hit = true;
            best.inst = ii;
            best.prim = prim;
            best_t = t;
            best_oo = oo;
            best_od = od;
            best.ov0 = v0; best.ov1 = v1; best.ov2 = v2;
        }
    }
    if (best.hit) wbw_f64(best_oo, best_od, best.ov0, best.ov1, best.ov2, &best.t, &best.u, &best.v, &best.front);
    return best;
}

}  // namespace oracle
