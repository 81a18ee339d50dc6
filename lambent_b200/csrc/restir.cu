// restir.cu - DataBuffers and the passes that follow rt_main:
//   temporal resampling   src/importance_sampling/temporal_resampling.wesl:37-65
//   spatial resampling    src/importance_sampling/spatial_resampling.wesl:35-194
//   end of frame          src/data_buffer/end_of_frame.wesl:14-99, TemporalBuffers::advance_frame
//                         (src/data_buffer/mod.rs:65-96, 272-349)
//   frame average         examples/cornell_box/src/average_to_buf.wgsl:11-21
// All are one thread per element; they are HBM-streaming kernels.
#include <algorithm>
#include <cstring>
#include <vector>

#include "device_math.cuh"
#include "guide.cuh"
#include "scene.h"
#include "tracer.h"

namespace lam {

constexpr int PASS_BLOCK = 256;

struct Samp {
    v3 vp;
    uint32_t vn;
    v3 sp;
    uint32_t sn;
    v3 orad;
    uint32_t ty;
    float rough;
};

LAM_DEV Samp sam_from(const lam_reservoir& r) {
    Samp s;
    s.vp = mk(r.visible_point[0], r.visible_point[1], r.visible_point[2]);
    s.vn = r.visible_normal;
    s.sp = mk(r.sample_point[0], r.sample_point[1], r.sample_point[2]);
    s.sn = r.sample_normal;
    s.orad = mk(r.out_radiance[0], r.out_radiance[1], r.out_radiance[2]);
    s.ty = r.ty;
    s.rough = r.roughness;
    return s;
}
LAM_DEV float p_hat(const Samp& s) { return fmaxf(len(s.orad), 0.00001f); }
LAM_DEV void assign(lam_reservoir& r, const Samp& s) {
    r.visible_point[0] = s.vp.x; r.visible_point[1] = s.vp.y; r.visible_point[2] = s.vp.z;
    r.visible_normal = s.vn;
    r.sample_point[0] = s.sp.x; r.sample_point[1] = s.sp.y; r.sample_point[2] = s.sp.z;
    r.sample_normal = s.sn;
    r.out_radiance[0] = s.orad.x; r.out_radiance[1] = s.orad.y; r.out_radiance[2] = s.orad.z;
    r.ty = s.ty;
    r.roughness = s.rough;
    r.packed_confidence_valid |= 0x80000000u;
}
// merge, shared.wesl:99-115
LAM_DEV bool merge(lam_reservoir& res, const lam_reservoir& r, float p, uint32_t seed) {
    uint32_t c = res.packed_confidence_valid & 0x7FFFFFFFu;
    uint32_t oc = r.packed_confidence_valid & 0x7FFFFFFFu;
    float w_new = p * r.W * __uint2float_rn(oc);
    res.packed_confidence_valid = ((c + oc) & 0x7FFFFFFFu) | (res.packed_confidence_valid & 0x80000000u);
    res.w = res.w + w_new;
    if (rand_f32(seed) * res.w < w_new) {
        assign(res, sam_from(r));
        return true;
    }
    return false;
}

__global__ void temporal_kernel(lam_reservoir* cur, const lam_reservoir* old, uint32_t width, uint32_t height,
                                uint32_t seed_offset) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= width * height) return;
    const uint32_t x = idx % width, y = idx / width;
    uint32_t own_seed = rand_u32(x * y) + rand_u32(seed_offset + y);
    lam_reservoir Rs = cur[idx];
    lam_reservoir R = old ? old[idx] : lam_reservoir{};
    if (dot(u32_to_normalised(R.sample_normal), u32_to_normalised(Rs.sample_normal)) < 0.95f) R = lam_reservoir{};
    if (Rs.ty == TY_SKY) return;
    float w = p_hat(sam_from(R));
    merge(Rs, R, w, own_seed);
    R = Rs;
    uint32_t c = R.packed_confidence_valid & 0x7FFFFFFFu;
    R.W = safe_div(R.w, __uint2float_rn(c) * p_hat(sam_from(R)));
    cur[idx] = R;
}

LAM_DEV float jacobian(const Samp& q, const Samp& r) {
    v3 q12 = q.sp - q.vp, r12 = r.sp - q.vp;
    v3 vn = u32_to_normalised(q.vn);
    float cr = dot(normalize(r12), vn), cq = dot(normalize(q12), vn);
    return safe_div(cr * len_sqrd(q12), cq * len_sqrd(r12));
}

// Neighbour confidences are summed on the fly (the reference keeps them in a private Q[129]).
__global__ void spatial_kernel(const lam_reservoir* __restrict__ cur, const lam_info* __restrict__ info, uint32_t width,
                               uint32_t height, uint32_t is_samples, uint32_t is_space, uint32_t seed_offset,
                               float4* __restrict__ out) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= width * height) return;
    const uint32_t x = idx % width, y = idx / width;
    uint32_t own_seed = rand_u32(x * y) + rand_u32(seed_offset) + y;
    lam_reservoir Rs = cur[idx];
    if (Rs.ty == TY_SKY) return;
    v3 Rs_normal = u32_to_normalised(Rs.sample_normal);
    uint32_t Z = (p_hat(sam_from(Rs)) > 0.0f) ? (Rs.packed_confidence_valid & 0x7FFFFFFFu) : 0u;
    const uint32_t max_val = is_space * is_space - 1u;
    const uint32_t min_space = is_space / 2u;
    const uint32_t self_idx = min_space + min_space * is_space;
    for (uint32_t i = 0; i < is_samples; ++i) {
        uint32_t rnd = rand_u32(own_seed) % max_val;
        if (rnd >= self_idx) rnd += 1u;
        int32_t nbx = (int32_t)(rnd % is_space) - (int32_t)min_space, nby = (int32_t)(rnd / is_space) - (int32_t)min_space;
        own_seed = rand_u32(own_seed);
        int32_t ox = (int32_t)x + nbx, oy = (int32_t)y + nby;
        if (ox < 0 || oy < 0 || (nbx == 0 && nby == 0)) continue;
        if ((uint32_t)ox >= width || (uint32_t)oy >= height) continue;
        const lam_reservoir Rn = cur[(uint32_t)ox + (uint32_t)oy * width];
        v3 Rn_normal = u32_to_normalised(Rn.sample_normal);
        if (dot(Rn_normal, Rs_normal) < 0.9f || Rn.ty != Rs.ty || fabsf(Rs.roughness - Rn.roughness) > 0.1f) continue;
        float jac = jacobian(sam_from(Rn), sam_from(Rs));
        if (Rs.ty != TY_DIFFUSE) continue;
        float pq = p_hat(sam_from(Rn)) * jac;
        bool picked = merge(Rs, Rn, pq, own_seed);
        own_seed = rand_u32(own_seed);
        if (picked) Rs_normal = u32_to_normalised(Rs.sample_normal);
        if (p_hat(sam_from(Rn)) > 0.0f) Z += Rn.packed_confidence_valid & 0x7FFFFFFFu;
        own_seed = rand_u32(own_seed);
    }
    float zp = __uint2float_rn(Z) * p_hat(sam_from(Rs));
    Rs.W = safe_div(Rs.w, zp);
    const float* a = info[idx].arr;
    v3 pix = fma3(mk(Rs.out_radiance[0], Rs.out_radiance[1], Rs.out_radiance[2]) * Rs.W, mk(a[6], a[7], a[8]),
                  mk(a[3], a[4], a[5]));
    out[idx] = make_float4(pix.x, pix.y, pix.z, 1.0f);
}

__global__ void eof_gi_kernel(lam_reservoir* r, uint64_t n, uint32_t cap) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t p = r[i].packed_confidence_valid;
    uint32_t c = p & 0x7FFFFFFFu;
    if (c > cap) {
        r[i].w *= __uint2float_rn(cap) / __uint2float_rn(c);
        r[i].packed_confidence_valid = (cap & 0x7FFFFFFFu) | (p & 0x80000000u);
    }
}

__global__ void eof_world_kernel(uint32_t* world, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t* e = world + i * W_STRIDE;
    if (e[W_TIMEOUT] == 0u) {
        e[W_SEC] = 0u;
        e[W_NUM] = 0u;
        e[W_LUM] = 0u;
        e[W_LUM + 1] = 0u;
        e[W_LUM + 2] = 0u;
        e[W_LOCK] = 0u;
        return;
    }
    uint32_t old_num = e[W_NUM];
    if (old_num != 0u) {
        uint32_t prod = old_num * 8u;
        uint32_t nn = prod / 9u + (prod % 9u != 0u ? 1u : 0u);
        float mul = __uint2float_rn(nn) / __uint2float_rn(old_num);
        for (int k = 0; k < 3; ++k) e[W_LUM + k] = __float_as_uint(__uint_as_float(e[W_LUM + k]) * mul);
        e[W_NUM] = nn;
    }
    e[W_TIMEOUT] = e[W_TIMEOUT] - 1u;
}

struct FramePtrs {
    const float4* f[64];
};

__global__ void average_kernel(FramePtrs fp, uint32_t n, uint32_t first, uint32_t count, uint64_t pixels, float* out,
                               uint32_t total) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    float4 a = first == 0u ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                           : make_float4(out[3 * i], out[3 * i + 1], out[3 * i + 2], 0.0f);
    const float nf = __uint2float_rn(total);
    for (uint32_t k = 0; k < count; ++k) {
        float4 v = fp.f[k][i];
        a.x = a.x + v.x / nf;
        a.y = a.y + v.y / nf;
        a.z = a.z + v.z / nf;
    }
    out[3 * i] = a.x;
    out[3 * i + 1] = a.y;
    out[3 * i + 2] = a.z;
    (void)n;
}

static int dalloc(void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (data buffers)");
    e = cudaMemset(*p, 0, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemset (data buffers)");
    return LAM_OK;
}

static void free_window(lam_data_buffers* b) {
    void* ps[] = {b->reservoirs, b->old_reservoirs, b->info, b->chains, b->old_chains, b->pixel_seed};
    for (void* p : ps) cudaFree(p);
    b->reservoirs = b->old_reservoirs = b->info = b->chains = b->old_chains = b->pixel_seed = nullptr;
}

static int alloc_window(lam_data_buffers* b, uint32_t w, uint32_t h) {
    const size_t pix = (size_t)w * h;
    b->width = w;
    b->height = h;
    b->pixels = pix;
    // reservoirs are always per pixel: rt_main writes gi_reservoirs[idx] in every ReSTIR mode
    b->reservoir_len = pix;
    b->chain_len = (b->types & LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE) ? pix : 1;
    int rc = 0;
    rc |= dalloc(&b->reservoirs, b->reservoir_len * sizeof(lam_reservoir));
    rc |= dalloc(&b->old_reservoirs, b->reservoir_len * sizeof(lam_reservoir));
    rc |= dalloc(&b->info, pix * sizeof(lam_info));
    rc |= dalloc(&b->chains, b->chain_len * sizeof(lam_markov_chain));
    rc |= dalloc(&b->old_chains, b->chain_len * sizeof(lam_markov_chain));
    rc |= dalloc(&b->pixel_seed, pix * sizeof(uint32_t));
    return rc ? LAM_ERR_CUDA : LAM_OK;
}

}  // namespace lam

using namespace lam;

extern "C" int lam_data_buffers_new(uint32_t width, uint32_t height, uint32_t world_size, uint32_t types,
                                    lam_data_buffers** out) {
    if (!out) return set_error(LAM_ERR_INVALID_ARGUMENT, "null output");
    if (types & ~LAM_BUFFER_ALL) return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown buffer type bits");
    lam_data_buffers* b = new lam_data_buffers();
    b->types = types;
    width = std::max(1u, width);
    height = std::max(1u, height);
    b->world_size = std::max(1u, world_size);
    b->world_len = (types & LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE) ? b->world_size : 1;
    int rc = alloc_window(b, width, height);
    if (!rc) rc |= dalloc(&b->world, b->world_len * sizeof(lam_world_markov_chain));
    if (!rc) rc |= dalloc(&b->old_world, b->world_len * sizeof(lam_world_markov_chain));
    if (rc) {
        free_window(b);
        cudaFree(b->world);
        cudaFree(b->old_world);
        delete b;
        return rc;
    }
    *out = b;
    return LAM_OK;
}

extern "C" int lam_data_buffers_resize(lam_data_buffers* b, uint32_t width, uint32_t height) {
    if (!b) return set_error(LAM_ERR_INVALID_ARGUMENT, "null buffers");
    width = std::max(1u, width);
    height = std::max(1u, height);
    cudaDeviceSynchronize();
    free_window(b);
    return alloc_window(b, width, height);
}

extern "C" int lam_data_buffers_advance_frame(lam_data_buffers* b, uint32_t adv, uint32_t cap, void* stream) {
    if (!b) return set_error(LAM_ERR_INVALID_ARGUMENT, "null buffers");
    if (cap == 0 || cap > 0xFFFF) return set_error(LAM_ERR_INVALID_ARGUMENT, "confidence_cap must be a NonZeroU16");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t res_bytes = b->reservoir_len * sizeof(lam_reservoir);
    const size_t chain_bytes = b->chain_len * sizeof(lam_markov_chain);
    const size_t world_bytes = b->world_len * sizeof(lam_world_markov_chain);
    if (adv & LAM_BUFFER_SPATIAL_RESAMPLING) {
        uint64_t n = b->reservoir_len;
        eof_gi_kernel<<<(unsigned)((n + PASS_BLOCK - 1) / PASS_BLOCK), PASS_BLOCK, 0, st>>>((lam_reservoir*)b->reservoirs, n, cap);
        cudaMemcpyAsync(b->old_reservoirs, b->reservoirs, res_bytes, cudaMemcpyDeviceToDevice, st);
        cudaMemsetAsync(b->reservoirs, 0, res_bytes, st);
    } else {
        cudaMemsetAsync(b->reservoirs, 0, res_bytes, st);
        cudaMemsetAsync(b->old_reservoirs, 0, res_bytes, st);
    }
    if (adv & LAM_BUFFER_MARKOV_CHAIN_SCREEN_SPACE) {
        cudaMemcpyAsync(b->old_chains, b->chains, chain_bytes, cudaMemcpyDeviceToDevice, st);
        cudaMemsetAsync(b->chains, 0, chain_bytes, st);
    } else {
        cudaMemsetAsync(b->chains, 0, chain_bytes, st);
        cudaMemsetAsync(b->old_chains, 0, chain_bytes, st);
    }
    if (adv & LAM_BUFFER_MARKOV_CHAIN_WORLD_SPACE) {
        uint64_t n = b->world_len;
        eof_world_kernel<<<(unsigned)((n + PASS_BLOCK - 1) / PASS_BLOCK), PASS_BLOCK, 0, st>>>((uint32_t*)b->world, n);
        cudaMemcpyAsync(b->old_world, b->world, world_bytes, cudaMemcpyDeviceToDevice, st);
    } else {
        cudaMemsetAsync(b->world, 0, world_bytes, st);
        cudaMemsetAsync(b->old_world, 0, world_bytes, st);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LAM_OK : cuda_error(e, "lam_data_buffers_advance_frame");
}

extern "C" int lam_data_buffers_get(const lam_data_buffers* b, uint32_t which, void** ptr, size_t* bytes) {
    if (!b || !ptr || !bytes) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    switch (which) {
        case 0: *ptr = b->reservoirs; *bytes = b->reservoir_len * sizeof(lam_reservoir); break;
        case 1: *ptr = b->old_reservoirs; *bytes = b->reservoir_len * sizeof(lam_reservoir); break;
        case 2: *ptr = b->info; *bytes = b->pixels * sizeof(lam_info); break;
        case 3: *ptr = b->chains; *bytes = b->chain_len * sizeof(lam_markov_chain); break;
        case 4: *ptr = b->old_chains; *bytes = b->chain_len * sizeof(lam_markov_chain); break;
        case 5: *ptr = b->world; *bytes = b->world_len * sizeof(lam_world_markov_chain); break;
        case 6: *ptr = b->old_world; *bytes = b->world_len * sizeof(lam_world_markov_chain); break;
        case 7: *ptr = b->pixel_seed; *bytes = b->pixels * sizeof(uint32_t); break;
        default: return set_error(LAM_ERR_INVALID_ARGUMENT, "unknown buffer index");
    }
    return LAM_OK;
}

extern "C" int lam_data_buffers_destroy(lam_data_buffers* b) {
    if (!b) return LAM_OK;
    free_window(b);
    cudaFree(b->world);
    cudaFree(b->old_world);
    delete b;
    return LAM_OK;
}

extern "C" int lam_temporal_resampling(lam_data_buffers* b, uint32_t width, uint32_t height, uint32_t seed_offset,
                                       void* stream) {
    if (!b) return set_error(LAM_ERR_INVALID_ARGUMENT, "null buffers");
    if (width != b->width || height != b->height) return set_error(LAM_ERR_INVALID_ARGUMENT, "size differs from the buffers");
    uint32_t n = width * height;
    temporal_kernel<<<(n + PASS_BLOCK - 1) / PASS_BLOCK, PASS_BLOCK, 0, (cudaStream_t)stream>>>(
        (lam_reservoir*)b->reservoirs, (const lam_reservoir*)b->old_reservoirs, width, height, seed_offset);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LAM_OK : cuda_error(e, "lam_temporal_resampling");
}

extern "C" int lam_spatial_resampling(lam_data_buffers* b, const lam_frame_targets* tg, uint32_t is_samples,
                                      uint32_t is_space, uint32_t seed_offset, void* stream) {
    if (!b || !tg || !tg->color) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    if (tg->width != b->width || tg->height != b->height) return set_error(LAM_ERR_INVALID_ARGUMENT, "size differs from the buffers");
    if (is_samples > 128) return set_error(LAM_ERR_INVALID_ARGUMENT, "IS_SAMPLES must be <= 128 (Q[129] in the reference)");
    if (is_space < 2) return set_error(LAM_ERR_INVALID_ARGUMENT, "IS_SPACE must be >= 2");
    uint32_t n = b->width * b->height;
    spatial_kernel<<<(n + PASS_BLOCK - 1) / PASS_BLOCK, PASS_BLOCK, 0, (cudaStream_t)stream>>>(
        (const lam_reservoir*)b->reservoirs, (const lam_info*)b->info, b->width, b->height, is_samples, is_space,
        seed_offset, (float4*)tg->color);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LAM_OK : cuda_error(e, "lam_spatial_resampling");
}

extern "C" int lam_average_frames(const float* const* frames, uint32_t n, uint32_t width, uint32_t height, float* out,
                                  void* stream) {
    if (!frames || !out || n == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_average_frames: bad argument");
    uint64_t pixels = (uint64_t)width * height;
    if (!pixels) return LAM_OK;
    // frames are summed in order in chunks of 64 pointers
    for (uint32_t first = 0; first < n; first += 64) {
        FramePtrs fp;
        uint32_t cnt = std::min(64u, n - first);
        for (uint32_t k = 0; k < cnt; ++k) {
            if (!frames[first + k]) return set_error(LAM_ERR_INVALID_ARGUMENT, "null frame pointer");
            fp.f[k] = (const float4*)frames[first + k];
        }
        average_kernel<<<(unsigned)((pixels + PASS_BLOCK - 1) / PASS_BLOCK), PASS_BLOCK, 0, (cudaStream_t)stream>>>(
            fp, n, first, cnt, pixels, out, n);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LAM_OK : cuda_error(e, "lam_average_frames");
}
