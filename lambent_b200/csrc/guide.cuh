// guide.cuh - the reference's vMF Markov-chain guiding on the device
// (src/path_tracing/general.wesl:147-500 and 984-1047).
//
// World grid: WorldMarcovChainState records (56 bytes, src/bindings.wesl:33-40) as 14 u32 words,
// updated with the same protocol as the shader: CAS-claim of the secondary hash, try-lock for
// the radiance sum (a locked cell is skipped, never waited on), relaxed stores of the chain.
#pragma once
#include "../../include/lambent.h"
#include "device_math.cuh"

namespace lam {

struct MC {
    v3 light;
    float mean_cosine, weight_sum;
    uint32_t num_samples;
    float score;
};

LAM_DEV MC mc_zero() {
    MC s;
    s.light = splat(0.0f);
    s.mean_cosine = 0.0f;
    s.weight_sum = 0.0f;
    s.num_samples = 0u;
    s.score = 0.0f;
    return s;
}

LAM_DEV MC mc_from(const lam_markov_chain& c) {
    MC s;
    s.light = mk(c.light_source[0], c.light_source[1], c.light_source[2]);
    s.mean_cosine = c.mean_cosine;
    s.weight_sum = c.weight_sum;
    s.num_samples = c.num_samples;
    s.score = c.score;
    return s;
}

LAM_DEV MC mc_load(const lam_markov_chain* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    float4 a = q[0], b = q[1];
    MC s;
    s.light = mk(a.x, a.y, a.z);
    s.mean_cosine = a.w;
    s.weight_sum = b.x;
    s.num_samples = __float_as_uint(b.y);
    s.score = b.z;
    return s;
}

LAM_DEV void mc_store(lam_markov_chain* p, const MC& s) {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(s.light.x, s.light.y, s.light.z, s.mean_cosine);
    q[1] = make_float4(s.weight_sum, __uint_as_float(s.num_samples), s.score, 0.0f);
}

constexpr int W_SEC = 0, W_NUM = 1, W_LUM = 2, W_LOCK = 5, W_CL = 6, W_CMEAN = 9, W_CWS = 10, W_CNUM = 11,
              W_CSCORE = 12, W_TIMEOUT = 13, W_STRIDE = 14;
constexpr uint32_t CACHE_TIMEOUT = 30u;
constexpr uint32_t MAX_NUM_SAMPLES = 0x0FFFFFFFu;
constexpr int NUM_RESAMPLES = 21;

LAM_DEV uint32_t vload(const uint32_t* p) { return *(const volatile uint32_t*)p; }
LAM_DEV void vstore(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }

struct Grid {
    uint32_t* world;
    const uint32_t* old_world;
    uint64_t len;      // cells (< 2^32: the buffer size is a u32)
    uint64_t mod_m;    // ~0 / len + 1 (computed on the host)
    v3 camera_loc;
};

// hash % len without a 64-bit division: Lemire's fast remainder for 32-bit operands (Lemire, Kaser
// and Kurz, "Faster remainder by direct computation", 2019) with m = floor((2^64 - 1) / len) + 1;
// exact for every 32-bit hash and 0 < len < 2^32 (len = 1 gives m = 0 and the remainder 0).
LAM_DEV uint64_t grid_index(const Grid& g, uint32_t hash) {
    return __umul64hi(g.mod_m * (uint64_t)hash, g.len);
}

struct IVec { int32_t x, y, z; };

LAM_DEV IVec grid_loc(const Grid& g, v3 pos) {
    v3 diff = pos - g.camera_loc;
    float len = fmaxf(fabsf(diff.x), fmaxf(fabsf(diff.y), fabsf(diff.z)));
    uint32_t shifts = f2u(log2f(fmaxf(len / 1.0f, 1.0f)));
    uint32_t mask = 0xFFFFFFFFu << min(shifts, 30u);
    IVec r{f2i(pos.x / 0.1f), f2i(pos.y / 0.1f), f2i(pos.z / 0.1f)};
    r.x &= (int32_t)mask;
    r.y &= (int32_t)mask;
    r.z &= (int32_t)mask;
    return r;
}

LAM_DEV uint32_t primary_hash(IVec l, v3 normal, v3 incoming) {
    uint32_t n = normalised_to_u32(normal) & 0xFF00FF00u;
    uint32_t ih = (uint32_t)(incoming.x > 0.0f) | ((uint32_t)(incoming.y > 0.0f) << 1) | ((uint32_t)(incoming.z > 0.0f) << 2);
    uint32_t inc = rand_u32(ih);
    return ((((uint32_t)l.x * 1u) ^ ((uint32_t)l.y * 687603047u)) ^ ((uint32_t)l.z * 571899763u)) ^ (n * 894271171u) ^
           (inc * 840057787u);
}

LAM_DEV uint32_t secondary_hash(IVec l, v3 normal) {
    uint32_t n = normalised_to_u32(normal) & 0xFF00FF00u;
    uint32_t h = (((uint32_t)l.x * 1699644091u) ^ ((uint32_t)l.y * 550105817u)) ^ ((uint32_t)l.z * 956114303u);
    return (rand_u32(h) ^ (n * 155096983u)) | 1u;
}

// Two adjacent words in one volatile access.  Grid cells are 56 bytes in cudaMalloc'd buffers and
// every pair starts at an even word, so the access is 8-byte aligned.  Reading two fields at once is
// one of the interleavings the reference's separate relaxed atomic loads allow.
LAM_DEV uint2 vload2(const uint32_t* p) {
    uint2 v;
    asm volatile("ld.volatile.global.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}

LAM_DEV void vstore2(uint32_t* p, uint32_t a, uint32_t b) {
    asm volatile("st.volatile.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"(a), "r"(b) : "memory");
}

LAM_DEV MC read_chain(const uint32_t* e) {
    MC s;
    const uint2 a = vload2(e + W_CL), b = vload2(e + W_CL + 2), c = vload2(e + W_CWS);
    s.light = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(b.x));
    s.mean_cosine = __uint_as_float(b.y);
    s.weight_sum = __uint_as_float(c.x);
    s.num_samples = c.y;
    s.score = __uint_as_float(vload(e + W_CSCORE));
    return s;
}

// A cell's score and timeout words (the timeout is only ever set to CACHE_TIMEOUT while shading;
// the end-of-frame pass lowers it).
LAM_DEV MC read_chain_timeout(const uint32_t* e, uint32_t* timeout) {
    MC s;
    const uint2 a = vload2(e + W_CL), b = vload2(e + W_CL + 2), c = vload2(e + W_CWS), d = vload2(e + W_CSCORE);
    s.light = mk(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(b.x));
    s.mean_cosine = __uint_as_float(b.y);
    s.weight_sum = __uint_as_float(c.x);
    s.num_samples = c.y;
    s.score = __uint_as_float(d.x);
    *timeout = d.y;
    return s;
}

LAM_DEV MC grid_load(const Grid& g, v3 pos, v3 normal, v3 incoming, bool force_old) {
    IVec l = grid_loc(g, pos);
    uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    uint32_t* e = g.world + idx * W_STRIDE;
    uint32_t sec = secondary_hash(l, normal);
    uint32_t timeout = 0u;
    MC s = read_chain_timeout(e, &timeout);
    if (vload(e + W_SEC) != sec || force_old) {
        const uint32_t* o = g.old_world ? g.old_world + idx * W_STRIDE : nullptr;
        if (o && vload(o + W_SEC) == sec) s = read_chain(o);
        else s = mc_zero();
    } else if (timeout != CACHE_TIMEOUT) {
        vstore(e + W_TIMEOUT, CACHE_TIMEOUT);  // writing the value the word already holds is skipped
    }
    s.light = strip_nan3(s.light);
    s.mean_cosine = strip_nan(s.mean_cosine);
    s.weight_sum = strip_nan(s.weight_sum);
    s.score = strip_nan(s.score);
    return s;
}

// grid_load of N cells (the world-space candidates of one bounce, general.wesl:389-398): every
// cell's words are read before any of them is examined, so the N reads are in flight together
// instead of one after another.  A cell's own words are read in grid_load's order.  When two
// candidates hash to one cell, the second read no longer sees the first one's timeout refresh;
// that refresh writes the value the word then holds, and the chain fields it returns are the same.
// Measured on the ReSTIR GI frame loop at 1080p: 19.45 / 19.86 against 20.03 / 20.22 ms per frame.
template <int N>
LAM_DEV void grid_load_n(const Grid& g, const v3* pos, v3 normal, v3 incoming, const bool* force_old, MC* out) {
    uint32_t* e[N];
    uint64_t idx[N];
    uint32_t sec[N], tmo[N], tag[N];
#pragma unroll
    for (int q = 0; q < N; ++q) {
        IVec l = grid_loc(g, pos[q]);
        idx[q] = grid_index(g, primary_hash(l, normal, incoming));
        e[q] = g.world + idx[q] * W_STRIDE;
        sec[q] = secondary_hash(l, normal);
    }
#pragma unroll
    for (int q = 0; q < N; ++q) {
        out[q] = read_chain_timeout(e[q], &tmo[q]);
        tag[q] = vload(e[q] + W_SEC);
    }
#pragma unroll
    for (int q = 0; q < N; ++q) {
        MC s = out[q];
        if (tag[q] != sec[q] || force_old[q]) {
            const uint32_t* o = g.old_world ? g.old_world + idx[q] * W_STRIDE : nullptr;
            if (o && vload(o + W_SEC) == sec[q]) s = read_chain(o);
            else s = mc_zero();
        } else if (tmo[q] != CACHE_TIMEOUT) {
            vstore(e[q] + W_TIMEOUT, CACHE_TIMEOUT);
        }
        s.light = strip_nan3(s.light);
        s.mean_cosine = strip_nan(s.mean_cosine);
        s.weight_sum = strip_nan(s.weight_sum);
        s.score = strip_nan(s.score);
        out[q] = s;
    }
}

LAM_DEV void grid_store(const Grid& g, v3 pos, v3 normal, v3 incoming, const MC& st) {
    IVec l = grid_loc(g, pos);
    uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    uint32_t* e = g.world + idx * W_STRIDE;
    uint32_t sec = secondary_hash(l, normal);
    if (vload(e + W_SEC) != sec) {
        if (atomicCAS(e + W_SEC, 0u, sec) != 0u) return;
    }
    vstore2(e + W_CL, __float_as_uint(st.light.x), __float_as_uint(st.light.y));
    vstore2(e + W_CL + 2, __float_as_uint(st.light.z), __float_as_uint(st.mean_cosine));
    vstore2(e + W_CWS, __float_as_uint(st.weight_sum), st.num_samples);
    vstore2(e + W_CSCORE, __float_as_uint(st.score), CACHE_TIMEOUT);
}

LAM_DEV v3 grid_radiance(const Grid& g, v3 pos, v3 normal, v3 incoming) {
    IVec l = grid_loc(g, pos);
    uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    uint32_t* e = g.world + idx * W_STRIDE;
    const uint2 sn = vload2(e + W_SEC), l01 = vload2(e + W_LUM);  // (tag, count), (radiance x, y)
    uint32_t num = sn.y;
    v3 rad = mk(__uint_as_float(l01.x), __uint_as_float(l01.y), __uint_as_float(vload(e + W_LUM + 2)));
    uint32_t sec = secondary_hash(l, normal);
    if (sn.x != sec) {
        const uint32_t* o = g.old_world ? g.old_world + idx * W_STRIDE : nullptr;
        if (o && vload(o + W_SEC) == sec) {
            num = vload(o + W_NUM);
            rad = mk(__uint_as_float(vload(o + W_LUM)), __uint_as_float(vload(o + W_LUM + 1)), __uint_as_float(vload(o + W_LUM + 2)));
        } else {
            return splat(0.0f);
        }
    } else if (vload(e + W_TIMEOUT) != CACHE_TIMEOUT) {
        vstore(e + W_TIMEOUT, CACHE_TIMEOUT);
    }
    if (num == 0u) return splat(0.0f);
    return clamp3(rad / __uint2float_rn(num), 0.0f, 1000.0f);
}

LAM_DEV void grid_add_radiance(const Grid& g, v3 pos, v3 normal, v3 incoming, v3 radiance) {
    IVec l = grid_loc(g, pos);
    uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    uint32_t* e = g.world + idx * W_STRIDE;
    uint32_t sec = secondary_hash(l, normal);
    v3 c = clamp3(radiance, 0.0f, 100.0f);
    if (vload(e + W_SEC) != sec) {
        if (atomicCAS(e + W_SEC, 0u, sec) != 0u) return;
    }
    // try-lock: a locked cell is skipped (the shader must make forward progress)
    if (atomicExch(e + W_LOCK, 1u) == 1u) return;
    __threadfence();
    uint32_t num = vload(e + W_NUM);
    if (num >= MAX_NUM_SAMPLES) {
        __threadfence();
        atomicExch(e + W_LOCK, 0u);
        vstore(e + W_TIMEOUT, CACHE_TIMEOUT);
        return;
    }
    atomicAdd(e + W_NUM, 1u);
    float cc[3] = {c.x, c.y, c.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float r = strip_nan(cc[k] + __uint_as_float(vload(e + W_LUM + k)));
        vstore(e + W_LUM + k, __float_as_uint(fmaxf(r, 0.0f)));
    }
    __threadfence();
    atomicExch(e + W_LOCK, 0u);
    vstore(e + W_TIMEOUT, CACHE_TIMEOUT);
}

// Warp-aggregated forms of grid_add_radiance and grid_store, for lanes of a warp that call them
// together.  Lanes whose updates address the same cell (primary index and secondary tag) act as
// one group.  For radiance, the group claims the cell and takes its try-lock once, and the leader
// applies every member's sample in lane order; for a chain store, the group's last lane writes.
// Either is the state that the members' own updates leave when they run one after another without
// contention, an outcome the reference's relaxed atomics allow (general.wesl:228-311).  Adjacent
// pixels, which share cells at the first bounces, then no longer queue on one lock and one line.
LAM_DEV void grid_add_radiance_warp(const Grid& g, v3 pos, v3 normal, v3 incoming, v3 radiance) {
    const IVec l = grid_loc(g, pos);
    const uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    const uint32_t sec = secondary_hash(l, normal);
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned grp = __match_any_sync(__activemask(), (idx << 32) | sec);
    const uint32_t leader = __ffs(grp) - 1u;
    uint32_t* e = g.world + idx * W_STRIDE;
    const v3 c = clamp3(radiance, 0.0f, 100.0f);
    int ok = 0;
    float lum[3] = {0.0f, 0.0f, 0.0f};
    uint32_t num = 0u;
    if (lane == leader) {
        ok = 1;
        if (vload(e + W_SEC) != sec && atomicCAS(e + W_SEC, 0u, sec) != 0u) ok = 0;
        // try-lock: a locked cell is skipped (the shader must make forward progress)
        if (ok && atomicExch(e + W_LOCK, 1u) == 1u) ok = 0;
        if (ok) {
            __threadfence();
            num = vload(e + W_NUM);
            const uint2 l01 = vload2(e + W_LUM);
            lum[0] = __uint_as_float(l01.x);
            lum[1] = __uint_as_float(l01.y);
            lum[2] = __uint_as_float(vload(e + W_LUM + 2));
        }
    }
    if (!__shfl_sync(grp, ok, leader)) return;
    uint32_t added = 0u;
    for (unsigned m = grp; m; m &= m - 1u) {
        const uint32_t src = __ffs(m) - 1u;
        const float cx = __shfl_sync(grp, c.x, src), cy = __shfl_sync(grp, c.y, src), cz = __shfl_sync(grp, c.z, src);
        if (lane == leader && num + added < MAX_NUM_SAMPLES) {
            ++added;
            lum[0] = fmaxf(strip_nan(cx + lum[0]), 0.0f);
            lum[1] = fmaxf(strip_nan(cy + lum[1]), 0.0f);
            lum[2] = fmaxf(strip_nan(cz + lum[2]), 0.0f);
        }
    }
    if (lane == leader) {
        if (added) {
            atomicAdd(e + W_NUM, added);
            vstore2(e + W_LUM, __float_as_uint(lum[0]), __float_as_uint(lum[1]));
            vstore(e + W_LUM + 2, __float_as_uint(lum[2]));
        }
        __threadfence();
        atomicExch(e + W_LOCK, 0u);
        vstore(e + W_TIMEOUT, CACHE_TIMEOUT);
    }
}

LAM_DEV void grid_store_warp(const Grid& g, v3 pos, v3 normal, v3 incoming, const MC& st) {
    const IVec l = grid_loc(g, pos);
    const uint64_t idx = grid_index(g, primary_hash(l, normal, incoming));
    const uint32_t sec = secondary_hash(l, normal);
    const unsigned grp = __match_any_sync(__activemask(), (idx << 32) | sec);
    if ((threadIdx.x & 31u) == 31u - __clz(grp)) grid_store(g, pos, normal, incoming, st);
}

LAM_DEV v3 light_dir(const MC& s, v3 cur) { return safe_div3(s.light, s.weight_sum) - cur; }

LAM_DEV float get_kappa(const MC& s) {
    const float Np = 0.2f, rp = 0.99f;
    float N2 = __uint2float_rn(s.num_samples * s.num_samples);
    float r = ((N2 * (s.mean_cosine / s.weight_sum)) + (Np * rp)) / (N2 + Np);
    return clampf(((3.0f * r) - ((r * r) * r)) / (1.0f - (r * r)), 0.001f, 8.50705867e37f);
}

LAM_DEV float exp_minus_one(float x) {
    float u = expf(x);
    if (u == 1.0f) return x;
    float y = u - 1.0f;
    if (fabsf(x) < 1.0f) return (x * y) / logf(u);
    return y;
}

// vmf_pdf with the fast hardware exponential, logarithm and division.  Their error bounds (CUDA:
// __expf 2 + 1.17|x| ulp, __logf 2^-21.41 absolute in [0.5, 2] and 3 ulp outside, __fdividef 2 ulp)
// lie within WGSL's accuracy requirements for exp (3 + 2|x| ulp), log (2^-21 absolute in [0.5, 2],
// 3 ulp outside) and division (2.5 ulp), which are all the reference's all_vmf_pdfs
// (general.wesl:984-1023) relies on.  Used for the mixture pdf, evaluated for every candidate of
// every guided bounce; the vMF draw itself keeps the precise functions.
LAM_DEV float vmf_pdf_fast(v3 mean, float kappa, v3 dir) {
    const float x = -2.0f * kappa;
    const float u = __expf(x);
    float frac = 1.0f;
    if (u != 1.0f) {
        const float y = u - 1.0f;
        frac = fabsf(x) < 1.0f ? __fdividef(__logf(u), y) : __fdividef(x, y);
    }
    return fmaxf(frac * (1.0f / (4.0f * PI_F)) * __expf(kappa * (dot(dir, mean) - 1.0f)), 0.0f);
}

// update_marcov_state, general.wesl:464-492 (sum_mc: the candidate weight sum of the last resample)
LAM_DEV MC update_chain(v3 x1, v3 x2, float p_hat, uint32_t seed, bool not_vmf, MC state, float confidence,
                        float sum_mc) {
    if (not_vmf) state = mc_zero();
    float score = p_hat;
    float rnd = rand_f32(seed);
    if ((rnd * sum_mc) < (p_hat * 21.0f)) {
        if (near_zero(len(light_dir(state, x1)))) return state;
        state.num_samples = min(state.num_samples + 1u, 1024u);
        float alpha = state.num_samples == 1u ? 1.0f : fmaxf(1.0f / __uint2float_rn(state.num_samples), 0.01f) * confidence;
        state.weight_sum = mixf(state.weight_sum, score, alpha);
        state.light = mix3(state.light, x2 * score, alpha);
        v3 mean = normalize(light_dir(state, x1));
        state.mean_cosine = mixf(state.mean_cosine, score * dot(normalize(x2 - x1), mean), alpha);
    }
    return state;
}

}  // namespace lam
