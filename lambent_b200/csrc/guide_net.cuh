// guide_net.cuh - the learned path-guiding network: a 4-layer MLP (64 -> 64 -> 64 -> 64 -> 40) whose
// output is an 8-lobe von Mises-Fisher mixture over incident directions, evaluated and trained with
// tcgen05 tensor-core MMAs (BF16 operands, FP32 accumulators in tensor memory).
//
// No counterpart in the reference: its guiding is the vMF Markov-chain cache
// (src/path_tracing/general.wesl:764-866).  The learned mixture is combined with the BSDF sampler by
// one-sample MIS (mixture pdf), so the estimator stays unbiased whatever the network outputs.
//
// Network.  Every layer is 64 x 64 (weights W[l][o][i], out x in).  Column 63 of every activation
// tile is the constant 1, so W[l][o][63] is the bias of unit o and the bias gradient comes out of the
// same weight-gradient product.  Hidden units 0..62 use ReLU; outputs 0..39 of the last layer are the
// head (logits 0-7, log-concentration 8-15, mean x/y/z 16-23 / 24-31 / 32-39).
//
// Shared-memory tiles use the canonical no-swizzle ("interleaved") UMMA layout: 8 rows x 16 bytes
// per core matrix, core matrices along K 128 bytes apart, 8-row groups `rg` bytes apart.  The same
// bytes are a K-major operand for X W^T and an MN-major operand (LBO/SBO swapped) for the transposed
// products of the backward pass, so no tile is ever transposed in memory.
#pragma once
#include <cuda_bf16.h>

#include "device_math.cuh"

namespace lam {
namespace net {

#define LAM_HD __host__ __device__ __forceinline__

constexpr int WIDTH = 64;
constexpr int LAYERS = 4;
constexpr int TILE = 128;                      // rows per MMA tile (M)
constexpr int OUT = 40;                        // head outputs used
constexpr int LOBES = 8;
constexpr int PARAMS = LAYERS * WIDTH * WIDTH; // 16384
constexpr uint32_t LAYER_BYTES = WIDTH * WIDTH * 2;   // 8 KB of bf16 per layer
constexpr uint32_t X_RG = 1024;                       // 8-row group stride of a 128 x 64 activation tile
constexpr uint32_t X_BYTES = TILE * WIDTH * 2;        // 16 KB
constexpr uint32_t G_RG = 2048;                       // gradient tile: 128 x 128 (columns 64..127 zero)
constexpr uint32_t G_BYTES = TILE * 128 * 2;          // 32 KB
constexpr uint32_t W_RG = 1024;                       // weight tile: 64 x 64
constexpr float KAPPA_LOG_MIN = -3.0f, KAPPA_LOG_MAX = 6.0f;

// Byte offset of element (row, col) in a core-matrix tile whose 8-row groups are `rg` bytes apart.
LAM_HD uint32_t core_off(uint32_t row, uint32_t col, uint32_t rg) {
    return (row >> 3) * rg + (col >> 3) * 128u + (row & 7u) * 16u + (col & 7u) * 2u;
}
// Index (in bf16 elements) of W[l][o][i] in the packed device weights (4 core-matrix tiles).
LAM_HD uint32_t packed_index(uint32_t l, uint32_t o, uint32_t i) {
    return l * (uint32_t)(WIDTH * WIDTH) + core_off(o, i, W_RG) / 2u;
}
// Trainable parameters: hidden unit 63 is the constant-1 unit, head rows 40..63 are unused.
LAM_HD bool trainable(uint32_t l, uint32_t o) { return l < 3 ? o < 63u : o < (uint32_t)OUT; }

// ---------------------------------------------------------------- tcgen05 / mbarrier primitives
LAM_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, SWIZZLE_NONE, sm100 version field = 1.
LAM_DEV uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: kind::f16 with BF16 A/B, F32 accumulator, dense.
constexpr uint32_t idesc_bf16(bool a_mn, bool b_mn, int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? (1u << 15) : 0u) | (b_mn ? (1u << 16) : 0u) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t ID_FWD = idesc_bf16(false, false, 128, 64);  // X W^T
constexpr uint32_t ID_DX = idesc_bf16(false, true, 128, 64);    // G W
constexpr uint32_t ID_DW = idesc_bf16(true, true, 128, 64);     // G^T X (rows 64..127 of D are zero)

LAM_DEV void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
LAM_DEV void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
LAM_DEV void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
LAM_DEV void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
LAM_DEV void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Whole warp: allocates `cols` TMEM columns and writes the base address to *slot.
LAM_DEV void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
LAM_DEV void tmem_free(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

LAM_DEV void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Polls of a completion barrier before a wait gives up (lam_guide_set_wait_limit), and the polls of
// the wait that, after a give-up, lets the MMAs still in flight finish before TMEM is read or freed.
constexpr uint32_t WAIT_TRIES = 1u << 20;
constexpr uint32_t DRAIN_TRIES = 1u << 22;
// Bounded wait for phase `parity` of the barrier; false when `tries` polls ran out (0: at once).
LAM_DEV bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t tries = WAIT_TRIES) {
    for (uint32_t it = 0; it < tries; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// 32 lanes x 16 consecutive f32 columns: this thread's row, columns [col, col + 16).  The wait is in
// the same statement so that no use of the registers can be scheduled before the load completes.
LAM_DEV void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
// 64 consecutive columns in one load and one wait.
LAM_DEV void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]),
          "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]),
          "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]),
          "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]),
          "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = __uint_as_float(r[k]);
}
// 32 + 8 columns (the head) in one statement and one wait.
LAM_DEV void tmem_ld40(uint32_t taddr, float* v) {
    uint32_t r[40];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%40];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%32, %33, %34, %35, %36, %37, %38, %39}, [%41];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]),
          "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39])
        : "r"(taddr), "r"(taddr + 32u));
#pragma unroll
    for (int k = 0; k < 40; ++k) v[k] = __uint_as_float(r[k]);
}
LAM_DEV void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __uint_as_float(r[k]);
}

LAM_DEV uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
LAM_DEV float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
LAM_DEV float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Writes 8 consecutive values (columns c8*8 .. c8*8+7) of `row` as one 16-byte chunk.
LAM_DEV void store_chunk(uint8_t* tile, uint32_t rg, uint32_t row, uint32_t c8, const float* v) {
    uint4 q = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    *reinterpret_cast<uint4*>(tile + core_off(row, c8 * 8u, rg)) = q;
}
LAM_DEV uint4 load_chunk(const uint8_t* tile, uint32_t rg, uint32_t row, uint32_t c8) {
    return *reinterpret_cast<const uint4*>(tile + core_off(row, c8 * 8u, rg));
}

// ---------------------------------------------------------------- input encoding
// 64 features: frequency encoding of the position normalised to the scene box (5 octaves, 30),
// the normal and outgoing direction (6), their 2-octave encodings (24), three zeros and the constant 1.
struct Query {
    v3 pos, n, wo;
};
LAM_DEV void encode_features(const Query& q, const float* box, float* f) {
    const float pc[3] = {q.pos.x, q.pos.y, q.pos.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ext = box[3 + a] - box[a];
        float u = ext > 0.0f ? (pc[a] - box[a]) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        float sv, cv;
        sincospif(u, &sv, &cv);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            f[6 * k + 2 * a] = sv;
            f[6 * k + 2 * a + 1] = cv;
            const float s2 = 2.0f * sv * cv, c2 = fmaf(-2.0f * sv, sv, 1.0f);  // next octave by angle doubling
            sv = s2;
            cv = c2;
        }
    }
    const float d[6] = {q.n.x, q.n.y, q.n.z, q.wo.x, q.wo.y, q.wo.z};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        f[30 + c] = d[c];
        float sv, cv;
        sincospif(d[c], &sv, &cv);
        f[36 + 4 * c] = sv;
        f[36 + 4 * c + 1] = cv;
        f[36 + 4 * c + 2] = 2.0f * sv * cv;
        f[36 + 4 * c + 3] = fmaf(-2.0f * sv, sv, 1.0f);
    }
    f[60] = 0.0f;
    f[61] = 0.0f;
    f[62] = 0.0f;
    f[63] = 1.0f;
}

// ---------------------------------------------------------------- lobe mixture
struct Lobes {
    float pi[LOBES], kappa[LOBES];
    float lognorm[LOBES];  // log(kappa / (2 pi (1 - e^{-2 kappa}))) - kappa
    v3 mu[LOBES];
};
LAM_DEV float clampf_(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

LAM_DEV void lobes_from_raw(const float* raw, Lobes& L) {
    float mx = raw[0];
#pragma unroll
    for (int j = 1; j < LOBES; ++j) mx = fmaxf(mx, raw[j]);
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) {
        L.pi[j] = __expf(raw[j] - mx);
        s += L.pi[j];
    }
    const float inv = 1.0f / s;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) {
        L.pi[j] *= inv;
        const float lk = clampf_(raw[8 + j], KAPPA_LOG_MIN, KAPPA_LOG_MAX);
        L.kappa[j] = __expf(lk);
        L.lognorm[j] = lk - 1.8378770664093453f - log1pf(-__expf(-2.0f * L.kappa[j])) - L.kappa[j];
        v3 m = mk(raw[16 + j], raw[24 + j], raw[32 + j]);
        const float l = len(m);
        L.mu[j] = l > 1e-12f ? m / l : mk(0.0f, 1.0f, 0.0f);
    }
}

// log of the vMF density kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.w - 1))
LAM_DEV float vmf_log_pdf(float kappa, float cos_mu) {
    return __logf(kappa) - 1.8378770664093453f - log1pf(-__expf(-2.0f * kappa)) + kappa * (cos_mu - 1.0f);
}

LAM_DEV float mixture_pdf(const Lobes& L, v3 w) {
    float p = 0.0f;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) p += L.pi[j] * __expf(fmaf(L.kappa[j], dot(L.mu[j], w), L.lognorm[j]));
    return p;
}

// Samples the mixture: u0 picks the lobe, (u1, u2) the direction inside it.
LAM_DEV v3 mixture_sample(const Lobes& L, float u0, float u1, float u2) {
    int j = LOBES - 1;
    float c = 0.0f;
#pragma unroll
    for (int k = 0; k < LOBES - 1; ++k) {
        c += L.pi[k];
        if (u0 < c) {
            j = k;
            break;
        }
    }
    float kappa = L.kappa[0];
    v3 mu = L.mu[0];
#pragma unroll
    for (int k = 1; k < LOBES; ++k)
        if (k == j) {
            kappa = L.kappa[k];
            mu = L.mu[k];
        }
    // W = 1 + log(u1 + (1 - u1) e^{-2 kappa}) / kappa (cosine to the mean), azimuth 2 pi u2
    const float W1 = log1pf(u1 * expm1f(-2.0f * kappa)) / kappa;
    const float W = fmaxf(1.0f + W1, -1.0f);
    const float sn = sqrtf(fmaxf(0.0f, -W1 * (2.0f + W1)));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    v3 other = fabsf(mu.x) > 0.9f ? mk(0.0f, 1.0f, 0.0f) : mk(1.0f, 0.0f, 0.0f);
    v3 b1 = normalize(cross(mu, other));
    v3 b2 = cross(mu, b1);
    return normalize(mu * W + b1 * (sn * cp) + b2 * (sn * sp));
}

// Gradient of  scale * (-weight * log q(w))  with respect to the 40 head outputs; returns the loss term.
LAM_DEV float head_grad(const float* raw, v3 w, float weight, float scale, float* g) {
    Lobes L;
    lobes_from_raw(raw, L);
    float lf[LOBES], mx = -3.0e38f;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) {
        lf[j] = __logf(fmaxf(L.pi[j], 1e-30f)) + vmf_log_pdf(L.kappa[j], dot(L.mu[j], w));
        mx = fmaxf(mx, lf[j]);
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) s += __expf(lf[j] - mx);
    const float logq = mx + __logf(s);
    const float c = -weight * scale;
#pragma unroll
    for (int j = 0; j < LOBES; ++j) {
        const float r = __expf(lf[j] - logq);
        const float k = L.kappa[j];
        const float cm = dot(L.mu[j], w);
        g[j] = c * (r - L.pi[j]);
        const float in_range = (raw[8 + j] > KAPPA_LOG_MIN && raw[8 + j] < KAPPA_LOG_MAX) ? 1.0f : 0.0f;
        const float dlogf_dk = 1.0f / k - 2.0f / expm1f(2.0f * k) + (cm - 1.0f);
        g[8 + j] = c * r * k * dlogf_dk * in_range;
        v3 m = mk(raw[16 + j], raw[24 + j], raw[32 + j]);
        const float ml = fmaxf(len(m), 1e-12f);
        v3 dm = (w - L.mu[j] * cm) * (c * r * k / ml);
        g[16 + j] = dm.x;
        g[24 + j] = dm.y;
        g[32 + j] = dm.z;
    }
    return -weight * scale * logq;
}

}  // namespace net
}  // namespace lam

namespace lam {
namespace net {

// ---------------------------------------------------------------- tile pipeline (128 threads, one row each)
struct TileCtx {
    uint32_t tmem;   // TMEM base (lane 0, first column)
    uint32_t bar;    // shared address of the completion mbarrier
    uint32_t phase;
    bool failed;
    uint32_t tries;  // polls of each completion wait before it gives up
};

// One MMA round: publishes this thread's shared-memory writes to the tensor core, lets thread 0 issue
// the MMAs and commit them to the barrier, then waits (bounded) for completion.  Returns false, on
// every thread, once any thread has seen a wait run out.
template <class Issue>
LAM_DEV bool mma_round(TileCtx& c, Issue issue) {
    fence_async_smem();
    fence_before();
    if (__syncthreads_or(c.failed ? 1 : 0)) {
        c.failed = true;
        return false;
    }
    if (threadIdx.x == 0) {
        fence_after();
        issue();
        mma_commit(c.bar);
    }
    if (!mbar_wait(c.bar, c.phase, c.tries)) c.failed = true;
    c.phase ^= 1u;
    fence_after();
    return true;
}

// acc[128 x 64] = X[128 x 64] . W^T  (4 MMAs of K = 16)
LAM_DEV void issue_fwd(uint32_t acc, uint32_t x_addr, uint32_t w_addr) {
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
        mma_bf16(acc, sdesc(x_addr + 256u * j, 128u, X_RG), sdesc(w_addr + 256u * j, 128u, W_RG), ID_FWD, j > 0u);
}
// dW[o][i] (+)= sum_rows G[row][o] X[row][i]: A = G as MN-major (o contiguous), B = X as MN-major
LAM_DEV void issue_dw(uint32_t acc, uint32_t g_addr, uint32_t x_addr, bool accumulate) {
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j)
        mma_bf16(acc, sdesc(g_addr + 4096u * j, G_RG, 128u), sdesc(x_addr + 2048u * j, X_RG, 128u), ID_DW,
                 (accumulate || j > 0u) ? 1u : 0u);
}
// dX[row][i] = sum_o G[row][o] W[o][i]: A = G as K-major, B = W as MN-major (i contiguous)
LAM_DEV void issue_dx(uint32_t acc, uint32_t g_addr, uint32_t w_addr) {
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
        mma_bf16(acc, sdesc(g_addr + 256u * j, 128u, G_RG), sdesc(w_addr + 2048u * j, W_RG, 128u), ID_DX, j > 0u);
}

LAM_DEV void store_row(uint8_t* tile, uint32_t rg, uint32_t row, const float* f) {
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) store_chunk(tile, rg, row, c, f + 8 * c);
}

// Hidden-layer epilogue: ReLU of this thread's accumulator row into `dst`; column 63 is the constant 1.
LAM_DEV void epilogue_relu(uint32_t t_row, uint8_t* dst, uint32_t row) {
    float v[64];
    tmem_ld64(t_row, v);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = fmaxf(v[k], 0.0f);
    v[63] = 1.0f;
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) store_chunk(dst, X_RG, row, c, v + 8 * c);
}
LAM_DEV void head_read(uint32_t t_row, float* raw) { tmem_ld40(t_row, raw); }

// Forward pass of a tile whose features are in X (overwritten layer by layer); raw = head outputs.
LAM_DEV bool forward_infer(TileCtx& c, uint8_t* X, uint32_t w_addr, float* raw) {
    const uint32_t x_addr = smem_u32(X);
    const uint32_t row = threadIdx.x;
    const uint32_t t_row = c.tmem + ((threadIdx.x & ~31u) << 16);
    for (uint32_t l = 0; l < (uint32_t)LAYERS; ++l) {
        if (!mma_round(c, [&] { issue_fwd(c.tmem, x_addr, w_addr + l * LAYER_BYTES); })) return false;
        if (l < 3u) epilogue_relu(t_row, X, row);
        else head_read(t_row, raw);
    }
    return true;
}

}  // namespace net
}  // namespace lam
