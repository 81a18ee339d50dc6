// guide_net.cu - evaluation and training kernels of the learned guiding network (guide_net.cuh) and
// the lam_guide_* entry points.  No counterpart in the reference.
//
//   guide_pack_kernel    f32 master weights -> BF16 core-matrix tiles
//   guide_eval_kernel    128-row tiles: features -> 4 tcgen05 layers -> 40 head outputs per query
//   guide_grad_kernel    forward + backward of 128-row tiles; weight gradients accumulate in TMEM
//                        across the tiles of a CTA and leave as one f32 partial per CTA
//   guide_update_kernel  sums the partials in a fixed order (deterministic) and applies Adam
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "guide_net.cuh"
#include "scene.h"
#include "tracer.h"

namespace lam {
namespace net {

constexpr uint32_t ERR_MMA_TIMEOUT = 1u << 8;
constexpr uint32_t EVAL_SMEM = LAYERS * LAYER_BYTES + X_BYTES + 64u + 128u;
// The last 32 KB are slack: every MMA operand extent stays inside its own tile, and the slack keeps
// even a misread of the MN-major gradient operand's strides inside this CTA's shared memory.
constexpr uint32_t GRAD_SMEM = LAYERS * LAYER_BYTES + 4u * X_BYTES + G_BYTES + 64u + 128u + 32768u;
constexpr uint32_t GRAD_TMEM_COLS = 512;  // acc 0..63, dW[l] at 64 (l + 1)
constexpr uint32_t EVAL_TMEM_COLS = 64;

LAM_DEV uint8_t* align128(uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 127u) & ~uintptr_t(127));
}

LAM_DEV void stage_weights(uint8_t* W, const uint16_t* packed) {
    const uint4* src = reinterpret_cast<const uint4*>(packed);
    uint4* dst = reinterpret_cast<uint4*>(W);
    for (uint32_t i = threadIdx.x; i < (uint32_t)(LAYERS * LAYER_BYTES / 16); i += blockDim.x) dst[i] = src[i];
}

__global__ void guide_pack_kernel(const float* __restrict__ master, uint16_t* __restrict__ packed) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (uint32_t)PARAMS) return;
    const uint32_t l = p / 4096u, o = (p / 64u) % 64u, i = p % 64u;
    const float w = trainable(l, o) ? master[p] : 0.0f;
    __nv_bfloat16 b = __float2bfloat16_rn(w);
    packed[packed_index(l, o, i)] = *reinterpret_cast<uint16_t*>(&b);
}

struct EvalArgs {
    const float* queries;  // n x 9
    uint32_t n;
    float box[6];
    const uint16_t* packed;
    float* out;            // n x 40
    uint32_t* err;
    uint32_t wait_tries;   // polls of each completion wait before it gives up
};

__global__ void __launch_bounds__(128) guide_eval_kernel(EvalArgs A) {
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = align128(smraw);
    uint8_t* W = sm;
    uint8_t* X = sm + LAYERS * LAYER_BYTES;
    uint64_t* bar = reinterpret_cast<uint64_t*>(X + X_BYTES);
    uint32_t* slot = reinterpret_cast<uint32_t*>(X + X_BYTES + 8);
    stage_weights(W, A.packed);
    if (threadIdx.x == 0) mbar_init(bar);
    if (threadIdx.x < 32) tmem_alloc(slot, EVAL_TMEM_COLS);
    fence_before();
    __syncthreads();
    fence_after();
    TileCtx c{*slot, smem_u32(bar), 0u, false, A.wait_tries};
    const uint32_t w_addr = smem_u32(W);
    const uint32_t tiles = (A.n + TILE - 1) / TILE;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t idx = tile * TILE + threadIdx.x;
        Query q{mk(0.0f, 0.0f, 0.0f), mk(0.0f, 1.0f, 0.0f), mk(0.0f, 1.0f, 0.0f)};
        if (idx < A.n) {
            const float* r = A.queries + (size_t)idx * 9u;
            q.pos = mk(r[0], r[1], r[2]);
            q.n = mk(r[3], r[4], r[5]);
            q.wo = mk(r[6], r[7], r[8]);
        }
        float f[WIDTH];
        encode_features(q, A.box, f);
        store_row(X, X_RG, threadIdx.x, f);
        float raw[OUT];
        if (!forward_infer(c, X, w_addr, raw)) break;
        if (idx < A.n)
            for (int k = 0; k < OUT; ++k) A.out[(size_t)idx * OUT + k] = raw[k];
    }
    if (c.failed) mbar_wait(c.bar, c.phase ^ 1u, DRAIN_TRIES);  // let an MMA in flight finish before TMEM is freed
    fence_before();
    c.failed = __syncthreads_or(c.failed ? 1 : 0) != 0;
    if (c.failed && threadIdx.x == 0) atomicOr(A.err, ERR_MMA_TIMEOUT);
    if (threadIdx.x < 32) {
        fence_after();
        tmem_free(c.tmem, EVAL_TMEM_COLS);
    }
}

struct GradArgs {
    const float* recs;      // records, `stride` floats each: pos, normal, wo, wi, weight
    uint32_t stride;
    uint32_t n;             // record count (used when n_dev is null)
    const uint32_t* n_dev;  // device record count, clamped to n
    uint32_t batch;         // rows (multiple of 128)
    uint32_t sequential;    // 1: row b reads record b (rows >= count weigh 0); 0: random records
    uint32_t seed, step;
    float scale;            // loss scale (1 / batch)
    float box[6];
    const uint16_t* packed;
    float* partial;         // gridDim x PARAMS
    float* partial_loss;    // gridDim
    uint32_t* err;
    uint32_t wait_tries;    // polls of each completion wait before it gives up
};

__global__ void __launch_bounds__(128, 1) guide_grad_kernel(GradArgs A) {
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = align128(smraw);
    uint8_t* W = sm;
    uint8_t* Xs[4];
    for (int l = 0; l < 4; ++l) Xs[l] = sm + LAYERS * LAYER_BYTES + l * X_BYTES;
    uint8_t* G = sm + LAYERS * LAYER_BYTES + 4 * X_BYTES;
    uint64_t* bar = reinterpret_cast<uint64_t*>(G + G_BYTES);
    uint32_t* slot = reinterpret_cast<uint32_t*>(G + G_BYTES + 8);
    float* sloss = reinterpret_cast<float*>(G + G_BYTES + 12);
    stage_weights(W, A.packed);
    {
        uint4* g4 = reinterpret_cast<uint4*>(G);
        for (uint32_t i = threadIdx.x; i < G_BYTES / 16u; i += blockDim.x) g4[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (threadIdx.x == 0) {
        mbar_init(bar);
        *sloss = 0.0f;
    }
    if (threadIdx.x < 32) tmem_alloc(slot, GRAD_TMEM_COLS);
    fence_before();
    __syncthreads();
    fence_after();
    TileCtx c{*slot, smem_u32(bar), 0u, false, A.wait_tries};
    const uint32_t row = threadIdx.x;
    const uint32_t t_row = c.tmem + ((threadIdx.x & ~31u) << 16);
    const uint32_t w_addr = smem_u32(W), g_addr = smem_u32(G);
    uint32_t n = A.n;
    if (A.n_dev) n = min(n, *A.n_dev);
    const uint32_t tiles = A.batch / TILE;
    bool any = false, stop = false;  // both uniform across the CTA
    float loss = 0.0f;
    for (uint32_t tile = blockIdx.x; tile < tiles && !stop; tile += gridDim.x) {
        const uint32_t b = tile * TILE + row;
        bool valid;
        uint32_t idx;
        if (A.sequential) {
            valid = b < n;
            idx = b;
        } else {
            valid = n > 0u;
            idx = valid ? rand_u32(A.seed ^ rand_u32(A.step * 0x9E3779B9u + b)) % n : 0u;
        }
        Query q{mk(0.0f, 0.0f, 0.0f), mk(0.0f, 1.0f, 0.0f), mk(0.0f, 1.0f, 0.0f)};
        v3 wi = mk(0.0f, 1.0f, 0.0f);
        float weight = 0.0f;
        if (valid) {
            const float* r = A.recs + (size_t)idx * A.stride;
            q.pos = mk(r[0], r[1], r[2]);
            q.n = mk(r[3], r[4], r[5]);
            q.wo = mk(r[6], r[7], r[8]);
            wi = mk(r[9], r[10], r[11]);
            weight = r[12];
            if (!(weight >= 0.0f) || !(weight < 3.0e38f)) weight = 0.0f;
        }
        float f[WIDTH];
        encode_features(q, A.box, f);
        store_row(Xs[0], X_RG, row, f);
        // forward, keeping every layer's input for the backward pass
        bool ok = true;
        for (uint32_t l = 0; l < 4u && ok; ++l) {
            ok = mma_round(c, [&] { issue_fwd(c.tmem, smem_u32(Xs[l]), w_addr + l * LAYER_BYTES); });
            if (!ok) {
                stop = true;
                break;
            }
            if (l < 3u) {
                epilogue_relu(t_row, Xs[l + 1], row);
            } else {
                float raw[OUT], g[WIDTH];
                head_read(t_row, raw);
                loss += head_grad(raw, wi, weight, A.scale, g);
                for (int k = OUT; k < WIDTH; ++k) g[k] = 0.0f;
                store_row(G, G_RG, row, g);
            }
        }
        // backward: dW[l] += G^T X[l]; G <- (G W[l]) * relu'(X[l])
        for (int l = 3; l >= 0 && ok; --l) {
            const bool acc_dw = any;
            ok = mma_round(c, [&] {
                issue_dw(c.tmem + 64u * (uint32_t)(l + 1), g_addr, smem_u32(Xs[l]), acc_dw);
                if (l > 0) issue_dx(c.tmem, g_addr, w_addr + (uint32_t)l * LAYER_BYTES);
            });
            if (!ok) {
                stop = true;
                break;
            }
            if (l > 0) {
                float v[64];
                tmem_ld64(t_row, v);
#pragma unroll
                for (uint32_t ch = 0; ch < 8; ++ch) {
                    const uint4 x = load_chunk(Xs[l], X_RG, row, ch);
                    const uint32_t xw[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (!(bf16_lo(xw[k]) > 0.0f)) v[8 * ch + 2 * k] = 0.0f;
                        if (!(bf16_hi(xw[k]) > 0.0f)) v[8 * ch + 2 * k + 1] = 0.0f;
                    }
                }
                v[63] = 0.0f;
#pragma unroll
                for (uint32_t ch = 0; ch < 8; ++ch) store_chunk(G, G_RG, row, ch, v + 8 * ch);
            }
        }
        any = true;
    }
    // loss: warp sums, then one shared-memory add per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xFFFFFFFFu, loss, o);
    if ((threadIdx.x & 31u) == 0u) atomicAdd(sloss, loss);
    if (c.failed) mbar_wait(c.bar, c.phase ^ 1u, DRAIN_TRIES);  // an MMA in flight finishes before TMEM is read or freed
    fence_before();
    c.failed = __syncthreads_or(c.failed ? 1 : 0) != 0;
    fence_after();
    // weight-gradient partials: rows 0..63 of each dW accumulator live in the lanes of warps 0 and 1
    float* part = A.partial + (size_t)blockIdx.x * PARAMS;
    if (threadIdx.x < 64) {
        const uint32_t o = threadIdx.x;
        for (uint32_t l = 0; l < 4u; ++l) {
            float v[64];
            tmem_ld64(t_row + 64u * (l + 1u), v);
            const bool use = any && !c.failed && trainable(l, o);
            float4* dst = reinterpret_cast<float4*>(part + l * 4096u + o * 64u);
#pragma unroll
            for (int k = 0; k < 16; ++k)
                dst[k] = use ? make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    if (threadIdx.x == 0) {
        A.partial_loss[blockIdx.x] = *sloss;
        if (c.failed) atomicOr(A.err, ERR_MMA_TIMEOUT);
    }
    fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        fence_after();
        tmem_free(c.tmem, GRAD_TMEM_COLS);
    }
}

struct UpdateArgs {
    const float* partial;
    const float* partial_loss;
    uint32_t parts;
    uint32_t mode;  // 0: write grad/loss, 1: Adam step
    float* grad;
    float* loss;
    float* master;
    float* m;
    float* v;
    uint16_t* packed;
    float lr_t, b1, b2, eps;
};

__global__ void guide_update_kernel(UpdateArgs A) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && A.loss) {
        float s = 0.0f;
        for (uint32_t c = 0; c < A.parts; ++c) s += A.partial_loss[c];
        *A.loss = s;
    }
    if (p >= (uint32_t)PARAMS) return;
    float g = 0.0f;
    for (uint32_t c = 0; c < A.parts; ++c) g += A.partial[(size_t)c * PARAMS + p];
    const uint32_t l = p / 4096u, o = (p / 64u) % 64u, i = p % 64u;
    if (!trainable(l, o)) g = 0.0f;
    if (A.mode == 0u) {
        A.grad[p] = g;
        return;
    }
    if (!trainable(l, o)) return;
    const float m = A.b1 * A.m[p] + (1.0f - A.b1) * g;
    const float v = A.b2 * A.v[p] + (1.0f - A.b2) * g * g;
    A.m[p] = m;
    A.v[p] = v;
    const float w = A.master[p] - A.lr_t * m / (sqrtf(v) + A.eps);
    A.master[p] = w;
    __nv_bfloat16 b = __float2bfloat16_rn(w);
    A.packed[packed_index(l, o, i)] = *reinterpret_cast<uint16_t*>(&b);
}

}  // namespace net

// ---------------------------------------------------------------- host side
static int galloc(lam_guide* g, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (guide)");
    g->allocs.push_back(*p);
    e = cudaMemset(*p, 0, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemset (guide)");
    return LAM_OK;
}

static void init_params(uint32_t seed, std::vector<float>& w) {
    // uniform(-a, a) with a = sqrt(6 / fan_in) for the hidden layers and a smaller head; zero biases
    w.assign(net::PARAMS, 0.0f);
    uint64_t s = 0x9E3779B97F4A7C15ull ^ (uint64_t)seed * 0xD1B54A32D192ED03ull;
    auto next = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    for (uint32_t l = 0; l < 4; ++l) {
        const double a = l < 3 ? std::sqrt(6.0 / 64.0) : 0.5 * std::sqrt(6.0 / 64.0);
        for (uint32_t o = 0; o < 64; ++o)
            for (uint32_t i = 0; i < 63; ++i) {
                const double r = (2.0 * next() - 1.0) * a;
                if (net::trainable(l, o)) w[l * 4096 + o * 64 + i] = (float)r;
            }
    }
}

static int upload_params(lam_guide* g, const float* host) {
    cudaError_t e = cudaMemcpy(g->master, host, net::PARAMS * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "lam_guide params upload");
    cudaMemset(g->adam_m, 0, net::PARAMS * sizeof(float));
    cudaMemset(g->adam_v, 0, net::PARAMS * sizeof(float));
    net::guide_pack_kernel<<<net::PARAMS / 256, 256>>>(g->master, g->packed);
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(e, "lam_guide pack");
    g->steps = 0;
    g->trained_spp = 0;
    return LAM_OK;
}

static int setup_kernels(lam_guide* g) {
    if (g->kernels_ready) return LAM_OK;
    cudaError_t e = cudaFuncSetAttribute(net::guide_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, net::GRAD_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(net::guide_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, net::EVAL_SMEM);
    if (e != cudaSuccess) return cuda_error(e, "guide kernel attributes");
    g->kernels_ready = true;
    return LAM_OK;
}

// Gradient partials of `batch` rows (one launch) and their reduction (mode 0: grad/loss, 1: Adam).
int guide_grad_and_update(lam_guide* g, const float* recs, uint32_t stride, uint32_t n, const uint32_t* n_dev,
                          uint32_t batch, bool sequential, float scale, const float box[6], uint32_t mode, float* grad,
                          float* loss, cudaStream_t st) {
    int rc = setup_kernels(g);
    if (rc) return rc;
    const uint32_t tiles = batch / net::TILE;
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, g->parts));
    net::GradArgs A;
    A.recs = recs;
    A.stride = stride;
    A.n = n;
    A.n_dev = n_dev;
    A.batch = batch;
    A.sequential = sequential ? 1u : 0u;
    A.seed = g->opts.seed;
    A.step = (uint32_t)g->steps;
    A.scale = scale;
    std::memcpy(A.box, box, sizeof(A.box));
    A.packed = g->packed;
    A.partial = g->partial;
    A.partial_loss = g->partial_loss;
    A.err = g->err;
    A.wait_tries = g->wait_tries;
    net::guide_grad_kernel<<<grid, 128, net::GRAD_SMEM, st>>>(A);
    net::UpdateArgs U;
    U.partial = g->partial;
    U.partial_loss = g->partial_loss;
    U.parts = grid;
    U.mode = mode;
    U.grad = grad;
    U.loss = loss;
    U.master = g->master;
    U.m = g->adam_m;
    U.v = g->adam_v;
    U.packed = g->packed;
    U.b1 = 0.9f;
    U.b2 = 0.99f;
    U.eps = 1e-8f;
    U.lr_t = 0.0f;
    if (mode == 1u) {
        g->steps++;
        const double t = (double)g->steps;
        U.lr_t = (float)(g->opts.learning_rate * std::sqrt(1.0 - std::pow((double)U.b2, t)) /
                         (1.0 - std::pow((double)U.b1, t)));
    }
    net::guide_update_kernel<<<net::PARAMS / 256, 256, 0, st>>>(U);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "guide training launch");
    return LAM_OK;
}

int guide_eval_launch(const lam_guide* g, const float* queries, uint32_t n, const float box[6], float* out,
                      cudaStream_t st) {
    int rc = setup_kernels(const_cast<lam_guide*>(g));
    if (rc) return rc;
    if (n == 0) return LAM_OK;
    net::EvalArgs A;
    A.queries = queries;
    A.n = n;
    std::memcpy(A.box, box, sizeof(A.box));
    A.packed = g->packed;
    A.out = out;
    A.err = g->err;
    A.wait_tries = g->wait_tries;
    const uint32_t tiles = (n + net::TILE - 1) / net::TILE;
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, (uint32_t)g->sms * 4u));
    net::guide_eval_kernel<<<grid, 128, net::EVAL_SMEM, st>>>(A);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "lam_guide_eval launch");
    return LAM_OK;
}

int guide_check_error(const lam_guide* g) {
    uint32_t h = 0;
    cudaError_t e = cudaMemcpy(&h, g->err, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "lam_guide error flags");
    if (h & net::ERR_MMA_TIMEOUT) {
        // reported once: the flags start clear again for the next kernels
        e = cudaMemset(g->err, 0, sizeof(h));
        if (e != cudaSuccess) return cuda_error(e, "lam_guide error flags");
        return set_error(LAM_ERR_DEVICE_TIMEOUT, "guide network: a tensor-core completion wait gave up");
    }
    return LAM_OK;
}

}  // namespace lam

using namespace lam;

extern "C" int lam_guide_options_default(lam_guide_options* o) {
    if (!o) return set_error(LAM_ERR_INVALID_ARGUMENT, "null options");
    o->train_spp = 32;
    o->steps_per_wave = 32;
    o->batch = 16384;
    o->record_capacity = 1u << 21;
    o->learning_rate = 2e-3f;
    o->guide_fraction = 0.5f;
    o->seed = 1;
    return LAM_OK;
}

extern "C" int lam_guide_create(const lam_guide_options* o, lam_guide** out) {
    if (!o || !out) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_guide_create: null argument");
    *out = nullptr;
    if (o->batch == 0 || o->batch % net::TILE != 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "batch must be a positive multiple of 128");
    if (!(o->guide_fraction >= 0.0f && o->guide_fraction < 1.0f))
        return set_error(LAM_ERR_INVALID_ARGUMENT, "guide_fraction must be in [0, 1)");
    if (!(o->learning_rate > 0.0f)) return set_error(LAM_ERR_INVALID_ARGUMENT, "learning_rate must be positive");
    lam_guide* g = new lam_guide();
    g->opts = *o;
    cudaGetDevice(&g->device);
    cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, g->device);
    g->parts = (uint32_t)std::max(1, g->sms);
    int rc = 0;
    rc |= galloc(g, (void**)&g->master, net::PARAMS * sizeof(float));
    rc |= galloc(g, (void**)&g->adam_m, net::PARAMS * sizeof(float));
    rc |= galloc(g, (void**)&g->adam_v, net::PARAMS * sizeof(float));
    rc |= galloc(g, (void**)&g->packed, net::PARAMS * sizeof(uint16_t));
    rc |= galloc(g, (void**)&g->partial, (size_t)g->parts * net::PARAMS * sizeof(float));
    rc |= galloc(g, (void**)&g->partial_loss, (size_t)g->parts * sizeof(float));
    rc |= galloc(g, (void**)&g->err, 16 * sizeof(uint32_t));
    if (o->record_capacity) rc |= galloc(g, (void**)&g->records, (size_t)o->record_capacity * GUIDE_RECORD_STRIDE * sizeof(float));
    if (rc) {
        lam_guide_destroy(g);
        return LAM_ERR_CUDA;
    }
    std::vector<float> w;
    init_params(o->seed, w);
    rc = upload_params(g, w.data());
    if (rc) {
        lam_guide_destroy(g);
        return rc;
    }
    *out = g;
    return LAM_OK;
}

extern "C" int lam_guide_destroy(lam_guide* g) {
    if (!g) return LAM_OK;
    for (void* p : g->allocs) cudaFree(p);
    delete g;
    return LAM_OK;
}

extern "C" int lam_guide_get_params(const lam_guide* g, float* params) {
    if (!g || !params) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    cudaError_t e = cudaMemcpy(params, g->master, net::PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "lam_guide_get_params");
    return LAM_OK;
}

extern "C" int lam_guide_set_params(lam_guide* g, const float* params) {
    if (!g || !params) return set_error(LAM_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<float> w(params, params + net::PARAMS);
    for (uint32_t l = 0; l < 4; ++l)
        for (uint32_t o = 0; o < 64; ++o)
            if (!net::trainable(l, o))
                for (uint32_t i = 0; i < 64; ++i) w[l * 4096 + o * 64 + i] = 0.0f;
    return upload_params(g, w.data());
}

extern "C" int lam_guide_eval(const lam_guide* g, const lam_guide_query* queries, uint32_t n, const float box[6],
                              float* outputs, void* stream) {
    if (!g || !box || (n && (!queries || !outputs))) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_guide_eval: null argument");
    return guide_eval_launch(g, reinterpret_cast<const float*>(queries), n, box, outputs, (cudaStream_t)stream);
}

extern "C" int lam_guide_loss_grad(lam_guide* g, const lam_guide_record* records, uint32_t n, const float box[6],
                                   float* grad, float* loss, void* stream) {
    if (!g || !box || !grad || !loss || (n && !records)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_guide_loss_grad: null argument");
    if (n == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_guide_loss_grad: no records");
    const uint32_t batch = (n + net::TILE - 1) / net::TILE * net::TILE;
    return guide_grad_and_update(g, reinterpret_cast<const float*>(records), 13u, n, nullptr, batch, true, 1.0f / (float)n,
                                 box, 0u, grad, loss, (cudaStream_t)stream);
}

extern "C" int lam_guide_train(lam_guide* g, const lam_guide_record* records, uint32_t n, uint32_t steps,
                               const float box[6], void* stream) {
    if (!g || !box || (n && !records)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_guide_train: null argument");
    for (uint32_t s = 0; s < steps && n; ++s) {
        int rc = guide_grad_and_update(g, reinterpret_cast<const float*>(records), 13u, n, nullptr, g->opts.batch, false,
                                       1.0f / (float)g->opts.batch, box, 1u, nullptr, nullptr, (cudaStream_t)stream);
        if (rc) return rc;
    }
    return LAM_OK;
}

extern "C" int lam_guide_set_wait_limit(lam_guide* g, uint32_t tries) {
    if (!g) return set_error(LAM_ERR_INVALID_ARGUMENT, "null guide");
    g->wait_tries = tries;
    return LAM_OK;
}

extern "C" int lam_guide_progress(const lam_guide* g, uint64_t* steps, uint32_t* trained_spp) {
    if (!g) return set_error(LAM_ERR_INVALID_ARGUMENT, "null guide");
    if (steps) *steps = g->steps;
    if (trained_spp) *trained_spp = g->trained_spp;
    return guide_check_error(g);
}
