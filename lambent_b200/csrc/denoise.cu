// denoise.cu - the denoiser hand-off of the reference's example (examples/cornell_box/src/main.rs:797-963).
//
// The reference keeps an OidnState: a device staging buffer holding the averaged frame as RGB f32
// (average_to_buf.wgsl writes it), a mappable read buffer and a mappable write buffer.  Each denoise
// copies the frame into the read buffer, maps it on the host, runs OIDN's RayTracing filter in place,
// writes the result into the write buffer and copies it back into the staging buffer.  Here a
// lam_denoiser owns the pinned host staging of one frame size; lam_denoiser_run copies the frame (and,
// when given, the first-hit normal and albedo images, repacked from rgba32f to RGB f32 on the device,
// the auxiliary images OIDN's RayTracing filter accepts) to the host, calls the caller's filter on
// them, and uploads the filtered colour into the frame in place.
#include <cstring>

#include "scene.h"

struct lam_denoiser {
    uint32_t width = 0, height = 0;
    float* host = nullptr;    // pinned: colour | normal | albedo, width * height * 3 floats each
    float* packed = nullptr;  // device: normal | albedo repacked to RGB
    int device = 0;
};

namespace lam {

__global__ void rgba_to_rgb_kernel(const float4* __restrict__ src, float* __restrict__ dst, uint64_t pixels) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    const float4 v = src[i];
    dst[3 * i + 0] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}

}  // namespace lam

using namespace lam;

extern "C" int lam_denoiser_create(uint32_t width, uint32_t height, lam_denoiser** out) {
    if (!out || width == 0 || height == 0) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_denoiser_create: bad argument");
    const uint64_t floats = (uint64_t)width * height * 3u;
    if (floats > (1ull << 33)) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_denoiser_create: frame too large");
    lam_denoiser* d = new lam_denoiser();
    d->width = width;
    d->height = height;
    cudaGetDevice(&d->device);
    cudaError_t e = cudaMallocHost((void**)&d->host, 3u * floats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d->packed, 2u * floats * sizeof(float));
    if (e != cudaSuccess) {
        if (d->host) cudaFreeHost(d->host);
        delete d;
        return cuda_error(e, "lam_denoiser_create");
    }
    *out = d;
    return LAM_OK;
}

extern "C" int lam_denoiser_destroy(lam_denoiser* d) {
    if (!d) return LAM_OK;
    if (d->host) cudaFreeHost(d->host);
    if (d->packed) cudaFree(d->packed);
    delete d;
    return LAM_OK;
}

extern "C" int lam_denoiser_run(lam_denoiser* d, float* rgb, const float* normal, const float* albedo,
                                lam_denoise_fn filter, void* user, void* stream) {
    if (!d || !rgb || !filter) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_denoiser_run: null argument");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_error(e, "lam_denoiser_run");
    if (device != d->device) return set_error(LAM_ERR_INVALID_ARGUMENT, "lam_denoiser_run: not the denoiser's device");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t pixels = (uint64_t)d->width * d->height;
    const uint64_t bytes = pixels * 3u * sizeof(float);
    float* h_rgb = d->host;
    float* h_normal = normal ? d->host + pixels * 3u : nullptr;
    float* h_albedo = albedo ? d->host + pixels * 6u : nullptr;
    const unsigned grid = (unsigned)((pixels + 255u) / 256u);
    const float* aux[2] = {normal, albedo};
    float* h_aux[2] = {h_normal, h_albedo};
    for (int k = 0; k < 2; ++k) {
        if (!aux[k]) continue;
        float* dst = d->packed + (uint64_t)k * pixels * 3u;
        rgba_to_rgb_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const float4*>(aux[k]), dst, pixels);
        e = cudaMemcpyAsync(h_aux[k], dst, bytes, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_error(e, "lam_denoiser_run: auxiliary image to the host");
    }
    e = cudaMemcpyAsync(h_rgb, rgb, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "lam_denoiser_run: frame to the host");
    const int rc = filter(user, h_rgb, h_normal, h_albedo, d->width, d->height);
    if (rc != 0) return set_error(LAM_ERR_CALLBACK, "lam_denoiser_run: the filter reported an error");
    e = cudaMemcpyAsync(rgb, h_rgb, bytes, cudaMemcpyHostToDevice, st);
    // the host staging is reused by the next call: the upload completes before this returns
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "lam_denoiser_run: filtered frame to the device");
    return LAM_OK;
}
