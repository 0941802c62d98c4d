// average.cu -- averaged intensity and per-event statistics of a batch of
// frames on the device: Detector::LoadAndAverageIntensity
// (IAC/Detector.cpp:687-790) after the frames are loaded.
//
// Per frame (in event order) the reference masks the frame
// (ParMultiplyElementwise, IAC/ArrayOperators.h:118-125), then either
//   * adds it to the running intensity where it reaches the threshold
//     (ParAdd with threshold, IAC/ArrayOperators.h:75-86), zeroing values below
//     a positive threshold first, or
//   * discretises it to photons (DiscretizeToPhotones: ceilf((v - thr) / step)
//     for v >= thr, else 0) and adds (long)floor(v + 0.5) to a running integer
//     count per pixel,
// and sets the event's MeanIntensity = Sum(frame) / npix and, when
// discretising, PhotonCount = (int)Sum(frame), Sum being the sequential FP32
// sum in pixel order (IAC/ArrayOperators.h:259-267).  At the end the
// intensity is the running value (as float) times 1 / nframes.
//
// Two kernels reproduce this bit for bit:
//   average_pixels_kernel  thread per pixel, frames in event order (the
//                          per-pixel FP32 accumulation order of the reference);
//   frame_sums_kernel      a warp per 32 frames: each 32 x 32 tile of (frame,
//                          pixel) is loaded coalesced into shared memory and
//                          every lane adds its frame's 32 values in pixel
//                          order, so each frame's sum is the sequential one.
#include <algorithm>
#include <cmath>

#include "iac_internal.cuh"

namespace iac {

namespace {

// the processed value of one pixel of one frame (masking, thresholding or
// photon discretisation), exactly as the reference computes it
__device__ __forceinline__ float frame_value(float v, const int *__restrict__ mask, uint64_t j, float thr, float step)
{
    if (mask) v = fmul(v, (float)mask[j]);
    if (step > 0.0f) return v >= thr ? ceilf(__fdiv_rn(fsub(v, thr), step)) : 0.0f;
    if (thr > 0.0f && v < thr) return 0.0f;
    return v;
}

__global__ void average_pixels_kernel(const float *__restrict__ frames, uint64_t npix, uint32_t nframes,
                                      const int *__restrict__ mask, float thr, float step, float *__restrict__ sum,
                                      long long *__restrict__ discr)
{
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < npix; j += (uint64_t)gridDim.x * blockDim.x) {
        if (step > 0.0f) {
            long long acc = discr[j];
            for (uint32_t f = 0; f < nframes; f++) {
                const float raw = frames[(size_t)f * npix + j];
                const float m = mask ? fmul(raw, (float)mask[j]) : raw;
                if (m >= thr) {
                    const float t = ceilf(__fdiv_rn(fsub(m, thr), step));
                    acc += (long long)floor(dadd((double)t, 0.5));
                }
            }
            discr[j] = acc;
        } else {
            float acc = sum[j];
            for (uint32_t f = 0; f < nframes; f++) {
                const float t = frame_value(frames[(size_t)f * npix + j], mask, j, thr, step);
                if (t >= thr) acc = fadd(acc, t);
            }
            sum[j] = acc;
        }
    }
}

__global__ void __launch_bounds__(32) frame_sums_kernel(const float *__restrict__ frames, uint64_t npix,
                                                        uint32_t nframes, const int *__restrict__ mask, float thr,
                                                        float step, float *__restrict__ mean,
                                                        float *__restrict__ count)
{
    __shared__ float tile[32][33];
    const uint32_t f0 = blockIdx.x * 32;
    const int lane = threadIdx.x;
    float acc = 0.0f;
    for (uint64_t p0 = 0; p0 < npix; p0 += 32) {
        const uint64_t j = p0 + lane;
        for (int r = 0; r < 32; r++) {
            const uint32_t f = f0 + r;
            float v = 0.0f;
            if (f < nframes && j < npix) v = frame_value(frames[(size_t)f * npix + j], mask, j, thr, step);
            tile[r][lane] = v;
        }
        __syncwarp();
        const int n = npix - p0 < 32 ? (int)(npix - p0) : 32;
        for (int c = 0; c < n; c++) acc = fadd(acc, tile[lane][c]);
        __syncwarp();
    }
    const uint32_t f = f0 + lane;
    if (f < nframes) {
        mean[f] = __fdiv_rn(acc, (float)npix);
        if (count) count[f] = acc;
    }
}

__global__ void average_finish_kernel(const float *__restrict__ sum, const long long *__restrict__ discr,
                                      uint64_t npix, float scale, float *__restrict__ out)
{
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < npix; j += (uint64_t)gridDim.x * blockDim.x)
        out[j] = fmul(discr ? (float)discr[j] : sum[j], scale);
}

}  // namespace
}  // namespace iac

using namespace iac;

extern "C" {

iac_status iac_average_frames(iac_ctx *ctx, const float *d_frames, uint64_t npix, uint32_t nframes,
                              const int32_t *d_mask, float threshold, float step, float *d_sum,
                              int64_t *d_discr, float *d_mean_intensity, float *d_photon_sum, void *stream)
{
    IAC_REQUIRE(ctx && d_frames && d_mean_intensity, "iac_average_frames: NULL argument");
    IAC_REQUIRE(npix > 0 && nframes > 0, "iac_average_frames: empty batch");
    IAC_REQUIRE(step > 0.0f ? d_discr != nullptr : d_sum != nullptr,
                "iac_average_frames: step > 0 accumulates into d_discr, else into d_sum");
    DeviceGuard g(ctx->device);
    cudaStream_t s = as_stream(stream);
    const unsigned grid = (unsigned)std::min<uint64_t>((npix + 255) / 256, (uint64_t)ctx->sm_count * 16);
    average_pixels_kernel<<<grid, 256, 0, s>>>(d_frames, npix, nframes, d_mask, threshold, step, d_sum,
                                               reinterpret_cast<long long *>(d_discr));
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    frame_sums_kernel<<<(nframes + 31) / 32, 32, 0, s>>>(d_frames, npix, nframes, d_mask, threshold, step,
                                                         d_mean_intensity, step > 0.0f ? d_photon_sum : nullptr);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_average_finish(iac_ctx *ctx, const float *d_sum, const int64_t *d_discr, uint64_t npix,
                              uint32_t nframes_total, float *d_intensity, void *stream)
{
    IAC_REQUIRE(ctx && d_intensity && (d_sum || d_discr), "iac_average_finish: NULL argument");
    IAC_REQUIRE(nframes_total > 0, "iac_average_finish: no frames");
    DeviceGuard g(ctx->device);
    const float scale = 1.0f / ((float)nframes_total);
    const unsigned grid = (unsigned)std::min<uint64_t>((npix + 255) / 256, (uint64_t)ctx->sm_count * 16);
    average_finish_kernel<<<grid, 256, 0, as_stream(stream)>>>(d_sum, reinterpret_cast<const long long *>(d_discr),
                                                                npix, scale, d_intensity);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

}  // extern "C"
