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
// Bit for bit on the device:
//   average_pixels_kernel  thread per 4 pixels (or 1), frames in event order
//                          (the reference's per-pixel accumulation order);
//                          with photon discretisation it also forms every
//                          frame's exact integer photon total;
//   photon_means_kernel    MeanIntensity / PhotonCount from those totals: the
//                          values are integers, so while a frame's total stays
//                          below 2^24 its sequential FP32 sum is that total;
//   frame_sums_kernel      the sequential FP32 sum in pixel order, a lane per
//                          frame fed by warps that stream and process the
//                          pixels: for every frame without discretisation and
//                          for frames of 2^24 photons or more.
#include <algorithm>
#include <cmath>

#include "iac_internal.cuh"

namespace iac {

namespace {

// Per-pixel accumulation, a thread per W pixels (W = 4 with 16-byte aligned
// rows, else 1), frames in event order, PIX_FB frames' loads in flight per
// thread and enough resident warps (<= 64 registers) for the whole grid to
// run in one wave.  PHOTON also forms every frame's exact photon total over
// the pixels: the counts are integers, taken exactly from their floats while
// below 2^23 (clamped to 2^24 above, which only has to push the total past
// 2^24); per batch a transposing butterfly over the warp leaves frame k's warp
// total in lanes 4k..4k+3, and the block's totals are added to total[] once
// per 32 frames.  POW2: step is a power of two and q * inv_step equals
// q / step exactly.  The per-element work is branch-free.
constexpr int PIX_THREADS = 128, PIX_FB = 8;

template <bool VEC, bool PHOTON, bool POW2>
__global__ void __launch_bounds__(PIX_THREADS, 8) average_pixels_kernel(
    const float *__restrict__ frames, uint64_t npix, uint32_t nframes, const int *__restrict__ mask, float thr,
    float step, float inv_step, float *__restrict__ sum, long long *__restrict__ discr,
    unsigned long long *__restrict__ total)
{
    constexpr int W = VEC ? 4 : 1;
    __shared__ uint32_t part[PIX_THREADS / 32][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t g = blockIdx.x * (uint64_t)PIX_THREADS + threadIdx.x;
    const bool live = g < npix / W;
    const uint64_t j = live ? g * W : 0;
    float mk[W], facc[W];
    long long dacc[W];
#pragma unroll
    for (int e = 0; e < W; e++) {
        mk[e] = mask && live ? (float)mask[j + e] : 1.0f;
        if constexpr (PHOTON) dacc[e] = live ? discr[j + e] : 0;
        else facc[e] = live ? sum[j + e] : 0.0f;
    }
#pragma unroll 1
    for (uint32_t f0 = 0; f0 < nframes; f0 += PIX_FB) {
        float v[PIX_FB][W];
#pragma unroll
        for (int k = 0; k < PIX_FB; k++) {
            const bool in = live && f0 + k < nframes;
            const float *src = frames + (size_t)(in ? f0 + k : 0) * npix + j;
            if constexpr (VEC) {
                const float4 x = in ? __ldcs(reinterpret_cast<const float4 *>(src)) : make_float4(0.f, 0.f, 0.f, 0.f);
                v[k][0] = x.x, v[k][1] = x.y, v[k][2] = x.z, v[k][3] = x.w;
            } else {
                v[k][0] = in ? __ldcs(src) : 0.0f;
            }
        }
        uint32_t fr[PIX_FB];
        int bacc[W];  // this batch's counts, each below 2^23
#pragma unroll
        for (int e = 0; e < W; e++) bacc[e] = 0;
#pragma unroll
        for (int k = 0; k < PIX_FB; k++) {
            const bool in = live && f0 + k < nframes;
            fr[k] = 0;
#pragma unroll
            for (int e = 0; e < W; e++) {
                const float m = mask ? fmul(v[k][e], mk[e]) : v[k][e];
                if constexpr (PHOTON) {
                    const float q = fsub(m, thr);
                    float t = ceilf(POW2 ? fmul(q, inv_step) : __fdiv_rn(q, step));
                    // t is integer-valued and >= 0 where counted, so
                    // (long)floor((double)t + 0.5), the reference's rounding, is t
                    t = (in && m >= thr) ? t : 0.0f;
                    const int it = __float_as_int(fadd(fminf(t, 8388607.0f), 8388608.0f)) - 0x4B000000;
                    bacc[e] += it;
                    fr[k] += (uint32_t)it;
                    if (t >= 8388608.0f) {  // rare: the exact count and a total past 2^24
                        dacc[e] += (long long)t - it;
                        fr[k] += (1u << 24) - (uint32_t)it;
                    }
                } else {
                    const float t = (thr > 0.0f && m < thr) ? 0.0f : m;
                    facc[e] = (in && t >= thr) ? fadd(facc[e], t) : facc[e];
                }
            }
        }
        if constexpr (PHOTON) {
#pragma unroll
            for (int e = 0; e < W; e++) dacc[e] += bacc[e];
            // 8 frames x 32 lanes -> frame k's warp total in lanes 4k..4k+3
            const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
            uint32_t a4[4], a2[2];
#pragma unroll
            for (int i = 0; i < 4; i++)
                a4[i] = (h16 ? fr[i + 4] : fr[i]) + __shfl_xor_sync(0xffffffffu, h16 ? fr[i] : fr[i + 4], 16);
#pragma unroll
            for (int i = 0; i < 2; i++)
                a2[i] = (h8 ? a4[i + 2] : a4[i]) + __shfl_xor_sync(0xffffffffu, h8 ? a4[i] : a4[i + 2], 8);
            uint32_t a1 = (h4 ? a2[1] : a2[0]) + __shfl_xor_sync(0xffffffffu, h4 ? a2[0] : a2[1], 4);
            a1 += __shfl_xor_sync(0xffffffffu, a1, 2);
            a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
            if ((lane & 3) == 0) part[warp][(f0 + (lane >> 2)) & 31] = a1;
            if (((f0 + PIX_FB) & 31) == 0 || f0 + PIX_FB >= nframes) {
                __syncthreads();
                const uint32_t f = (f0 & ~31u) + threadIdx.x;
                if (threadIdx.x < 32 && f < nframes) {
                    unsigned long long t = 0;
#pragma unroll
                    for (int w = 0; w < PIX_THREADS / 32; w++) t += part[w][threadIdx.x];
                    atomicAdd(&total[f], t);
                }
                __syncthreads();
            }
        }
    }
    if (live) {
#pragma unroll
        for (int e = 0; e < W; e++) {
            if constexpr (PHOTON) discr[j + e] = dacc[e];
            else sum[j + e] = facc[e];
        }
    }
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}
// bounded wait: false after 2^20 polls, each of which suspends for a bounded time
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity)
{
    for (uint32_t i = 0; i < (1u << 20); i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Sequential per-frame FP32 sums of FPC frames per CTA.  Warp SUM_WARP sums:
// lane i < FPC adds frame f0 + i's processed values in pixel order, one
// dependent add per pixel, which is the reference's sequential sum and the
// bound of the kernel.  The four warps before it keep that chain fed: each
// thread owns FPC / 4 frame rows x one 16-byte granule (VEC) or 4 scalar
// columns of every 128-pixel chunk, copies them (and the matching mask
// entries) with cp.async
// SUM_RAW - 1 chunks ahead into a raw ring, processes what it copied itself
// (mask, threshold or photon discretisation, exactly as the reference) and
// stores the results into a ring of SUM_COOKED processed chunks, handed to
// the summing warp through mbarriers (bounded waits).  Rows are padded to
// SUM_PITCH floats so that every access pattern is free of bank conflicts.
// Each lane's frame streams through its own DRAM pages, so few frames per CTA
// spread the streams over many SMs (FPC is chosen for the grid to cover them).
constexpr int SUM_COLS = 128, SUM_PITCH = SUM_COLS + 4, SUM_RAW = 7, SUM_COOKED = 4, SUM_WARP = 4;
template <int FPC>
struct SumCfg {
    static constexpr int RAW_FLOATS = (FPC + SUM_WARP) * SUM_PITCH;  // frame rows + one mask row per copying warp
    static constexpr int COOKED_FLOATS = FPC * SUM_PITCH;
    static constexpr size_t SMEM = (size_t)(SUM_RAW * RAW_FLOATS + SUM_COOKED * COOKED_FLOATS) * 4 + 2 * SUM_COOKED * 8;
};

template <bool VEC, int FPC>
__global__ void __launch_bounds__(32 * (SUM_WARP + 1)) frame_sums_kernel(
    const float *__restrict__ frames, uint64_t npix, uint32_t nframes, const int *__restrict__ mask, float thr,
    float step, const int *__restrict__ only, float *__restrict__ mean, float *__restrict__ count,
    DeviceCounters *ctr)
{
    using C = SumCfg<FPC>;
    constexpr int RPW = FPC / SUM_WARP;  // frame rows per copying thread
    extern __shared__ __align__(16) float ring[];
    float *raw = ring;
    float *cooked = ring + SUM_RAW * C::RAW_FLOATS;
    const uint32_t bars = smem_addr(cooked + SUM_COOKED * C::COOKED_FLOATS);  // full[SUM_COOKED], empty[SUM_COOKED]
    __shared__ int s_err;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t f0 = blockIdx.x * FPC;
    {
        const uint32_t f = f0 + lane;
        const int need = warp == 0 && lane < FPC && f < nframes && (!only || only[f]);
        if (!__syncthreads_or(need)) return;
    }
    if (threadIdx.x == 0) {
        s_err = 0;
        for (int c = 0; c < SUM_COOKED; c++) {
            mbar_init(bars + 8 * c, 32 * SUM_WARP);                 // full: every processing thread
            mbar_init(bars + 8 * (SUM_COOKED + c), 32);             // empty: every summing lane
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const uint64_t nch = (npix + SUM_COLS - 1) / SUM_COLS;
    bool ok = true;
    if (warp < SUM_WARP) {
        const int r0 = RPW * warp;
        auto issue = [&](uint64_t ch) {
            if (ch < nch) {
                float *st = raw + (ch % SUM_RAW) * C::RAW_FLOATS;
                const uint64_t p0 = ch * SUM_COLS;
#pragma unroll
                for (int i = 0; i <= RPW; i++) {
                    // rows r0..r0+RPW-1: frames f0 + r; the last: this warp's mask row
                    const int r = i < RPW ? r0 + i : FPC + warp;
                    const bool live = i < RPW ? f0 + r < nframes : mask != nullptr;
                    const float *row = i < RPW ? frames + (size_t)(live ? f0 + r : 0) * npix : (const float *)mask;
                    if constexpr (VEC) {
                        const uint64_t j = p0 + 4 * lane;
                        const bool in = live && j < npix;  // npix % 4 == 0: a granule is whole or absent
                        cp_async16(smem_addr(st + r * SUM_PITCH + 4 * lane), in ? (const void *)(row + j) : frames,
                                   in ? 16u : 0u);
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const uint64_t j = p0 + 32 * q + lane;
                            const bool in = live && j < npix;
                            cp_async4(smem_addr(st + r * SUM_PITCH + 32 * q + lane),
                                      in ? (const void *)(row + j) : frames, in ? 4u : 0u);
                        }
                    }
                }
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        };
        auto process = [&](float t, float m) {
            if (mask) t = fmul(t, m);
            if (step > 0.0f) return t >= thr ? ceilf(__fdiv_rn(fsub(t, thr), step)) : 0.0f;
            return (thr > 0.0f && t < thr) ? 0.0f : t;
        };
#pragma unroll 1
        for (int k = 0; k < SUM_RAW - 1; k++) issue(k);
#pragma unroll 1
        for (uint64_t ch = 0; ch < nch; ch++) {
            asm volatile("cp.async.wait_group %0;\n" ::"n"(SUM_RAW - 2) : "memory");  // own copies of chunk ch
            const int c = (int)(ch % SUM_COOKED);
            if (ch >= SUM_COOKED && !mbar_wait(bars + 8 * (SUM_COOKED + c), (uint32_t)(ch / SUM_COOKED - 1) & 1)) {
                ok = false;
                break;
            }
            const float *st = raw + (ch % SUM_RAW) * C::RAW_FLOATS;
            float *out = cooked + c * C::COOKED_FLOATS;
            if constexpr (VEC) {
                float4 m = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                if (mask) {
                    const int4 mi = *reinterpret_cast<const int4 *>(st + (FPC + warp) * SUM_PITCH + 4 * lane);
                    m = make_float4((float)mi.x, (float)mi.y, (float)mi.z, (float)mi.w);
                }
#pragma unroll
                for (int i = 0; i < RPW; i++) {
                    const float4 v = *reinterpret_cast<const float4 *>(st + (r0 + i) * SUM_PITCH + 4 * lane);
                    *reinterpret_cast<float4 *>(out + (r0 + i) * SUM_PITCH + 4 * lane) =
                        make_float4(process(v.x, m.x), process(v.y, m.y), process(v.z, m.z), process(v.w, m.w));
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float m = mask ? (float)__float_as_int(st[(FPC + warp) * SUM_PITCH + 32 * q + lane]) : 1.0f;
#pragma unroll
                    for (int i = 0; i < RPW; i++)
                        out[(r0 + i) * SUM_PITCH + 32 * q + lane] = process(st[(r0 + i) * SUM_PITCH + 32 * q + lane], m);
                }
            }
            mbar_arrive(bars + 8 * c);
            issue(ch + SUM_RAW - 1);  // into the raw stage of chunk ch - 1, read by this thread alone
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    } else {
        float acc = 0.0f;
#pragma unroll 1
        for (uint64_t ch = 0; ch < nch; ch++) {
            const int c = (int)(ch % SUM_COOKED);
            if (!mbar_wait(bars + 8 * c, (uint32_t)(ch / SUM_COOKED) & 1)) {
                ok = false;
                break;
            }
            const float4 *row = reinterpret_cast<const float4 *>(cooked + c * C::COOKED_FLOATS + lane * SUM_PITCH);
            const uint64_t p0 = ch * SUM_COLS;
            if (lane >= FPC) {
            } else if (npix - p0 >= (uint64_t)SUM_COLS) {
#pragma unroll
                for (int g = 0; g < SUM_COLS / 4; g++) {
                    const float4 v = row[g];
                    acc = fadd(fadd(fadd(fadd(acc, v.x), v.y), v.z), v.w);
                }
            } else {
                const float *rs = reinterpret_cast<const float *>(row);
                for (int k = 0; k < (int)(npix - p0); k++) acc = fadd(acc, rs[k]);
            }
            mbar_arrive(bars + 8 * (SUM_COOKED + c));
        }
        const uint32_t f = f0 + lane;
        if (ok && lane < FPC && f < nframes && (!only || only[f])) {
            mean[f] = __fdiv_rn(acc, (float)npix);
            if (count) count[f] = acc;
        }
    }
    if (!ok) s_err = 1;
    __syncthreads();
    if (threadIdx.x == 0 && s_err) note_timeout(ctr, SITE_AVERAGE);
}

__global__ void photon_means_kernel(const unsigned long long *__restrict__ total, uint32_t nframes, uint64_t npix,
                                    float *__restrict__ mean, float *__restrict__ count, int *__restrict__ redo)
{
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nframes) return;
    const unsigned long long t = total[f];
    const bool exact = t < (1ull << 24);
    redo[f] = exact ? 0 : 1;
    if (exact) {
        const float s = (float)t;
        mean[f] = __fdiv_rn(s, (float)npix);
        if (count) count[f] = s;
    }
}

__global__ void average_finish_kernel(const float *__restrict__ sum, const long long *__restrict__ discr,
                                      uint64_t npix, float scale, float *__restrict__ out)
{
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < npix; j += (uint64_t)gridDim.x * blockDim.x)
        out[j] = fmul(discr ? (float)discr[j] : sum[j], scale);
}

template <bool VEC, int FPC>
iac_status launch_sums(const float *frames, uint64_t npix, uint32_t nframes, const int *mask, float thr, float step,
                       const int *only, float *mean, float *count, DeviceCounters *ctr, cudaStream_t s)
{
    const size_t smem = SumCfg<FPC>::SMEM;
    IAC_CUDA(cudaFuncSetAttribute(frame_sums_kernel<VEC, FPC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    frame_sums_kernel<VEC, FPC><<<(nframes + FPC - 1) / FPC, 32 * (SUM_WARP + 1), smem, s>>>(
        frames, npix, nframes, mask, thr, step, only, mean, count, ctr);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

template <bool VEC>
iac_status launch_sums_fpc(int sms, const float *frames, uint64_t npix, uint32_t nframes, const int *mask, float thr,
                           float step, const int *only, float *mean, float *count, DeviceCounters *ctr,
                           cudaStream_t s)
{
    // the most frames per CTA (at most 32, at least 4) that still give every SM a CTA
    if (nframes >= 32u * sms) return launch_sums<VEC, 32>(frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s);
    if (nframes >= 16u * sms) return launch_sums<VEC, 16>(frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s);
    if (nframes >= 8u * sms) return launch_sums<VEC, 8>(frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s);
    return launch_sums<VEC, 4>(frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s);
}

iac_status launch_frame_sums(int sms, const float *frames, uint64_t npix, uint32_t nframes, const int *mask,
                             float thr, float step, const int *only, float *mean, float *count, DeviceCounters *ctr,
                             cudaStream_t s)
{
    const bool vec = npix % 4 == 0 && ((uintptr_t)frames & 15) == 0 && ((uintptr_t)mask & 15) == 0;
    return vec ? launch_sums_fpc<true>(sms, frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s)
               : launch_sums_fpc<false>(sms, frames, npix, nframes, mask, thr, step, only, mean, count, ctr, s);
}

}  // namespace
}  // namespace iac

using namespace iac;

extern "C" {

iac_status iac_average_frames(iac_ctx *ctx, const float *d_frames, uint64_t npix, uint32_t nframes,
                              const int32_t *d_mask, float threshold, float step, float *d_sum,
                              int64_t *d_discr, float *d_mean_intensity, float *d_photon_sum, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_frames && d_mean_intensity, "iac_average_frames: NULL argument");
    IAC_REQUIRE(npix > 0 && nframes > 0, "iac_average_frames: empty batch");
    IAC_REQUIRE(step > 0.0f ? d_discr != nullptr : d_sum != nullptr,
                "iac_average_frames: step > 0 accumulates into d_discr, else into d_sum");
    DeviceGuard g(ctx->device);
    cudaStream_t s = as_stream(stream);
    const bool vec = npix % 4 == 0 && ((uintptr_t)d_frames & 15) == 0;
    const uint64_t threads = vec ? npix / 4 : npix;
    IAC_REQUIRE(threads <= (uint64_t)PIX_THREADS * 0x7fffffffull, "iac_average_frames: too many pixels");
    const unsigned grid = (unsigned)((threads + PIX_THREADS - 1) / PIX_THREADS);
    long long *discr = reinterpret_cast<long long *>(d_discr);
    // a power-of-two step 2^k (|k| <= 126): dividing by it and multiplying by
    // 2^-k round the same real number
    int ex = 0;
    const float mant = step > 0.0f ? std::frexp(step, &ex) : 0.0f;
    const float inv_step = (mant == 0.5f && ex >= -125 && ex <= 127) ? std::ldexp(1.0f, 1 - ex) : 0.0f;
    if (step > 0.0f) {
        // exact integer photon totals per frame, formed with the per-pixel counts;
        // frames of 2^24 photons or more get the sequential sum in pixel order
        void *scratch = nullptr;
        const size_t tb = ((size_t)nframes * 8 + 255) & ~(size_t)255;
        iac_status st = stream_scratch(ctx, stream, SLOT_AUX0, tb + 4 * (size_t)nframes, &scratch);
        if (st != IAC_OK) return st;
        unsigned long long *total = (unsigned long long *)scratch;
        int *redo = (int *)((char *)scratch + tb);
        IAC_CUDA(cudaMemsetAsync(total, 0, 8 * (size_t)nframes, s));
        auto kern = vec ? (inv_step != 0.0f ? average_pixels_kernel<true, true, true> : average_pixels_kernel<true, true, false>)
                        : (inv_step != 0.0f ? average_pixels_kernel<false, true, true>
                                            : average_pixels_kernel<false, true, false>);
        kern<<<grid, PIX_THREADS, 0, s>>>(d_frames, npix, nframes, d_mask, threshold, step, inv_step, d_sum, discr,
                                          total);
        IAC_LAUNCHED(ctx);
        IAC_CUDA(cudaGetLastError());
        photon_means_kernel<<<(nframes + 127) / 128, 128, 0, s>>>(total, nframes, npix, d_mean_intensity,
                                                                 d_photon_sum, redo);
        IAC_LAUNCHED(ctx);
        IAC_CUDA(cudaGetLastError());
        // frames of 2^24 photons or more: the sequential sum in pixel order
        st = launch_frame_sums(ctx->sm_count, d_frames, npix, nframes, d_mask, threshold, step, redo, d_mean_intensity,
                               d_photon_sum, ctx->d_counters, s);
        if (st != IAC_OK) return st;
        IAC_LAUNCHED(ctx);
    } else {
        auto kern = vec ? average_pixels_kernel<true, false, false> : average_pixels_kernel<false, false, false>;
        kern<<<grid, PIX_THREADS, 0, s>>>(d_frames, npix, nframes, d_mask, threshold, step, 0.0f, d_sum, discr,
                                          nullptr);
        IAC_LAUNCHED(ctx);
        IAC_CUDA(cudaGetLastError());
        iac_status st = launch_frame_sums(ctx->sm_count, d_frames, npix, nframes, d_mask, threshold, step, nullptr,
                                          d_mean_intensity, nullptr, ctx->d_counters, s);
        if (st != IAC_OK) return st;
        IAC_LAUNCHED(ctx);
    }
    return IAC_OK;
}

iac_status iac_average_finish(iac_ctx *ctx, const float *d_sum, const int64_t *d_discr, uint64_t npix,
                              uint32_t nframes_total, float *d_intensity, void *stream)
{
    IAC_TRACE();
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
