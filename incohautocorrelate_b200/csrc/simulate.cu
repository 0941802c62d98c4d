// simulate.cu -- (d) the Simulator's emitter-phase intensity sum, photon
// statistics and device-side photonisation, batched over frames.
//
// Replaces Simulator::SimulatePart (IAC/Simulator.cpp:662-944) with its kernel
// SimulateCrystal (IAC/kernel.cl:768-859), Crystal::GetEmitters
// (IAC/Crystal.cpp:29-184), ArrayOperators::ScalarPoissonSampling
// (IAC/ArrayOperators.h:25-55) and Detector::CreateSparseHitList
// (IAC/Detector.cpp:926-977), so that simulated frames reach the pair
// correlator without leaving the GPU.
//
//  crystal_emitters_kernel   one CTA per (frame, mode): the frame's random
//                            orientation (axis uniform in the unit ball scaled
//                            by the isotropy, angle uniform), the rotated atom
//                            positions, per-mode fluorescence roll and phases;
//                            the event matrix is the inverse rotation.
//  simulate_kernel           one thread per pixel, grid over (pixels, frames):
//                            per mode and sub-pixel, Psi = sum_j exp(i(k.r_j +
//                            phi_j)) with the phase argument formed in FP32 in
//                            the reference's order, then |Psi| (reference) or
//                            |Psi|^2 summed over modes as the host does.
//  frame_sum_kernel          per-frame integrated intensity (double).
//  photon_kernel             rescale to the expected photon number, Poisson
//                            draw (inversion below 25, clipped Box-Muller above),
//                            optional ADU noise, value per photon.
//  sparsify_*                stream compaction of photon frames into the
//                            (k, count) photon lists of the pair correlator,
//                            pixel order kept.
//
// Sine and cosine: the phase argument (|arg| up to ~10^2 rad) is reduced to
// [-pi, pi] explicitly with a two-word Cody-Waite split of 2*pi (the split is
// computed from pi in double below) and evaluated with the SFU's __sincosf, or
// (accurate mode) with sincosf.  Accuracy against an FP64 evaluation is
// measured by the tests.
#include <algorithm>
#include <cmath>

#include "iac_internal.cuh"
#include "rng.cuh"

namespace iac {

constexpr double TWO_PI_D = 6.283185307179586476925286766559;
constexpr float TWO_PI_HI = (float)TWO_PI_D;
constexpr float TWO_PI_LO = (float)(TWO_PI_D - (double)TWO_PI_HI);
constexpr float INV_TWO_PI = (float)(1.0 / TWO_PI_D);

// the whole number of turns in a phase, rintf(arg / 2 pi) with ties to even, by
// two FP32 adds on the FMA pipe: x + 1.5 * 2^23 rounds x to an integer in the
// float's last place for |x| < 2^22 (phases below 2.6e7 rad; past that an FP32
// phase has lost every fraction of a turn anyway).  rintf is a conversion-unit
// instruction, and that unit also runs the two MUFU operations of every term,
// which bound the simulator.
__device__ __forceinline__ float phase_turns(float arg)
{
    return fsub(fadd(fmul(arg, INV_TWO_PI), ROUND_MAGIC), ROUND_MAGIC);
}

struct CrystalArgs {
    const double *__restrict__ atoms;  // 3 doubles per atom
    uint32_t natoms, nframes, nmodes;
    uint64_t seed;
    float yield;
    float isotropy;
    int rand_orientation;
    int incoherent;
    float4 *__restrict__ em;        // [frame][mode][atom] (x, y, z, phase)
    uint32_t *__restrict__ em_count;  // [frame][mode]
    float *__restrict__ rot_event;  // 9 per frame (inverse of the crystal rotation)
    float *__restrict__ rot_crystal;  // 9 per frame (may be null)
};

// Crystal::RotateVectors matrix (IAC/Crystal.cpp:125-157) in double.
__device__ void axis_angle(double alpha, double ax0, double ax1, double ax2, double m[9])
{
    const double N = sqrt(ax0 * ax0 + ax1 * ax1 + ax2 * ax2);
    ax0 /= N;
    ax1 /= N;
    ax2 /= N;
    const double c = cos(alpha), s = sin(alpha);
    m[0] = ax0 * ax0 * (1 - c) + c;
    m[1] = ax1 * ax0 * (1 - c) - ax2 * s;
    m[2] = ax2 * ax0 * (1 - c) + ax1 * s;
    m[3] = ax0 * ax1 * (1 - c) + ax2 * s;
    m[4] = ax1 * ax1 * (1 - c) + c;
    m[5] = ax2 * ax1 * (1 - c) - ax0 * s;
    m[6] = ax0 * ax2 * (1 - c) - ax1 * s;
    m[7] = ax1 * ax2 * (1 - c) + ax0 * s;
    m[8] = ax2 * ax2 * (1 - c) + c;
}

__global__ void crystal_emitters_kernel(const CrystalArgs a)
{
    const uint32_t f = blockIdx.x / a.nmodes, mode = blockIdx.x % a.nmodes;
    __shared__ double s_m[9];
    __shared__ uint32_t s_count;
    if (threadIdx.x == 0) {
        double m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (a.rand_orientation) {
            // IAC/Crystal.cpp:53-69: axis uniform in the unit ball (rejection,
            // bounded; the acceptance rate is pi/6), angle uniform in [0, 2 pi)
            double v0 = 0, v1 = 0, v2 = 1;
            for (uint32_t t = 0; t < 256; t++) {
                double u0, u1, u2, u3;
                uniform2(a.seed, RNG_ROTATION | f, 2 * (uint64_t)t, u0, u1);
                uniform2(a.seed, RNG_ROTATION | f, 2 * (uint64_t)t + 1, u2, u3);
                v0 = u0 * 2. - 1.;
                v1 = (u1 * 2. - 1.) * a.isotropy;
                v2 = (u2 * 2. - 1.) * a.isotropy;
                if (!(v0 * v0 + v1 * v1 + v2 * v2 > 1) && (v0 != 0 || v1 != 0 || v2 != 0)) break;
            }
            double ua, ub;
            uniform2(a.seed, RNG_ROTATION | f, 1u << 20, ua, ub);
            axis_angle(ua * 2 * 3.14159265358979323846, v0, v1, v2, m);
        }
        // the crystal matrix is kept in float, as the reference's array<float,9>
        float R[9];
        for (int k = 0; k < 9; k++) R[k] = (float)m[k];
        for (int k = 0; k < 9; k++) s_m[k] = m[k];
        if (mode == 0) {
            // event matrix = inverse of the float crystal matrix, in double
            const double A = R[0], B = R[1], C = R[2], D = R[3], E = R[4], F = R[5], G = R[6],
                         H = R[7], I = R[8];
            const double c0 = E * I - F * H, c1 = -(D * I - F * G), c2 = D * H - E * G;
            const double det = A * c0 + B * c1 + C * c2;
            float *o = a.rot_event + 9 * (size_t)f;
            o[0] = (float)(c0 / det);
            o[1] = (float)(-(B * I - C * H) / det);
            o[2] = (float)((B * F - C * E) / det);
            o[3] = (float)(c1 / det);
            o[4] = (float)((A * I - C * G) / det);
            o[5] = (float)(-(A * F - C * D) / det);
            o[6] = (float)(c2 / det);
            o[7] = (float)(-(A * H - B * G) / det);
            o[8] = (float)((A * E - B * D) / det);
            if (a.rot_crystal)
                for (int k = 0; k < 9; k++) a.rot_crystal[9 * (size_t)f + k] = R[k];
        }
        s_count = 0;
    }
    __syncthreads();
    const size_t base = ((size_t)f * a.nmodes + mode) * a.natoms;
    // atoms kept with probability FlYield (IAC/Crystal.cpp:35-43), in order
    for (uint32_t i0 = 0; i0 < a.natoms; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        bool keep = false;
        double phase = 0.0;
        if (i < a.natoms) {
            keep = true;
            if (a.yield < 1.0f) {
                double y0, y1;
                uniform2(a.seed, RNG_YIELD | ((uint64_t)mode << 32) | f, i, y0, y1);
                keep = y0 <= (double)a.yield;
            }
            if (a.incoherent) {
                double p0, p1;
                uniform2(a.seed, RNG_PHASE | ((uint64_t)mode << 32) | f, i, p0, p1);
                phase = p0 * 2.0 * 3.14159265358979323846;
            }
        }
        // order-preserving compaction within the chunk
        const unsigned ball = __ballot_sync(0xffffffffu, keep);
        __shared__ uint32_t s_w[32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) s_w[w] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = s_count;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
                const uint32_t c = s_w[k];
                s_w[k] = t;
                t += c;
            }
            s_count = t;
        }
        __syncthreads();
        if (keep) {
            const double *p = a.atoms + 3 * (size_t)i;
            const double x = s_m[0] * p[0] + s_m[1] * p[1] + s_m[2] * p[2];
            const double y = s_m[3] * p[0] + s_m[4] * p[1] + s_m[5] * p[2];
            const double z = s_m[6] * p[0] + s_m[7] * p[1] + s_m[8] * p[2];
            a.em[base + s_w[w] + __popc(ball & ((1u << lane) - 1))] =
                make_float4((float)x, (float)y, (float)z, (float)phase);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) a.em_count[(size_t)f * a.nmodes + mode] = s_count;
}

struct SimArgs {
    const float *__restrict__ pm;  // pixel map, 3 floats per pixel
    const float4 *__restrict__ em;
    const uint32_t *__restrict__ em_count;
    uint64_t npix;
    uint32_t natoms, nmodes, nframes;
    int susa;
    float us[3], vs[3];
    float wavelength;
    int amplitude_sq;  // 0: |Psi| as the reference, 1: |Psi|^2
    int accurate;      // 1: sincosf instead of explicit reduction + SFU
    float *__restrict__ out;  // [frame][pixel]
};

constexpr int SIM_THREADS = 128;
constexpr int SIM_MAX_EM = 1024;  // emitters per (frame, mode) staged in shared memory

// pixels per thread of simulate_kernel: pixels p and p + SIM_THREADS share
// every emitter load and the loop overhead; each pixel's sums keep their order
constexpr int SIM_PIX = 2;

__global__ void __launch_bounds__(SIM_THREADS) simulate_kernel(const SimArgs a)
{
    extern __shared__ float4 s_em[];  // [mode][SIM_MAX_EM window]
    const uint32_t f = blockIdx.y;
    const uint64_t p0 = blockIdx.x * (uint64_t)(SIM_PIX * SIM_THREADS) + threadIdx.x;
    const uint32_t ncap = min(a.natoms, (uint32_t)SIM_MAX_EM);
    for (uint32_t m = 0; m < a.nmodes; m++) {
        const uint32_t n = min(a.em_count[(size_t)f * a.nmodes + m], ncap);
        const float4 *src = a.em + ((size_t)f * a.nmodes + m) * a.natoms;
        for (uint32_t i = threadIdx.x; i < n; i += SIM_THREADS) s_em[m * ncap + i] = src[i];
    }
    __syncthreads();
    if (p0 >= a.npix) return;
    uint64_t px[SIM_PIX];
    float pc[SIM_PIX][3];
#pragma unroll
    for (int q = 0; q < SIM_PIX; q++) {
        px[q] = p0 + (uint64_t)q * SIM_THREADS;
        const uint64_t pp = px[q] < a.npix ? px[q] : p0;  // a pixel past the end repeats p0, unwritten
#pragma unroll
        for (int d = 0; d < 3; d++) pc[q][d] = a.pm[3 * pp + d];
    }
    const float nsub = (float)((2 * a.susa + 1) * (2 * a.susa + 1));
    float total[SIM_PIX];
#pragma unroll
    for (int q = 0; q < SIM_PIX; q++) total[q] = 0.0f;
    for (uint32_t m = 0; m < a.nmodes; m++) {
        const uint32_t n = min(a.em_count[(size_t)f * a.nmodes + m], ncap);
        const float4 *E = s_em + m * ncap;
        float acc[SIM_PIX];
#pragma unroll
        for (int q = 0; q < SIM_PIX; q++) acc[q] = 0.0f;
        for (int v = -a.susa; v <= a.susa; v++)
            for (int u = -a.susa; u <= a.susa; u++) {
                float k[SIM_PIX][3], re[SIM_PIX], im[SIM_PIX];
#pragma unroll
                for (int q = 0; q < SIM_PIX; q++) {
                    // IAC/kernel.cl:823-832
                    const float c0 = fadd(fadd(pc[q][0], fmul((float)v, a.vs[0])), fmul((float)u, a.us[0]));
                    const float c1 = fadd(fadd(pc[q][1], fmul((float)v, a.vs[1])), fmul((float)u, a.us[1]));
                    const float c2 = fadd(fadd(pc[q][2], fmul((float)v, a.vs[2])), fmul((float)u, a.us[2]));
                    float nk = (float)(1.0 / (double)norm3(c0, c1, c2));
                    nk = (float)((double)nk * ((2.0 * 3.1415926535897932) / (double)a.wavelength));
                    k[q][0] = fmul(c0, nk);
                    k[q][1] = fmul(c1, nk);
                    k[q][2] = fmul(c2, nk);
                    re[q] = 0.0f;
                    im[q] = 0.0f;
                }
                for (uint32_t i = 0; i < n; i++) {
                    const float4 e = E[i];
#pragma unroll
                    for (int q = 0; q < SIM_PIX; q++) {
                        float arg = fmul(k[q][0], e.x);
                        arg = fadd(arg, fmul(k[q][1], e.y));
                        arg = fadd(arg, fmul(k[q][2], e.z));
                        arg = fadd(arg, e.w);
                        float sn, cs;
                        if (a.accurate) {
                            sincosf(arg, &sn, &cs);
                        } else {
                            const float kk = phase_turns(arg);
                            const float r = fmaf(-kk, TWO_PI_LO, fmaf(-kk, TWO_PI_HI, arg));
                            __sincosf(r, &sn, &cs);
                        }
                        re[q] = fadd(re[q], cs);
                        im[q] = fadd(im[q], sn);
                    }
                }
#pragma unroll
                for (int q = 0; q < SIM_PIX; q++) {
                    const float a2 = fadd(fmul(re[q], re[q]), fmul(im[q], im[q]));
                    acc[q] = fadd(acc[q], a.amplitude_sq ? a2 : __fsqrt_rn(a2));
                }
            }
#pragma unroll
        for (int q = 0; q < SIM_PIX; q++) total[q] = fadd(total[q], __fdiv_rn(acc[q], nsub));  // as ParAdd sums modes
    }
#pragma unroll
    for (int q = 0; q < SIM_PIX; q++)
        if (px[q] < a.npix) a.out[(size_t)f * a.npix + px[q]] = total[q];
}

// simulate_kernel for crystals whose emitters do not fit the shared-memory
// stage (more than SIM_MAX_EM, or modes x emitters past 200 KB): per mode and
// sub-pixel the emitters stream through a stage of SIM_MAX_EM, chunk by chunk
// in emitter order, so every pixel's phase sum adds the same terms in the same
// order as the staged kernel
__global__ void __launch_bounds__(SIM_THREADS) simulate_chunked_kernel(const SimArgs a)
{
    __shared__ float4 s_em[SIM_MAX_EM];
    const uint32_t f = blockIdx.y;
    const uint64_t p = blockIdx.x * (uint64_t)SIM_THREADS + threadIdx.x;
    const bool live = p < a.npix;
    const float pc0 = live ? a.pm[3 * p] : 0.0f, pc1 = live ? a.pm[3 * p + 1] : 0.0f,
                pc2 = live ? a.pm[3 * p + 2] : 0.0f;
    const float nsub = (float)((2 * a.susa + 1) * (2 * a.susa + 1));
    float total = 0.0f;
    for (uint32_t m = 0; m < a.nmodes; m++) {
        const uint32_t n = min(a.em_count[(size_t)f * a.nmodes + m], a.natoms);
        const float4 *src = a.em + ((size_t)f * a.nmodes + m) * a.natoms;
        float acc = 0.0f;
        for (int v = -a.susa; v <= a.susa; v++)
            for (int u = -a.susa; u <= a.susa; u++) {
                const float c0 = fadd(fadd(pc0, fmul((float)v, a.vs[0])), fmul((float)u, a.us[0]));
                const float c1 = fadd(fadd(pc1, fmul((float)v, a.vs[1])), fmul((float)u, a.us[1]));
                const float c2 = fadd(fadd(pc2, fmul((float)v, a.vs[2])), fmul((float)u, a.us[2]));
                float nk = live ? (float)(1.0 / (double)norm3(c0, c1, c2)) : 0.0f;
                nk = (float)((double)nk * ((2.0 * 3.1415926535897932) / (double)a.wavelength));
                const float k0 = fmul(c0, nk), k1 = fmul(c1, nk), k2 = fmul(c2, nk);
                float re = 0.0f, im = 0.0f;
                for (uint32_t c = 0; c < n; c += SIM_MAX_EM) {
                    const uint32_t cn = min(n - c, (uint32_t)SIM_MAX_EM);
                    __syncthreads();  // the previous chunk is read
                    for (uint32_t i = threadIdx.x; i < cn; i += SIM_THREADS) s_em[i] = src[c + i];
                    __syncthreads();
                    if (!live) continue;
                    for (uint32_t i = 0; i < cn; i++) {
                        const float4 e = s_em[i];
                        float arg = fmul(k0, e.x);
                        arg = fadd(arg, fmul(k1, e.y));
                        arg = fadd(arg, fmul(k2, e.z));
                        arg = fadd(arg, e.w);
                        float sn, cs;
                        if (a.accurate) {
                            sincosf(arg, &sn, &cs);
                        } else {
                            const float kk = phase_turns(arg);
                            const float r = fmaf(-kk, TWO_PI_LO, fmaf(-kk, TWO_PI_HI, arg));
                            __sincosf(r, &sn, &cs);
                        }
                        re = fadd(re, cs);
                        im = fadd(im, sn);
                    }
                }
                const float a2 = fadd(fmul(re, re), fmul(im, im));
                acc = fadd(acc, a.amplitude_sq ? a2 : __fsqrt_rn(a2));
            }
        total = fadd(total, __fdiv_rn(acc, nsub));
    }
    if (live) a.out[(size_t)f * a.npix + p] = total;
}

// per-frame double sum, one CTA per frame
__global__ void frame_sum_kernel(const float *__restrict__ I, uint64_t npix, double *__restrict__ sums)
{
    const uint32_t f = blockIdx.x;
    const float *x = I + (size_t)f * npix;
    double s = 0;
    for (uint64_t i = threadIdx.x; i < npix; i += blockDim.x) s += (double)x[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; w++) t += sh[w];
        sums[f] = t;
    }
}

// ScalarPoissonSampling, IAC/ArrayOperators.h:25-55; the sequential search
// stops once the term underflows to zero (a draw the rounded cumulative sum
// never reaches would otherwise not end).
__device__ __forceinline__ uint32_t poisson_draw(double mean, uint64_t seed, uint64_t stream, uint64_t idx)
{
    double u0, u1;
    uniform2(seed, stream, idx, u0, u1);
    double ret;
    if (mean < 25) {
        int i = 0;
        double r = exp(-mean);
        double pcum = r;
        while (pcum < u0 && r > 0) {
            i++;
            r *= mean / i;
            pcum += r;
        }
        ret = i;
    } else {
        const double u = 1 - u0, v = 1 - u1;
        ret = (mean + sqrt(mean) * sqrt(-2. * log(u)) * cos(2. * 3.14159265358979323846 * v));
        if (ret < 0) ret = 0;
    }
    return (uint32_t)ret;
}

struct PhotonArgs {
    float *__restrict__ I;  // in: intensity, out: photon image
    const double *__restrict__ sums;
    uint64_t npix;
    uint32_t nframes;
    uint64_t frame0;        // global index of the first frame (random streams)
    double expected;        // AveragePhotonesPerEmitterOnDetector * FlYield * atoms
    int poisson;
    float adu_noise;
    float value_per_photon;
    uint64_t seed;
};

__global__ void photon_kernel(const PhotonArgs a)
{
    const uint32_t f = blockIdx.y;
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= a.npix) return;
    const uint64_t gf = a.frame0 + f;
    // IAC/Simulator.cpp:871-894: factor in double, applied as float
    const float factor = (float)(a.expected / a.sums[f]);
    float v = fmul(a.I[(size_t)f * a.npix + p], factor);
    if (a.poisson) v = (float)poisson_draw((double)v, a.seed, RNG_POISSON | gf, p);
    if (a.adu_noise != 0.0f) {
        double n0, n1;
        uniform2(a.seed, RNG_NOISE | gf, p, n0, n1);
        v = fadd(v, (float)((2 * n0 - 1) * a.adu_noise));
    }
    a.I[(size_t)f * a.npix + p] = fmul(v, a.value_per_photon);
}

// ---------------------------------------------------------------------------
// CreateSparseHitList on the device: photons = pixels with I >= Threshold and
// I > 0 (after the pixel mask), value photonised as ceil((I - T) / Step).
// Pass 1 counts per (frame, block); the host-side scan is replaced by a
// device exclusive scan over the counts; pass 2 writes in pixel order.
// ---------------------------------------------------------------------------
constexpr int SPARSE_THREADS = 256;
constexpr int SPARSE_PIX = 4096;  // pixels per block

__global__ void sparsify_count_kernel(const float *__restrict__ I, const int *__restrict__ mask,
                                      uint64_t npix, float thr, uint32_t *__restrict__ counts)
{
    const uint32_t f = blockIdx.y;
    const uint64_t p0 = (uint64_t)blockIdx.x * SPARSE_PIX;
    uint32_t c = 0;
    for (uint64_t p = p0 + threadIdx.x; p < min(npix, p0 + SPARSE_PIX); p += SPARSE_THREADS) {
        const float v = fmul(I[(size_t)f * npix + p], mask ? (float)mask[p] : 1.0f);
        c += (v >= thr && v > 0.0f) ? 1 : 0;
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ uint32_t s[SPARSE_THREADS / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < SPARSE_THREADS / 32; w++) t += s[w];
        counts[(size_t)f * gridDim.x + blockIdx.x] = t;
    }
}

// exclusive scan of counts (n entries) into offs (n + 1 entries), one CTA
__global__ void __launch_bounds__(1024) scan_u32_kernel(const uint32_t *__restrict__ counts, uint64_t n,
                                                         uint64_t *__restrict__ offs, uint64_t base)
{
    __shared__ unsigned long long ws[32];
    const uint32_t tid = threadIdx.x;
    const uint64_t chunk = (n + 1023) / 1024;
    const uint64_t i0 = min(n, tid * chunk), i1 = min(n, i0 + chunk);
    unsigned long long local = 0;
    for (uint64_t i = i0; i < i1; i++) local += counts[i];
    const int lane = tid & 31, w = tid >> 5;
    unsigned long long incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        const unsigned long long v = ws[lane];
        unsigned long long s = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += u;
        }
        ws[lane] = s - v;
    }
    __syncthreads();
    unsigned long long run = base + ws[w] + incl - local;
    for (uint64_t i = i0; i < i1; i++) {
        offs[i] = run;
        run += counts[i];
    }
    if (tid == 1023) offs[n] = base + ws[w] + incl;
}

__global__ void sparsify_write_kernel(const float *__restrict__ I, const int *__restrict__ mask,
                                      const float *__restrict__ kmap, uint64_t npix, float thr,
                                      float step, int photonize, const uint64_t *__restrict__ block_off,
                                      float4 *__restrict__ out, uint64_t capacity)
{
    const uint32_t f = blockIdx.y;
    const uint64_t p0 = (uint64_t)blockIdx.x * SPARSE_PIX;
    __shared__ uint32_t s_w[SPARSE_THREADS / 32];
    __shared__ uint32_t s_round;
    __shared__ uint64_t s_base;
    if (threadIdx.x == 0) s_base = block_off[(size_t)f * gridDim.x + blockIdx.x];
    __syncthreads();
    for (uint64_t q0 = p0; q0 < min(npix, p0 + SPARSE_PIX); q0 += SPARSE_THREADS) {
        const uint64_t p = q0 + threadIdx.x;
        float v = 0.0f;
        bool keep = false;
        if (p < min(npix, p0 + SPARSE_PIX)) {
            v = fmul(I[(size_t)f * npix + p], mask ? (float)mask[p] : 1.0f);
            keep = v >= thr && v > 0.0f;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, keep);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) s_w[w] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int k = 0; k < SPARSE_THREADS / 32; k++) {
                const uint32_t c = s_w[k];
                s_w[k] = t;
                t += c;
            }
            s_round = t;
        }
        __syncthreads();
        if (keep) {
            const uint64_t o = s_base + s_w[w] + __popc(ball & ((1u << lane) - 1));
            // IAC/ArrayOperators.h:144: ceil((I - T) / Step) * (I >= T)
            const float val = photonize ? ceilf(__fdiv_rn(fsub(v, thr), step)) : v;
            if (o < capacity) out[o] = make_float4(kmap[3 * p], kmap[3 * p + 1], kmap[3 * p + 2], val);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += s_round;
        __syncthreads();
    }
}

// frame offsets, clamped to the capacity so that no consumer reads past the
// photons actually written; a clamp is counted as an overflow
__global__ void frame_offsets_kernel(const uint64_t *__restrict__ block_off, uint32_t blocks_per_frame,
                                     uint32_t nframes, uint64_t capacity,
                                     uint64_t *__restrict__ frame_off, DeviceCounters *counters)
{
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f > nframes) return;
    const uint64_t o = block_off[(size_t)f * blocks_per_frame];
    frame_off[f] = o < capacity ? o : capacity;
    if (f == nframes && o > capacity) atomicAdd(&counters->photon_overflow, o - capacity);
}

}  // namespace iac

using namespace iac;

extern "C" {

iac_status iac_crystal_emitters(iac_ctx *ctx, const double *d_atoms, uint32_t natoms,
                                uint32_t nframes, uint32_t nmodes, const iac_crystal_params *cp,
                                uint64_t seed, float *d_emitters, uint32_t *d_em_count,
                                float *d_rot_event, float *d_rot_crystal, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_atoms && cp && d_emitters && d_em_count && d_rot_event,
                "iac_crystal_emitters: NULL argument");
    IAC_REQUIRE(natoms > 0 && nmodes > 0, "iac_crystal_emitters: no atoms or modes");
    IAC_REQUIRE(cp->fluorescence_yield > 0 && cp->fluorescence_yield <= 1,
                "FluorescenceYield must be in (0, 1]");
    if (nframes == 0) return IAC_OK;
    DeviceGuard g(ctx->device);
    CrystalArgs a;
    a.atoms = d_atoms;
    a.natoms = natoms;
    a.nframes = nframes;
    a.nmodes = nmodes;
    a.seed = seed;
    a.yield = cp->fluorescence_yield;
    a.isotropy = cp->isotropy;
    a.rand_orientation = cp->random_orientation;
    a.incoherent = cp->incoherent;
    a.em = (float4 *)d_emitters;
    a.em_count = d_em_count;
    a.rot_event = d_rot_event;
    a.rot_crystal = d_rot_crystal;
    crystal_emitters_kernel<<<nframes * nmodes, 128, 0, as_stream(stream)>>>(a);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_simulate_intensity(iac_ctx *ctx, const float *d_pixel_map, uint64_t npix,
                                  const float *d_emitters, const uint32_t *d_em_count,
                                  uint32_t natoms, uint32_t nmodes, uint32_t nframes,
                                  const iac_sim_params *sp, float *d_intensity, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_pixel_map && d_emitters && d_em_count && sp && d_intensity,
                "iac_simulate_intensity: NULL argument");
    IAC_REQUIRE(npix > 0 && natoms > 0 && nmodes > 0, "iac_simulate_intensity: empty input");
    IAC_REQUIRE(sp->subsampling >= 0 && sp->subsampling <= 16, "SubSampling out of range");
    IAC_REQUIRE(sp->wavelength > 0, "wavelength must be positive");
    IAC_REQUIRE(nframes <= 65535, "at most 65535 frames per call");
    if (nframes == 0) return IAC_OK;
    DeviceGuard g(ctx->device);
    SimArgs a;
    a.pm = d_pixel_map;
    a.em = (const float4 *)d_emitters;
    a.em_count = d_em_count;
    a.npix = npix;
    a.natoms = natoms;
    a.nmodes = nmodes;
    a.nframes = nframes;
    a.susa = sp->subsampling;
    for (int d = 0; d < 3; d++) {
        a.us[d] = (float)sp->u_step[d];
        a.vs[d] = (float)sp->v_step[d];
    }
    a.wavelength = (float)sp->wavelength;
    a.amplitude_sq = sp->intensity_squared;
    a.accurate = sp->accurate_sincos;
    a.out = d_intensity;
    dim3 grid((unsigned)((npix + SIM_THREADS - 1) / SIM_THREADS), nframes);
    if (natoms <= (uint32_t)SIM_MAX_EM && (uint64_t)nmodes * natoms * 16 <= 200 * 1024) {
        // every mode's emitters staged at once
        const size_t smem = sizeof(float4) * nmodes * natoms;
        IAC_CUDA(cudaFuncSetAttribute(simulate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const dim3 grid2((unsigned)((npix + SIM_PIX * SIM_THREADS - 1) / (SIM_PIX * SIM_THREADS)), nframes);
        simulate_kernel<<<grid2, SIM_THREADS, smem, as_stream(stream)>>>(a);
    } else {
        simulate_chunked_kernel<<<grid, SIM_THREADS, 0, as_stream(stream)>>>(a);
    }
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_simulate_photons(iac_ctx *ctx, float *d_intensity, uint64_t npix, uint32_t nframes,
                                uint64_t first_frame, const iac_photon_params *pp, uint64_t seed,
                                void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_intensity && pp, "iac_simulate_photons: NULL argument");
    IAC_REQUIRE(nframes <= 65535, "at most 65535 frames per call");
    if (nframes == 0 || npix == 0) return IAC_OK;
    DeviceGuard g(ctx->device);
    void *scr = nullptr;
    iac_status st = stream_scratch(ctx, stream, SLOT_AUX0, sizeof(double) * nframes, &scr);
    if (st != IAC_OK) return st;
    cudaStream_t s = as_stream(stream);
    frame_sum_kernel<<<nframes, 256, 0, s>>>(d_intensity, npix, (double *)scr);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    PhotonArgs a;
    a.I = d_intensity;
    a.sums = (const double *)scr;
    a.npix = npix;
    a.nframes = nframes;
    a.frame0 = first_frame;
    a.expected = pp->expected_photons;
    a.poisson = pp->poisson;
    a.adu_noise = pp->adu_noise;
    a.value_per_photon = pp->value_per_photon;
    a.seed = seed;
    dim3 grid((unsigned)((npix + 255) / 256), nframes);
    photon_kernel<<<grid, 256, 0, s>>>(a);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    return IAC_OK;
}

iac_status iac_sparsify_frames(iac_ctx *ctx, const float *d_intensity, const int *d_mask,
                               const float *d_kmap, uint64_t npix, uint32_t nframes, float threshold,
                               float step, int photonize, float *d_photons, uint64_t capacity,
                               uint64_t *d_frame_offsets, uint64_t *h_total, void *stream)
{
    IAC_TRACE();
    IAC_REQUIRE(ctx && d_intensity && d_kmap && d_photons && d_frame_offsets,
                "iac_sparsify_frames: NULL argument");
    IAC_REQUIRE(!photonize || step > 0, "photon step must be positive");
    IAC_REQUIRE(nframes <= 65535, "at most 65535 frames per call");
    DeviceGuard g(ctx->device);
    cudaStream_t s = as_stream(stream);
    if (nframes == 0 || npix == 0) {
        IAC_CUDA(cudaMemsetAsync(d_frame_offsets, 0, sizeof(uint64_t) * (nframes + 1), s));
        if (h_total) *h_total = 0;
        return IAC_OK;
    }
    const uint32_t bpf = (uint32_t)((npix + SPARSE_PIX - 1) / SPARSE_PIX);
    const uint64_t nb = (uint64_t)bpf * nframes;
    void *scr = nullptr;
    const size_t counts_bytes = ((sizeof(uint32_t) * nb + 15) / 16) * 16;
    iac_status st = stream_scratch(ctx, stream, SLOT_AUX1, counts_bytes + sizeof(uint64_t) * (nb + 2), &scr);
    if (st != IAC_OK) return st;
    uint32_t *counts = (uint32_t *)scr;
    uint64_t *boff = (uint64_t *)((char *)scr + counts_bytes);
    dim3 grid(bpf, nframes);
    sparsify_count_kernel<<<grid, SPARSE_THREADS, 0, s>>>(d_intensity, d_mask, npix, threshold, counts);
    IAC_LAUNCHED(ctx);
    scan_u32_kernel<<<1, 1024, 0, s>>>(counts, nb, boff, 0);
    IAC_LAUNCHED(ctx);
    sparsify_write_kernel<<<grid, SPARSE_THREADS, 0, s>>>(d_intensity, d_mask, d_kmap, npix, threshold, step,
                                                          photonize, boff, (float4 *)d_photons, capacity);
    IAC_LAUNCHED(ctx);
    frame_offsets_kernel<<<(nframes + 256) / 256, 256, 0, s>>>(boff, bpf, nframes, capacity,
                                                               d_frame_offsets, ctx->d_counters);
    IAC_LAUNCHED(ctx);
    IAC_CUDA(cudaGetLastError());
    if (h_total) {
        IAC_CUDA(cudaMemcpyAsync(h_total, boff + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        IAC_CUDA(cudaStreamSynchronize(s));
        if (*h_total > capacity) {
            set_error("photon lists need %llu entries, capacity is %llu",
                      (unsigned long long)*h_total, (unsigned long long)capacity);
            return IAC_ERR_INVALID_ARG;
        }
    }
    return IAC_OK;
}

}  // extern "C"
